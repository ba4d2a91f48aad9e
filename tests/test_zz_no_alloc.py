"""vapor_advect_noalloc: MacCormack/semi-Lagrangian advection whose scratch is
a fixed array in the library's device image, for callers that must not
allocate device memory while they advect (a frame loop that cannot afford the
device-wide synchronization of cudaFree, or a host that owns all device memory
and only lends buffers to plugins).

Checked through the C ABI against the existing staged entry point
(vapor_stage_advect_*_device) on two calls in a row, bit for bit (the bar of
the other advection tests). The second call must not change the device's
free memory; the first may commit the fixed array itself (its module loads
lazily) and nothing more. This file is collected last so a failure here comes after every
other test has run; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import vapor_b200 as vb
from oracle_lib import random_fields
from vapor_b200.abi import MACCORMACK, SEMI_LAGRANGIAN

pytestmark = pytest.mark.gpu


def _lib():
    lib = vb.library()
    fn = lib.vapor_advect_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32, C.c_float, C.c_int32, C.c_float, C.c_float, C.c_int32, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def _stage_reference(n, box, loc, dt, cfl, method, src, flow):
    """The existing entry point on device memory (it allocates its workspace)."""
    import torch
    stage = vb.StageBackend(n, box)
    out = torch.empty_like(src)
    if loc == 0:
        out.copy_(src)
        vb.check(vb.library().vapor_stage_advect_scalar_device(stage._h, dt, cfl, method, out.data_ptr(),
                                                               *[f.data_ptr() for f in flow]))
    else:
        vb.check(vb.library().vapor_stage_advect_face_device(stage._h, loc - 1, dt, cfl, method, src.data_ptr(),
                                                             *[f.data_ptr() for f in flow], out.data_ptr()))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("method", [MACCORMACK, SEMI_LAGRANGIAN])
def test_noalloc_matches_existing_entry_point_twice(method):
    import torch
    lib = _lib()
    n, box, dt, cfl = 48, 2.0, 0.05, 3.0
    fields = random_fields(n, seed=77, scale=1.5)
    dev = [torch.from_numpy(a.copy()).cuda() for a in fields]
    flow = dev[1:]
    for loc, src in enumerate(dev):
        expected = _stage_reference(n, box, loc, dt, cfl, method, src, flow)
        outs = []
        for call in range(2):
            out = torch.full_like(src, float("nan"))
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            st = lib.vapor_advect_noalloc(n, box, loc, dt, cfl, method, src.data_ptr(), flow[0].data_ptr(),
                                          flow[1].data_ptr(), flow[2].data_ptr(), out.data_ptr(), None)
            assert st == 0, vb.library().vapor_last_error()
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            if call == 0:
                # the first call may load the array's module (lazy loading),
                # which commits at most the 4 MiB array (2 MiB pages)
                assert free_before - free_after <= (4 << 20) + (2 << 20)
            else:
                assert free_after == free_before
            outs.append(out.cpu().numpy())
        for got in outs:
            assert np.array_equal(got.view(np.uint32), expected.view(np.uint32)), f"loc {loc}"


def test_noalloc_rejects_oversize_and_aliasing():
    import torch
    lib = _lib()
    n = 102  # 102*102*103 face values exceed the fixed scratch
    big = torch.zeros(n * n * (n + 1), device="cuda")
    out = torch.zeros_like(big)
    st = lib.vapor_advect_noalloc(n, 1.0, 1, 0.01, 3.0, MACCORMACK, big.data_ptr(), big.data_ptr(),
                                  big.data_ptr(), big.data_ptr(), out.data_ptr(), None)
    assert st == vb.abi.VAPOR_LENGTH_ERROR
    assert b"scratch capacity" in vb.library().vapor_last_error()
    small = torch.zeros(8 * 8 * 9, device="cuda")
    st = lib.vapor_advect_noalloc(8, 1.0, 1, 0.01, 3.0, MACCORMACK, small.data_ptr(), small.data_ptr(),
                                  small.data_ptr(), small.data_ptr(), small.data_ptr(), None)
    assert st == vb.abi.VAPOR_INVALID_ARGUMENT
