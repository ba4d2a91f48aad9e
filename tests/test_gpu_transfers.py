"""Streamed host transfers of the resident simulation (vapor_mac3d_upload_async,
vapor_mac3d_download_async, vapor_mac3d_wait_transfers): the same steps and
the same host results as the synchronous upload / advance / download, with
the copies on their own streams."""
import numpy as np
import pytest

import vapor_b200 as vb
from vapor_b200.abi import field_shapes

pytestmark = pytest.mark.gpu
DT = 1 / 60


def _params():
    p = vb.algorithm_params(vb.abi.REFLECTION_MACCORMACK)
    p.emitter_radius, p.emitter_center_z = .2, .3
    return p


def _states(n, count, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        fields = [rng.random(s, dtype=np.float32) * .5 if k == 0 else
                  (rng.standard_normal(s) * .3).astype(np.float32) for k, s in enumerate(field_shapes(n))]
        out.append(fields)
    return out


def _pinned_like(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True).numpy()
    t[...] = a
    return t


def _bits(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("pinned", [True, False])
def test_streamed_steps_equal_synchronous_steps(pinned):
    """Each step's inputs uploaded from the host and its result downloaded:
    the streamed calls give the synchronous calls' bits, step after step."""
    n = 32
    inputs = _states(n, 5)
    if pinned:
        inputs = [[_pinned_like(a) for a in fields] for fields in inputs]
    sync = vb.MacSimulation3D(n, 1.0, _params())
    want = []
    for fields in inputs:
        sync.upload(*fields)
        sync.advance(DT)
        want.append(sync.download())
    streamed = vb.MacSimulation3D(n, 1.0, _params())
    got = [[np.empty(s, np.float32) if not pinned else _pinned_like(np.zeros(s, np.float32))
            for s in field_shapes(n)] for _ in inputs]
    for fields, out in zip(inputs, got):
        streamed.upload_async(*fields)
        streamed.advance(DT)
        streamed.download_async(out)
    streamed.wait_transfers()
    for k, (g, w) in enumerate(zip(got, want)):
        for name, a, b in zip(("density", "u", "v", "w"), g, w):
            assert _bits(a, b), (k, name)
    assert streamed.byte_counters() == sync.byte_counters()
    sync.close()
    streamed.close()


def test_downloads_snapshot_the_steps_issued_before_them():
    """Downloads after every step of a run without uploads, one output
    buffer reused: each snapshot is its step's state."""
    n = 32
    a = vb.MacSimulation3D(n, 1.0, _params())
    b = vb.MacSimulation3D(n, 1.0, _params())
    outs = [[np.empty(s, np.float32) for s in field_shapes(n)] for _ in range(4)]
    want = []
    for out in outs:
        a.advance(DT)
        a.download_async(out)
        b.advance(DT)
        want.append(b.download())
    a.wait_transfers()
    for g, w in zip(outs, want):
        for x, y in zip(g, w):
            assert _bits(x, y)
    a.close()
    b.close()


def test_a_synchronous_upload_replaces_a_staged_one():
    n = 16
    s1, s2 = _states(n, 2)
    a = vb.MacSimulation3D(n, 1.0, _params())
    a.upload_async(*s1)
    a.upload(*s2)  # replaces the staged snapshot
    a.advance(DT)
    got = a.download()
    b = vb.MacSimulation3D(n, 1.0, _params())
    b.upload(*s2)
    b.advance(DT)
    for x, y in zip(got, b.download()):
        assert _bits(x, y)
    a.wait_transfers()
    a.close()
    b.close()
