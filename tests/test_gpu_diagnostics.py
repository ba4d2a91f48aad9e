"""Device comparison metrics (vapor_mac3d_comparison_metrics) and the raw
density dump, against the oracle's restatement of the reference's diagnostic
harness (tests/ReflectionComparison.hpp:32-75) on the same state: counts and
maxima exactly, the FP64 sums to FP64 rounding of a different summation
order (relative 1e-12)."""
import os

import numpy as np
import pytest

from oracle_lib import comparison_metrics
from vapor_b200 import MacSimulation3D
from vapor_b200.diagnostics import harness_params, read_density, write_density

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", [0, 3])
def test_device_metrics_match_the_harness_restatement(variant):
    n = 32
    p = harness_params(variant, 40)
    sim = MacSimulation3D(n, 1.0, p)
    for _ in range(30):
        sim.advance(1.0 / 60.0)
    got = sim.comparison_metrics(60.0)
    d, u, v, w = sim.download()
    want = comparison_metrics(n, 1.0, d, u, v, w, 60.0, p.cfl_mc)
    assert want["smoke_cells"] > 0
    for key in ("smoke_cells", "cfl_fallback", "boundary_fallback"):
        assert got[key] == want[key], key
    for key in ("max_div", "max_cfl"):
        assert got[key] == want[key], key
    for key in ("mass_sum", "mass", "grad_per_mass", "square_per_mass", "rms_div"):
        assert got[key] == pytest.approx(want[key], rel=1e-12, abs=1e-300), key
    sim.close()


def test_density_dump_is_the_raw_fp32_field(tmp_path):
    n = 16
    sim = MacSimulation3D(n, 1.0, harness_params(1, 20))
    for _ in range(5):
        sim.advance(1.0 / 60.0)
    d = sim.download()[0]
    path = os.path.join(tmp_path, "v1_f5.density")
    write_density(path, d)
    assert os.path.getsize(path) == n ** 3 * 4
    assert np.array_equal(read_density(path, n).view(np.uint32), d.view(np.uint32))
    sim.close()


def test_device_render_matches_the_shader_restatement():
    """The CUDA ray-march of a plume's density against the oracle's FP32
    restatement of the volume shader on the same density and camera: the
    same operations except the exponential of the shadow (CUDA's expf against
    the C library's), so channels agree to 1e-4 except where a compositing
    cut-off (alpha > .99, shadow > 3) flips, which the bound on the fraction
    of differing pixels covers."""
    from oracle_lib import render_volume
    from vapor_b200.abi import RenderParams
    n = 32
    sim = MacSimulation3D(n, 1.0, harness_params(3, 40))
    for _ in range(40):
        sim.advance(1.0 / 60.0)
    params = RenderParams.harness(160, 120)
    got = sim.render(params)
    want = render_volume(n, 1.0, sim.download()[0], params)
    bg = np.array([0.03, 0.04, 0.07], np.float32)
    assert (np.abs(want - bg).max(axis=2) > 1e-3).sum() > 100  # the plume is visible
    diff = np.abs(got - want)
    assert (diff > 1e-4).mean() < 1e-3, float(diff.max())
    assert float(diff.max()) < 0.05
    sim.close()
