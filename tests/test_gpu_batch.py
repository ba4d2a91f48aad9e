"""Batched scenes and the sweep tuning hook: same bits as the scenes stepped
one by one."""
import numpy as np
import pytest

import vapor_b200 as vb
from oracle_lib import algorithm_params
from vapor_b200.abi import LinearSolveOptions

pytestmark = pytest.mark.gpu


def _scene(n, alg, k):
    p = algorithm_params(alg)
    p.stir_strength = 0.5
    p.emitter_center_x = 0.3 + 0.1 * k
    p.use_solve_options = 1
    p.solve = LinearSolveOptions.defaults(max_iterations=3000, relative_tolerance=1e-6, absolute_tolerance=0.0)
    p.solver_kind = vb.abi.SOLVER_MIXED_REFINEMENT
    return vb.MacSimulation3D(n, 1.0, p)


def test_batched_graph_equals_separate_steps():
    sizes = [(16, 3), (24, 1), (32, 2), (20, 0)]
    single = [_scene(n, a, k) for k, (n, a) in enumerate(sizes)]
    grouped = [_scene(n, a, k) for k, (n, a) in enumerate(sizes)]
    batch = vb.Batch(grouped)
    for _ in range(4):
        for s in single:
            s.advance(0.01)
        batch.advance(0.01)
    batch.synchronize()
    for a, b in zip(single, grouped):
        assert a.total_iterations() == b.total_iterations()
        for x, y in zip(a.download(), b.download()):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    # the scenes stay usable one by one after batching
    grouped[0].advance(0.01)
    single[0].advance(0.01)
    for x, y in zip(single[0].download(), grouped[0].download()):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    batch.close()


def test_sor_plane_tuning_changes_no_bits():
    n = 32
    ref = _scene(n, 3, 0)
    for _ in range(2):
        ref.advance(0.01)
    vb.tune_sor_planes(n, 8)
    try:
        tuned = _scene(n, 3, 0)
        for _ in range(2):
            tuned.advance(0.01)
    finally:
        vb.tune_sor_planes(n, 0)
    assert ref.total_iterations() == tuned.total_iterations()
    for x, y in zip(ref.download(), tuned.download()):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_batch_rejects_duplicates():
    s = _scene(16, 0, 0)
    with pytest.raises(vb.InvalidArgument):
        vb.Batch([s, s])
