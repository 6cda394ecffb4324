"""The batched workload: seeded cantilevers of uneven sizes, each an
independent SimpLoop on its own stream, driven by several host threads.
Running them concurrently must give exactly what running them one at a time
gives (the designs share nothing but the GPU).  FP64 with a fixed fine-operator
shape, so both runs execute the same kernels on the same data."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_seeded_batch_has_the_workload_ranges():
    from pytopo3d_b200.batch import batched_cantilevers

    specs = batched_cantilevers(64, seed=0)
    assert len(specs) == 64
    for s in specs:
        assert 24 <= s.nelx <= 96 and s.nely == s.nelx // 2 and 12 <= s.nelz <= 48
        assert 0.15 <= s.volfrac <= 0.4 and 1.5 <= s.rmin <= 3.5
        assert 0 <= len(s.cylinders) <= 3 and all(2 <= c[3] <= 8 for c in s.cylinders)
    assert any(s.load_mid for s in specs) and not all(s.load_mid for s in specs)
    assert batched_cantilevers(64, seed=0)[5] == specs[5]  # seeded


def test_concurrent_designs_match_sequential_runs():
    from pytopo3d_b200.batch import BatchRunner, batched_cantilevers, design_problem
    from pytopo3d_b200.optimizer import SimpLoop
    from pytopo3d_b200.stiffness import lk_H8

    specs = batched_cantilevers(6, seed=1)
    opts = {"fine_operator": 3}
    br = BatchRunner(specs, precision="fp64", workers=3, solver_options=opts, tune=None)
    stats = br.run(2)
    assert stats["designs"] == 6 and stats["simp_iterations_per_s"] > 0
    KE = lk_H8(elem_size=1.0)
    for i, spec in enumerate(specs):
        shape, solid, void, F, fixed = design_problem(spec)
        loop = SimpLoop(spec.nelx, spec.nely, spec.nelz, spec.volfrac, spec.penal, spec.rmin, KE, F, fixed,
                        solid, void, precision="fp64", solver_options=opts)
        loop.set_beta(1.0)
        for _ in range(2):
            st = loop.step()
        c = float(st[0])
        assert c == pytest.approx(br.compliance[i], rel=1e-10), i
        np.testing.assert_allclose(loop.design().cpu().numpy(), br.design(i).cpu().numpy(), rtol=0, atol=1e-10)
        loop.close()
    br.close()


def test_batch_designs_are_autotuned_one_by_one():
    """With tuning on (the default), every design gets smoothing degrees searched
    on its own grid, and the batch still runs."""
    from pytopo3d_b200.batch import BatchRunner, batched_cantilevers

    specs = batched_cantilevers(3, seed=7)
    br = BatchRunner(specs, precision="mixed", workers=3)
    assert len(br.tuning) == 3
    for t, loop in zip(br.tuning, br.loops):
        assert t["degree_fine"] in (1, 2) and t["degree_deep"] in (2, 4, 6)
        assert loop.solver.stats()["autotuned"] in (1, 2)
    stats = br.run(2)
    assert np.isfinite(br.compliance).all() and stats["dof_cg_iterations_per_s"] > 0
    br.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_graph_matches_host_runs(precision):
    """All designs advanced by one graph launch (each design's loop body in a
    WHILE node of its own, parallel branches) give exactly what each design's
    host-driven loop gives, and a second launch continues them."""
    from pytopo3d_b200.batch import BatchRunner, batched_cantilevers, design_problem
    from pytopo3d_b200.optimizer import SimpLoop
    from pytopo3d_b200.stiffness import lk_H8

    specs = batched_cantilevers(5, seed=3)
    opts = {"fine_operator": 3}
    br = BatchRunner(specs, precision=precision, workers=1, solver_options=opts, tune=None)
    br.run(1)
    stats = br.run_graph(2)
    assert stats["designs"] == 5 and stats["handed_back"] == 0
    br.run_graph(2)
    KE = lk_H8(elem_size=1.0)
    for i, spec in enumerate(specs):
        shape, solid, void, F, fixed = design_problem(spec)
        loop = SimpLoop(spec.nelx, spec.nely, spec.nelz, spec.volfrac, spec.penal, spec.rmin, KE, F, fixed,
                        solid, void, precision=precision, solver_options=opts)
        loop.set_beta(1.0)
        for _ in range(5):
            st = loop.step()
        assert float(st[0]) == br.compliance[i], i
        np.testing.assert_array_equal(loop.design().cpu().numpy(), br.design(i).cpu().numpy())
        loop.close()
    br.close()
