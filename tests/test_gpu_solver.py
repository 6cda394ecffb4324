"""Matrix-free operator and multigrid PCG against the oracle's assembled CSR K and spsolve.

Tolerances: apply FP64 1e-13 relative to max|y|; apply FP32 2e-6; FP64 solve to
relative residual 1e-10 compared with spsolve at 1e-8 (displacement) and
1e-9 (compliance); mixed-precision compliance within 1e-6 of FP64 (displacements
within 1e-5 at the mixed form's default rtol 1e-6, 1e-6 at rtol 1e-10).
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from oracle import simp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def P():
    import pytopo3d_b200 as P
    from pytopo3d_b200 import _lib

    _lib.lib()
    return P


def _problem(nx, ny, nz, seed=0, support_mask=None, lo=0.0):
    rng = np.random.default_rng(seed)
    shape = (ny, nx, nz)
    rho = rng.uniform(lo, 1.0, size=shape)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    free, fixed = O.build_supports(nx, ny, nz, ndof, support_mask)
    fmask = np.ones(ndof, np.uint8)
    fmask[free] = 0
    return rho, free, fmask


def _oracle_apply(rho, KE, penal, nx, ny, nz, fmask, u):
    K, _ = O.assemble_K(rho, KE, penal, nx, ny, nz)
    z = 1.0 - fmask
    return z * (K @ (z * u)) + fmask * u


# fine_operator 1: dense-KE kernel; 2: Walsh-Hadamard block kernel.  The
# larger grids span several tiles in x and y and several z chunks.
@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("dims", [(6, 4, 3), (5, 7, 2), (1, 1, 1), (13, 3, 4), (8, 33, 3), (41, 70, 9),
                                  (70, 9, 41)])
def test_apply_matches_assembled_matrix(P, dims, form):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=nx)
    u = np.random.default_rng(1).normal(size=fmask.size)
    y_ref = _oracle_apply(rho, KE, 3.0, nx, ny, nz, fmask, u)
    for prec in ("fp64", "mixed"):
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, fine_operator=form)
        s.set_density(to_flat(rho), 3.0)
        st = s.stats()
        assert (st["fine_form_fp64"] == 0) if form == 1 else (st["fine_form_fp64"] >= 1)
        y = s.apply(torch.as_tensor(u).cuda()).cpu().numpy()
        np.testing.assert_allclose(y, y_ref, rtol=0, atol=1e-13 * np.abs(y_ref).max())
        if prec == "mixed":
            # FP32 operator (FP32 moduli) against the FP64 assembled operator
            u32 = u.astype(np.float32).astype(float)
            y32_ref = _oracle_apply(rho, KE, 3.0, nx, ny, nz, fmask, u32)
            y32 = s.apply(torch.as_tensor(u, dtype=torch.float32).cuda()).double().cpu().numpy()
            np.testing.assert_allclose(y32, y32_ref, rtol=0, atol=2e-6 * np.abs(y32_ref).max())
        s.close()
    # BF16-density FP32 operator against the operator of the rounded densities
    s = HexSolver(nx, ny, nz, KE, fmask, precision="mixed", inner_density=1, fine_operator=form)
    s.set_density(to_flat(rho), 3.0)
    rho16 = torch.as_tensor(rho).to(torch.bfloat16).double().numpy()
    y16_ref = _oracle_apply(rho16, KE, 3.0, nx, ny, nz, fmask, u.astype(np.float32).astype(float))
    y16 = s.apply(torch.as_tensor(u, dtype=torch.float32).cuda()).double().cpu().numpy()
    np.testing.assert_allclose(y16, y16_ref, rtol=0, atol=2e-6 * np.abs(y16_ref).max())
    s.close()


# FP32 Walsh-Hadamard shapes: 0-2 the packed two-plane kernel (paired FP32
# instructions), 3-5 the scalar two-barrier kernel, 6-7 the one-barrier kernel.
# Odd plane counts per block and grids spanning several tiles and z chunks; the
# apply against the assembled FP64 operator, and a mixed solve (every epilogue
# mode of the kernel) against FP64.
@pytest.mark.parametrize("shape", range(8))
@pytest.mark.parametrize("dims", [(5, 7, 2), (13, 3, 4), (41, 70, 9), (70, 9, 41), (24, 12, 13)])
def test_fp32_operator_shapes(P, dims, shape):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=nx + ny, lo=0.05)
    u = np.random.default_rng(2).normal(size=fmask.size)
    u32 = u.astype(np.float32).astype(float)
    y_ref = _oracle_apply(rho, KE, 3.0, nx, ny, nz, fmask, u32)
    s = HexSolver(nx, ny, nz, KE, fmask, precision="mixed", fine_operator=3 + shape)
    s.set_density(to_flat(rho), 3.0)
    assert s.stats()["fine_form_fp32"] == 1 + shape
    y = s.apply(torch.as_tensor(u, dtype=torch.float32).cuda()).double().cpu().numpy()
    np.testing.assert_allclose(y, y_ref, rtol=0, atol=2e-6 * np.abs(y_ref).max())
    ndof = fmask.size
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, ndof)).cuda()
    U = s.solve(F)
    r64 = HexSolver(nx, ny, nz, KE, fmask, precision="fp64", rtol=1e-12)
    r64.set_density(to_flat(rho), 3.0)
    U64 = r64.solve(F)
    c, c64 = float(F @ U), float(F @ U64)
    assert abs(c - c64) <= 1e-6 * abs(c64)
    assert s.stats()["fp64_fallback"] == 0
    s.close()
    r64.close()


# The one-barrier kernel (FP32 shapes 6-7) does the two-barrier kernel's
# arithmetic in the same order: its Apply output is bit-identical to the
# two-barrier kernel's, whatever the tile or slab depth, and its solves (every
# epilogue mode) give the same compliance.
@pytest.mark.parametrize("dims", [(5, 7, 2), (41, 70, 9), (70, 9, 41), (24, 12, 13)])
def test_one_barrier_kernel_is_bit_identical(P, dims):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=3 * nx + nz, lo=0.05)
    u = torch.as_tensor(np.random.default_rng(4).normal(size=fmask.size), dtype=torch.float32).cuda()
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    outs, comps = [], []
    for shape in (5, 6, 7):
        s = HexSolver(nx, ny, nz, KE, fmask, precision="mixed", fine_operator=3 + shape)
        s.set_density(to_flat(rho), 3.0)
        st = s.stats()
        assert st["fine_form_fp32"] == 1 + shape
        # the tile the timed choice kept covers the grid with whole node rows
        assert 2 <= st["fine_tile_y"] and 2 <= st["fine_tile_x"]
        assert (st["fine_tile_y"] + 2) * (st["fine_tile_x"] + 2) <= st["fine_threads"]
        outs.append(s.apply(u).cpu())
        comps.append(float(F @ s.solve(F)))
        s.close()
    # a pinned slab depth (node planes per block) changes the tiling, not the result
    for depth in (1, 3):
        s = HexSolver(nx, ny, nz, KE, fmask, precision="mixed", fine_operator=9, fine_slab_depth=depth)
        s.set_density(to_flat(rho), 3.0)
        assert s.stats()["fine_slab_depth"] == min(depth, nz + 1)
        outs.append(s.apply(u).cpu())
        comps.append(float(F @ s.solve(F)))
        s.close()
    for y, c in zip(outs[1:], comps[1:]):
        assert torch.equal(y, outs[0])
        assert c == pytest.approx(comps[0], rel=1e-9)


@pytest.mark.parametrize("tag", ["8x4x4", "32x16x16"])
def test_fp64_solve_matches_reference_direct_solve(P, golden, tag):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = (int(v) for v in golden[f"it{tag}_dims"][:3])
    KE = P.lk_H8(elem_size=1.0)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    F = O.build_force_vector(nx, ny, nz, ndof)
    free, _ = O.build_supports(nx, ny, nz, ndof)
    s = HexSolver.from_freedofs(nx, ny, nz, KE, free, precision="fp64")
    s.set_density(to_flat(golden[f"it{tag}_rho_p"]), 3.0)
    U = s.solve(torch.as_tensor(F).cuda()).cpu().numpy()
    Uref = golden[f"it{tag}_U"]
    assert s.last_relres <= 1e-10
    np.testing.assert_allclose(U, Uref, rtol=0, atol=1e-8 * np.abs(Uref).max())
    assert F @ U == pytest.approx(F @ Uref, rel=1e-9)
    s.close()


# The mixed form stops at its default rtol (1e-6) unless a tighter one is
# given; either way its compliance must stay within 1e-6 of the FP64 form's.
@pytest.mark.parametrize("dims,opts", [((16, 8, 8), {}), ((24, 12, 12), {}), ((20, 7, 9), {}),
                                       ((24, 12, 12), {"inner_density": 1}), ((16, 8, 8), {"rtol": 1e-10}),
                                       ((24, 12, 12), {"inner_density": 1, "rtol": 1e-10}),
                                       ((24, 12, 12), {"coarse_bf16": 0}), ((40, 20, 20), {"coarse_bf16": 1}),
                                       ((16, 8, 8), {"coarse_bf16": 1, "rtol": 1e-10}),
                                       ((40, 20, 20), {"coarse_bf16": 4})])
def test_mixed_precision_matches_fp64(P, dims, opts):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=2, lo=0.0)
    rho[rho < 0.3] = 0.0  # void pockets: E = 1e-9
    ndof = fmask.size
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, ndof)).cuda()
    out = {}
    for prec in ("fp64", "mixed"):
        o = dict(opts)
        if prec == "fp64":
            o.pop("rtol", None)
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, **o)
        rtol = s.opts.rtol
        assert rtol == (1e-10 if prec == "fp64" else opts.get("rtol", 1e-6))
        s.set_density(to_flat(rho), 3.0)
        U = s.solve(F)
        assert s.stats()["device_loop"] == 1.0  # one graph launch per solve, no host polling
        st = s.stats()
        # bf16 stencils on levels 1 .. coarse_bf16, never on the dense coarsest level
        n16 = max(0, min(opts.get("coarse_bf16", 99), int(st["levels"]) - 2)) if prec == "mixed" else 0
        assert st["coarse_bf16"] == n16, st
        # 1e-9 void pockets put an attainable floor on the true residual; the
        # solver accepts it only once restarts / reliable updates stop gaining
        assert s.last_relres <= rtol or (s.stats()["residual_floor"] and s.last_relres <= max(rtol, 1e-7))
        out[prec] = U.cpu().numpy()
        s.close()
    Fh = F.cpu().numpy()
    c64, c32 = Fh @ out["fp64"], Fh @ out["mixed"]
    assert abs(c32 - c64) <= 1e-6 * abs(c64)
    tol_u = 1e-6 if opts.get("rtol", 1e-6) <= 1e-10 else 1e-5
    assert np.linalg.norm(out["mixed"] - out["fp64"]) <= tol_u * np.linalg.norm(out["fp64"])


# The coarse end of the V-cycle as one cooperative launch runs the same
# per-DOF operations as one launch per phase: same iterations, same solution.
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("dims,smoother", [((24, 12, 12), 0), ((48, 24, 24), 0), ((20, 7, 9), 0),
                                           ((24, 12, 12), 1)])
def test_fused_coarse_cycle_matches_per_phase_launches(P, dims, smoother, prec):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    # damped Jacobi needs a mild contrast to converge in few iterations; long
    # runs amplify rounding differences between otherwise identical paths
    rho, free, fmask = _problem(nx, ny, nz, seed=3, lo=0.3 if smoother else 0.0)
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    its, Us = [], []
    for fused in (0, 65536):
        # one thread per DOF on every level: the fused cycle's order of additions
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, fused_cycle_dofs=fused, smoother=smoother,
                      split_dofs=0)
        s.set_density(to_flat(rho), 3.0)
        U = s.solve(F)
        st = s.stats()
        assert (st["fused_cycle_level"] >= 1) == bool(fused), st
        its.append(s.last_iterations)
        Us.append(U.cpu().numpy())
        s.close()
    # rounding may differ where the compiler contracts differently; the long
    # damped-Jacobi runs (hundreds of iterations) may then end a few apart
    assert abs(its[0] - its[1]) <= max(1, 0.02 * its[0]), its
    tol = 1e-9 if prec == "fp64" else 1e-5
    np.testing.assert_allclose(Us[1], Us[0], rtol=0, atol=tol * np.abs(Us[0]).max())


# The small levels' stencil with four lanes per DOF is the same operator as
# one thread per DOF, summed in another order: same iterations (within one or
# 2%), same solution to rounding.
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("dims", [(48, 24, 24), (20, 7, 9), (33, 17, 9)])
def test_split_stencil_matches_one_thread_per_dof(P, dims, prec):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=7, lo=0.0)
    rho[rho < 0.25] = 0.0
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    its, Us = [], []
    for split in (0, 1 << 30):
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, split_dofs=split, fine_operator=3,
                      coarse_node_major=0)
        s.set_density(to_flat(rho), 3.0)
        U = s.solve(F)
        its.append(s.last_iterations)
        Us.append(U.cpu().numpy())
        s.close()
    assert abs(its[0] - its[1]) <= max(1, 0.02 * its[0]), its
    tol = 1e-9 if prec == "fp64" else 1e-5
    np.testing.assert_allclose(Us[1], Us[0], rtol=0, atol=tol * np.abs(Us[0]).max())


# The last smoothed level and the coarsest solve as one block (mixed form)
# compute what the per-phase launches compute (the stencil rows summed in one
# thread's order rather than four lanes'): same iterations within one or 2%,
# same solution to the mixed form's rounding.  The block holds the level's
# operator in shared memory, so it is used when that fits: a last smoothed
# level of at most about 380 nodes with bf16 stencils (64x32x32: 9x5x5 nodes;
# 16x8x8: 9x5x5), not for 40x20x20 (11x6x6 = 396 nodes) or 48x24x24
# (13x7x7), and not with damped Jacobi, whose levels keep FP32 stencils
# (twice the bytes).
@pytest.mark.parametrize("smoother", [0, 1])
@pytest.mark.parametrize("dims,fits", [((64, 32, 32), True), ((40, 20, 20), False), ((16, 8, 8), True),
                                       ((48, 24, 24), False)])
def test_deep_block_cycle_matches_per_phase_launches(P, dims, fits, smoother):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=8, lo=0.3 if smoother else 0.0)
    if not smoother:
        rho[rho < 0.25] = 0.0
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    its, Us = [], []
    for deep in (0, 1):
        s = HexSolver(nx, ny, nz, KE, fmask, precision="mixed", deep_cta=deep, smoother=smoother, fine_operator=3)
        s.set_density(to_flat(rho), 3.0)
        st = s.stats()
        assert st["deep_cta_level"] == (st["levels"] - 2 if deep and fits and not smoother else 0), st
        U = s.solve(F)
        its.append(s.last_iterations)
        Us.append(U.cpu().numpy())
        s.close()
    assert abs(its[0] - its[1]) <= max(1, 0.02 * its[0]), its
    np.testing.assert_allclose(Us[1], Us[0], rtol=0, atol=1e-5 * np.abs(Us[0]).max())


# The two last smoothed levels and the coarsest solve as one thread-block
# cluster (cluster_cycle) against the same levels as per-phase launches plus
# the one-block deep cycle: the same operations, the level before the block
# summed in another order, so the same iterations (within one or 2%) and the
# same solution to rounding.  (16, 8, 8) has too few levels for a cluster.
@pytest.mark.parametrize("dims,used", [((64, 32, 32), True), ((32, 16, 16), True), ((128, 64, 64), True),
                                       ((62, 30, 34), True), ((16, 8, 8), False)])
def test_cluster_cycle_matches_block_cycle(P, dims, used):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=9)
    rho[rho < 0.25] = 0.0
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    its, Us = [], []
    for clu in (0, 1):
        s = HexSolver(nx, ny, nz, KE, fmask, precision="mixed", cluster_cycle=clu, fine_operator=3)
        s.set_density(to_flat(rho), 3.0)
        st = s.stats()
        if clu and used:
            assert st["cluster_level"] == st["levels"] - 3 and st["cluster_ctas"] in (8, 16), st
        else:
            assert st["cluster_level"] == 0, st
        U = s.solve(F)
        its.append(s.last_iterations)
        Us.append(U.cpu().numpy())
        s.close()
    assert abs(its[0] - its[1]) <= max(1, 0.02 * its[0]), its
    np.testing.assert_allclose(Us[1], Us[0], rtol=0, atol=1e-5 * np.abs(Us[0]).max())


# Coarse levels from the node-major bf16 stencil (three lanes per node) against
# the packed bf16 stencil (one thread per DOF): the same coefficients summed in
# another order, so each level's operator agrees to FP32 rounding, and the mixed
# solves agree with each other and with FP64.  split_dofs=0 keeps the packed
# solver's small levels at one thread per DOF; odd sizes give ragged last warps.  The level
# builders write the node-major rows themselves (galerkin 0); the stencil triple
# product (galerkin 1) is permuted from the packed layout.
@pytest.mark.parametrize("galerkin", [0, 1])
@pytest.mark.parametrize("dims", [(24, 12, 13), (41, 18, 22), (64, 32, 32)])
def test_node_major_coarse_levels_match_packed(P, dims, galerkin):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=nx + 2 * nz, lo=0.01)
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    solvers = [HexSolver(nx, ny, nz, KE, fmask, precision="mixed", split_dofs=0, coarse_node_major=nm,
                         galerkin=galerkin) for nm in (0, 1)]
    for s in solvers:
        s.set_density(to_flat(rho), 3.0)
    nlev = int(solvers[0].stats()["levels"])
    assert nlev >= 3
    gen = torch.Generator(device="cuda").manual_seed(7)
    g = list(solvers[0].grid)
    for L in range(1, nlev - 1):
        g = [(v + 1) // 2 for v in g]
        nn = (g[0] + 1) * (g[1] + 1) * (g[2] + 1)
        u = torch.randn(3 * nn, device="cuda", generator=gen, dtype=torch.float32)
        y0, y1 = (s.apply_level(L, u) for s in solvers)
        assert torch.isfinite(y1).all()
        tol = 2e-6 * float(y0.abs().max())
        assert float((y1 - y0).abs().max()) <= tol, (L, float((y1 - y0).abs().max()), tol)
    r64 = HexSolver(nx, ny, nz, KE, fmask, precision="fp64", rtol=1e-12)
    r64.set_density(to_flat(rho), 3.0)
    c64 = float(F @ r64.solve(F))
    its = []
    for s in solvers:
        c = float(F @ s.solve(F))
        its.append(s.last_iterations)
        assert abs(c - c64) <= 1e-6 * abs(c64)
        assert s.stats()["fp64_fallback"] == 0
        s.close()
    r64.close()
    assert abs(its[0] - its[1]) <= max(1, 0.05 * its[0]), its


# Residual and restriction in one launch on the small levels are the same
# operations as the two launches, summed in another order: same iterations
# (within one or 2%), same solution to rounding.
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("dims", [(48, 24, 24), (33, 17, 9)])
def test_fused_residual_restriction_matches_two_launches(P, dims, prec):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=12, lo=0.0)
    rho[rho < 0.25] = 0.0
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    its, Us = [], []
    for thr in (0, 1 << 30):
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, resid_restrict_dofs=thr, fine_operator=3)
        s.set_density(to_flat(rho), 3.0)
        U = s.solve(F)
        its.append(s.last_iterations)
        Us.append(U.cpu().numpy())
        s.close()
    assert abs(its[0] - its[1]) <= max(1, 0.02 * its[0]), its
    tol = 1e-9 if prec == "fp64" else 1e-5
    np.testing.assert_allclose(Us[1], Us[0], rtol=0, atol=tol * np.abs(Us[0]).max())


# The split solve (queue, let the caller queue work on U, then wait) gives the
# blocking solve's result; when the mixed form has to finish in FP64 (here: an
# iteration cap it cannot meet) the FP64 solve runs after the caller's queued
# work and reports that U was replaced.
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("cap", [5000, 4])
def test_split_solve_matches_blocking_solve(P, prec, cap):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 24, 12, 12
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=10, lo=0.0)
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    out = []
    for split in (False, True):
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, max_iterations=cap, fine_operator=3)
        s.set_density(to_flat(rho), 3.0)
        U = torch.zeros_like(F)
        seen = None
        if split:
            s.solve_begin(F, U)
            seen = torch.dot(U, F)  # queued behind the solve
            replaced = s.solve_end(raise_on_fail=False)
            assert replaced == (prec == "mixed" and cap == 4)
        else:
            s.solve(F, U, raise_on_fail=False)
        out.append((U.cpu().numpy(), s.last_iterations, seen))
        s.close()
    (U0, it0, _), (U1, it1, seen) = out
    assert it0 == it1
    np.testing.assert_array_equal(U1, U0)
    if not (prec == "mixed" and cap == 4):
        assert float(seen) == float(np.dot(U0, F.cpu().numpy())) or abs(float(seen) - float(np.dot(U0, F.cpu().numpy()))) <= 1e-12 * abs(float(seen))


# Programmatic dependent launch only changes when a kernel may be scheduled,
# never what it computes or in which order the kernels' writes land: every
# mask gives bit-identical iterations and solutions, with the device loop.
# (The fine operator's launch shape is fixed: the timed choice may pick
# another shape per solver, which rounds differently.)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_programmatic_launch_is_bitwise_neutral(P, prec):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 40, 20, 20
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=6, lo=0.0)
    rho[rho < 0.3] = 0.0
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    its, Us = [], []
    for mask in (0, 1, 2, 3):
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, pdl=mask, fine_operator=3)
        s.set_density(to_flat(rho), 3.0)
        U = s.solve(F)
        st = s.stats()
        assert st["pdl"] == mask and st["device_loop"] == 1.0, st
        its.append(s.last_iterations)
        Us.append(U.cpu().numpy())
        s.close()
    assert len(set(its)) == 1, its
    for U in Us[1:]:
        np.testing.assert_array_equal(U, Us[0])


# Levels >= 2 from element-wise Galerkin products (default) and from the
# stencil triple product P^T A P are the same operators up to rounding: same
# iterations, same solution.  Odd grids exercise the padded coarse elements.
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("dims", [(48, 24, 24), (33, 17, 9), (40, 12, 21)])
def test_element_galerkin_matches_stencil_galerkin(P, dims, prec):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = dims
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=5, lo=0.0)
    rho[rho < 0.25] = 0.0
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    its, Us = [], []
    for gal in (1, 0):
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, galerkin=gal)
        s.set_density(to_flat(rho), 3.0)
        assert s.stats()["levels"] >= 3
        U = s.solve(F)
        its.append(s.last_iterations)
        Us.append(U.cpu().numpy())
        s.close()
    assert abs(its[0] - its[1]) <= 1, its
    tol = 1e-9 if prec == "fp64" else 1e-5
    np.testing.assert_allclose(Us[1], Us[0], rtol=0, atol=tol * np.abs(Us[0]).max())


def test_damped_jacobi_smoother_option(P):
    # damped Jacobi (omega 0.6) is stable for grey designs without voids
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 16, 8, 8
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=3, lo=0.2)
    F = O.build_force_vector(nx, ny, nz, fmask.size)
    Uref, _ = O.solve_displacement(rho, KE, 3.0, F, free, nx, ny, nz)
    for prec in ("fp64", "mixed"):
        s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, smoother=1)
        s.set_density(to_flat(rho), 3.0)
        U = s.solve(torch.as_tensor(F).cuda()).cpu().numpy()
        np.testing.assert_allclose(U, Uref, rtol=0, atol=1e-7 * np.abs(Uref).max())
        s.close()


def test_multigrid_and_jacobi_agree_with_spsolve(P):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 10, 5, 6
    KE = P.lk_H8(elem_size=0.01)
    sm = np.zeros((ny, nx, nz), bool)
    sm[1:3, 0, 2:4] = True  # small clamp patch: coarse levels need the dilation rule
    rho, free, fmask = _problem(nx, ny, nz, seed=4, support_mask=sm, lo=0.05)
    ndof = fmask.size
    F = O.build_force_vector(nx, ny, nz, ndof)
    Uref, _ = O.solve_displacement(rho, KE, 3.0, F, free, nx, ny, nz)
    for opts in (dict(), dict(max_levels=1, max_iterations=20000)):
        s = HexSolver(nx, ny, nz, KE, fmask, precision="fp64", **opts)
        s.set_density(to_flat(rho), 3.0)
        U = s.solve(torch.as_tensor(F).cuda()).cpu().numpy()
        np.testing.assert_allclose(U, Uref, rtol=0, atol=1e-7 * np.abs(Uref).max())
        s.close()


def test_iteration_cap_raises_runtime_error(P):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 12, 6, 6
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=6, lo=0.01)
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    s = HexSolver(nx, ny, nz, KE, fmask, precision="fp64", max_iterations=1)
    s.set_density(to_flat(rho), 3.0)
    with pytest.raises(RuntimeError, match="converge"):
        s.solve(F)
    s.close()


# The coarsest dense inverse handles a failed elimination on the device: an
# operator with negative moduli (negative densities, E = -1) has a negative
# first pivot, every shifted attempt fails too, and the inverse falls back to
# the inverse diagonal (zero where the diagonal is not positive); a normal
# operator takes the first attempt.
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_coarsest_inverse_falls_back_on_the_device(P, prec):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 16, 8, 8
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=9, lo=0.1)
    s = HexSolver(nx, ny, nz, KE, fmask, precision=prec, smoother=1)
    s.set_density(to_flat(rho), 3.0)
    st = s.stats()
    assert st["coarsest_status"] == 0 and st["coarse_fallback"] == 0, st
    s.set_density(to_flat(-np.ones_like(rho)), 3.0)
    st = s.stats()
    assert st["coarsest_status"] == 4 and st["coarse_fallback"] == 1, st
    s.set_density(to_flat(rho), 3.0)  # and back
    st = s.stats()
    assert st["coarsest_status"] == 0 and st["coarse_fallback"] == 0, st
    s.close()


def test_nonfinite_density_reports_an_error_not_a_hang(P):
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 8, 4, 4
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=7, lo=0.1)
    rho[1, 2, 1] = np.nan
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    s = HexSolver(nx, ny, nz, KE, fmask, precision="fp64", max_iterations=50)
    s.set_density(to_flat(rho), 3.0)
    with pytest.raises(RuntimeError):
        s.solve(F)
    s.close()


@pytest.mark.parametrize("precision,criterion", [("fp64", "time"), ("mixed", "time"), ("mixed", "bytes")])
def test_autotune_picks_measured_degrees_and_caches_them(P, precision, criterion):
    """tp3d_solver_autotune searches the smoothing degrees by timing solves on
    the grid at hand (a coordinate search of at most 7 candidates), keeps the
    fastest, records it in stats(), caches it per (grid, precision), and
    leaves the solution unchanged within the solver's tolerance."""
    from pytopo3d_b200.solver import HexSolver
    from pytopo3d_b200._tensors import to_flat

    nx, ny, nz = 26, 13, 11  # a grid no other test tunes (the cache is per grid, precision, criterion)
    rho, free, fmask = _problem(nx, ny, nz, seed=4, lo=0.05)
    KE = P.lk_H8(elem_size=1.0)
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, ndof)).cuda()
    rd = to_flat(rho)
    ref = HexSolver(nx, ny, nz, KE, fmask, precision=precision)
    ref.set_density(rd, 3.0)
    U_ref = ref.solve(F)
    s = HexSolver(nx, ny, nz, KE, fmask, precision=precision)
    s.set_density(rd, 3.0)
    t = s.autotune(F, criterion=criterion)
    assert not t["from_cache"] and 1 <= t["tried"] <= 7
    assert t["degree_fine"] in (1, 2) and t["degree_level1"] in (1, 2, 3) and t["degree_deep"] in (2, 4, 6)
    assert 0 < t["best"] <= t["start"], t
    st = s.stats()
    assert st["autotuned"] == 1 and st["degree_fine"] == t["degree_fine"]
    assert st["degree_level1"] == t["degree_level1"] and st["degree_level2"] == t["degree_deep"]
    U = s.solve(F)
    tol = 1e-8 if precision == "fp64" else 1e-5
    assert float((U - U_ref).norm() / U_ref.norm()) <= tol
    s2 = HexSolver(nx, ny, nz, KE, fmask, precision=precision)
    s2.set_density(rd, 3.0)
    t2 = s2.autotune(F, criterion=criterion)
    assert t2["from_cache"] and (t2["degree_fine"], t2["degree_level1"], t2["degree_deep"]) == (
        t["degree_fine"], t["degree_level1"], t["degree_deep"])
    assert s2.stats()["autotuned"] == 2
    for h in (ref, s, s2):
        h.close()


# Rayleigh-Ritz start (tp3d_solver_ritz_start): for the new operator, the
# combination of the last two solutions has an energy x'Kx/2 - F'x no higher
# than the linear extrapolation 2 U1 - U2 or U1 (both lie in the same span), the
# history is rotated (U_prev <- U1), and without history U is left as it is.
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_ritz_start_lowers_the_energy_of_the_initial_guess(P, prec):
    from pytopo3d_b200 import _lib
    from pytopo3d_b200._tensors import to_flat
    from pytopo3d_b200.solver import HexSolver

    nx, ny, nz = 24, 12, 12
    KE = P.lk_H8(elem_size=1.0)
    rho, free, fmask = _problem(nx, ny, nz, seed=21, lo=0.05)
    F = torch.as_tensor(O.build_force_vector(nx, ny, nz, fmask.size)).cuda()
    s = HexSolver(nx, ny, nz, KE, fmask, precision=prec)
    assert s.opts.ritz_start == 1
    sols = []
    for scale in (1.0, 0.97, 0.94):
        r = np.clip(rho * scale, 0.01, 1.0)
        s.set_density(to_flat(r), 3.0)
        sols.append(s.solve(F).clone())
    U1, U2 = sols[1], sols[0]
    # the third density's operator is current (its solve is in sols[2])

    def energy(x):
        y = s.apply(x)
        return 0.5 * float(x @ y) - float(F @ x)

    L = _lib.lib()
    U, Up = U1.clone(), U2.clone()
    _lib.check(L.tp3d_solver_ritz_start(s._h, F.data_ptr(), U.data_ptr(), Up.data_ptr(), 1), "ritz_start")
    torch.cuda.synchronize()
    assert torch.equal(Up, U1)
    e_ritz, e_ext, e_last = energy(U), energy(2 * U1 - U2), energy(U1)
    assert e_ritz <= e_ext + 1e-12 * abs(e_ext) and e_ritz <= e_last + 1e-12 * abs(e_last)
    # no history: U unchanged, U_prev takes it
    U, Up = U1.clone(), torch.zeros_like(U1)
    _lib.check(L.tp3d_solver_ritz_start(s._h, F.data_ptr(), U.data_ptr(), Up.data_ptr(), 0), "ritz_start")
    torch.cuda.synchronize()
    assert torch.equal(U, U1) and torch.equal(Up, U1)
    s.close()
    # without the option the entry point is refused and the loops use the extrapolation
    s0 = HexSolver(nx, ny, nz, KE, fmask, precision=prec, ritz_start=0)
    s0.set_density(to_flat(rho), 3.0)
    assert L.tp3d_solver_ritz_start(s0._h, F.data_ptr(), U.data_ptr(), Up.data_ptr(), 1) == _lib.TP3D_ERR_ARG
    s0.close()
