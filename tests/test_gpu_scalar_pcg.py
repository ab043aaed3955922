"""FP64 PCG on scalar matrices, whose SpMV is the TMA-staged tiled kernel
whenever its tiles fit (cg.rs:40-149 arithmetic up to the order of the dot
products), against the oracle's CG: P1 rows of ~7 entries (256-row tiles)
and P2 rows of ~28 (64-row tiles), and the repeatability the kernel choice
rule is there for.

Tolerances: iteration counts within max(3, 2 %) of the oracle's; solutions
within 1e-8 relative L2 of a direct solve at a 1e-12 tolerance; the
recurrence reaches 1e-12 and the true residual of the returned x is below
1e-10; repeated solves, on the same matrix and on a second matrix of the
same shape (which takes the remembered kernel choice), bit-identical.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle as O

pytestmark = pytest.mark.gpu


def _system_p1(n):
    om = O.unit_square(n, n)
    rng = np.random.default_rng(5)
    kappa = np.exp(rng.standard_normal(om.nc))
    A = O.assemble_stiffness_2d(om, kappa)
    b = O.assemble_rhs_2d(om, lambda x, y: np.sin(3 * x) + y)
    bd = O.boundary_dofs_2d(om)
    return om, kappa, bd, O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))


def _device_p1(fcu, ctx, om, kappa, bd):
    V = fcu.FunctionSpace(ctx, fcu.Mesh(om.coords, om.cells), fcu.FCU_SPACE_P1)
    M = fcu.Matrix(ctx, V).assemble_stiffness(kappa)
    return V, M


@pytest.mark.parametrize("n", [96, 200])
def test_p1_fp64_pcg_matches_oracle(fcu, ctx, n):
    om, kappa, bd, (Ab, bb) = _system_p1(n)
    V, M = _device_p1(fcu, ctx, om, kappa, bd)
    b = np.asarray(O.assemble_rhs_2d(om, lambda x, y: np.sin(3 * x) + y))
    M.apply_dirichlet(b, bd, np.zeros(len(bd)))
    assert np.max(np.abs(b - bb)) <= 1e-14 * np.max(np.abs(bb))
    x, info = M.pcg(b, tol=1e-12, max_iter=20000)
    _, it_o, _ = O.solve_cg(Ab, bb, None, 1e-12, 20000)
    assert abs(info.iterations - it_o) <= max(3, 0.02 * it_o), (info.iterations, it_o)
    S = Ab.to_scipy().tocsc()
    xd = spla.spsolve(S, bb)
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    assert info.rel_residual < 1e-12
    assert np.linalg.norm(bb - S @ x) / np.linalg.norm(bb) < 1e-10
    M.close()
    V.close()


def test_p2_fp64_pcg_matches_oracle(fcu, ctx):
    om = O.unit_cube(10, 10, 10)
    cd, ev = O.p2_dofmap(om)
    nd = om.nv + len(ev)
    rng = np.random.default_rng(8)
    kappa = np.exp(rng.standard_normal(om.nc))
    A = O.assemble_p2_stiffness_3d(om, cd, nd, kappa)
    bd = O.p2_boundary_dofs(om)
    b0 = np.cos(np.arange(nd) * 0.01)
    Ab, bb = O.apply_dirichlet_bc(A, b0, bd, np.zeros(len(bd)))
    V = fcu.FunctionSpace(ctx, fcu.Mesh(om.coords, om.cells), fcu.FCU_SPACE_P2)
    assert V.ndofs == nd
    M = fcu.Matrix(ctx, V).assemble_stiffness(kappa)
    b = b0.copy()
    M.apply_dirichlet(b, bd, np.zeros(len(bd)))
    assert np.max(np.abs(b - bb)) <= 1e-14 * np.max(np.abs(bb))
    x, info = M.pcg(b, tol=1e-12, max_iter=20000)
    _, it_o, _ = O.solve_cg(Ab, bb, None, 1e-12, 20000)
    assert abs(info.iterations - it_o) <= max(3, 0.02 * it_o), (info.iterations, it_o)
    S = Ab.to_scipy().tocsc()
    xd = spla.spsolve(S, bb)
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    M.close()
    V.close()


def test_fp64_scalar_pcg_repeats_bit_for_bit(fcu, ctx):
    om, kappa, bd, (Ab, bb) = _system_p1(160)
    b = np.asarray(O.assemble_rhs_2d(om, lambda x, y: np.sin(3 * x) + y))
    runs = []
    for _ in range(2):  # a second matrix of the same shape takes the remembered choice
        V, M = _device_p1(fcu, ctx, om, kappa, bd)
        bb2 = b.copy()
        M.apply_dirichlet(bb2, bd, np.zeros(len(bd)))
        for _ in range(2):
            x, info = M.pcg(bb2, tol=1e-10, max_iter=20000)
            runs.append((x.copy(), info.iterations, info.rel_residual))
        M.close()
        V.close()
    x0, it0, r0 = runs[0]
    for x, it, r in runs[1:]:
        assert it == it0 and r == r0
        assert np.array_equal(x, x0)
