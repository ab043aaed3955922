"""The 3x3 block CSR operators (GpuBsr3Context, solve_bsr3_pcg_gpu,
spmv_bsr3_multi_gpu; gpu.rs:434-1141) on the device, against the oracle's
restatement, on the reference's own synthetic case (gpu.rs:1666-1760) and on
an assembled, clamped elasticity matrix exported in the same layout.

Tolerances: products within 1e-12 of |A| |x| (summation order differs); PCG
iteration counts within 1 and solutions within 1e-8 relative of the oracle's
(same recurrence, different reduction order)."""
import numpy as np
import pytest

import oracle as O
from bsr3_cases import synthetic_bsr3

pytestmark = pytest.mark.gpu


def test_reference_case_spmv_multi_gpu_and_pcg(fcu, ctx):
    nn, rp, ci, va, dinv = synthetic_bsr3(15)
    x_in = (np.arange(3 * nn) % 17) * 0.1
    g = fcu.GpuBsr3Context(nn, rp, ci, va, dinv, ctx=ctx)
    assert g.nnz_blocks() == len(ci)
    y = np.empty(3 * nn)
    g.spmv(x_in, y)
    yo = O.bsr3_spmv(nn, rp, ci, va, x_in)
    assert np.max(np.abs(y - yo)) <= 1e-12 * np.max(np.abs(yo))
    ym, devs = fcu.spmv_bsr3_multi_gpu(nn, rp, ci, va, x_in, 3)
    assert len(devs) >= 1
    assert np.max(np.abs(ym - y)) <= 1e-12 * np.max(np.abs(y))
    b = np.ones(3 * nn)
    res = fcu.solve_bsr3_pcg_gpu(nn, rp, ci, va, dinv, b, None, 1e-9, 500, ctx=ctx)
    assert res.final_residual < 1e-9
    xo, ito, relo = O.solve_bsr3_pcg(nn, rp, ci, va, dinv, b, None, 1e-9, 500)
    assert abs(res.iterations - ito) <= 1
    assert np.linalg.norm(res.solution - xo) <= 1e-8 * np.linalg.norm(xo)
    g.close()


def test_pcg_edge_cases(fcu, ctx):
    nn, rp, ci, va, dinv = synthetic_bsr3(4)
    z = fcu.solve_bsr3_pcg_gpu(nn, rp, ci, va, dinv, np.zeros(3 * nn), ctx=ctx)
    assert z.iterations == 0 and not z.solution.any()
    # iteration limit: Ok with the residual reached so far
    b = np.sin(np.arange(3 * nn))
    lim = fcu.solve_bsr3_pcg_gpu(nn, rp, ci, va, dinv, b, None, 1e-14, 3, ctx=ctx)
    xo, ito, relo = O.solve_bsr3_pcg(nn, rp, ci, va, dinv, b, None, 1e-14, 3)
    assert lim.iterations == 3 == ito
    assert lim.final_residual == pytest.approx(relo, rel=1e-9)
    # warm start from x0
    x0 = np.cos(np.arange(3 * nn))
    w = fcu.solve_bsr3_pcg_gpu(nn, rp, ci, va, dinv, b, x0, 1e-10, 500, ctx=ctx)
    xw, itw, _ = O.solve_bsr3_pcg(nn, rp, ci, va, dinv, b, x0, 1e-10, 500)
    assert abs(w.iterations - itw) <= 1 and np.linalg.norm(w.solution - xw) <= 1e-8 * np.linalg.norm(xw)
    bad = ci.copy()
    bad[5] = nn
    with pytest.raises(fcu.FcuError):
        fcu.solve_bsr3_pcg_gpu(nn, rp, bad, va, dinv, b, ctx=ctx)


@pytest.mark.parametrize("zero_initial_z", [True, False])
def test_jacobi_smooth_matches_oracle(fcu, ctx, zero_initial_z):
    nn, rp, ci, va, dinv = synthetic_bsr3(6)
    g = fcu.GpuBsr3Context(nn, rp, ci, va, dinv, ctx=ctx)
    r = np.sin(np.arange(3 * nn))
    for sweeps in (0, 1, 3):
        z0 = np.cos(np.arange(3 * nn))
        z = z0.copy()
        g.jacobi_smooth(r, z, sweeps, 0.7, zero_initial_z)
        zo = O.bsr3_jacobi_smooth(nn, rp, ci, va, dinv, r, z0, sweeps, 0.7, zero_initial_z)
        assert np.max(np.abs(z - zo)) <= 1e-13 * max(1.0, np.max(np.abs(zo)))
    g.close()


def test_assembled_elasticity_block_jacobi(fcu, ctx):
    m = O.box_beam(4.0, 1.0, 1.0, 24, 6, 6)
    fm = fcu.Mesh(m.coords, m.cells)
    V = fcu.FunctionSpace(ctx, fm, fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
    dofs = O.clamp_dofs(m)
    b = V.body_force([0.0, 0.0, -7.8e4])
    M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
    M.block_jacobi(True)
    rp, ci, va, dinv = M.export_bsr3(with_dinv=True)
    nn = m.nv
    # the exported blocks are the assembled matrix; dinv inverts its diagonal blocks
    Kb, bb = O.apply_dirichlet_bc(O.assemble_elasticity_3d(m, 210e9, 0.3), O.body_force_3d(m, [0, 0, -7.8e4]),
                                  dofs, np.zeros(len(dofs)))
    x = np.random.default_rng(2).standard_normal(3 * nn)
    Ax = Kb.to_scipy() @ x
    assert np.max(np.abs(O.bsr3_spmv(nn, rp, ci, va, x) - Ax)) <= 1e-12 * np.max(np.abs(Ax))
    assert np.max(np.abs(dinv - O.bsr3_block_inverse(nn, rp, ci, va))) <= 1e-12 * np.max(np.abs(dinv))
    # block-Jacobi PCG: the reference's entry point and fcu_pcg on the resident matrix
    res = fcu.solve_bsr3_pcg_gpu(nn, rp, ci, va, dinv, b, None, 1e-8, 20000, ctx=ctx)
    xo, ito, relo = O.solve_bsr3_pcg(nn, rp, ci, va, O.bsr3_block_inverse(nn, rp, ci, va), b, None, 1e-8, 20000)
    assert res.final_residual < 1e-8 and abs(res.iterations - ito) <= max(2, ito // 100)
    assert np.linalg.norm(res.solution - xo) <= 1e-6 * np.linalg.norm(xo)
    xb, info_b = M.pcg(b, tol=1e-8, max_iter=20000)
    assert abs(info_b.iterations - res.iterations) <= max(2, ito // 100)
    assert np.linalg.norm(xb - xo) <= 1e-6 * np.linalg.norm(xo)
    # point Jacobi needs more iterations on elasticity
    M.block_jacobi(False)
    xp, info_p = M.pcg(b, tol=1e-8, max_iter=20000)
    assert info_p.iterations > info_b.iterations
    assert np.linalg.norm(xp - xo) <= 1e-6 * np.linalg.norm(xo)
    # block-Jacobi is an FP64 preconditioner
    M.block_jacobi(True)
    with pytest.raises(fcu.FcuError):
        M.pcg(b, tol=1e-8, precision=fcu.FCU_MIXED)
    M.close()
    V.close()
