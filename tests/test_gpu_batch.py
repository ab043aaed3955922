"""Batched PCG (fcu_batch_pcg): independent 2D P1 Poisson instances of uneven
sizes, per-cell kappa = exp(N(0,1)), nodal f ~ U[-1, 1], u = 0 on each
boundary, solved as the diagonal blocks of one system.

Each instance is checked against the oracle run on that instance alone
(assemble_stiffness_2d with kappa, assemble_rhs_2d from f at the quadrature
points, apply_dirichlet_bc, solve_cg: poisson.rs:23-263, cg.rs:40-149).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _instances(nb, nmin, nmax, seed):
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=nb)
    meshes, kappas, fs = [], [], []
    for n in ns:
        m = O.unit_square(int(n), int(n))
        meshes.append(m)
        kappas.append(np.exp(rng.standard_normal(m.cells.shape[0])))
        fs.append(rng.uniform(-1.0, 1.0, m.coords.shape[0]))
    return meshes, kappas, fs


def _fq(m, f):
    """Nodal interpolant sum_j f_j phi_j at the oracle's quadrature points."""
    q = O.quadrature_points_2d(m).reshape(m.cells.shape[0], -1, 2)
    v = m.coords[m.cells]                       # nc x 3 x 2
    T = np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]], axis=2)  # nc x 2 x 2
    lam12 = np.linalg.solve(T[:, None], (q - v[:, None, 0])[..., None])[..., 0]
    lam = np.concatenate([1.0 - lam12.sum(-1, keepdims=True), lam12], axis=-1)
    return np.einsum("cqk,ck->cq", lam, f[m.cells])


def _oracle_solve(m, kappa, f, tol):
    A = O.assemble_stiffness_2d(m, kappa)
    b = O.assemble_rhs_2d_values(m, _fq(m, f))
    bd = O.boundary_dofs_2d(m)
    Ab, bb = O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))
    x, it, _ = O.solve_cg(Ab, bb, None, tol, 100000)
    return x, it, Ab, bb


def _fcu_meshes(fcu, meshes):
    return [fcu.Mesh(m.coords, m.cells) for m in meshes]


def test_batch_fp64_matches_oracle_per_instance(fcu, ctx):
    meshes, kappas, fs = _instances(12, 3, 24, seed=5)
    tol = 1e-10
    sol = fcu.solve_poisson_batch(_fcu_meshes(fcu, meshes), kappas, fs, tol=tol, ctx=ctx, precision=fcu.FCU_FP64)
    assert np.all(sol.statuses == 0)
    for i, m in enumerate(meshes):
        x_o, it_o, Ab, bb = _oracle_solve(m, kappas[i], fs[i], tol)
        x = sol.solutions[i]
        assert np.linalg.norm(x - x_o) <= 1e-8 * np.linalg.norm(x_o)
        assert abs(int(sol.iterations[i]) - it_o) <= max(3, 0.02 * it_o)
        r = bb - Ab.to_scipy() @ x
        assert np.linalg.norm(r) / np.linalg.norm(bb) < 10 * tol
        assert sol.rel_residuals[i] < tol


def test_batch_mixed_reaches_fp64_residual(fcu, ctx):
    meshes, kappas, fs = _instances(16, 4, 40, seed=9)
    tol = 1e-8
    sol = fcu.solve_poisson_batch(_fcu_meshes(fcu, meshes), kappas, fs, tol=tol, ctx=ctx, precision=fcu.FCU_MIXED)
    assert np.all(sol.statuses == 0)
    import scipy.sparse.linalg as spl
    for i, m in enumerate(meshes):
        _, _, Ab, bb = _oracle_solve(m, kappas[i], fs[i], 1e-8)
        x_o = spl.spsolve(Ab.to_scipy().tocsc(), bb)
        x = sol.solutions[i]
        # the residual the batch reports is the FP64 one, and it is true
        r = bb - Ab.to_scipy() @ x
        assert np.linalg.norm(r) / np.linalg.norm(bb) < 2 * tol
        assert np.linalg.norm(x - x_o) <= 1e-5 * np.linalg.norm(x_o)


def test_batch_replay_is_bit_identical_and_tuned(fcu, ctx):
    meshes, kappas, fs = _instances(8, 5, 30, seed=3)
    fm = _fcu_meshes(fcu, meshes)
    mesh, offs = fcu.concat_meshes(fm)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
    M = fcu.Matrix(ctx, V).assemble_stiffness(np.concatenate(kappas))
    b = V.rhs_source(fcu.FCU_SRC_NODAL, nodal=np.concatenate(fs))
    bd = V.boundary_dofs()
    M.apply_dirichlet(b, bd, np.zeros(len(bd)))
    for prec in (fcu.FCU_FP64, fcu.FCU_MIXED):
        x1, it1, _, st1, _ = M.batch_pcg(offs, b, tol=1e-9, precision=prec)
        x2, it2, _, st2, _ = M.batch_pcg(offs, b, tol=1e-9, precision=prec)
        assert np.array_equal(x1, x2) and np.array_equal(it1, it2)
        assert np.all(st1 == 0)
        v, t, c = M.batch_config(prec)
        assert v in (1, 2, 4) and t in (512, 1024) and c in (1, 2, 4, 8)
    M.close()
    V.close()


def test_batch_zero_rhs_and_iteration_limit(fcu, ctx):
    meshes, kappas, fs = _instances(5, 6, 20, seed=1)
    fs[2] = np.zeros_like(fs[2])
    sol = fcu.solve_poisson_batch(_fcu_meshes(fcu, meshes), kappas, fs, tol=1e-10, ctx=ctx,
                                  precision=fcu.FCU_FP64)
    assert sol.statuses[2] == 0 and sol.iterations[2] == 0
    assert np.all(sol.solutions[2] == 0.0)
    # a limit below what the larger instances need: they report no convergence
    lim = fcu.solve_poisson_batch(_fcu_meshes(fcu, meshes), kappas, fs, tol=1e-12, max_iter=4, ctx=ctx,
                                  precision=fcu.FCU_FP64, raise_on_error=False)
    assert np.all(lim.iterations <= 4)
    assert np.any(lim.statuses == fcu._abi.FCU_ERR_NO_CONVERGENCE)
    assert lim.statuses[2] == 0


def test_batch_rejects_bad_offsets(fcu, ctx):
    meshes, kappas, fs = _instances(3, 4, 8, seed=2)
    mesh, offs = fcu.concat_meshes(_fcu_meshes(fcu, meshes))
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
    M = fcu.Matrix(ctx, V).assemble_stiffness(None)
    b = np.ones(V.ndofs)
    with pytest.raises(fcu.FcuError):
        M.batch_pcg([0, offs[-1] - 1], b)          # does not span the rows
    bad = offs.copy()
    bad[1] += 3                                    # splits instance 0's block
    with pytest.raises(fcu.FcuError, match="block diagonal"):
        M.batch_pcg(bad, b)
    M.close()
    V.close()


def test_batch_p2_instances_match_single_solves(fcu, ctx):
    """The batched solver is generic over scalar block-diagonal matrices: two
    P2 unit cubes of different sizes (rows of ~28 entries) in one batch,
    FP64 and mixed, each instance against a direct solve of its block."""
    rng = np.random.default_rng(6)
    parts = [fcu.unit_cube(3, 3, 3), fcu.unit_cube(5, 4, 4)]
    mesh, _ = fcu.concat_meshes(parts)
    kappa = np.exp(rng.standard_normal(mesh.nc))
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P2)
    M = fcu.Matrix(ctx, V).assemble_stiffness(kappa)
    b = V.rhs_source(fcu.FCU_SRC_CONSTANT, params=(1.0,))
    bd = V.boundary_dofs()
    M.apply_dirichlet(b, bd, np.zeros(len(bd)))
    # P2 dofs: all vertices first, then all edges; the concatenated mesh's
    # numbering is not block diagonal per instance, so permute rows into blocks
    A = M.export_csc().to_scipy().tocsr()
    nv = [p.nv for p in parts]
    V0 = fcu.FunctionSpace(ctx, parts[0], fcu.FCU_SPACE_P2)
    ne0 = V0.ndofs - nv[0]
    V0.close()
    ne1 = V.ndofs - sum(nv) - ne0
    perm = np.concatenate([np.arange(nv[0]), sum(nv) + np.arange(ne0),
                           nv[0] + np.arange(nv[1]), sum(nv) + ne0 + np.arange(ne1)])
    Ap = A[perm][:, perm].tocsc()
    bp = b[perm]
    Cm = fcu.Matrix.from_csc(ctx, fcu.CscMatrix(Ap.shape[0], Ap.indptr.astype(np.int64),
                                               Ap.indices.astype(np.int64), Ap.data))
    offs = np.array([0, nv[0] + ne0, Ap.shape[0]])
    for prec in (fcu.FCU_FP64, fcu.FCU_MIXED):
        x, it, rel, st, _ = Cm.batch_pcg(offs, bp, tol=1e-10, precision=prec)
        assert np.all(st == 0) and np.all(rel < 1e-10)
        import scipy.sparse.linalg as spl
        for i in range(2):
            sl = slice(offs[i], offs[i + 1])
            xi_direct = spl.spsolve(Ap[sl, sl].tocsc(), bp[sl])
            assert np.linalg.norm(x[sl] - xi_direct) <= 1e-7 * np.linalg.norm(xi_direct)
    M.close()
    V.close()
