"""Mass matrices, matrix combinations, Dirichlet folding, the transient
stepper and the vibration-mode solver on the device, against the oracle's
restatement (mass.rs, transient.rs, heat_solver.rs, direct.rs, eigen.rs) and
the reference's own assertions (mass.rs:271-323, transient.rs:104-127,
heat_solver.rs:107-171, tests/modal_tests.rs).

Tolerances: assembled values within 1e-13 of the largest entry (the device
evaluates the same products; only the determinant's rounding may differ),
patterns bit-exact; the stepper solves with PCG to a relative residual of
1e-12 where the oracle factorises, so states agree to 1e-9 relative.
"""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _perturbed_cube(n, seed):
    m = O.unit_cube(n, n, n)
    rng = np.random.default_rng(seed)
    inner = np.all((m.coords > 1e-9) & (m.coords < 1 - 1e-9), axis=1)
    m.coords[inner] += rng.uniform(-0.2 / n, 0.2 / n, (inner.sum(), 3))
    return m


def _same(A, B, tol=1e-13):
    assert A.n == B.n
    assert np.array_equal(np.asarray(A.colptr), np.asarray(B.colptr))
    assert np.array_equal(np.asarray(A.rowidx), np.asarray(B.rowidx))
    scale = max(np.max(np.abs(B.vals)), 1e-300)
    assert np.max(np.abs(np.asarray(A.vals) - B.vals)) <= tol * scale


def test_mass_matrices_match_oracle(fcu, ctx):
    rng = np.random.default_rng(7)
    m2 = O.unit_square(9, 6)
    _same(fcu.assemble_mass_2d(fcu.Mesh(m2.coords, m2.cells), ctx), O.assemble_mass_2d(m2))
    m3 = _perturbed_cube(4, 3)
    fm3 = fcu.Mesh(m3.coords, m3.cells)
    _same(fcu.assemble_mass_3d(fm3, ctx), O.assemble_mass_3d(m3))
    _same(fcu.assemble_elasticity_mass_3d(fm3, 7850.0, ctx), O.assemble_elasticity_mass_3d(m3, 7850.0))
    # scalar P2 and a per-cell coefficient
    coef = np.exp(rng.standard_normal(m3.nc))
    V = fcu.FunctionSpace(ctx, fm3, fcu.FCU_SPACE_P2)
    M = fcu.Matrix(ctx, V).assemble_mass(2.5, coef)
    cd, ev = O.p2_dofmap(m3)
    _same(M.export_csc(), O.assemble_p2_mass_3d(m3, cd, m3.nv + len(ev), 2.5, coef))
    M.close()
    V.close()


def test_p2_one_tet_products(fcu, ctx):
    # mass.rs:305-323: identity map, M(0,0) = 1/420, 1^T M 1 = 1/6
    fm = fcu.Mesh(np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]), np.array([[0, 1, 2, 3]]))
    A = fcu.assemble_mass_p2_3d(fm, 1.0, ctx).to_scipy()
    assert A[0, 0] == pytest.approx(1.0 / 420.0, abs=1e-15)
    assert float(np.ones(10) @ (A @ np.ones(10))) == pytest.approx(1.0 / 6.0, abs=1e-15)
    # global numbering: vertices, then edges by (min, max) vertex pair; the
    # cell's dofmap gives the element's local order
    m = O.Mesh(fm.coords, fm.cells.astype(np.int64))
    cd, _ = O.p2_dofmap(m)
    P = O.p2_mass_products()
    assert np.max(np.abs(A.toarray()[np.ix_(cd[0], cd[0])] - P)) <= 1e-16


def test_vector_p2_mass_on_caller_nodes(fcu, ctx):
    # assemble_elasticity_mass_p2_3d (mass.rs:137-180): the reference element
    # (mass.rs:305-323), then a perturbed cube's P2 node mesh, vs the oracle
    v = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0],
                  [0, 0, 0.5], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    A = fcu.assemble_elasticity_mass_p2_3d(v, np.arange(10).reshape(1, 10), 1.0, ctx)
    _same(A, O.assemble_elasticity_mass_p2_3d(v, np.arange(10).reshape(1, 10), 1.0))
    S = A.to_scipy()
    assert float(np.ones(30) @ (S @ np.ones(30))) == pytest.approx(0.5, abs=1e-14)
    m = _perturbed_cube(3, 8)
    verts, c10 = O.p2_node_mesh(m)
    # the caller's own numbering: permute the nodes
    perm = np.random.default_rng(9).permutation(len(verts))
    inv = np.argsort(perm)
    verts_p, c10_p = verts[perm], inv[c10]
    _same(fcu.assemble_elasticity_mass_p2_3d(verts_p, c10_p, 7850.0, ctx),
          O.assemble_elasticity_mass_p2_3d(verts_p, c10_p, 7850.0))
    # a space on caller nodes refuses what it does not support
    fm = fcu.Mesh(verts_p, np.ascontiguousarray(c10_p[:, :4]))
    V = fcu.FunctionSpace(ctx, fm, fcu._abi.FCU_SPACE_P2_NODES, cells10=c10_p)
    with pytest.raises(fcu.FcuError):
        V.body_force([0.0, 0.0, 1.0])
    Ms = fcu.Matrix(ctx, V).assemble_mass(1.0)
    assert Ms.export_csc().vals.sum() == pytest.approx(1.0, abs=1e-12)   # the cube's volume
    Ms.close()
    V.close()
    bad = c10_p.copy()
    bad[0, 0] = bad[0, 1]
    with pytest.raises(fcu.FcuError):
        fcu.FunctionSpace(ctx, fm, fcu._abi.FCU_SPACE_P2_NODES_VEC3, cells10=bad)


def test_add_scaled_scale_and_fold(fcu, ctx):
    m = _perturbed_cube(3, 5)
    fm = fcu.Mesh(m.coords, m.cells)
    V = fcu.FunctionSpace(ctx, fm, fcu.FCU_SPACE_P1_VEC3)
    K = fcu.Matrix(ctx, V).assemble_elasticity(1.0e7, 0.3)
    Mm = fcu.Matrix(ctx, V).assemble_mass(1000.0)
    Ko, Mo = O.assemble_elasticity_3d(m, 1.0e7, 0.3), O.assemble_elasticity_mass_3d(m, 1000.0)
    # lhs of a step: union pattern = the stiffness pattern
    S = Mm.clone().set_add_scaled(Mm, K, 0.125)
    _same(S.export_csc(), O.add_scaled_matrices(Mo, Ko, 0.125))
    # scaling
    Ks = K.clone().scale(0.7)
    _same(Ks.export_csc(), O.Csc(Ko.n, Ko.colptr, Ko.rowidx, 0.7 * Ko.vals))
    # folding, with repeated and out-of-range dofs; idempotent
    fixed = np.concatenate([O.clamp_dofs(m), [5, 5, 10 ** 9]]).astype(np.int64)
    # The folded pattern drops exact zeros, so where a stiffness entry cancels
    # to zero in one evaluation and to round-off in the other the patterns
    # may differ by such entries: compare densely, and the patterns on the
    # entries above round-off.
    Kf = K.clone().fold_dirichlet(fixed, True)
    Fo = O.fold_dirichlet(Ko, fixed, True)
    for _ in range(2):
        Fd = Kf.export_csc()
        Ad, Ao = Fd.to_scipy().toarray(), Fo.to_scipy().toarray()
        scale = np.max(np.abs(Ao))
        assert np.max(np.abs(Ad - Ao)) <= 1e-13 * scale
        assert np.all(Fd.vals != 0.0)
        assert np.array_equal(np.abs(Ad) > 1e-10 * scale, np.abs(Ao) > 1e-10 * scale)
        Kf.fold_dirichlet(fixed, True)   # idempotent
    Mf = Mm.clone().fold_dirichlet(fixed, False)
    _same(Mf.export_csc(), O.fold_dirichlet(Mo, fixed, False))
    # wrapped CSC operands with the same layout; different layouts refused
    A = fcu.CscMatrix(Mo.n, Mo.colptr, Mo.rowidx, Mo.vals)
    B = fcu.CscMatrix(Mo.n, Mo.colptr, Mo.rowidx, 3.0 * Mo.vals)
    _same(fcu.add_scaled_matrices(A, B, -0.5, ctx), O.add_scaled_matrices(Mo, O.Csc(Mo.n, Mo.colptr, Mo.rowidx,
                                                                                   3.0 * Mo.vals), -0.5))
    # different layouts: the union pattern, as the triplet build gives it
    _exact(fcu.add_scaled_matrices(A, fcu.CscMatrix(Ko.n, Ko.colptr, Ko.rowidx, Ko.vals), 1.0, ctx),
           O.add_scaled_matrices(Mo, Ko, 1.0))
    with pytest.raises(fcu.FcuError):
        K.clone().fold_dirichlet(np.array([-1], np.int64), True)
    for x in (S, Ks, Kf, Mf, K, Mm):
        x.close()
    V.close()


def _exact(A, B):
    """Same pattern and identical values (a zero's sign aside)."""
    assert A.n == B.n
    assert np.array_equal(np.asarray(A.colptr), np.asarray(B.colptr))
    assert np.array_equal(np.asarray(A.rowidx), np.asarray(B.rowidx))
    assert np.array_equal(np.asarray(A.vals), np.asarray(B.vals))


def _random_csc(n, density, seed, zeros=True):
    """A faer-layout CSC with sorted rows, a full diagonal and, optionally,
    explicit zeros among its entries."""
    rng = np.random.default_rng(seed)
    mask = rng.random((n, n)) < density
    np.fill_diagonal(mask, True)
    vals = rng.standard_normal((n, n))
    if zeros:
        vals[rng.random((n, n)) < 0.1] = 0.0
    colptr = np.zeros(n + 1, np.int64)
    rows, vs = [], []
    for j in range(n):
        r = np.nonzero(mask[:, j])[0]
        rows.append(r)
        vs.append(vals[r, j])
        colptr[j + 1] = colptr[j] + len(r)
    return O.Csc(n, colptr, np.concatenate(rows).astype(np.int64), np.concatenate(vs))


def test_add_scaled_union_matches_oracle(fcu, ctx):
    """add_scaled_matrices (transient.rs:72-97) on operands whose patterns
    differ: the union build against the oracle's faer-style triplet build,
    pattern and values bit for bit."""
    # wrapped CSC operands with explicit zeros, empty columns on one side
    n = 57
    Ao, Bo = _random_csc(n, 0.08, 1), _random_csc(n, 0.05, 2)
    A = fcu.CscMatrix(n, Ao.colptr, Ao.rowidx, Ao.vals)
    B = fcu.CscMatrix(n, Bo.colptr, Bo.rowidx, Bo.vals)
    for alpha in (1.0, -0.37, 0.0):
        _exact(fcu.add_scaled_matrices(A, B, alpha, ctx), O.add_scaled_matrices(Ao, Bo, alpha))
    # two spaces of one order: P1 stiffness on a mesh, P1 mass on the same
    # vertices renumbered (another pattern)
    m = O.unit_square(9, 7)
    perm = np.random.default_rng(3).permutation(m.nv)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(m.nv)
    m2 = O.Mesh(np.ascontiguousarray(m.coords[perm]), np.ascontiguousarray(inv[m.cells]).astype(m.cells.dtype))
    V1 = fcu.FunctionSpace(ctx, fcu.Mesh(m.coords, m.cells), fcu.FCU_SPACE_P1)
    V2 = fcu.FunctionSpace(ctx, fcu.Mesh(m2.coords, m2.cells), fcu.FCU_SPACE_P1)
    K = fcu.Matrix(ctx, V1).assemble_stiffness(None)
    Mm = fcu.Matrix(ctx, V2).assemble_mass(2.5)
    Ko, Mo = K.export_csc(), Mm.export_csc()
    _exact(fcu.add_scaled_matrices(K, Mm, 0.01, ctx), O.add_scaled_matrices(Ko, Mo, 0.01))
    # one space, one operand with Dirichlet rows eliminated: its exported
    # matrix is the operand
    K2 = fcu.Matrix(ctx, V1).assemble_stiffness(None)
    bd = V1.boundary_dofs().astype(np.int64)
    rhs = np.ones(V1.ndofs)
    K2.apply_dirichlet(rhs, bd, np.zeros(len(bd)))
    K2o = K2.export_csc()
    _exact(fcu.add_scaled_matrices(K, K2, -2.0, ctx), O.add_scaled_matrices(Ko, K2o, -2.0))
    # the handle-level entry point; order mismatch refused
    U = fcu.Matrix.add_scaled_union(K, Mm, 0.5)
    _exact(U.export_csc(), O.add_scaled_matrices(Ko, Mo, 0.5))
    with pytest.raises(fcu.FcuError) as e:
        fcu.add_scaled_matrices(A, fcu.CscMatrix(1, np.array([0, 1]), np.array([0]), np.array([1.0])), 1.0, ctx)
    assert e.value.code == fcu._abi.FCU_ERR_BAD_ARG
    for x in (U, K, K2, Mm):
        x.close()
    V1.close()
    V2.close()


def test_transient_exponential_decay(fcu, ctx):
    # transient.rs:108-127
    M = fcu.CscMatrix(1, np.array([0, 1]), np.array([0]), np.array([1.0]))
    K = fcu.CscMatrix(1, np.array([0, 1]), np.array([0]), np.array([2.0]))
    solver = fcu.TransientHeatSolver(fcu.TimeSteppingScheme.CrankNicolson, 0.01, ctx)
    u = np.array([1.0])
    uo = np.array([1.0])
    Mo = O.csc_from_triplets(1, [0], [0], [1.0])
    Ko = O.csc_from_triplets(1, [0], [0], [2.0])
    f = np.zeros(1)
    for _ in range(100):
        u = solver.step(M, K, u, f, f)
        uo = O.transient_step(1, 0.01, Mo, Ko, uo, f, f)
    solver.close()
    assert abs(u[0] - math.exp(-2.0)) < 1e-4
    assert abs(u[0] - uo[0]) <= 1e-13


def _walls(m):
    x = m.coords[:, 0]
    left = np.nonzero(np.abs(x) < 1e-6)[0]
    right = np.nonzero(np.abs(x - 1.0) < 1e-6)[0]
    return left, right


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_transient_heat_steady_state_matches_oracle(fcu, ctx, precision):
    # heat_solver.rs:112-171
    m = O.unit_square(8, 8)
    left, right = _walls(m)
    bcs = [fcu.DirichletBC(list(left), [100.0] * len(left)), fcu.DirichletBC(list(right), [0.0] * len(right))]
    prec = fcu.FCU_FP64 if precision == "fp64" else fcu.FCU_MIXED
    sol = fcu.solve_transient_heat_2d(fcu.Mesh(m.coords, m.cells), 1.0, np.zeros(m.nv), bcs, 0.05, 40,
                                      fcu.TimeSteppingScheme.CrankNicolson, None, ctx, precision=prec)
    mid = np.abs(m.coords[:, 0] - 0.5) < 1e-6
    assert np.all(np.abs(sol.final_temperature[mid] - 50.0) <= 1.5)
    times, hist, final = O.solve_transient_heat_2d(m, 1.0, np.zeros(m.nv), [(left, np.full(len(left), 100.0)),
                                                                           (right, np.zeros(len(right)))],
                                                   0.05, 40, 1)
    assert sol.time_steps == pytest.approx(times)
    assert len(sol.temperature_history) == 41
    err = max(np.max(np.abs(a - b)) for a, b in zip(sol.temperature_history, hist))
    assert err <= 1e-9 * 100.0


def test_backward_euler_with_source_matches_oracle(fcu, ctx):
    m = O.unit_square(12, 10)
    left, _ = _walls(m)
    src = lambda t, p: (1.0 + t) * math.sin(math.pi * p[0]) * math.cos(0.5 * math.pi * p[1])  # noqa: E731
    u0 = np.cos(m.coords[:, 0]) * m.coords[:, 1]
    sol = fcu.solve_transient_heat_2d(fcu.Mesh(m.coords, m.cells), 0.3, u0, [fcu.DirichletBC(list(left),
                                      [1.0] * len(left))], 0.02, 12, fcu.TimeSteppingScheme.BackwardEuler, src, ctx)
    _, hist, final = O.solve_transient_heat_2d(m, 0.3, u0, [(left, np.ones(len(left)))], 0.02, 12, 0, src)
    assert np.max(np.abs(sol.final_temperature - final)) <= 1e-9 * np.max(np.abs(final))
    with pytest.raises(ValueError):
        fcu.solve_transient_heat_2d(fcu.Mesh(m.coords, m.cells), 1.0, np.zeros(3), [], 0.1, 1,
                                    fcu.TimeSteppingScheme.BackwardEuler, None, ctx)


def _cantilever(fcu, ctx, nx, ny, nz, density=1000.0):
    m = O.box_beam(1.0, 0.1, 0.1, nx, ny, nz)
    fm = fcu.Mesh(m.coords, m.cells)
    V = fcu.FunctionSpace(ctx, fm, fcu.FCU_SPACE_P1_VEC3)
    K = fcu.Matrix(ctx, V).assemble_elasticity(1.0e7, 0.3)
    M = fcu.Matrix(ctx, V).assemble_mass(density)
    return m, V, K, M, O.clamp_dofs(m)


def test_cantilever_modes_match_oracle(fcu, ctx):
    # modal_tests.rs:9-87, and the oracle's restatement of the iteration
    m, V, K, M, fixed = _cantilever(fcu, ctx, 16, 2, 2)
    modes, pit, info = fcu.solve_vibration_modes(K, M, fixed, 3, 30, 1e-5, ctx, return_stats=True)
    f = [md.frequency_hz for md in modes]
    assert 1.0 < f[0] < 3.0 and 1.5 < f[1] < 3.5 and 8.0 < f[2] < 20.0
    ref = O.solve_vibration_modes(O.assemble_elasticity_3d(m, 1.0e7, 0.3), O.assemble_elasticity_mass_3d(m, 1000.0),
                                  fixed, 3, 30, 1e-5)
    for md, (lam, v, its), p in zip(modes, ref, pit):
        assert abs(md.eigenvalue - lam) <= 1e-4 * lam
        assert abs(int(p) - its) <= 1
        assert md.omega_rad_s == pytest.approx(math.sqrt(md.eigenvalue), rel=1e-15)
        assert np.all(md.mode_shape[fixed] == 0.0)
    # the third (well separated) mode shape, up to sign, mass-normalised
    Mo = O.assemble_elasticity_mass_3d(m, 1000.0).to_scipy()
    v3, r3 = modes[2].mode_shape, ref[2][1]
    assert abs(abs(float(v3 @ (Mo @ r3))) / math.sqrt(float(v3 @ (Mo @ v3)) * float(r3 @ (Mo @ r3))) - 1.0) < 1e-6
    assert info.iterations > 0
    for x in (K, M, V):
        x.close()


def test_frequencies_scale_and_custom_inner(fcu, ctx):
    # modal_tests.rs:89-156
    m, V, K, M1, fixed = _cantilever(fcu, ctx, 8, 1, 1, 1000.0)
    M2 = fcu.Matrix(ctx, V).assemble_mass(1000.0 * 10000.0)
    a = fcu.solve_vibration_modes(K, M1, fixed, 2, 60, 1e-8, ctx)
    b = fcu.solve_vibration_modes(K, M2, fixed, 2, 60, 1e-8, ctx)
    for hi, lo in zip(b, a):
        assert hi.frequency_hz / lo.frequency_hz == pytest.approx(0.01, abs=1e-4)
    d = fcu.solve_vibration_modes(K, M1, fixed, 3, 60, 1e-8, ctx)
    Kd = K.clone().fold_dirichlet(fixed, True)
    calls = []

    def inner(bv, x0):
        calls.append(1)
        return Kd.pcg(bv, x0=x0, tol=1e-9, max_iter=1000)[0]

    c = fcu.solve_vibration_modes_with_inner(K, M1, fixed, 3, 60, 1e-8, inner, ctx)
    assert calls
    for rd, rc in zip(d, c):
        assert rc.frequency_hz / rd.frequency_hz == pytest.approx(1.0, abs=1e-9)
    # the mixed inner solve reaches the same modes
    mx = fcu.solve_vibration_modes(K, M1, fixed, 3, 60, 1e-8, ctx, precision=fcu.FCU_MIXED)
    for rd, rm in zip(d, mx):
        assert rm.eigenvalue == pytest.approx(rd.eigenvalue, rel=1e-6)

    def failing(bv, x0):
        raise RuntimeError("inner solve gave up")

    with pytest.raises(RuntimeError, match="gave up"):
        fcu.solve_vibration_modes_with_inner(K, M1, fixed, 1, 5, 1e-8, failing, ctx)
    with pytest.raises(fcu.FcuError, match="No free degrees"):
        fcu.solve_vibration_modes(K, M1, np.arange(K.n), 1, 5, 1e-8, ctx)
    for x in (Kd, K, M1, M2, V):
        x.close()
