"""Pins the oracle's restatement of the mass matrices, the transient stepper
and the vibration-mode solver to the reference's own tests:

- mass.rs:271-323 (P2 reference products in closed form, one-tet volume);
- transient.rs:104-127 (Crank-Nicolson exponential decay);
- heat_solver.rs:107-171 (heated wall -> linear steady state);
- tests/modal_tests.rs:9-156 (cantilever frequencies, 1/sqrt(density)
  scaling, custom inner solve equal to the default);
- eigen.rs:55-79 (fold_dirichlet) against a direct numpy construction.
"""
import math

import numpy as np
import pytest

import oracle as O


def test_p2_reference_products_closed_forms():
    # mass.rs:281-300
    P = O.p2_mass_products()
    assert P[0, 0] == pytest.approx(1.0 / 420.0, abs=1e-14)
    assert P[4, 4] == pytest.approx(4.0 / 315.0, abs=1e-14)
    assert P[0, 1] == pytest.approx(1.0 / 2520.0, abs=1e-14)
    assert P[0, 4] == pytest.approx(-1.0 / 630.0, abs=1e-14)
    assert P[4, 6] == pytest.approx(2.0 / 315.0, abs=1e-14)
    assert P[4, 9] == pytest.approx(1.0 / 315.0, abs=1e-14)
    rows = P.sum(axis=1)
    assert np.allclose(rows[:4], -1.0 / 120.0, atol=1e-14, rtol=0)
    assert np.allclose(rows[4:], 1.0 / 30.0, atol=1e-14, rtol=0)
    assert P.sum() == pytest.approx(1.0 / 6.0, abs=1e-13)
    assert np.array_equal(P, P.T)


def test_p2_mass_one_tet_conserves_volume():
    # mass.rs:305-323 on the scalar P2 space: 1^T M 1 = |T| = 1/6, M(0,0) = 1/420
    m = O.Mesh(np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]), np.array([[0, 1, 2, 3]]))
    cd, ev = O.p2_dofmap(m)
    M = O.assemble_p2_mass_3d(m, cd, m.nv + len(ev))
    A = M.to_scipy()
    assert float(np.ones(10) @ (A @ np.ones(10))) == pytest.approx(1.0 / 6.0, abs=1e-13)
    assert A[0, 0] == pytest.approx(1.0 / 420.0, abs=1e-13)


def test_vector_p2_mass_one_tet():
    # mass.rs:305-323: the reference element with its ten nodes, density 1:
    # 1^T M 1 = 3 / 6 (three components), M(0,0) = 1/420
    v = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0],
                  [0, 0, 0.5], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    A = O.assemble_elasticity_mass_p2_3d(v, np.arange(10).reshape(1, 10), 1.0).to_scipy()
    assert A.shape == (30, 30)
    assert float(np.ones(30) @ (A @ np.ones(30))) == pytest.approx(3.0 / 6.0, abs=1e-13)
    assert A[0, 0] == pytest.approx(1.0 / 420.0, abs=1e-13)


def test_mass_matrices_measure_and_patterns():
    m2 = O.unit_square(5, 3)
    M = O.assemble_mass_2d(m2)
    assert M.vals.sum() == pytest.approx(1.0, abs=1e-14)
    K = O.assemble_stiffness_2d(m2)
    assert np.array_equal(M.colptr, K.colptr) and np.array_equal(M.rowidx, K.rowidx)
    m3 = O.box_beam(2.0, 1.0, 0.5, 4, 2, 2)
    assert O.assemble_mass_3d(m3).vals.sum() == pytest.approx(1.0, abs=1e-13)
    Me = O.assemble_elasticity_mass_3d(m3, 7850.0)
    assert Me.n == 3 * m3.nv
    # each component carries the density times the volume
    A = Me.to_scipy()
    for c in range(3):
        e = np.zeros(Me.n)
        e[c::3] = 1.0
        assert float(e @ (A @ e)) == pytest.approx(7850.0, rel=1e-13)
    # same-component entries only (mass.rs:118-123): three per vertex pair
    Ms = O.assemble_mass_3d(m3)
    assert Me.nnz == 3 * Ms.nnz
    assert np.all(Me.rowidx % 3 == np.repeat(np.arange(Me.n) % 3, np.diff(Me.colptr)))


def test_transient_exponential_decay():
    # transient.rs:108-127: du/dt + 2u = 0, CN, dt = 0.01, 100 steps
    M = O.csc_from_triplets(1, [0], [0], [1.0])
    K = O.csc_from_triplets(1, [0], [0], [2.0])
    u = np.array([1.0])
    for _ in range(100):
        u = O.transient_step(1, 0.01, M, K, u, [0.0], [0.0])
    assert abs(u[0] - math.exp(-2.0)) < 1e-4


def _heat_walls(m):
    x = m.coords[:, 0]
    left = np.nonzero(np.abs(x) < 1e-6)[0]
    right = np.nonzero(np.abs(x - 1.0) < 1e-6)[0]
    return [(left, np.full(len(left), 100.0)), (right, np.zeros(len(right)))]


def test_transient_heat_steady_state():
    # heat_solver.rs:112-171: CN, dt = 0.05, 40 steps, center 50 within 1.5
    m = O.unit_square(8, 8)
    _, _, u = O.solve_transient_heat_2d(m, 1.0, np.zeros(m.nv), _heat_walls(m), 0.05, 40, 1)
    mid = np.abs(m.coords[:, 0] - 0.5) < 1e-6
    assert np.all(np.abs(u[mid] - 50.0) <= 1.5)


def test_add_scaled_and_fold_against_dense():
    rng = np.random.default_rng(1)
    m = O.unit_square(4, 3)
    M, K = O.assemble_mass_2d(m), O.assemble_stiffness_2d(m)
    S = O.add_scaled_matrices(M, K, 0.3)
    assert np.array_equal(S.colptr, M.colptr)
    assert np.array_equal(S.vals, M.vals + 0.3 * K.vals)
    fixed = [0, 3, 7, 3, 1000]   # repeated and out-of-range dofs (eigen.rs:63-66)
    F = O.fold_dirichlet(K, fixed, True)
    D = K.to_scipy().toarray()
    fx = np.zeros(m.nv, bool)
    fx[[0, 3, 7]] = True
    D[fx, :] = 0.0
    D[:, fx] = 0.0
    D[fx, fx] = 1.0
    assert np.array_equal(F.to_scipy().toarray(), D)
    assert np.all(F.vals != 0.0)          # zero entries dropped
    G = O.fold_dirichlet(F, fixed, True)  # idempotent
    assert np.array_equal(G.colptr, F.colptr) and np.array_equal(G.vals, F.vals)
    Fm = O.fold_dirichlet(M, fixed, False)
    assert Fm.to_scipy().toarray()[fx].sum() == 0.0 and Fm.nnz < M.nnz
    del rng


def _cantilever(nx, ny, nz, density=1000.0):
    m = O.box_beam(1.0, 0.1, 0.1, nx, ny, nz)
    k = O.assemble_elasticity_3d(m, 1.0e7, 0.3)
    mm = O.assemble_elasticity_mass_3d(m, density)
    fixed = O.clamp_dofs(m)
    return m, k, mm, fixed


def _freq(lam):
    return math.sqrt(lam) / (2.0 * math.pi)


def test_cantilever_natural_frequencies():
    # modal_tests.rs:9-87
    _, k, mm, fixed = _cantilever(16, 2, 2)
    modes = O.solve_vibration_modes(k, mm, fixed, 3, 30, 1e-5)
    f = [_freq(lam) for lam, _, _ in modes]
    assert 1.0 < f[0] < 3.0
    assert 1.5 < f[1] < 3.5
    assert 8.0 < f[2] < 20.0


def test_frequencies_scale_as_one_over_sqrt_density():
    # modal_tests.rs:89-118
    _, k, m1, fixed = _cantilever(8, 1, 1, 1000.0)
    _, _, m2, _ = _cantilever(8, 1, 1, 1000.0 * 10000.0)
    a = O.solve_vibration_modes(k, m1, fixed, 2, 60, 1e-8)
    b = O.solve_vibration_modes(k, m2, fixed, 2, 60, 1e-8)
    for hi, lo in zip(b, a):
        assert _freq(hi[0]) / _freq(lo[0]) == pytest.approx(0.01, abs=1e-4)


def test_custom_inner_solver_matches_default():
    # modal_tests.rs:120-156
    _, k, mm, fixed = _cantilever(8, 1, 1)
    d = O.solve_vibration_modes(k, mm, fixed, 3, 60, 1e-8)

    def inner(kd, b, x0):
        return O.solve_cg(kd, b, x0, 1e-9, 1000)[0]

    c = O.solve_vibration_modes_with_inner(k, mm, fixed, 3, 60, 1e-8, inner)
    for a, b in zip(d, c):
        assert _freq(b[0]) / _freq(a[0]) == pytest.approx(1.0, abs=1e-9)
