"""Pins the oracle (CPU restatement) to the reference's own known answers.

Every constant below is taken from a test in the reference repository and
cited by file:line; together they are the golden values for the path (the
reference stores no golden vectors). A second group cross-checks the oracle
against an independent numpy/scipy computation.
"""
import math

import numpy as np
import pytest

import oracle as O

PI = math.pi


# -- fenics-mesh: generators.rs:135-157 -------------------------------------

def test_unit_square_counts():
    m = O.unit_square(4, 4)
    assert m.nv == 25 and m.nc == 32
    v, _, _ = O.boundary_facets_2d(m)
    assert len(v) == 16
    # total_volume / boundary_measure (mesh.rs:116-143)
    c = m.coords[m.cells]
    area = 0.5 * np.abs((c[:, 1, 0] - c[:, 0, 0]) * (c[:, 2, 1] - c[:, 0, 1])
                        - (c[:, 1, 1] - c[:, 0, 1]) * (c[:, 2, 0] - c[:, 0, 0]))
    assert abs(area.sum() - 1.0) < 1e-12
    e = m.coords[v[:, 1]] - m.coords[v[:, 0]]
    assert abs(np.linalg.norm(e, axis=1).sum() - 4.0) < 1e-12


def test_unit_cube_counts():
    m = O.unit_cube(3, 3, 3)
    assert m.nv == 64 and m.nc == 162
    v, _, _ = O.boundary_facets_3d(m)
    assert len(v) == 108
    p = m.coords[v]
    cr = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    assert abs(0.5 * np.linalg.norm(cr, axis=1).sum() - 6.0) < 1e-12
    # Outward orientation (mesh.rs:166-192): normals point away from the centre.
    centroid = p.mean(axis=1) - 0.5
    assert np.all((cr * centroid).sum(axis=1) > 0)


def test_box_beam_vertex_and_cell_order():
    # generators.rs:69-108: x fastest, then y, then z; Kuhn split around p0-p7.
    m = O.box_beam(2.0, 1.0, 1.0, 2, 1, 1)
    assert np.allclose(m.coords[1], [1.0, 0.0, 0.0]) and np.allclose(m.coords[3], [0.0, 1.0, 0.0])
    assert m.cells[0].tolist() == [0, 1, 4, 10]
    assert m.cells[5].tolist() == [0, 7, 1, 10]


# -- fenics-element: jacobian.rs:107-147 -------------------------------------

def test_jacobian_triangle_kat():
    ok, det, invT = O.affine_map([[1.0, 1.0], [3.0, 1.0], [1.0, 4.0]])
    assert ok and abs(det - 6.0) < 1e-12
    g = invT @ np.array([6.0, 15.0])
    assert np.allclose(g, [3.0, 5.0], atol=1e-12)
    # map_to_physical of (0.5, 0.5) is (2, 2.5): second point of the 3-point rule
    m = O.Mesh(np.array([[1.0, 1.0], [3.0, 1.0], [1.0, 4.0]]), np.array([[0, 1, 2]], np.int64))
    q = O.quadrature_points_2d(m)
    assert np.allclose(q[1], [2.0, 2.5], atol=1e-12)


def test_jacobian_tet_kat():
    ok, det, invT = O.affine_map([[0, 0, 0], [2, 0, 0], [0, 3, 0], [0, 0, 4]])
    assert ok and abs(det - 24.0) < 1e-12
    assert np.allclose(invT @ np.array([2.0, 6.0, 12.0]), [1.0, 2.0, 3.0], atol=1e-12)


def test_degenerate_cell_rejected():
    ok, det, _ = O.affine_map([[0, 0], [1, 0], [2, 0]])
    assert not ok and abs(det) < 1e-14


# -- fenics-element: quadrature.rs:226-273 -----------------------------------

def test_quadrature_polynomial_exactness():
    # sum_i b_i = int f (partition of unity); degree-2 rules are exact.
    tri = O.Mesh(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]], np.int64))
    b = O.assemble_rhs_2d(tri, lambda x, y: x * x + 2.0 * y)
    assert abs(b.sum() - 5.0 / 12.0) < 1e-12
    tet = O.Mesh(np.eye(4, 3, k=-1), np.array([[0, 1, 2, 3]], np.int64))
    b3 = O.assemble_rhs_3d(tet, lambda x, y, z: x * x)
    assert abs(b3.sum() - 1.0 / 60.0) < 1e-12
    b1 = O.assemble_rhs_3d(tet, lambda x, y, z: np.ones_like(x))
    assert abs(b1.sum() - 1.0 / 6.0) < 1e-12


# -- fenics-element: lagrange.rs:480-559 (P2 tetrahedron) --------------------

P2_NODES = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [.5, 0, 0],
                     [.5, .5, 0], [0, .5, 0], [0, 0, .5], [.5, 0, .5], [0, .5, .5]])


def test_p2_kronecker_and_partition_of_unity():
    for i, node in enumerate(P2_NODES):
        phi = O.p2_basis(node)
        assert np.allclose(phi, np.eye(10)[i], atol=1e-12)
    for pt in ([.25, .25, .25], [.1, .2, .3], [.5, .1, .1]):
        assert abs(O.p2_basis(pt).sum() - 1.0) < 1e-12
        assert np.allclose(O.p2_grads(pt).sum(axis=0), 0.0, atol=1e-12)


def _tet_gauss(n=6):
    """Collapsed-coordinate Gauss rule on the unit tetrahedron (exact to 2n-1-ish)."""
    g, w = np.polynomial.legendre.leggauss(n)
    g = 0.5 * (g + 1)
    w = 0.5 * w
    pts, wts = [], []
    for a, wa in zip(g, w):
        for b, wb in zip(g, w):
            for c, wc in zip(g, w):
                x = a
                y = b * (1 - a)
                z = c * (1 - a) * (1 - b)
                pts.append([x, y, z])
                wts.append(wa * wb * wc * (1 - a) ** 2 * (1 - b))
    return np.array(pts), np.array(wts)


def test_p2_node_order_pinned_by_mass_products():
    # mass.rs:271-294 closed forms pin the corner/edge order 01,12,02,03,13,23.
    pts, wts = _tet_gauss()
    phi = np.array([O.p2_basis(p) for p in pts])
    M = (phi * wts[:, None]).T @ phi
    assert abs(M[0, 0] - 1 / 420) < 1e-14
    assert abs(M[4, 4] - 4 / 315) < 1e-14
    assert abs(M[0, 1] - 1 / 2520) < 1e-14
    assert abs(M[0, 4] - (-1 / 630)) < 1e-14
    assert abs(M[4, 6] - 2 / 315) < 1e-14   # edges 01 and 02 share corner 0
    assert abs(M[4, 9] - 1 / 315) < 1e-14   # edges 01 and 23 are opposite
    assert abs(M.sum() - 1 / 6) < 1e-13


# -- fenics-form/src/lib.rs:36-71: P1 stiffness on the reference triangle ----

def test_p1_reference_triangle_stiffness():
    tri = O.Mesh(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]], np.int64))
    K = O.assemble_stiffness_2d(tri).to_scipy().toarray()
    assert np.allclose(K, [[1.0, -0.5, -0.5], [-0.5, 0.5, 0.0], [-0.5, 0.0, 0.5]], atol=1e-12)


# -- fenics-solver/src/cg.rs:156-169 ----------------------------------------

def test_cg_2x2():
    A = O.csc_from_triplets(2, [0, 0, 1, 1], [0, 1, 0, 1], [4.0, -1.0, -1.0, 4.0])
    x, it, res = O.solve_cg(A, [3.0, 3.0], None, 1e-10, 100)
    assert it <= 2 and res < 1e-10 and np.allclose(x, [1.0, 1.0], atol=1e-8)


def test_cg_errors_like_reference():
    # Non-convergence is Err (cg.rs:139-148); breakdown is Err (cg.rs:102-107).
    m = O.unit_square(8, 8)
    A = O.assemble_stiffness_2d(m)
    b = O.assemble_rhs_2d(m, lambda x, y: np.ones_like(x))
    bd = O.boundary_dofs_2d(m)
    Ab, bb = O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))
    with pytest.raises(O.CgError):
        O.solve_cg(Ab, bb, None, 1e-12, 1)
    Z = O.csc_from_triplets(2, [0, 1], [0, 1], [0.0, 0.0])
    with pytest.raises(O.CgError):
        O.solve_cg(Z, [1.0, 1.0], None, 1e-10, 10)


def test_faer_triplet_semantics():
    # duplicates summed, rows sorted per column, explicit zeros kept
    A = O.csc_from_triplets(3, [2, 0, 2, 1], [0, 0, 0, 2], [1.0, 2.0, 3.0, 0.0])
    assert A.colptr.tolist() == [0, 2, 2, 3]
    assert A.rowidx.tolist() == [0, 2, 1]
    assert A.vals.tolist() == [2.0, 4.0, 0.0]


# -- fenics-solver/tests/poisson_tests.rs:5-73 -------------------------------

def _u2(x, y):
    return np.sin(PI * x) * np.sin(PI * y)


def _f2(x, y):
    return 2.0 * PI * PI * np.sin(PI * x) * np.sin(PI * y)


def test_poisson_2d_quadratic_rate():
    errs = []
    for n in (8, 16, 32):
        m = O.unit_square(n, n)
        x, _, _ = O.solve_poisson_2d(m, _f2, _u2, 1e-10, 500)
        errs.append(O.l2_error_2d(m, x, _u2))
    r1, r2 = errs[0] / errs[1], errs[1] / errs[2]
    assert 3.8 < r1 < 4.2 and 3.8 < r2 < 4.2


def test_poisson_3d_error():
    u = lambda x, y, z: np.sin(PI * x) * np.sin(PI * y) * np.sin(PI * z)
    f = lambda x, y, z: 3.0 * PI * PI * u(x, y, z)
    m = O.unit_cube(8, 8, 8)
    x, _, _ = O.solve_poisson_3d(m, f, u, 1e-10, 1000)
    assert O.l2_error_3d(m, x, u) < 0.05


# -- fenics-solver/tests/ab_benchmarks.rs:13-100 -----------------------------

def test_ab_poisson_2d_vs_dolfinx():
    m = O.unit_square(16, 16)
    x, _, _ = O.solve_poisson_2d(m, _f2, _u2, 1e-12, 1000)
    l2 = O.l2_error_2d(m, x, _u2)
    assert abs(l2 - 5.377435e-3) / 5.377435e-3 < 0.05
    assert abs(x.max() - 0.996793) / 0.996793 < 1e-3


def test_ab_cantilever_vs_dolfinx():
    m = O.box_beam(1.0, 0.1, 0.1, 10, 2, 2)
    dofs = O.clamp_dofs(m)
    x, _, _ = O.solve_elasticity_3d(m, 1e7, 0.3, [0.0, -1000.0, 0.0], dofs, 1e-8, 1000)
    tip = np.abs(m.coords[:, 0] - 1.0) < 1e-6
    uy = x[3 * np.nonzero(tip)[0] + 1].mean()
    assert abs(uy - (-0.005339)) / 0.005339 < 0.01


# -- fenics-solver/tests/elasticity_tests.rs:6-126 ---------------------------

def test_axial_bar_extension():
    m = O.box_beam(1.0, 0.1, 0.1, 10, 2, 2)
    dofs = O.clamp_dofs(m)
    x, _, _ = O.solve_elasticity_3d(m, 1.0e6, 0.0, [1000.0, 0.0, 0.0], dofs, 1e-10, 1000)
    tip = np.abs(m.coords[:, 0] - 1.0) < 1e-6
    ux = x[3 * np.nonzero(tip)[0]].mean()
    assert abs(ux - 5e-4) / 5e-4 < 0.03


def test_cantilever_bending_vs_dolfinx():
    m = O.box_beam(1.0, 0.1, 0.1, 20, 3, 3)
    dofs = O.clamp_dofs(m)
    x, _, _ = O.solve_elasticity_3d(m, 1.0e6, 0.3, [0.0, 0.0, -1000.0], dofs, 1e-9, 2000)
    tip = np.abs(m.coords[:, 0] - 1.0) < 1e-6
    uz = x[3 * np.nonzero(tip)[0] + 2].mean()
    assert abs(uz - (-0.0890)) / 0.0890 < 0.06 and uz < 0
    _, vvm = O.von_mises(m, x, 1.0e6, 0.3)
    assert vvm.max() > 1e4


# -- Independent cross-checks (numpy / scipy) --------------------------------

def _numpy_p1_stiffness(coords, cells):
    """Vectorised P1 stiffness built independently of the oracle."""
    import scipy.sparse as sp
    d = coords.shape[1]
    X = coords[cells]                                  # [nc, d+1, d]
    J = np.transpose(X[:, 1:, :] - X[:, :1, :], (0, 2, 1))   # columns v_i - v0
    det = np.linalg.det(J)
    G = np.linalg.inv(J).transpose(0, 2, 1)            # J^{-T}
    ref = np.vstack([-np.ones(d), np.eye(d)])          # [d+1, d]
    g = np.einsum("cij,kj->cki", G, ref)               # [nc, d+1, d]
    meas = np.abs(det) / math.factorial(d)
    K = np.einsum("cid,cjd->cij", g, g) * meas[:, None, None]
    n = coords.shape[0]
    r = np.repeat(cells, d + 1, axis=1).ravel()
    c = np.tile(cells, (1, d + 1)).ravel()
    return sp.csc_matrix((K.ravel(), (r, c)), shape=(n, n))


def test_stiffness_vs_numpy_on_perturbed_meshes():
    rng = np.random.default_rng(7)
    for m in (O.unit_square(7, 5), O.unit_cube(4, 3, 2)):
        h = 0.15 / max(m.cells.shape)
        m.coords[:] += rng.uniform(-h, h, m.coords.shape)
        A = (O.assemble_stiffness_2d(m) if m.dim == 2 else O.assemble_stiffness_3d(m)).to_scipy()
        B = _numpy_p1_stiffness(m.coords, m.cells)
        B.sum_duplicates()
        B.sort_indices()
        assert np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices)
        assert np.max(np.abs(A.data - B.data)) <= 1e-12 * np.max(np.abs(B.data))


def test_cg_vs_scipy_spsolve_fd_laplacian():
    # gpu.rs:1610-1663: 20^3 7-point FD Laplacian, b = 1, CG to 1e-9.
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    nx = 20
    n = nx ** 3
    idx = np.arange(n).reshape(nx, nx, nx)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [np.full(n, 6.0)]
    for ax in range(3):
        a = np.take(idx, range(nx - 1), axis=ax).ravel()
        b = np.take(idx, range(1, nx), axis=ax).ravel()
        rows += [a, b]
        cols += [b, a]
        vals += [-np.ones(len(a)), -np.ones(len(a))]
    r, c, v = (np.concatenate(t) for t in (rows, cols, vals))
    A = O.csc_from_triplets(n, r, c, v)
    x, it, _ = O.solve_cg(A, np.ones(n), None, 1e-9, 1000)
    xd = spl.spsolve(sp.csc_matrix((v, (r, c)), shape=(n, n)), np.ones(n))
    assert np.allclose(x, xd, rtol=1e-5, atol=1e-5)


def test_elasticity_matrix_properties():
    # Rigid-body modes lie in the kernel of the unconstrained stiffness.
    m = O.box_beam(2.0, 1.0, 1.0, 3, 2, 2)
    K = O.assemble_elasticity_3d(m, 210e9, 0.3).to_scipy()
    assert abs(K - K.T).max() == 0.0
    t = np.tile([1.0, 0.0, 0.0], m.nv)
    rot = np.column_stack([-m.coords[:, 1], m.coords[:, 0], np.zeros(m.nv)]).ravel()
    scale = abs(K).max()
    assert np.abs(K @ t).max() < 1e-9 * scale
    assert np.abs(K @ rot).max() < 1e-9 * scale


def test_p2_patch_test():
    # P2 reproduces a quadratic solution exactly: u = x^2 + y z, -lap u = -2.
    m = O.unit_cube(3, 3, 3)
    cd, ev = O.p2_dofmap(m)
    nd = m.nv + len(ev)
    xyz = np.vstack([m.coords, 0.5 * (m.coords[ev[:, 0]] + m.coords[ev[:, 1]])])
    u = xyz[:, 0] ** 2 + xyz[:, 1] * xyz[:, 2]
    K = O.assemble_p2_stiffness_3d(m, cd, nd)
    q = O.quadrature_points_3d(m)
    b = O.assemble_p2_rhs_3d(m, cd, nd, np.full(len(q), -2.0))
    bd = O.p2_boundary_dofs(m)
    Kb, bb = O.apply_dirichlet_bc(K, b, bd, u[bd])
    x, _, _ = O.solve_cg(Kb, bb, None, 1e-13, 2000)
    assert np.abs(x - u).max() < 1e-9


def test_p2_boundary_dof_count():
    m = O.unit_cube(4, 4, 4)
    bd = O.p2_boundary_dofs(m)
    nbv = 5 ** 3 - 3 ** 3
    per_face_edges = 2 * 4 * 5 + 4 * 4
    assert len(bd) == nbv + 6 * per_face_edges - 12 * 4
    assert np.all(np.diff(bd) > 0)


def test_adjoint_compliance_identity_small():
    # dJ/dtheta for J = f^T u equals -3 theta^2 E0 u_e^T K_e^1 u_e. Checked two
    # ways on a small clamped beam: against -u^T (dK/dtheta_e) u built by the
    # assembler itself (exact to round-off), and against central differences.
    # FD uses h = 1e-4: at h = 1e-6 the assembly round-off in J(theta +- h)
    # (~1e-14 |J|) divided by 2h is ~1e-5 of the gradient on this mesh, so 1e-6
    # agreement is not reachable in FP64 there; h = 1e-4 keeps both the noise
    # and the O(h^2) truncation below 1e-6.
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    rng = np.random.default_rng(3)
    m = O.box_beam(3.0, 1.0, 1.0, 6, 2, 2)
    theta = rng.uniform(0.3, 1.0, m.nc)
    nu, E0 = 0.3, 1.0
    dofs = O.clamp_dofs(m)
    f = O.body_force_3d(m, [0.0, 0.0, -1.0])

    def J(th):
        K = O.assemble_elasticity_3d(m, E0, nu, cell_E=E0 * th ** 3)
        Kb, fb = O.apply_dirichlet_bc(K, f, dofs, np.zeros(len(dofs)))
        S = Kb.to_scipy().tocsc()
        lu = spl.splu(S)
        u = lu.solve(fb)
        u += lu.solve(fb - S @ u)          # one refinement step
        return fb @ u, u

    j0, u = J(theta)
    g = O.adjoint_grad(m, nu, E0, theta, u, u)
    unit_diag = sp.diags(np.isin(np.arange(3 * m.nv), dofs).astype(float))
    for c in rng.choice(m.nc, 6, replace=False):
        sel = np.where(np.arange(m.nc) == c, 3 * theta[c] ** 2 * E0, 0.0)
        dK, _ = O.apply_dirichlet_bc(O.assemble_elasticity_3d(m, 1.0, nu, cell_E=sel), f, dofs,
                                     np.zeros(len(dofs)))
        direct = -u @ ((dK.to_scipy() - unit_diag) @ u)
        assert abs(direct - g[c]) <= 1e-10 * abs(g[c])
        h = 1e-4
        tp, tm = theta.copy(), theta.copy()
        tp[c] += h
        tm[c] -= h
        fd = (J(tp)[0] - J(tm)[0]) / (2 * h)
        assert abs(fd - g[c]) <= 1e-6 * abs(g[c]) + 1e-15 * abs(j0) / h


def test_add_scaled_matrices_union_semantics():
    """add_scaled_matrices (transient.rs:72-97) on operands of different
    patterns, as restated by the oracle: the union pattern with rows sorted
    per column, explicit zeros of either operand kept, an entry held by both
    a + (alpha * b) and one held by b alone alpha * b (checked against a
    dense restatement; scipy's sum would drop the explicit zeros)."""
    rng = np.random.default_rng(11)
    n = 23

    def rand_csc(density, seed):
        r = np.random.default_rng(seed)
        mask = r.random((n, n)) < density
        vals = r.standard_normal((n, n))
        vals[r.random((n, n)) < 0.15] = 0.0
        cp = np.zeros(n + 1, np.int64)
        rows, vs = [], []
        for j in range(n):
            rr = np.nonzero(mask[:, j])[0]
            rows.append(rr)
            vs.append(vals[rr, j])
            cp[j + 1] = cp[j] + len(rr)
        return O.Csc(n, cp, np.concatenate(rows).astype(np.int64), np.concatenate(vs)), mask, vals

    A, ma, va = rand_csc(0.2, 1)
    B, mb, vb = rand_csc(0.1, 2)
    alpha = float(rng.uniform(-2, 2))
    C = O.add_scaled_matrices(A, B, alpha)
    union = ma | mb
    assert np.array_equal(np.diff(C.colptr), union.sum(axis=0))
    for j in range(n):
        rows = np.asarray(C.rowidx[C.colptr[j]:C.colptr[j + 1]])
        assert np.array_equal(rows, np.nonzero(union[:, j])[0])
        for k, i in enumerate(rows):
            v = C.vals[C.colptr[j] + k]
            if ma[i, j] and mb[i, j]:
                assert v == va[i, j] + alpha * vb[i, j]
            elif ma[i, j]:
                assert v == va[i, j]
            else:
                assert v == alpha * vb[i, j]
