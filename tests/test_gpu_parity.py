"""Parity of the CUDA path with the oracle (CPU restatement of the reference).

Bars (from the reference's own test tolerances and the hot-path contract):
  * sparsity pattern, dof maps, boundary-dof and facet sets: bit-exact
  * FP64 matrix entries: |a - b| <= 1e-12 * max|row| (per-cell round-off in
    structurally zero entries makes a purely relative test meaningless there)
  * load vectors: bit-exact (the RHS kernels keep the reference's order)
  * solutions: within 1e-8 relative L2 of a direct solve when solved tightly
All calls go through the C ABI (libfenics_cuda.so).
"""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

PI = math.pi


def _perturbed(mesh_fn, *args, seed=0, frac=0.2):
    m = mesh_fn(*args)
    rng = np.random.default_rng(seed)
    h = frac / max(args[-3:]) if len(args) >= 3 else frac / max(args)
    inner = np.all((m.coords > 1e-9) & (m.coords < m.coords.max(axis=0) - 1e-9), axis=1)
    m.coords[inner] += rng.uniform(-h, h, (inner.sum(), m.coords.shape[1])) * 0.5
    return m


def _assert_csc_equal(A, B, tol=1e-12):
    """A from the device, B from the oracle."""
    assert A.n == B.n
    assert np.array_equal(A.colptr, B.colptr), "column pointers differ"
    assert np.array_equal(A.rowidx, B.rowidx), "row indices differ"
    scale = np.maximum.reduceat(np.abs(B.vals), B.colptr[:-1]) if B.nnz else np.zeros(0)
    colscale = np.repeat(scale, np.diff(B.colptr))
    assert np.all(np.abs(A.vals - B.vals) <= tol * np.maximum(colscale, 1e-300)), \
        f"max rel dev {np.max(np.abs(A.vals - B.vals) / np.maximum(colscale, 1e-300)):.3e}"


def _fmesh(fcu, om):
    return fcu.Mesh(om.coords, om.cells)


# ---------------------------------------------------------------------------
# assembly
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n", [1, 4, 16, 33])
def test_p1_2d_stiffness(fcu, ctx, n):
    om = O.unit_square(n, n)
    A = fcu.assemble_stiffness_2d(_fmesh(fcu, om), ctx)
    _assert_csc_equal(A, O.assemble_stiffness_2d(om))


def test_p1_2d_stiffness_perturbed_with_kappa(fcu, ctx):
    om = _perturbed(O.unit_square, 20, 13, seed=1)
    kappa = np.exp(np.random.default_rng(2).normal(size=om.nc))
    A = fcu.assemble_stiffness_2d(_fmesh(fcu, om), ctx, kappa=kappa)
    _assert_csc_equal(A, O.assemble_stiffness_2d(om, kappa=kappa))


def test_p1_2d_degenerate_cells_skipped(fcu, ctx):
    om = O.unit_square(6, 6)
    # collapse one vertex onto a neighbour: two cells become degenerate
    om.coords[8] = om.coords[9]
    A = fcu.assemble_stiffness_2d(_fmesh(fcu, om), ctx)
    B = O.assemble_stiffness_2d(om)
    _assert_csc_equal(A, B)


@pytest.mark.parametrize("dims", [(1, 1, 1), (3, 3, 3), (7, 5, 4)])
def test_p1_3d_stiffness(fcu, ctx, dims):
    om = _perturbed(O.unit_cube, *dims, seed=3)
    A = fcu.assemble_stiffness_3d(_fmesh(fcu, om), ctx)
    _assert_csc_equal(A, O.assemble_stiffness_3d(om))


def test_p1_3d_stiffness_kappa(fcu, ctx):
    om = O.unit_cube(6, 6, 6)
    kappa = np.exp(np.random.default_rng(4).normal(size=om.nc))
    A = fcu.assemble_stiffness_3d(_fmesh(fcu, om), ctx, kappa=kappa)
    _assert_csc_equal(A, O.assemble_stiffness_3d(om, kappa=kappa))


@pytest.mark.parametrize("dims", [(1, 1, 1), (4, 2, 2), (9, 3, 3)])
def test_elasticity_stiffness(fcu, ctx, dims):
    om = O.box_beam(4.0, 1.0, 1.0, *dims)
    mat = fcu.ElasticMaterial(210e9, 0.3)
    A = fcu.assemble_elasticity_stiffness_3d(_fmesh(fcu, om), mat, ctx)
    _assert_csc_equal(A, O.assemble_elasticity_3d(om, 210e9, 0.3))


def _star_mesh():
    """Tetrahedra joining the centre of the unit cube to each boundary
    triangle of its 3x3x3 Kuhn subdivision: the centre's row couples to all
    56 boundary vertices (57 blocks), so the row kernels take 32 lanes per
    row and two chunks, which the box meshes (15 blocks per row at most)
    never reach."""
    box = O.unit_cube(3, 3, 3)
    tri, _, _ = O.boundary_facets_3d(box)
    used = np.unique(tri)
    remap = np.full(box.nv, -1, np.int64)
    remap[used] = np.arange(len(used))
    coords = np.vstack([box.coords[used], [[0.5, 0.5, 0.5]]])
    centre = len(used)
    cells = np.column_stack([np.full(len(tri), centre), remap[tri]]).astype(box.cells.dtype)
    return O.Mesh(np.ascontiguousarray(coords), np.ascontiguousarray(cells))


def test_long_rows_star_mesh(fcu, ctx):
    om = _star_mesh()
    fm = _fmesh(fcu, om)
    V = fcu.FunctionSpace(ctx, fm, fcu.FCU_SPACE_P1_VEC3)
    K = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
    _assert_csc_equal(K.export_csc(), O.assemble_elasticity_3d(om, 210e9, 0.3))
    Mm = fcu.Matrix(ctx, V).assemble_mass(7850.0)
    _assert_csc_equal(Mm.export_csc(), O.assemble_elasticity_mass_3d(om, 7850.0))
    kappa = np.random.default_rng(8).uniform(0.5, 2.0, om.nc)
    _assert_csc_equal(fcu.assemble_stiffness_3d(fm, ctx, kappa=kappa), O.assemble_stiffness_3d(om, kappa))
    for x in (K, Mm):
        x.close()
    V.close()


def test_elasticity_stiffness_per_cell_modulus_perturbed(fcu, ctx):
    om = _perturbed(O.box_beam, 3.0, 1.0, 1.0, 6, 3, 3, seed=5)
    th = np.random.default_rng(6).uniform(0.01, 1.0, om.nc)
    A = fcu.assemble_elasticity_stiffness_3d(_fmesh(fcu, om), fcu.ElasticMaterial(1.0, 0.3), ctx, cell_E=th ** 3)
    _assert_csc_equal(A, O.assemble_elasticity_3d(om, 1.0, 0.3, cell_E=th ** 3))


def test_elasticity_rejects_bad_poisson_ratio(fcu, ctx):
    om = O.box_beam(1.0, 1.0, 1.0, 1, 1, 1)
    V = fcu.FunctionSpace(ctx, _fmesh(fcu, om), fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V)
    with pytest.raises(fcu.FcuError):
        M.assemble_elasticity(1.0, 0.5)


@pytest.mark.parametrize("dims", [(1, 1, 1), (3, 3, 3), (5, 4, 3)])
def test_p2_dofmap_stiffness_boundary(fcu, ctx, dims):
    om = _perturbed(O.unit_cube, *dims, seed=7)
    kappa = np.exp(np.random.default_rng(8).normal(size=om.nc))
    cd, ev = O.p2_dofmap(om)
    nd = om.nv + len(ev)
    V = fcu.FunctionSpace(ctx, _fmesh(fcu, om), fcu.FCU_SPACE_P2)
    assert V.ndofs == nd
    dcd, dev = V.p2_dofmap()
    assert np.array_equal(dcd, cd) and np.array_equal(dev, ev)
    assert np.array_equal(V.boundary_dofs(), O.p2_boundary_dofs(om))
    M = fcu.Matrix(ctx, V).assemble_stiffness(kappa)
    _assert_csc_equal(M.export_csc(), O.assemble_p2_stiffness_3d(om, cd, nd, kappa))


# ---------------------------------------------------------------------------
# boundary sets, load vectors
# ---------------------------------------------------------------------------

def test_boundary_dofs_and_facets(fcu, ctx):
    for om in (O.unit_square(9, 5), _perturbed(O.unit_cube, 4, 3, 5, seed=9)):
        fm = _fmesh(fcu, om)
        bd = fcu.boundary_dofs_2d(fm, ctx) if om.dim == 2 else fcu.boundary_dofs_3d(fm, ctx)
        ref = O.boundary_dofs_2d(om) if om.dim == 2 else O.boundary_dofs_3d(om)
        assert np.array_equal(bd, ref)
        v, c, lo = fcu.extract_boundary_facets(fm, ctx)
        rv, rc, rl = O.boundary_facets_2d(om) if om.dim == 2 else O.boundary_facets_3d(om)
        assert np.array_equal(v, rv) and np.array_equal(c, rc) and np.array_equal(lo, rl)


def test_rhs_2d_bitexact(fcu, ctx):
    om = _perturbed(O.unit_square, 17, 11, seed=10)
    f = lambda x, y: 2.0 * PI * PI * np.sin(PI * x) * np.sin(PI * y)
    b = fcu.assemble_rhs_2d(_fmesh(fcu, om), f, ctx)
    assert np.array_equal(b, O.assemble_rhs_2d(om, f))


def test_rhs_3d_bitexact(fcu, ctx):
    om = _perturbed(O.unit_cube, 5, 4, 3, seed=11)
    f = lambda x, y, z: x * x - y * z + 1.0
    b = fcu.assemble_rhs_3d(_fmesh(fcu, om), f, ctx)
    assert np.array_equal(b, O.assemble_rhs_3d(om, f))


def test_rhs_p2_and_device_sources(fcu, ctx):
    om = O.unit_cube(4, 4, 4)
    cd, ev = O.p2_dofmap(om)
    nd = om.nv + len(ev)
    V = fcu.FunctionSpace(ctx, _fmesh(fcu, om), fcu.FCU_SPACE_P2)
    q = V.quadrature_points()
    assert np.array_equal(q, O.quadrature_points_3d(om))
    fq = 1.0 + q[:, 0] * q[:, 1]
    assert np.array_equal(V.rhs_values(fq), O.assemble_p2_rhs_3d(om, cd, nd, fq))
    # constant source evaluated on the device equals the values path
    b1 = V.rhs_source(fcu.FCU_SRC_CONSTANT, (1.0,))
    assert np.array_equal(b1, O.assemble_p2_rhs_3d(om, cd, nd, np.ones(len(q))))
    # analytic sine product: device sin vs libm sin, so allow last-bit noise
    m2 = O.unit_square(16, 16)
    V2 = fcu.FunctionSpace(ctx, _fmesh(fcu, m2), fcu.FCU_SPACE_P1)
    bs = V2.rhs_source(fcu.FCU_SRC_SIN_PRODUCT, (2.0 * PI * PI, PI))
    ref = O.assemble_rhs_2d(m2, lambda x, y: 2.0 * PI * PI * np.sin(PI * x) * np.sin(PI * y))
    assert np.max(np.abs(bs - ref)) <= 1e-14 * np.max(np.abs(ref))
    # nodal source: b = M f through the 3-point rule
    fn = np.random.default_rng(12).uniform(-1, 1, m2.nv)
    bn = V2.rhs_source(fcu.FCU_SRC_NODAL, nodal=fn)
    qq = O.quadrature_points_2d(m2)
    cells = m2.cells
    # interpolate f at the edge midpoints of each triangle: (0.5,0), (0.5,0.5), (0,0.5)
    f0, f1, f2 = fn[cells[:, 0]], fn[cells[:, 1]], fn[cells[:, 2]]
    fq2 = np.stack([0.5 * f0 + 0.5 * f1, 0.5 * f1 + 0.5 * f2, 0.5 * f0 + 0.5 * f2], 1).ravel()
    assert qq.shape[0] == fq2.shape[0]
    assert np.max(np.abs(bn - O.assemble_rhs_2d_values(m2, fq2))) <= 1e-15 * np.max(np.abs(bn))


def test_body_force_and_traction_bitexact(fcu, ctx):
    om = _perturbed(O.box_beam, 3.0, 1.0, 1.0, 6, 2, 3, seed=13)
    fm = _fmesh(fcu, om)
    f = fcu.assemble_elasticity_body_force_3d(fm, [0.5, -2.0, -7.8e4], ctx)
    assert np.array_equal(f, O.body_force_3d(om, [0.5, -2.0, -7.8e4]))
    v, _, _ = O.boundary_facets_3d(om)
    tip = v[np.all(np.abs(om.coords[v][:, :, 0] - 3.0) < 1e-9, axis=1)]
    assert len(tip) == 2 * 2 * 3
    t = lambda x, y, z: (0.0 * x, 0.1 * y, -1.0 + 0.0 * z)
    bt = fcu.assemble_surface_traction_3d(fm, tip, t, ctx)
    assert np.array_equal(bt, O.surface_traction_3d(om, tip, t))


# ---------------------------------------------------------------------------
# Dirichlet
# ---------------------------------------------------------------------------

def test_dirichlet_scalar_matches_oracle(fcu, ctx):
    om = _perturbed(O.unit_square, 12, 9, seed=14)
    A = O.assemble_stiffness_2d(om)
    b = O.assemble_rhs_2d(om, lambda x, y: 1.0 + x)
    bd = O.boundary_dofs_2d(om)
    g = np.sin(om.coords[bd, 0]) + om.coords[bd, 1]
    # repeated dofs: the diagonal counts them, the last value wins
    dofs = np.concatenate([bd, bd[:3]])
    vals = np.concatenate([g, g[:3] + 1.0])
    Ab, bb = O.apply_dirichlet_bc(A, b, dofs, vals)
    # device: assemble on the space, eliminate in place, export
    V = fcu.FunctionSpace(ctx, _fmesh(fcu, om), fcu.FCU_SPACE_P1)
    M = fcu.Matrix(ctx, V).assemble_stiffness()
    bdev = V.rhs_values(np.asarray(1.0 + O.quadrature_points_2d(om)[:, 0]))
    assert np.array_equal(bdev, b)
    M.apply_dirichlet(bdev, dofs, vals)
    _assert_csc_equal(M.export_csc(), Ab)
    assert np.max(np.abs(bdev - bb)) <= 1e-12 * np.max(np.abs(bb))
    # the drop-in function on a caller CSC
    A2, b2 = fcu.apply_dirichlet_bc(A, b, fcu.DirichletBC(dofs, vals), ctx)
    _assert_csc_equal(A2, Ab)
    assert np.array_equal(b2, bb)


def test_dirichlet_vector_matches_oracle(fcu, ctx):
    om = O.box_beam(2.0, 1.0, 1.0, 4, 2, 2)
    K = O.assemble_elasticity_3d(om, 1e6, 0.25)
    f = O.body_force_3d(om, [0.0, 0.0, -1.0])
    dofs = O.clamp_dofs(om)
    # partial clamp on another face: only the y component
    extra = 3 * np.nonzero(om.coords[:, 0] > 2.0 - 1e-9)[0] + 1
    d = np.concatenate([dofs, extra])
    v = np.concatenate([np.zeros(len(dofs)), 0.01 * np.ones(len(extra))])
    Kb, fb = O.apply_dirichlet_bc(K, f, d, v)
    V = fcu.FunctionSpace(ctx, _fmesh(fcu, om), fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V).assemble_elasticity(1e6, 0.25)
    fd = V.body_force([0.0, 0.0, -1.0])
    M.apply_dirichlet(fd, d, v)
    _assert_csc_equal(M.export_csc(), Kb)
    assert np.max(np.abs(fd - fb)) <= 1e-12 * np.max(np.abs(fb))
    bc = fcu.VectorDirichletBC(list(zip(d.tolist(), v.tolist())))
    K2, f2 = fcu.apply_vector_dirichlet_bc(K, f, bc, ctx)
    _assert_csc_equal(K2, Kb)


def test_dirichlet_rejects_out_of_range(fcu, ctx):
    om = O.unit_square(3, 3)
    A = O.assemble_stiffness_2d(om)
    with pytest.raises(fcu.FcuError):
        fcu.apply_dirichlet_bc(A, np.zeros(om.nv), fcu.DirichletBC(np.array([om.nv]), np.array([0.0])), ctx)


# ---------------------------------------------------------------------------
# solvers
# ---------------------------------------------------------------------------

def _direct(A, b):
    import scipy.sparse.linalg as spl
    return spl.spsolve(A.to_scipy().tocsc(), b)


def test_cg_2x2(fcu, ctx):
    A = O.csc_from_triplets(2, [0, 0, 1, 1], [0, 1, 0, 1], [4.0, -1.0, -1.0, 4.0])
    x, it, res = fcu.solve_cg(A, [3.0, 3.0], None, 1e-10, 100, ctx)
    assert it <= 2 and res < 1e-10 and np.allclose(x, [1.0, 1.0], atol=1e-8)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cg_poisson_matches_direct(fcu, ctx, precision):
    om = _perturbed(O.unit_square, 40, 40, seed=15)
    A = O.assemble_stiffness_2d(om)
    b = O.assemble_rhs_2d(om, lambda x, y: np.ones_like(x))
    bd = O.boundary_dofs_2d(om)
    Ab, bb = O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))
    xd = _direct(Ab, bb)
    prec = fcu.FCU_FP64 if precision == "fp64" else fcu.FCU_MIXED
    x, it, res = fcu.solve_cg(Ab, bb, None, 1e-13, 5000, ctx, precision=prec)
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    # the FP64 residual the solver reports is the true one
    r = bb - Ab.to_scipy() @ x
    assert np.linalg.norm(r) / np.linalg.norm(bb) < 1e-13 * 10
    if precision == "fp64":
        _, it_o, _ = O.solve_cg(Ab, bb, None, 1e-13, 5000)
        assert abs(it - it_o) <= max(3, 0.02 * it_o)


def test_cg_iterations_track_oracle_elasticity(fcu, ctx):
    om = O.box_beam(4.0, 1.0, 1.0, 16, 4, 4)
    dofs = O.clamp_dofs(om)
    K = O.assemble_elasticity_3d(om, 210e9, 0.3)
    f = O.body_force_3d(om, [0.0, 0.0, -7.8e4])
    Kb, fb = O.apply_dirichlet_bc(K, f, dofs, np.zeros(len(dofs)))
    x_o, it_o, _ = O.solve_cg(Kb, fb, None, 1e-8, 20000)
    V = fcu.FunctionSpace(ctx, _fmesh(fcu, om), fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
    fd = V.body_force([0.0, 0.0, -7.8e4])
    M.apply_dirichlet(fd, dofs, np.zeros(len(dofs)))
    x, info = M.pcg(fd, tol=1e-8, max_iter=20000)
    assert abs(info.iterations - it_o) <= max(3, 0.02 * it_o)
    assert np.linalg.norm(x - x_o) <= 1e-6 * np.linalg.norm(x_o)
    xm, im = M.pcg(fd, tol=1e-8, max_iter=20000, precision=fcu.FCU_MIXED)
    r = fb - Kb.to_scipy() @ xm
    assert np.linalg.norm(r) / np.linalg.norm(fb) < 1e-8
    assert im.outer_updates >= 1


def test_cg_error_behaviour(fcu, ctx):
    om = O.unit_square(8, 8)
    A = O.assemble_stiffness_2d(om)
    b = O.assemble_rhs_2d(om, lambda x, y: np.ones_like(x))
    bd = O.boundary_dofs_2d(om)
    Ab, bb = O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))
    with pytest.raises(fcu.CgError) as e:
        fcu.solve_cg(Ab, bb, None, 1e-12, 1, ctx)
    assert e.value.code == 3
    Z = O.csc_from_triplets(2, [0, 1], [0, 1], [0.0, 0.0])
    with pytest.raises(fcu.CgError) as e2:
        fcu.solve_cg(Z, [1.0, 1.0], None, 1e-10, 10, ctx)
    assert e2.value.code == 4
    # zero right-hand side converges at iteration 0 (cg.rs:87-90)
    x, it, res = fcu.solve_cg(Ab, np.zeros(Ab.n), None, 1e-10, 10, ctx)
    assert it == 0 and np.all(x == 0)


def test_cg_with_initial_guess(fcu, ctx):
    om = O.unit_square(10, 10)
    A = O.assemble_stiffness_2d(om)
    b = O.assemble_rhs_2d(om, lambda x, y: x)
    bd = O.boundary_dofs_2d(om)
    Ab, bb = O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))
    xd = _direct(Ab, bb)
    x, it, _ = fcu.solve_cg(Ab, bb, xd, 1e-10, 100, ctx)
    assert it == 0 and np.array_equal(x, xd)


def test_solve_csr_cg_gpu_fd_laplacian(fcu, ctx):
    # gpu.rs:1610-1663: 20^3 7-point Laplacian, b = 1, rtol 1e-9, vs CPU CG at 1e-5
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
    x_cpu, _, _ = O.solve_cg(A, np.ones(n), None, 1e-9, 1000)
    # CSR == CSC for this symmetric matrix (gpu.rs:1551-1583)
    inv = 1.0 / A.to_scipy().diagonal()
    res = fcu.solve_csr_cg_gpu(A.colptr.astype(np.uint32), A.rowidx.astype(np.uint32), A.vals, inv,
                               np.ones(n), None, 1e-9, 1000)
    assert np.allclose(res.solution, x_cpu, rtol=1e-5, atol=1e-5)
    assert res.final_residual < 1e-9
    g = fcu.solve_cg_gpu_or_cpu(A, np.ones(n), None, 1e-9, 1000)
    assert np.allclose(g.solution, x_cpu, rtol=1e-5, atol=1e-5)
    # the reference returns Ok with a zero solution for b = 0 and Ok at the limit
    z = fcu.solve_csr_cg_gpu(A.colptr.astype(np.uint32), A.rowidx.astype(np.uint32), A.vals, inv,
                             np.zeros(n), None, 1e-9, 1000)
    assert z.iterations == 0 and np.all(z.solution == 0)
    lim = fcu.solve_csr_cg_gpu(A.colptr.astype(np.uint32), A.rowidx.astype(np.uint32), A.vals, inv,
                               np.ones(n), None, 1e-14, 3)
    assert lim.iterations == 3 and lim.final_residual > 1e-14


def test_spmv_matches_oracle(fcu, ctx):
    om = _perturbed(O.unit_cube, 5, 5, 5, seed=16)
    A = O.assemble_stiffness_3d(om)
    x = np.random.default_rng(17).normal(size=A.n)
    y = fcu.spmv(A, x, ctx)
    yo = O.spmv(A, x)
    assert np.max(np.abs(y - yo)) <= 1e-13 * np.max(np.abs(yo))


# ---------------------------------------------------------------------------
# the reference's end-to-end known answers, through the device path
# ---------------------------------------------------------------------------

def _u2(x, y):
    return np.sin(PI * x) * np.sin(PI * y)


def _f2(x, y):
    return 2.0 * PI * PI * np.sin(PI * x) * np.sin(PI * y)


def test_ab_poisson_2d_vs_dolfinx_device(fcu, ctx):
    # ab_benchmarks.rs:13-48
    om = O.unit_square(16, 16)
    sol = fcu.solve_poisson_2d(_fmesh(fcu, om), _f2, _u2, 1e-12, 1000, ctx)
    l2 = O.l2_error_2d(om, sol.u, _u2)
    assert abs(l2 - 5.377435e-3) / 5.377435e-3 < 0.05
    assert abs(sol.u.max() - 0.996793) / 0.996793 < 1e-3
    x_o, it_o, _ = O.solve_poisson_2d(om, _f2, _u2, 1e-12, 1000)
    assert np.max(np.abs(sol.u - x_o)) < 1e-10


def test_poisson_rates_device(fcu, ctx):
    # poisson_tests.rs:5-52
    errs = []
    for n in (8, 16, 32):
        om = O.unit_square(n, n)
        sol = fcu.solve_poisson_2d(_fmesh(fcu, om), _f2, _u2, 1e-10, 500, ctx)
        errs.append(O.l2_error_2d(om, sol.u, _u2))
    assert 3.8 < errs[0] / errs[1] < 4.2 and 3.8 < errs[1] / errs[2] < 4.2


def test_ab_cantilever_device(fcu, ctx):
    # ab_benchmarks.rs:51-100
    om = O.box_beam(1.0, 0.1, 0.1, 10, 2, 2)
    dofs = O.clamp_dofs(om)
    bc = fcu.VectorDirichletBC([(int(d), 0.0) for d in dofs])
    sol = fcu.solve_elasticity_3d(_fmesh(fcu, om), fcu.ElasticMaterial(1e7, 0.3), [0.0, -1000.0, 0.0], bc, 1e-8,
                                  1000, ctx)
    tip = np.abs(om.coords[:, 0] - 1.0) < 1e-6
    uy = sol.displacements[3 * np.nonzero(tip)[0] + 1].mean()
    assert abs(uy - (-0.005339)) / 0.005339 < 0.01


def test_cantilever_bending_device(fcu, ctx):
    # elasticity_tests.rs:51-126
    om = O.box_beam(1.0, 0.1, 0.1, 20, 3, 3)
    dofs = O.clamp_dofs(om)
    bc = fcu.VectorDirichletBC([(int(d), 0.0) for d in dofs])
    # The FP32 inner iteration converges more slowly on this ill-conditioned
    # beam, so the mixed solve gets a larger iteration budget.
    for prec, budget in ((fcu.FCU_FP64, 2000), (fcu.FCU_MIXED, 20000)):
        sol = fcu.solve_elasticity_3d(_fmesh(fcu, om), fcu.ElasticMaterial(1e6, 0.3), [0.0, 0.0, -1000.0], bc,
                                      1e-9, budget, ctx, precision=prec)
        tip = np.abs(om.coords[:, 0] - 1.0) < 1e-6
        uz = sol.displacements[3 * np.nonzero(tip)[0] + 2].mean()
        assert abs(uz - (-0.0890)) / 0.0890 < 0.06


# ---------------------------------------------------------------------------
# adjoint
# ---------------------------------------------------------------------------

def test_adjoint_gradient_matches_oracle(fcu, ctx):
    om = _perturbed(O.box_beam, 3.0, 1.0, 1.0, 6, 2, 2, seed=18)
    rng = np.random.default_rng(19)
    theta = rng.uniform(0.01, 1.0, om.nc)
    u = rng.normal(size=3 * om.nv)
    lam = rng.normal(size=3 * om.nv)
    V = fcu.FunctionSpace(ctx, _fmesh(fcu, om), fcu.FCU_SPACE_P1_VEC3)
    g = V.adjoint_gradient(1.0, 0.3, theta, u, lam)
    go = O.adjoint_grad(om, 0.3, 1.0, theta, u, lam)
    assert np.max(np.abs(g - go)) <= 1e-12 * np.max(np.abs(go))
