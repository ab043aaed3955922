"""ORACLE — test infrastructure only.

numpy/ctypes front end of ``oracle.cpp``, the CPU FP64 restatement of the
GlassOnTin/fenics-rs assembly + Jacobi-PCG path. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs
import this module, and only as the checker or the timed CPU baseline; the
product (``fenics-rs_b200``) never imports it.

Each wrapper names the reference function it restates; ``oracle.cpp`` cites
the reference file:line for the arithmetic.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

i64 = C.c_int64
dbl = C.c_double
vp = C.c_void_p
P = np.ctypeslib.ndpointer


def build() -> str:
    """Compile liboracle.so from oracle.cpp (make; no reference sources involved)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def _load() -> C.CDLL:
    if not os.path.exists(_SO):
        build()
    lib = C.CDLL(_SO)
    f64p = P(np.float64, flags="C_CONTIGUOUS")
    i64p = P(np.int64, flags="C_CONTIGUOUS")
    sig = {
        "orc_csc_from_triplets": (vp, [i64, i64, i64p, i64p, f64p]),
        "orc_csc_from_arrays": (vp, [i64, i64p, i64p, f64p]),
        "orc_csc_n": (i64, [vp]),
        "orc_csc_nnz": (i64, [vp]),
        "orc_csc_export": (None, [vp, i64p, i64p, f64p]),
        "orc_csc_free": (None, [vp]),
        "orc_unit_square": (None, [i64, i64, f64p, i64p]),
        "orc_box_beam": (None, [dbl, dbl, dbl, i64, i64, i64, f64p, i64p]),
        "orc_boundary_facets_2d": (i64, [i64, i64p, vp, vp, vp]),
        "orc_boundary_facets_3d": (i64, [f64p, i64, i64p, vp, vp, vp]),
        "orc_boundary_dofs_2d": (i64, [i64, i64p, vp]),
        "orc_boundary_dofs_3d": (i64, [f64p, i64, i64p, vp]),
        "orc_assemble_stiffness_2d": (vp, [i64, f64p, i64, i64p, vp, C.c_int]),
        "orc_assemble_stiffness_3d": (vp, [i64, f64p, i64, i64p, vp, C.c_int]),
        "orc_assemble_elasticity_3d": (vp, [i64, f64p, i64, i64p, dbl, dbl, vp, C.c_int]),
        "orc_elasticity_element_unit": (C.c_int, [f64p, i64p, dbl, f64p]),
        "orc_quadrature_points_2d": (None, [f64p, i64, i64p, f64p]),
        "orc_assemble_rhs_2d": (None, [i64, f64p, i64, i64p, f64p, f64p]),
        "orc_quadrature_points_3d": (None, [f64p, i64, i64p, f64p]),
        "orc_assemble_rhs_3d": (None, [i64, f64p, i64, i64p, f64p, f64p]),
        "orc_body_force_3d": (None, [i64, f64p, i64, i64p, f64p, f64p]),
        "orc_traction_points_3d": (None, [f64p, i64, i64p, f64p]),
        "orc_surface_traction_3d": (None, [i64, f64p, i64, i64p, f64p, f64p]),
        "orc_p2_num_edges": (i64, [i64, i64p]),
        "orc_p2_dofmap": (None, [i64, i64, i64p, i64p, vp]),
        "orc_assemble_p2_stiffness_3d": (vp, [i64, f64p, i64, i64p, i64p, vp, C.c_int]),
        "orc_assemble_p2_rhs_3d": (None, [i64, f64p, i64, i64p, i64p, f64p, f64p]),
        "orc_p2_boundary_dofs": (i64, [i64, f64p, i64, i64p, vp]),
        "orc_apply_dirichlet": (vp, [vp, f64p, i64, i64p, f64p, f64p]),
        "orc_spmv": (None, [vp, f64p, f64p]),
        "orc_solve_cg": (C.c_int, [vp, f64p, vp, dbl, i64, f64p, C.POINTER(i64), C.POINTER(dbl)]),
        "orc_cg_fixed_iters": (dbl, [vp, f64p, i64, f64p]),
        "orc_l2_points_2d": (None, [f64p, i64, i64p, f64p]),
        "orc_l2_error_2d": (dbl, [f64p, i64, i64p, f64p, f64p]),
        "orc_l2_points_3d": (None, [f64p, i64, i64p, f64p]),
        "orc_l2_error_3d": (dbl, [f64p, i64, i64p, f64p, f64p]),
        "orc_von_mises": (None, [i64, f64p, i64, i64p, f64p, dbl, dbl, f64p, f64p]),
        "orc_adjoint_grad": (None, [f64p, i64, i64p, dbl, dbl, f64p, f64p, f64p, f64p, C.c_int]),
        "orc_affine_map_2d": (C.c_int, [f64p, C.POINTER(dbl), f64p]),
        "orc_affine_map_3d": (C.c_int, [f64p, C.POINTER(dbl), f64p]),
        "orc_p2_basis": (None, [f64p, f64p]),
        "orc_p2_grads": (None, [f64p, f64p]),
        "orc_p2_mass_products": (None, [f64p]),
        "orc_cg_fixed_iters_mt": (dbl, [vp, f64p, i64, f64p, C.c_int]),
        "orc_solve_cg_mt": (C.c_int, [vp, f64p, vp, dbl, i64, C.c_int, f64p, C.POINTER(i64), C.POINTER(dbl)]),
        "orc_assemble_mass": (vp, [i64, f64p, i64, i64p, vp, C.c_int, dbl, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


# ---------------------------------------------------------------------------
# Sparse matrix (faer SparseColMat semantics)
# ---------------------------------------------------------------------------

@dataclass
class Csc:
    """Column-compressed matrix as faer stores it: rows sorted per column."""
    n: int
    colptr: np.ndarray
    rowidx: np.ndarray
    vals: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self.vals, self.rowidx, self.colptr), shape=(self.n, self.n))


def _take_csc(h) -> Csc:
    L = lib()
    n = L.orc_csc_n(h)
    nnz = L.orc_csc_nnz(h)
    cp = np.empty(n + 1, np.int64)
    ri = np.empty(nnz, np.int64)
    va = np.empty(nnz, np.float64)
    L.orc_csc_export(h, cp, ri, va)
    L.orc_csc_free(h)
    return Csc(n, cp, ri, va)


class _Handle:
    """Temporary oracle-side CSC handle for a Python Csc."""

    def __init__(self, m: Csc):
        self.h = lib().orc_csc_from_arrays(m.n, _i64(m.colptr), _i64(m.rowidx), _f64(m.vals))

    def __enter__(self):
        return self.h

    def __exit__(self, *a):
        lib().orc_csc_free(self.h)


def csc_from_triplets(n, rows, cols, vals) -> Csc:
    """faer SparseColMat::try_new_from_triplets (sum duplicates, sort rows)."""
    rows, cols, vals = _i64(rows), _i64(cols), _f64(vals)
    return _take_csc(lib().orc_csc_from_triplets(n, len(rows), rows, cols, vals))


# ---------------------------------------------------------------------------
# Meshes (generators.rs)
# ---------------------------------------------------------------------------

@dataclass
class Mesh:
    coords: np.ndarray  # [nv, dim] float64
    cells: np.ndarray   # [nc, nodes] int64

    @property
    def nv(self) -> int:
        return self.coords.shape[0]

    @property
    def nc(self) -> int:
        return self.cells.shape[0]

    @property
    def dim(self) -> int:
        return self.coords.shape[1]


def unit_square(nx: int, ny: int) -> Mesh:
    co = np.empty(((nx + 1) * (ny + 1), 2))
    ce = np.empty((2 * nx * ny, 3), np.int64)
    lib().orc_unit_square(nx, ny, co, ce)
    return Mesh(co, ce)


def box_beam(L, W, H, nx, ny, nz) -> Mesh:
    co = np.empty(((nx + 1) * (ny + 1) * (nz + 1), 3))
    ce = np.empty((6 * nx * ny * nz, 4), np.int64)
    lib().orc_box_beam(L, W, H, nx, ny, nz, co, ce)
    return Mesh(co, ce)


def unit_cube(nx, ny, nz) -> Mesh:
    return box_beam(1.0, 1.0, 1.0, nx, ny, nz)


def boundary_facets_2d(m: Mesh):
    L = lib()
    ce = _i64(m.cells)
    nf = L.orc_boundary_facets_2d(m.nc, ce, None, None, None)
    v = np.empty((nf, 2), np.int64)
    c = np.empty(nf, np.int64)
    lo = np.empty(nf, np.int64)
    L.orc_boundary_facets_2d(m.nc, ce, _ptr(v), _ptr(c), _ptr(lo))
    return v, c, lo


def boundary_facets_3d(m: Mesh):
    L = lib()
    co, ce = _f64(m.coords), _i64(m.cells)
    nf = L.orc_boundary_facets_3d(co, m.nc, ce, None, None, None)
    v = np.empty((nf, 3), np.int64)
    c = np.empty(nf, np.int64)
    lo = np.empty(nf, np.int64)
    L.orc_boundary_facets_3d(co, m.nc, ce, _ptr(v), _ptr(c), _ptr(lo))
    return v, c, lo


def boundary_dofs_2d(m: Mesh) -> np.ndarray:
    L = lib()
    ce = _i64(m.cells)
    out = np.empty(m.nv, np.int64)
    k = L.orc_boundary_dofs_2d(m.nc, ce, _ptr(out))
    return out[:k].copy()


def boundary_dofs_3d(m: Mesh) -> np.ndarray:
    L = lib()
    out = np.empty(m.nv, np.int64)
    k = L.orc_boundary_dofs_3d(_f64(m.coords), m.nc, _i64(m.cells), _ptr(out))
    return out[:k].copy()


# ---------------------------------------------------------------------------
# Assembly
# ---------------------------------------------------------------------------

def assemble_stiffness_2d(m: Mesh, kappa=None, threads: int = 0) -> Csc:
    k = None if kappa is None else _f64(kappa)
    return _take_csc(lib().orc_assemble_stiffness_2d(m.nv, _f64(m.coords), m.nc, _i64(m.cells), _ptr(k), threads))


def assemble_stiffness_3d(m: Mesh, kappa=None, threads: int = 0) -> Csc:
    k = None if kappa is None else _f64(kappa)
    return _take_csc(lib().orc_assemble_stiffness_3d(m.nv, _f64(m.coords), m.nc, _i64(m.cells), _ptr(k), threads))


def assemble_elasticity_3d(m: Mesh, E: float, nu: float, cell_E=None, threads: int = 0) -> Csc:
    ce = None if cell_E is None else _f64(cell_E)
    return _take_csc(lib().orc_assemble_elasticity_3d(m.nv, _f64(m.coords), m.nc, _i64(m.cells), E, nu,
                                                      _ptr(ce), threads))


def elasticity_element_unit(m: Mesh, c: int, nu: float) -> np.ndarray:
    Ke = np.empty(144)
    lib().orc_elasticity_element_unit(_f64(m.coords), _i64(m.cells[c]), nu, Ke)
    return Ke.reshape(12, 12)


def quadrature_points_2d(m: Mesh) -> np.ndarray:
    out = np.empty((m.nc * 3, 2))
    lib().orc_quadrature_points_2d(_f64(m.coords), m.nc, _i64(m.cells), out)
    return out


def quadrature_points_3d(m: Mesh) -> np.ndarray:
    out = np.empty((m.nc * 4, 3))
    lib().orc_quadrature_points_3d(_f64(m.coords), m.nc, _i64(m.cells), out)
    return out


def assemble_rhs_2d(m: Mesh, f) -> np.ndarray:
    """assemble_rhs_2d with a vectorised f(x, y) evaluated at the rule's points."""
    q = quadrature_points_2d(m)
    fq = _f64(f(q[:, 0], q[:, 1]))
    b = np.empty(m.nv)
    lib().orc_assemble_rhs_2d(m.nv, _f64(m.coords), m.nc, _i64(m.cells), fq, b)
    return b


def assemble_rhs_2d_values(m: Mesh, fq) -> np.ndarray:
    b = np.empty(m.nv)
    lib().orc_assemble_rhs_2d(m.nv, _f64(m.coords), m.nc, _i64(m.cells), _f64(fq), b)
    return b


def assemble_rhs_3d(m: Mesh, f) -> np.ndarray:
    q = quadrature_points_3d(m)
    fq = _f64(f(q[:, 0], q[:, 1], q[:, 2]))
    b = np.empty(m.nv)
    lib().orc_assemble_rhs_3d(m.nv, _f64(m.coords), m.nc, _i64(m.cells), fq, b)
    return b


def body_force_3d(m: Mesh, f) -> np.ndarray:
    b = np.empty(3 * m.nv)
    lib().orc_body_force_3d(m.nv, _f64(m.coords), m.nc, _i64(m.cells), _f64(f), b)
    return b


def traction_points_3d(m: Mesh, facets) -> np.ndarray:
    fa = _i64(facets)
    out = np.empty((len(fa) * 3, 3))
    lib().orc_traction_points_3d(_f64(m.coords), len(fa), fa, out)
    return out


def surface_traction_3d(m: Mesh, facets, t) -> np.ndarray:
    """assemble_surface_traction_3d with a vectorised t(x, y, z) -> (tx, ty, tz)."""
    fa = _i64(facets)
    pts = traction_points_3d(m, fa)
    tq = np.stack(np.broadcast_arrays(*t(pts[:, 0], pts[:, 1], pts[:, 2])), axis=1)
    b = np.zeros(3 * m.nv)
    lib().orc_surface_traction_3d(m.nv, _f64(m.coords), len(fa), fa, _f64(tq), b)
    return b


# P2 extension ---------------------------------------------------------------

def p2_dofmap(m: Mesh):
    L = lib()
    ce = _i64(m.cells)
    ne = L.orc_p2_num_edges(m.nc, ce)
    cd = np.empty((m.nc, 10), np.int64)
    ev = np.empty((ne, 2), np.int64)
    L.orc_p2_dofmap(m.nv, m.nc, ce, cd, _ptr(ev))
    return cd, ev


def assemble_p2_stiffness_3d(m: Mesh, cell_dofs, ndofs, kappa=None, threads: int = 0) -> Csc:
    k = None if kappa is None else _f64(kappa)
    return _take_csc(lib().orc_assemble_p2_stiffness_3d(ndofs, _f64(m.coords), m.nc, _i64(m.cells),
                                                        _i64(cell_dofs), _ptr(k), threads))


def assemble_p2_rhs_3d(m: Mesh, cell_dofs, ndofs, fq) -> np.ndarray:
    b = np.empty(ndofs)
    lib().orc_assemble_p2_rhs_3d(ndofs, _f64(m.coords), m.nc, _i64(m.cells), _i64(cell_dofs), _f64(fq), b)
    return b


def p2_boundary_dofs(m: Mesh) -> np.ndarray:
    L = lib()
    ne = L.orc_p2_num_edges(m.nc, _i64(m.cells))
    out = np.empty(m.nv + ne, np.int64)
    k = L.orc_p2_boundary_dofs(m.nv, _f64(m.coords), m.nc, _i64(m.cells), _ptr(out))
    return out[:k].copy()


# ---------------------------------------------------------------------------
# Dirichlet + CG
# ---------------------------------------------------------------------------

def apply_dirichlet_bc(A: Csc, rhs, dofs, vals):
    """apply_dirichlet_bc / apply_vector_dirichlet_bc -> (Csc, b)."""
    nb = np.empty(A.n)
    d, v = _i64(dofs), _f64(vals)
    with _Handle(A) as h:
        out = lib().orc_apply_dirichlet(h, _f64(rhs), len(d), d, v, nb)
    return _take_csc(out), nb


def spmv(A: Csc, x) -> np.ndarray:
    y = np.empty(A.n)
    with _Handle(A) as h:
        lib().orc_spmv(h, _f64(x), y)
    return y


class CgError(RuntimeError):
    pass


def solve_cg(A: Csc, b, x0=None, tol=1e-10, max_iter=1000):
    """solve_cg (cg.rs:40-149): returns (x, iterations, absolute residual); raises
    CgError on breakdown or non-convergence as the reference returns Err."""
    x = np.empty(A.n)
    it = i64(0)
    res = dbl(0.0)
    x0a = None if x0 is None else _f64(x0)
    with _Handle(A) as h:
        st = lib().orc_solve_cg(h, _f64(b), _ptr(x0a), tol, max_iter, x, C.byref(it), C.byref(res))
    if st == 1:
        raise CgError(f"Breakdown in CG: curvature p^T A p is near zero at iteration {it.value}")
    if st == 2:
        raise CgError(f"CG failed to converge within {max_iter} iterations")
    return x, it.value, res.value


def solve_cg_mt(A: Csc, b, x0=None, tol=1e-10, max_iter=1000, threads: int = 0):
    """solve_cg's recurrence and stopping rules (cg.rs:40-149) with the SpMV,
    vector loops and dot products on `threads` OpenMP threads (0 = all): a
    multi-threaded CSR variant, labelled as such (the reference's CG is
    sequential). A must be symmetric. Returns (x, iterations, absolute
    residual); raises CgError like solve_cg."""
    x = np.empty(A.n)
    it = i64(0)
    res = dbl(0.0)
    x0a = None if x0 is None else _f64(x0)
    with _Handle(A) as h:
        st = lib().orc_solve_cg_mt(h, _f64(b), _ptr(x0a), tol, max_iter, threads, x, C.byref(it), C.byref(res))
    if st == 1:
        raise CgError(f"Breakdown in CG: curvature p^T A p is near zero at iteration {it.value}")
    if st == 2:
        raise CgError(f"CG failed to converge within {max_iter} iterations")
    return x, it.value, res.value


def cg_fixed_iters_mt(A: Csc, b, iters: int, threads: int = 0):
    """cg_fixed_iters with an OpenMP row-gather SpMV and parallel vector work
    (a multi-threaded CSR variant for the CPU baseline; A symmetric)."""
    x = np.empty(A.n)
    with _Handle(A) as h:
        rel = lib().orc_cg_fixed_iters_mt(h, _f64(b), iters, x, threads)
    return x, rel


def cg_fixed_iters(A: Csc, b, iters: int):
    x = np.empty(A.n)
    with _Handle(A) as h:
        rel = lib().orc_cg_fixed_iters(h, _f64(b), iters, x)
    return x, rel


def l2_error_2d(m: Mesh, uh, u_exact) -> float:
    pts = np.empty((m.nc * 4, 2))
    lib().orc_l2_points_2d(_f64(m.coords), m.nc, _i64(m.cells), pts)
    ue = _f64(u_exact(pts[:, 0], pts[:, 1]))
    return lib().orc_l2_error_2d(_f64(m.coords), m.nc, _i64(m.cells), _f64(uh), ue)


def l2_error_3d(m: Mesh, uh, u_exact) -> float:
    pts = np.empty((m.nc * 5, 3))
    lib().orc_l2_points_3d(_f64(m.coords), m.nc, _i64(m.cells), pts)
    ue = _f64(u_exact(pts[:, 0], pts[:, 1], pts[:, 2]))
    return lib().orc_l2_error_3d(_f64(m.coords), m.nc, _i64(m.cells), _f64(uh), ue)


def von_mises(m: Mesh, u, E, nu):
    cv = np.empty(m.nc)
    vv = np.empty(m.nv)
    lib().orc_von_mises(m.nv, _f64(m.coords), m.nc, _i64(m.cells), _f64(u), E, nu, cv, vv)
    return cv, vv


def adjoint_grad(m: Mesh, nu, E0, theta, u, lam, threads: int = 0) -> np.ndarray:
    g = np.empty(m.nc)
    lib().orc_adjoint_grad(_f64(m.coords), m.nc, _i64(m.cells), nu, E0, _f64(theta), _f64(u), _f64(lam), g, threads)
    return g


def affine_map(verts):
    """AffineSimplexMap::from_{triangle,tetrahedron}_vertices -> (ok, det, J^{-T})."""
    v = _f64(verts)
    d = v.shape[1]
    det = dbl(0.0)
    inv = np.zeros((d, d))
    fn = lib().orc_affine_map_2d if d == 2 else lib().orc_affine_map_3d
    ok = fn(v.reshape(-1).copy(), C.byref(det), inv.reshape(-1))
    return bool(ok), det.value, inv


def p2_basis(xi) -> np.ndarray:
    out = np.empty(10)
    lib().orc_p2_basis(_f64(xi), out)
    return out


def p2_grads(xi) -> np.ndarray:
    out = np.empty(30)
    lib().orc_p2_grads(_f64(xi), out)
    return out.reshape(10, 3)


# ---------------------------------------------------------------------------
# Reference-level drivers (poisson_solver.rs, elasticity_solver.rs)
# ---------------------------------------------------------------------------

def solve_poisson_2d(m: Mesh, f, g, tol, max_iter):
    A = assemble_stiffness_2d(m)
    b = assemble_rhs_2d(m, f)
    bd = boundary_dofs_2d(m)
    bv = g(m.coords[bd, 0], m.coords[bd, 1])
    Ab, bb = apply_dirichlet_bc(A, b, bd, bv)
    return solve_cg(Ab, bb, None, tol, max_iter)


def solve_poisson_3d(m: Mesh, f, g, tol, max_iter):
    A = assemble_stiffness_3d(m)
    b = assemble_rhs_3d(m, f)
    bd = boundary_dofs_3d(m)
    bv = g(m.coords[bd, 0], m.coords[bd, 1], m.coords[bd, 2])
    Ab, bb = apply_dirichlet_bc(A, b, bd, bv)
    return solve_cg(Ab, bb, None, tol, max_iter)


def clamp_dofs(m: Mesh, x0: float = 1e-6) -> np.ndarray:
    """Clamp set of the reference's elasticity tests (elasticity_tests.rs:22-28):
    all three components of every vertex with x < x0, in vertex order."""
    v = np.nonzero(m.coords[:, 0] < x0)[0]
    return (3 * v[:, None] + np.arange(3)[None, :]).reshape(-1).astype(np.int64)


def solve_elasticity_3d(m: Mesh, E, nu, f_body, dofs, tol, max_iter):
    K = assemble_elasticity_3d(m, E, nu)
    f = body_force_3d(m, f_body)
    Kb, fb = apply_dirichlet_bc(K, f, dofs, np.zeros(len(dofs)))
    return solve_cg(Kb, fb, None, tol, max_iter)


# ---------------------------------------------------------------------------
# Mass matrices, matrix combinations, transient heat, vibration modes
# (mass.rs, transient.rs, heat_solver.rs, direct.rs, eigen.rs)
# ---------------------------------------------------------------------------

def p2_mass_products() -> np.ndarray:
    """build_reference_mass_products_p2 (mass.rs:195-250), 10x10."""
    out = np.empty(100)
    lib().orc_p2_mass_products(out)
    return out.reshape(10, 10)


def _mass(m: Mesh, kind: int, density: float, coef=None, cell_dofs=None, ndofs=None) -> Csc:
    nd = ndofs if ndofs is not None else (3 * m.nv if kind == 2 else m.nv)
    cd = None if cell_dofs is None else _i64(cell_dofs)
    cf = None if coef is None else _f64(coef)
    h = lib().orc_assemble_mass(nd, _f64(m.coords), m.nc, _i64(m.cells), _ptr(cd), kind, float(density), _ptr(cf))
    return _take_csc(h)


def assemble_mass_2d(m: Mesh, coef=None) -> Csc:
    """assemble_mass_2d (mass.rs:10-44)."""
    return _mass(m, 0, 1.0, coef)


def assemble_mass_3d(m: Mesh, coef=None) -> Csc:
    """assemble_mass_3d (mass.rs:47-81)."""
    return _mass(m, 1, 1.0, coef)


def assemble_elasticity_mass_3d(m: Mesh, density: float, coef=None) -> Csc:
    """assemble_elasticity_mass_3d (mass.rs:84-127)."""
    return _mass(m, 2, density, coef)


def assemble_p2_mass_3d(m: Mesh, cell_dofs, ndofs, density: float = 1.0, coef=None) -> Csc:
    """Scalar P2 mass: density |det J| times the reference products
    (one component of assemble_elasticity_mass_p2_3d, mass.rs:137-180)."""
    return _mass(m, 3, density, coef, cell_dofs, ndofs)


def assemble_elasticity_mass_p2_3d(vertices, cells10, density: float) -> Csc:
    """assemble_elasticity_mass_p2_3d (mass.rs:137-180): vertices = every P2
    node, cells10 = ten nodes per cell in P2Tetrahedron order."""
    c10 = _i64(cells10)
    m = Mesh(np.ascontiguousarray(vertices, dtype=np.float64), np.ascontiguousarray(c10[:, :4]))
    return _mass(m, 4, density, None, c10, 3 * m.nv)


def p2_node_mesh(m: Mesh):
    """(vertices, cells10) of the P2 node mesh over a tetrahedron mesh: the
    vertices, then the edge midpoints in this build's edge order."""
    cd, ev = p2_dofmap(m)
    mid = 0.5 * (m.coords[ev[:, 0]] + m.coords[ev[:, 1]])
    return np.concatenate([m.coords, mid]), cd


def _triplets(A: Csc):
    cols = np.repeat(np.arange(A.n, dtype=np.int64), np.diff(A.colptr))
    return A.rowidx.astype(np.int64), cols, A.vals


def add_scaled_matrices(a: Csc, b: Csc, alpha: float) -> Csc:
    """add_scaled_matrices (transient.rs:72-97): per column, a's triplets then
    alpha * b's, summed by the triplet build."""
    ra, ca, va = _triplets(a)
    rb, cb, vb = _triplets(b)
    # interleave per column: all of a's entries of column c, then b's
    key_a = ca * 2
    key_b = cb * 2 + 1
    rows = np.concatenate([ra, rb])
    cols = np.concatenate([ca, cb])
    vals = np.concatenate([va, alpha * vb])
    order = np.argsort(np.concatenate([key_a, key_b]), kind="stable")
    return csc_from_triplets(a.n, rows[order], cols[order], vals[order])


def fold_dirichlet(mat: Csc, fixed_dofs, unit_diag: bool) -> Csc:
    """fold_dirichlet (eigen.rs:55-79)."""
    n = mat.n
    fixed = np.zeros(n, bool)
    fd = np.asarray(fixed_dofs, dtype=np.int64)
    fixed[fd[fd < n]] = True
    rows, cols, vals = _triplets(mat)
    keep = ~(fixed[rows] | fixed[cols] | (vals == 0.0))
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    if unit_diag:
        fc = np.nonzero(fixed)[0]
        # the unit diagonal follows the column's kept entries
        rows = np.concatenate([rows, fc])
        cols = np.concatenate([cols, fc])
        vals = np.concatenate([vals, np.ones(len(fc))])
        order = np.argsort(cols, kind="stable")
        rows, cols, vals = rows[order], cols[order], vals[order]
    return csc_from_triplets(n, rows, cols, vals)


def solve_direct(A: Csc, b) -> np.ndarray:
    """solve_direct (direct.rs:26-53): dense partial-pivoting LU (LAPACK
    gesv through numpy), for systems of a few thousand dofs at most."""
    return np.linalg.solve(A.to_scipy().toarray(), np.asarray(b, dtype=np.float64))


def transient_step(scheme: int, dt: float, mass: Csc, stiff: Csc, u_n, f_n, f_next) -> np.ndarray:
    """TransientHeatSolver::step (transient.rs:32-68); scheme 0 = backward
    Euler, 1 = Crank-Nicolson."""
    u_n = np.asarray(u_n, dtype=np.float64)
    if scheme == 0:
        lhs = add_scaled_matrices(mass, stiff, dt)
        rhs = spmv(mass, u_n) + dt * np.asarray(f_next, dtype=np.float64)
    else:
        half_dt = 0.5 * dt
        lhs = add_scaled_matrices(mass, stiff, half_dt)
        rhs_mat = add_scaled_matrices(mass, stiff, -half_dt)
        rhs = spmv(rhs_mat, u_n) + half_dt * (np.asarray(f_n, dtype=np.float64) + np.asarray(f_next, dtype=np.float64))
    return solve_direct(lhs, rhs)


def solve_transient_heat_2d(m: Mesh, diffusivity, u_initial, bcs, dt, num_steps, scheme, heat_source=None):
    """solve_transient_heat_2d (heat_solver.rs:23-104); bcs: [(dofs, values)].
    Returns (times, history, final)."""
    n = m.nv
    mass = assemble_mass_2d(m)
    k = assemble_stiffness_2d(m)
    stiff = Csc(k.n, k.colptr, k.rowidx, diffusivity * k.vals)
    u = np.asarray(u_initial, dtype=np.float64).copy()
    times, hist = [0.0], [u.copy()]
    for step in range(1, num_steps + 1):
        t0, t1 = (step - 1) * dt, step * dt
        f0 = np.zeros(n) if heat_source is None else np.array([heat_source(t0, m.coords[i]) for i in range(n)])
        f1 = np.zeros(n) if heat_source is None else np.array([heat_source(t1, m.coords[i]) for i in range(n)])
        for dofs, vals in bcs:
            for d, v in zip(dofs, vals):
                u[d] = v
        un = transient_step(scheme, dt, mass, stiff, u, f0, f1)
        for dofs, vals in bcs:
            for d, v in zip(dofs, vals):
                un[d] = v
        u = un
        times.append(t1)
        hist.append(u.copy())
    return times, hist, u


def _mean_abs_diag(A: Csc) -> float:
    acc, found = 0.0, 0
    for c in range(A.n):
        for p in range(A.colptr[c], A.colptr[c + 1]):
            if A.rowidx[p] == c:
                acc += abs(A.vals[p])
                found += 1
                break
    return acc / found if found else 0.0


def solve_vibration_modes_with_inner(k: Csc, m: Csc, fixed_dofs, num_modes, max_power_iters, tol, inner):
    """solve_vibration_modes_with_inner (eigen.rs:94-271). Returns a list of
    (eigenvalue, mode_shape, power_iterations)."""
    kd = fold_dirichlet(k, fixed_dofs, True)
    md = fold_dirichlet(m, fixed_dofs, False)
    n = kd.n
    is_fixed = np.zeros(n, bool)
    fd = np.asarray(fixed_dofs, dtype=np.int64)
    is_fixed[fd[fd < n]] = True
    if n - int(is_fixed.sum()) == 0:
        raise ValueError("No free degrees of freedom in system")
    kdg, mdg = _mean_abs_diag(kd), _mean_abs_diag(md)
    s = kdg / mdg if kdg > 0.0 and mdg > 0.0 else 1.0
    modes, vecs = [], []
    idx = np.arange(n, dtype=np.int64)
    for mode in range(num_modes):
        v = (((idx + 1) * 31 + (mode + 1) * 97) % 1000).astype(np.float64) / 1000.0 - 0.5
        v[is_fixed] = 0.0
        m_prev = [spmv(md, p) * s for p in vecs]
        for mp, prev in zip(m_prev, vecs):
            v = v - float(np.dot(v, mp)) * prev
        mv = spmv(md, v) * s
        norm_m = math.sqrt(float(np.dot(v, mv)))
        if norm_m > 1e-14:
            v = v / norm_m
        prev_r = 0.0
        its = 0
        for it in range(max_power_iters):
            its = it + 1
            mv = spmv(md, v) * s
            w = np.array(inner(kd, mv, v), dtype=np.float64)
            w[is_fixed] = 0.0
            for mp, prev in zip(m_prev, vecs):
                w = w - float(np.dot(w, mp)) * prev
            mw = spmv(md, w)
            mw_norm = math.sqrt(float(np.dot(w, mw))) * math.sqrt(s)
            if mw_norm < 1e-15:
                break
            w = w / mw_norm
            r = float(np.dot(w, spmv(kd, w)))
            v = w
            denom = max(abs(r), abs(prev_r))
            if denom == 0.0 or abs(r - prev_r) / denom < tol:
                break
            prev_r = r
        lam = max(float(np.dot(v, spmv(kd, v))) / float(np.dot(v, spmv(md, v))), 0.0)
        vecs.append(v)
        modes.append((lam, v, its))
    return modes


def solve_vibration_modes(k: Csc, m: Csc, fixed_dofs, num_modes, max_power_iters, tol,
                          inner_tol=1e-9, inner_max_iter=1000):
    """solve_vibration_modes (eigen.rs:286-300): inner solve = solve_cg on
    the folded stiffness from x0 at 1e-9 / 1000 iterations."""
    def inner(kd, b, x0):
        x, _, _ = solve_cg(kd, b, x0, inner_tol, inner_max_iter)
        return x
    return solve_vibration_modes_with_inner(k, m, fixed_dofs, num_modes, max_power_iters, tol, inner)


# ---------------------------------------------------------------------------
# 3x3 block CSR (gpu.rs:434-1141): spmv, block-Jacobi sweeps, block-Jacobi PCG
# ---------------------------------------------------------------------------

def bsr3_spmv(n_nodes, row_ptr, cols, vals_flat, x) -> np.ndarray:
    """y = A x with row-major 3x3 blocks: y[3i+a] = sum_k sum_b V[k][a][b] x[3 cols[k] + b]."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    ci = np.asarray(cols, dtype=np.int64)
    V = np.asarray(vals_flat, dtype=np.float64).reshape(-1, 3, 3)
    X = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    rows = np.repeat(np.arange(n_nodes), np.diff(rp))
    contrib = np.einsum("kab,kb->ka", V, X[ci])
    Y = np.zeros((n_nodes, 3))
    np.add.at(Y, rows, contrib)
    return Y.ravel()


def bsr3_apply_dinv(dinv_flat, r) -> np.ndarray:
    """bsr3_apply_dinv: z = D^-1 r per block row."""
    D = np.asarray(dinv_flat, dtype=np.float64).reshape(-1, 3, 3)
    return np.einsum("kab,kb->ka", D, np.asarray(r, dtype=np.float64).reshape(-1, 3)).ravel()


def bsr3_jacobi_smooth(n_nodes, row_ptr, cols, vals_flat, dinv_flat, r, z, sweeps, omega, zero_initial_z):
    """GpuBsr3Context::jacobi_smooth (gpu.rs:547-657)."""
    z = np.array(z, dtype=np.float64)
    if sweeps == 0:
        return z
    start = 0
    if zero_initial_z:
        z = bsr3_apply_dinv(dinv_flat, r)
        start = 1
    for _ in range(start, sweeps):
        y = bsr3_spmv(n_nodes, row_ptr, cols, vals_flat, z)
        z = z + omega * bsr3_apply_dinv(dinv_flat, np.asarray(r) - y)
    return z


def bsr3_block_inverse(n_nodes, row_ptr, cols, vals_flat) -> np.ndarray:
    """Inverse diagonal blocks (numpy LAPACK inverse) of a block CSR matrix."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    ci = np.asarray(cols, dtype=np.int64)
    V = np.asarray(vals_flat, dtype=np.float64).reshape(-1, 3, 3)
    out = np.empty((n_nodes, 3, 3))
    for i in range(n_nodes):
        k = rp[i] + int(np.nonzero(ci[rp[i]:rp[i + 1]] == i)[0][0])
        out[i] = np.linalg.inv(V[k])
    return out.ravel()


def solve_bsr3_pcg(n_nodes, row_ptr, cols, vals_flat, dinv_flat, b, x0=None, rtol=1e-8, max_iter=1000):
    """solve_bsr3_pcg_gpu (gpu.rs:775-1141): block-Jacobi PCG; returns
    (x, iterations, final relative residual). Ok at the limit, x = 0 for
    b = 0, stop on p.Ap <= 1e-30."""
    b = np.asarray(b, dtype=np.float64)
    n = 3 * n_nodes
    bnorm = math.sqrt(float(np.dot(b, b)))
    if bnorm == 0.0:
        return np.zeros(n), 0, 0.0
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    r = b.copy()
    if x0 is not None:
        r = r - bsr3_spmv(n_nodes, row_ptr, cols, vals_flat, x)
    z = bsr3_apply_dinv(dinv_flat, r)
    p = z.copy()
    rz = float(np.dot(r, z))
    final_rel, iters = 1.0, 0
    for it in range(1, max_iter + 1):
        iters = it
        ap = bsr3_spmv(n_nodes, row_ptr, cols, vals_flat, p)
        pap = float(np.dot(p, ap))
        if pap <= 1e-30:
            break
        alpha = rz / pap
        x = x + alpha * p
        r = r - alpha * ap
        final_rel = math.sqrt(max(float(np.dot(r, r)), 0.0)) / bnorm
        if final_rel < rtol:
            break
        z = bsr3_apply_dinv(dinv_flat, r)
        rz_new = float(np.dot(r, z))
        beta = rz_new / max(rz, 1e-30)
        rz = rz_new
        p = z + beta * p
    return x, iters, final_rel


def bsr3_from_csc(A: Csc):
    """The 3x3 block CSR of a vector matrix given as CSC (dof = 3 node + a):
    block pattern = node pairs with any stored entry."""
    S = A.to_scipy().tocsr()
    B = S.tobsr(blocksize=(3, 3))
    B.sort_indices()
    return (S.shape[0] // 3, B.indptr.astype(np.uint32), B.indices.astype(np.uint32),
            np.ascontiguousarray(B.data).ravel())
