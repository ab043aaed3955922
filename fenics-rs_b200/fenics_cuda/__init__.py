"""fenics_cuda — B200 FEM assembly + Jacobi-PCG behind the fenics-rs interface.

Python mirror of the reference's hot-path API over the C ABI of
``libfenics_cuda.so`` (include/fenics_cuda.h). Function names, argument
meaning and error behaviour follow GlassOnTin/fenics-rs:

  crates/fenics-mesh       unit_square, box_beam, unit_cube  (generators.rs)
  crates/fenics-assembly   assemble_stiffness_2d/3d, assemble_rhs_2d/3d,
                           apply_dirichlet_bc, boundary_dofs_2d/3d,
                           assemble_elasticity_stiffness_3d,
                           assemble_elasticity_body_force_3d,
                           apply_vector_dirichlet_bc, assemble_surface_traction_3d
  crates/fenics-assembly   assemble_mass_2d/3d, assemble_elasticity_mass_3d (mass.rs)
  crates/fenics-solver     solve_cg, solve_csr_cg_gpu, solve_cg_gpu_or_cpu,
                           solve_poisson_2d/3d, solve_elasticity_3d,
                           add_scaled_matrices, TransientHeatSolver,
                           solve_transient_heat_2d, fold_dirichlet,
                           solve_vibration_modes(_with_inner)

All compute runs in CUDA kernels on the device; there is no CPU fallback (a
missing library or device raises). Arrays may be numpy (host), DeviceArray (device memory the library allocates), or torch CUDA
tensors (device); device arrays are used in place.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import (FCU_BACKWARD_EULER, FCU_CRANK_NICOLSON, FCU_FP64, FCU_MIXED, FCU_SPACE_P1, FCU_SPACE_P1_VEC3,
                   FCU_SPACE_P2, FCU_SRC_CONSTANT, FCU_SRC_NODAL, FCU_SRC_SIN_PRODUCT, SolveInfo)

__all__ = [
    "Context", "Mesh", "FunctionSpace", "Matrix", "CscMatrix", "FcuError", "CgError",
    "unit_square", "box_beam", "unit_cube", "default_context",
    "assemble_stiffness_2d", "assemble_stiffness_3d", "assemble_rhs_2d", "assemble_rhs_3d",
    "apply_dirichlet_bc", "boundary_dofs_2d", "boundary_dofs_3d", "DirichletBC",
    "ElasticMaterial", "VectorDirichletBC", "assemble_elasticity_stiffness_3d",
    "assemble_elasticity_body_force_3d", "apply_vector_dirichlet_bc", "assemble_surface_traction_3d",
    "extract_boundary_facets", "solve_cg", "solve_csr_cg_gpu", "solve_cg_gpu_or_cpu", "GpuSolveResult",
    "solve_poisson_2d", "solve_poisson_3d", "solve_elasticity_3d", "spmv",
    "assemble_mass_2d", "assemble_mass_3d", "assemble_elasticity_mass_3d", "assemble_mass_p2_3d",
    "assemble_elasticity_mass_p2_3d",
    "add_scaled_matrices", "TimeSteppingScheme", "TransientHeatSolver", "TransientHeatSolution",
    "solve_transient_heat_2d", "fold_dirichlet", "VibrationMode", "solve_vibration_modes",
    "solve_vibration_modes_with_inner", "GpuBsr3Context", "solve_bsr3_pcg_gpu", "spmv_bsr3_multi_gpu",
    "FCU_FP64", "FCU_MIXED",
]


class FcuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[fcu error {code}] {msg}")
        self.code = code


class CgError(FcuError):
    """Err(String) of solve_cg (cg.rs:102-107, 139-148)."""


def _L():
    return _abi.lib()


# ---------------------------------------------------------------------------
# pointers: numpy (host), DeviceArray or any CUDA tensor with data_ptr() (device)
# ---------------------------------------------------------------------------

def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a, dtype=None):
    """(address, keepalive) of a contiguous array, converting numpy dtypes."""
    if a is None:
        return None, None
    if isinstance(a, DeviceArray):
        if dtype is not None and np.dtype(dtype) != a.dtype:
            raise TypeError(f"device array of {a.dtype} where {np.dtype(dtype)} is expected")
        return a.ptr, a
    if _is_torch(a):
        if not a.is_contiguous():
            raise ValueError("torch tensors must be contiguous")
        return a.data_ptr(), a
    arr = np.ascontiguousarray(a, dtype=dtype) if dtype is not None else np.ascontiguousarray(a)
    return arr.ctypes.data, arr


class DeviceArray:
    """A one-dimensional array in device memory, allocated by the library
    (fcu_buffer_alloc on the context's stream) for callers that have no CUDA
    array type of their own; the mirror of a Rust caller passing memory from
    its own arena. Every function of this module accepts it wherever it
    accepts a host array, and then leaves the data on the device."""

    def __init__(self, ctx: "Context", n: int, dtype=np.float64):
        self.ctx = ctx
        self.dtype = np.dtype(dtype)
        self.n = int(n)
        h = C.c_void_p()
        _check(ctx, _L().fcu_buffer_alloc(ctx.h, self.nbytes, C.byref(h)))
        self.ptr = h.value

    @classmethod
    def from_numpy(cls, ctx: "Context", a, dtype=None) -> "DeviceArray":
        a = np.ascontiguousarray(a, dtype=dtype)
        d = cls(ctx, a.size, a.dtype)
        d.copy_from(a)
        return d

    @property
    def nbytes(self) -> int:
        return self.n * self.dtype.itemsize

    @property
    def shape(self):
        return (self.n,)

    def __len__(self):
        return self.n

    def copy_from(self, a):
        """Copy from a host array or another device array of the same size."""
        if isinstance(a, DeviceArray):
            src, keep = a.ptr, a
        else:
            keep = np.ascontiguousarray(a, dtype=self.dtype)
            src = keep.ctypes.data
        if (keep.nbytes if not isinstance(keep, DeviceArray) else keep.nbytes) != self.nbytes:
            raise ValueError("size mismatch")
        _check(self.ctx, _L().fcu_buffer_copy(self.ctx.h, C.c_void_p(self.ptr), C.c_void_p(src), self.nbytes))
        return self

    def zero_(self):
        _check(self.ctx, _L().fcu_buffer_memset(self.ctx.h, C.c_void_p(self.ptr), 0, self.nbytes))
        return self

    def numpy(self) -> np.ndarray:
        """Host copy (waits for the context's stream)."""
        out = np.empty(self.n, self.dtype)
        _check(self.ctx, _L().fcu_buffer_copy(self.ctx.h, C.c_void_p(out.ctypes.data), C.c_void_p(self.ptr),
                                               self.nbytes))
        return out

    def clone(self) -> "DeviceArray":
        return DeviceArray(self.ctx, self.n, self.dtype).copy_from(self)

    def free(self):
        if self.ptr and self.ctx.h:
            _L().fcu_buffer_free(self.ctx.h, C.c_void_p(self.ptr))
        self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def device_count() -> int:
    n = C.c_int(0)
    rc = _L().fcu_device_count(C.byref(n))
    return n.value if rc == _abi.FCU_OK else 0


def device_name(device: int = 0) -> str:
    buf = C.create_string_buffer(256)
    if _L().fcu_device_name(device, buf, 256) != _abi.FCU_OK:
        return f"cuda:{device}"
    return buf.value.decode()


def _check(ctx: "Context", rc: int):
    if rc != _abi.FCU_OK:
        msg = _L().fcu_last_error(ctx.h if ctx else None)
        msg = msg.decode() if msg else ""
        if rc in (_abi.FCU_ERR_NO_CONVERGENCE, _abi.FCU_ERR_BREAKDOWN):
            raise CgError(rc, msg)
        raise FcuError(rc, msg)


# ---------------------------------------------------------------------------
# context
# ---------------------------------------------------------------------------

class Context:
    """A device, a stream and the library state on them (CudaSession, gpu.rs:325-430)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = _L().fcu_ctx_create(device, C.byref(h))
        if rc != _abi.FCU_OK:
            raise FcuError(rc, (_L().fcu_last_error(None) or b"").decode())
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            _L().fcu_ctx_destroy(self.h)
            self.h = None

    def synchronize(self):
        _check(self, _L().fcu_ctx_synchronize(self.h))

    @property
    def stream(self) -> int:
        return _L().fcu_ctx_stream(self.h) or 0

    @property
    def kernel_launches(self) -> int:
        return _L().fcu_ctx_kernel_launches(self.h)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# ---------------------------------------------------------------------------
# meshes (fenics-mesh)
# ---------------------------------------------------------------------------

class Mesh:
    """SimplicialMesh<DIM, NODES> (mesh.rs:11-20): host vertices and cells, with
    device copies created per context on first use."""

    def __init__(self, coords, cells):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.cells = np.ascontiguousarray(cells, dtype=np.int64)
        if self.coords.ndim != 2 or self.cells.ndim != 2 or self.cells.shape[1] != self.coords.shape[1] + 1:
            raise ValueError("coords must be [nv, dim] and cells [nc, dim+1]")
        self._dev = {}

    @property
    def dim(self) -> int:
        return self.coords.shape[1]

    def num_vertices(self) -> int:
        return self.coords.shape[0]

    def num_cells(self) -> int:
        return self.cells.shape[0]

    nv = property(num_vertices)
    nc = property(num_cells)

    def handle(self, ctx: Context):
        key = id(ctx)
        if key not in self._dev:
            h = C.c_void_p()
            _check(ctx, _L().fcu_mesh_create(ctx.h, self.dim, self.nv, self.coords.ctypes.data, self.nc,
                                             self.cells.ctypes.data, C.byref(h)))
            self._dev[key] = (ctx, h)
        return self._dev[key][1]

    def release(self):
        for ctx, h in self._dev.values():
            _L().fcu_mesh_destroy(h)
        self._dev.clear()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def unit_square(nx: int, ny: int) -> Mesh:
    """generators.rs:24-55: vertices row by row, each square split along v00-v11."""
    if nx <= 0 or ny <= 0:
        raise ValueError("nx and ny must be at least 1")
    j, i = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    coords = np.stack([i.ravel() / nx, j.ravel() / ny], axis=1)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    v00 = (jj * (nx + 1) + ii).ravel()
    v10, v01, v11 = v00 + 1, v00 + nx + 1, v00 + nx + 2
    cells = np.empty((2 * nx * ny, 3), np.int64)
    cells[0::2] = np.stack([v00, v10, v11], 1)
    cells[1::2] = np.stack([v00, v11, v01], 1)
    return Mesh(coords, cells)


def concat_meshes(meshes) -> tuple[Mesh, np.ndarray]:
    """One mesh holding several meshes side by side (vertex ranges disjoint,
    cells renumbered), and the vertex offsets of each: the layout of a batch,
    whose scalar P1 matrix is block diagonal over these offsets."""
    meshes = list(meshes)
    if not meshes:
        raise ValueError("no meshes")
    dims = {m.dim for m in meshes}
    if len(dims) != 1:
        raise ValueError("meshes of one dimension expected")
    nvs = np.array([m.nv for m in meshes], np.int64)
    offs = np.concatenate([[0], np.cumsum(nvs)])
    coords = np.concatenate([m.coords for m in meshes])
    cells = np.concatenate([m.cells + o for m, o in zip(meshes, offs[:-1])])
    return Mesh(coords, cells), offs


def box_beam(length, width, height, nx, ny, nz) -> Mesh:
    """generators.rs:58-111: x fastest, Kuhn split of each hexahedron into 6 tets."""
    if nx <= 0 or ny <= 0 or nz <= 0:
        raise ValueError("nx, ny, and nz must be at least 1")
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    coords = np.stack([(i.ravel() / nx) * length, (j.ravel() / ny) * width, (k.ravel() / nz) * height], axis=1)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    p0 = (kk * sz + jj * sy + ii).ravel()
    p1, p2, p3 = p0 + sx, p0 + sy, p0 + sx + sy
    p4, p5, p6, p7 = p0 + sz, p0 + sz + sx, p0 + sz + sy, p0 + sz + sx + sy
    tets = [(p0, p1, p3, p7), (p0, p3, p2, p7), (p0, p2, p6, p7), (p0, p6, p4, p7), (p0, p4, p5, p7), (p0, p5, p1, p7)]
    cells = np.empty((6 * nx * ny * nz, 4), np.int64)
    for t, tet in enumerate(tets):
        cells[t::6] = np.stack(tet, 1)
    return Mesh(coords, cells)


def unit_cube(nx, ny, nz) -> Mesh:
    return box_beam(1.0, 1.0, 1.0, nx, ny, nz)


def extract_boundary_facets(mesh: Mesh, ctx: Context | None = None):
    """extract_boundary_facets (mesh.rs:79-113, 145-210) on the device.
    Returns (vertices [nf, dim], cell_idx [nf], local_facet_idx [nf]), sorted by
    facet key; 3D facets are oriented outward."""
    ctx = ctx or default_context()
    h = mesh.handle(ctx)
    n = C.c_int64(0)
    _check(ctx, _L().fcu_boundary_facets(ctx.h, h, None, None, None, C.byref(n)))
    v = np.empty((n.value, mesh.dim), np.int64)
    c = np.empty(n.value, np.int64)
    lo = np.empty(n.value, np.int64)
    if n.value:
        _check(ctx, _L().fcu_boundary_facets(ctx.h, h, v.ctypes.data, c.ctypes.data, lo.ctypes.data, C.byref(n)))
    return v, c, lo


# ---------------------------------------------------------------------------
# spaces and matrices
# ---------------------------------------------------------------------------

class FunctionSpace:
    """Dof map + sparsity pattern of P1 / P2 / vector-P1 on a mesh, on the device."""

    def __init__(self, ctx: Context, mesh: Mesh, kind: int, cells10=None):
        self.ctx, self.mesh, self.kind = ctx, mesh, kind
        h = C.c_void_p()
        if kind in (_abi.FCU_SPACE_P2_NODES, _abi.FCU_SPACE_P2_NODES_VEC3):
            pc, kc = _ptr(cells10, np.int64)
            _check(ctx, _L().fcu_space_create_p2_nodes(ctx.h, mesh.handle(ctx), pc,
                                                       1 if kind == _abi.FCU_SPACE_P2_NODES_VEC3 else 0,
                                                       C.byref(h)))
        else:
            _check(ctx, _L().fcu_space_create(ctx.h, mesh.handle(ctx), kind, C.byref(h)))
        self.h = h
        nd, nz, ne = C.c_int64(), C.c_int64(), C.c_int64()
        _L().fcu_space_info(h, C.byref(nd), C.byref(nz), C.byref(ne))
        self.ndofs, self.nnz, self.nedges = nd.value, nz.value, ne.value

    def close(self):
        if getattr(self, "h", None):
            _L().fcu_space_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def boundary_dofs(self) -> np.ndarray:
        n = C.c_int64(0)
        _check(self.ctx, _L().fcu_space_boundary_dofs(self.ctx.h, self.h, None, C.byref(n)))
        out = np.empty(n.value, np.int64)
        if n.value:
            _check(self.ctx, _L().fcu_space_boundary_dofs(self.ctx.h, self.h, out.ctypes.data, C.byref(n)))
        return out

    def p2_dofmap(self):
        cd = np.empty((self.mesh.nc, 10), np.int64)
        ev = np.empty((self.nedges, 2), np.int64)
        _check(self.ctx, _L().fcu_space_p2_dofmap(self.ctx.h, self.h, cd.ctypes.data, ev.ctypes.data))
        return cd, ev

    def quadrature_points(self) -> np.ndarray:
        nq = 3 if self.mesh.dim == 2 else 4
        out = np.empty((self.mesh.nc * nq, self.mesh.dim))
        _check(self.ctx, _L().fcu_quadrature_points(self.ctx.h, self.h, out.ctypes.data))
        return out

    def rhs_values(self, fq, out=None):
        out = np.empty(self.ndofs) if out is None else out
        pf, kf = _ptr(fq, np.float64)
        pb, kb = _ptr(out)
        _check(self.ctx, _L().fcu_assemble_rhs_values(self.ctx.h, self.h, pf, pb))
        return out

    def rhs_source(self, kind, params=(), nodal=None, out=None):
        out = np.empty(self.ndofs) if out is None else out
        par = np.ascontiguousarray(list(params) + [0.0, 0.0], dtype=np.float64)
        pn, kn = _ptr(nodal, np.float64)
        pb, kb = _ptr(out)
        _check(self.ctx, _L().fcu_assemble_rhs_source(self.ctx.h, self.h, kind, par.ctypes.data, pn, pb))
        return out

    def body_force(self, f_body, out=None):
        out = np.empty(self.ndofs) if out is None else out
        f = np.ascontiguousarray(f_body, dtype=np.float64)
        pb, kb = _ptr(out)
        _check(self.ctx, _L().fcu_assemble_body_force(self.ctx.h, self.h, f.ctypes.data, pb))
        return out

    def surface_traction(self, facets, tq, out=None):
        out = np.empty(self.ndofs) if out is None else out
        pf, kf = _ptr(facets, np.int64)
        pt, kt = _ptr(tq, np.float64)
        pb, kb = _ptr(out)
        nf = len(facets)
        _check(self.ctx, _L().fcu_assemble_surface_traction(self.ctx.h, self.h, nf, pf, pt, pb))
        return out

    def element_stresses(self, E, nu, u, stress=None, strain=None, von_mises=None, trace=None):
        """Per-cell stress, strain (nc x 9), von Mises stress and trace (nc) into
        the given outputs (numpy or CUDA tensors; None skips an output)."""
        pu, ku = _ptr(u, np.float64)
        ps, ks = _ptr(stress)
        pe, ke = _ptr(strain)
        pv, kv = _ptr(von_mises)
        pt, kt = _ptr(trace)
        _check(self.ctx, _L().fcu_element_stresses(self.ctx.h, self.h, float(E), float(nu), pu, ps, pe, pv, pt))

    def vertex_von_mises(self, cell_von_mises, out=None):
        out = np.empty(self.mesh.nv) if out is None else out
        pc, kc = _ptr(cell_von_mises, np.float64)
        po, ko = _ptr(out)
        _check(self.ctx, _L().fcu_vertex_von_mises(self.ctx.h, self.h, pc, po))
        return out

    def adjoint_gradient(self, E0, nu, theta, u, lam, out=None):
        out = np.empty(self.mesh.nc) if out is None else out
        pt, kt = _ptr(theta, np.float64)
        pu, ku = _ptr(u, np.float64)
        pl, kl = _ptr(lam, np.float64)
        pg, kg = _ptr(out)
        _check(self.ctx, _L().fcu_adjoint_gradient(self.ctx.h, self.h, E0, nu, pt, pu, pl, pg))
        return out


@dataclass
class CscMatrix:
    """faer SparseColMat<usize, f64> as exported: column pointers, row indices
    sorted inside each column, explicit zeros kept."""
    n: int
    colptr: np.ndarray
    rowidx: np.ndarray
    vals: np.ndarray
    _device: object = field(default=None, repr=False, compare=False)

    def nrows(self) -> int:
        return self.n

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self.vals, self.rowidx, self.colptr), shape=(self.n, self.n))


class Matrix:
    """A matrix on the device: FP64 values and their FP32 copy on a space's
    pattern, or a wrapped caller CSC."""

    def __init__(self, ctx: Context, space: FunctionSpace | None = None, h=None):
        self.ctx, self.space = ctx, space
        if h is None:
            h = C.c_void_p()
            _check(ctx, _L().fcu_matrix_create(ctx.h, space.h, C.byref(h)))
        self.h = h
        n = C.c_int64()
        _L().fcu_matrix_info(h, C.byref(n), None)
        self.n = n.value

    @classmethod
    def from_csc(cls, ctx: Context, A: CscMatrix) -> "Matrix":
        h = C.c_void_p()
        cp, kc = _ptr(A.colptr, np.int64)
        ri, kr = _ptr(A.rowidx, np.int64)
        va, kv = _ptr(A.vals, np.float64)
        _check(ctx, _L().fcu_matrix_from_csc(ctx.h, A.n, cp, ri, va, C.byref(h)))
        return cls(ctx, None, h)

    def close(self):
        if getattr(self, "h", None):
            _L().fcu_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nnz(self) -> int:
        z = C.c_int64()
        _check(self.ctx, _L().fcu_matrix_info(self.h, None, C.byref(z)))
        return z.value

    def assemble_stiffness(self, coef=None):
        pc, kc = _ptr(coef, np.float64)
        _check(self.ctx, _L().fcu_assemble_stiffness(self.ctx.h, self.h, pc))
        return self

    def assemble_elasticity(self, E, nu, cell_E=None):
        pc, kc = _ptr(cell_E, np.float64)
        _check(self.ctx, _L().fcu_assemble_elasticity(self.ctx.h, self.h, float(E), float(nu), pc))
        return self

    def assemble_mass(self, rho=1.0, coef=None):
        """Mass matrix (mass.rs:10-250): rho = density of the vector space,
        1 for the scalar reference matrices; coef multiplies per cell."""
        pc, kc = _ptr(coef, np.float64)
        _check(self.ctx, _L().fcu_assemble_mass(self.ctx.h, self.h, float(rho), pc))
        return self

    def clone(self) -> "Matrix":
        h = C.c_void_p()
        _check(self.ctx, _L().fcu_matrix_clone(self.ctx.h, self.h, C.byref(h)))
        return Matrix(self.ctx, self.space, h)

    def set_add_scaled(self, a: "Matrix", b: "Matrix", alpha):
        """self = a + alpha * b on one pattern (add_scaled_matrices, transient.rs:72-97)."""
        _check(self.ctx, _L().fcu_matrix_add_scaled(self.ctx.h, self.h, a.h, b.h, float(alpha)))
        return self

    @classmethod
    def add_scaled_union(cls, a: "Matrix", b: "Matrix", alpha) -> "Matrix":
        """A new wrapped CSC matrix a + alpha * b on the union of the two
        exported patterns (add_scaled_matrices, transient.rs:72-97)."""
        h = C.c_void_p()
        _check(a.ctx, _L().fcu_matrix_add_scaled_union(a.ctx.h, a.h, b.h, float(alpha), C.byref(h)))
        return cls(a.ctx, None, h)

    def scale(self, s):
        _check(self.ctx, _L().fcu_matrix_scale(self.ctx.h, self.h, float(s)))
        return self

    def fold_dirichlet(self, fixed_dofs, unit_diag: bool):
        """fold_dirichlet (eigen.rs:55-79), in place."""
        pd, kd = _ptr(fixed_dofs, np.int64)
        _check(self.ctx, _L().fcu_matrix_fold_dirichlet(self.ctx.h, self.h, len(fixed_dofs), pd, 1 if unit_diag else 0))
        return self

    @classmethod
    def from_bsr3(cls, ctx: Context, n_nodes, row_ptr, cols, vals_flat, dinv_flat=None) -> "Matrix":
        """A resident 3x3 block CSR matrix (GpuBsr3Context::new, gpu.rs:453-494)."""
        h = C.c_void_p()
        pr, kr = _ptr(row_ptr, np.uint32)
        pc, kc = _ptr(cols, np.uint32)
        pv, kv = _ptr(vals_flat, np.float64)
        pd, kd = _ptr(dinv_flat, np.float64)
        _check(ctx, _L().fcu_bsr3_create(ctx.h, int(n_nodes), pr, pc, pv, pd, C.byref(h)))
        return cls(ctx, None, h)

    def block_jacobi(self, enable=True):
        """Block-Jacobi preconditioning from the 3x3 diagonal blocks (FP64 PCG)."""
        _check(self.ctx, _L().fcu_matrix_block_jacobi(self.ctx.h, self.h, 1 if enable else 0))
        return self

    def export_bsr3(self, with_dinv=False):
        """(row_ptr u32, cols u32, vals_flat, dinv_flat or None): the reference's
        block CSR inputs of solve_bsr3_pcg_gpu."""
        nn = self.n // 3
        rp = np.empty(nn + 1, np.uint32)
        _check(self.ctx, _L().fcu_matrix_export_bsr3(self.ctx.h, self.h, rp.ctypes.data, None, None, None))
        nb = int(rp[-1])
        ci = np.empty(nb, np.uint32)
        va = np.empty(9 * nb)
        di = np.empty(9 * nn) if with_dinv else None
        _check(self.ctx, _L().fcu_matrix_export_bsr3(self.ctx.h, self.h, None, ci.ctypes.data, va.ctypes.data,
                                                     di.ctypes.data if di is not None else None))
        return rp, ci, va, di

    def apply_dirichlet(self, b, dofs, vals):
        """In place on the matrix and b (numpy array or CUDA tensor)."""
        pb, kb = _ptr(b)
        pd, kd = _ptr(dofs, np.int64)
        pv, kv = _ptr(vals, np.float64)
        _check(self.ctx, _L().fcu_apply_dirichlet(self.ctx.h, self.h, pb, len(dofs), pd, pv))
        return b

    def export_csc(self) -> CscMatrix:
        nnz = self.nnz
        cp = np.empty(self.n + 1, np.int64)
        ri = np.empty(nnz, np.int64)
        va = np.empty(nnz, np.float64)
        _check(self.ctx, _L().fcu_matrix_export_csc(self.ctx.h, self.h, cp.ctypes.data, ri.ctypes.data,
                                                    va.ctypes.data))
        return CscMatrix(self.n, cp, ri, va)

    def spmv(self, x, y=None):
        y = np.empty(self.n) if y is None else y
        px, kx = _ptr(x, np.float64)
        py, ky = _ptr(y)
        _check(self.ctx, _L().fcu_spmv(self.ctx.h, self.h, px, py))
        return y

    def time_spmv(self, precision=FCU_FP64, reps=20, cold=False, flush_bytes=0):
        """(ms per launch, algorithmic bytes per launch) of the PCG SpMV kernel:
        the mean of `reps` back-to-back launches, or with cold=True the mean
        of `reps` single launches each after an L2 flush of `flush_bytes`
        (0: 256 MiB)."""
        ms, by = C.c_double(), C.c_double()
        if cold:
            rc = _L().fcu_time_spmv_cold(self.ctx.h, self.h, precision, reps, flush_bytes, C.byref(ms), C.byref(by))
        else:
            rc = _L().fcu_time_spmv(self.ctx.h, self.h, precision, reps, C.byref(ms), C.byref(by))
        _check(self.ctx, rc)
        return ms.value, by.value

    def time_pcg(self, precision=FCU_MIXED, iterations=200, reps=3, flush_bytes=0):
        """(ms per launch, algorithmic bytes per launch) of the persistent PCG
        loop running exactly `iterations` iterations from x = 0 on b = 1, the
        mean of `reps` launches each after an L2 flush. Overwrites the solver's
        work vectors."""
        ms, by = C.c_double(), C.c_double()
        rc = _L().fcu_time_pcg(self.ctx.h, self.h, precision, int(iterations), reps, flush_bytes, C.byref(ms),
                               C.byref(by))
        _check(self.ctx, rc)
        return ms.value, by.value

    def pcg(self, b, x=None, x0=None, tol=1e-8, max_iter=10000, precision=FCU_FP64, raise_on_error=True):
        """Jacobi-PCG (cg.rs:40-149). Returns (x, SolveInfo)."""
        x = np.empty(self.n) if x is None else x
        pb, kb = _ptr(b, np.float64)
        p0, k0 = _ptr(x0, np.float64)
        px, kx = _ptr(x)
        info = SolveInfo()
        rc = _L().fcu_pcg(self.ctx.h, self.h, pb, p0, px, float(tol), int(max_iter), precision, C.byref(info))
        if raise_on_error:
            _check(self.ctx, rc)
        return x, info

    def batch_pcg(self, offsets, b, x=None, tol=1e-8, max_iter=10000, precision=FCU_MIXED, raise_on_error=True):
        """Batched Jacobi-PCG over the diagonal blocks [offsets[i], offsets[i+1])
        of this matrix, each solved from zero to its own tolerance in one
        persistent launch. Returns (x, iterations, rel_residual, status, SolveInfo)."""
        offs = np.ascontiguousarray(offsets, dtype=np.int64)
        nb = len(offs) - 1
        x = np.empty(self.n) if x is None else x
        pb, kb = _ptr(b, np.float64)
        px, kx = _ptr(x)
        it = np.zeros(nb, np.int64)
        rel = np.zeros(nb)
        st = np.zeros(nb, np.int32)
        info = SolveInfo()
        rc = _L().fcu_batch_pcg(self.ctx.h, self.h, nb, offs.ctypes.data, pb, px, float(tol), int(max_iter),
                                precision, it.ctypes.data, rel.ctypes.data, st.ctypes.data, C.byref(info))
        if raise_on_error:
            _check(self.ctx, rc)
        return x, it, rel, st, info

    def batch_config(self, precision=FCU_MIXED):
        """(lanes per row, threads per CTA, CTAs per instance) the batched solver
        tuned for this matrix."""
        v, t, c = C.c_int(), C.c_int(), C.c_int()
        _L().fcu_batch_config(self.h, precision, C.byref(v), C.byref(t), C.byref(c))
        return v.value, t.value, c.value


# ---------------------------------------------------------------------------
# fenics-assembly mirror
# ---------------------------------------------------------------------------

def _assembled(kind, mesh, ctx, fill) -> CscMatrix:
    ctx = ctx or default_context()
    V = FunctionSpace(ctx, mesh, kind)
    M = Matrix(ctx, V)
    fill(M)
    A = M.export_csc()
    M.close()
    V.close()
    return A


def assemble_stiffness_2d(mesh: Mesh, ctx: Context | None = None, kappa=None) -> CscMatrix:
    """assemble_stiffness_2d (poisson.rs:23-69)."""
    if mesh.dim != 2:
        raise ValueError("triangle mesh expected")
    return _assembled(FCU_SPACE_P1, mesh, ctx, lambda M: M.assemble_stiffness(kappa))


def assemble_stiffness_3d(mesh: Mesh, ctx: Context | None = None, kappa=None) -> CscMatrix:
    """assemble_stiffness_3d (poisson.rs:124-165)."""
    if mesh.dim != 3:
        raise ValueError("tetrahedron mesh expected")
    return _assembled(FCU_SPACE_P1, mesh, ctx, lambda M: M.assemble_stiffness(kappa))


def _rhs(mesh: Mesh, f, ctx):
    ctx = ctx or default_context()
    V = FunctionSpace(ctx, mesh, FCU_SPACE_P1)
    q = V.quadrature_points()
    fq = np.asarray(f(*[q[:, d] for d in range(mesh.dim)]), dtype=np.float64)
    fq = np.broadcast_to(fq, (len(q),)).copy()
    return V.rhs_values(fq)


def assemble_rhs_2d(mesh: Mesh, f, ctx: Context | None = None) -> np.ndarray:
    """assemble_rhs_2d (poisson.rs:72-121); f is evaluated (vectorised) at the
    rule's physical points, as the reference evaluates its closure there."""
    return _rhs(mesh, f, ctx)


def assemble_rhs_3d(mesh: Mesh, f, ctx: Context | None = None) -> np.ndarray:
    """assemble_rhs_3d (poisson.rs:168-218)."""
    return _rhs(mesh, f, ctx)


@dataclass
class DirichletBC:
    """poisson.rs:15-20"""
    dofs: np.ndarray
    values: np.ndarray


def _apply_bc(mat: CscMatrix, rhs, dofs, vals, ctx):
    ctx = ctx or default_context()
    M = Matrix.from_csc(ctx, mat)
    b = np.array(rhs, dtype=np.float64, copy=True)
    M.apply_dirichlet(b, np.asarray(dofs, np.int64), np.asarray(vals, np.float64))
    A = M.export_csc()
    M.close()
    return A, b


def apply_dirichlet_bc(mat: CscMatrix, rhs, bc: DirichletBC, ctx: Context | None = None):
    """apply_dirichlet_bc (poisson.rs:222-263) -> (matrix, rhs)."""
    return _apply_bc(mat, rhs, bc.dofs, bc.values, ctx)


def boundary_dofs_2d(mesh: Mesh, ctx: Context | None = None) -> np.ndarray:
    """boundary_dofs_2d (poisson.rs:266-275): sorted, unique."""
    return _boundary_dofs(mesh, ctx)


def boundary_dofs_3d(mesh: Mesh, ctx: Context | None = None) -> np.ndarray:
    """boundary_dofs_3d (poisson.rs:278-287)."""
    return _boundary_dofs(mesh, ctx)


def _boundary_dofs(mesh: Mesh, ctx):
    ctx = ctx or default_context()
    h = mesh.handle(ctx)
    n = C.c_int64(0)
    _check(ctx, _L().fcu_boundary_dofs(ctx.h, h, None, C.byref(n)))
    out = np.empty(n.value, np.int64)
    if n.value:
        _check(ctx, _L().fcu_boundary_dofs(ctx.h, h, out.ctypes.data, C.byref(n)))
    return out


@dataclass
class ElasticMaterial:
    """elasticity.rs:14-48"""
    youngs_modulus: float
    poissons_ratio: float

    def __post_init__(self):
        if not (-1.0 < self.poissons_ratio < 0.5):
            raise ValueError("Poisson's ratio must be in (-1.0, 0.5) for physical stability")

    def lame_lambda(self) -> float:
        e, nu = self.youngs_modulus, self.poissons_ratio
        return (e * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu))

    def lame_mu(self) -> float:
        return self.youngs_modulus / (2.0 * (1.0 + self.poissons_ratio))


@dataclass
class VectorDirichletBC:
    """elasticity.rs:65-69: list of (dof, value)."""
    prescribed_dofs: list

    def arrays(self):
        if len(self.prescribed_dofs) == 0:
            return np.empty(0, np.int64), np.empty(0)
        d, v = zip(*self.prescribed_dofs)
        return np.asarray(d, np.int64), np.asarray(v, np.float64)


def assemble_elasticity_stiffness_3d(mesh: Mesh, material: ElasticMaterial, ctx: Context | None = None,
                                     cell_E=None) -> CscMatrix:
    """assemble_elasticity_stiffness_3d (elasticity.rs:73-149)."""
    return _assembled(FCU_SPACE_P1_VEC3, mesh, ctx,
                      lambda M: M.assemble_elasticity(material.youngs_modulus, material.poissons_ratio, cell_E))


def assemble_elasticity_body_force_3d(mesh: Mesh, f_body, ctx: Context | None = None) -> np.ndarray:
    """assemble_elasticity_body_force_3d (elasticity.rs:153-185)."""
    ctx = ctx or default_context()
    return FunctionSpace(ctx, mesh, FCU_SPACE_P1_VEC3).body_force(f_body)


def apply_vector_dirichlet_bc(mat: CscMatrix, rhs, bc: VectorDirichletBC, ctx: Context | None = None):
    """apply_vector_dirichlet_bc (elasticity.rs:188-227) -> (matrix, rhs)."""
    d, v = bc.arrays()
    return _apply_bc(mat, rhs, d, v, ctx)


def assemble_surface_traction_3d(mesh: Mesh, facets, traction_fn, ctx: Context | None = None) -> np.ndarray:
    """assemble_surface_traction_3d (boundary.rs:48-108). `facets` is an [nf, 3]
    vertex array (e.g. from extract_boundary_facets); traction_fn(x, y, z) is
    evaluated (vectorised) at each facet's three edge midpoints."""
    ctx = ctx or default_context()
    fa = np.ascontiguousarray(facets, dtype=np.int64).reshape(-1, 3)
    X = mesh.coords
    p0, p1, p2 = X[fa[:, 0]], X[fa[:, 1]], X[fa[:, 2]]
    mids = np.stack([0.5 * (p0 + p1), 0.5 * (p1 + p2), 0.5 * (p2 + p0)], axis=1).reshape(-1, 3)
    t = traction_fn(mids[:, 0], mids[:, 1], mids[:, 2])
    tq = np.stack(np.broadcast_arrays(*t), axis=1).astype(np.float64)
    return FunctionSpace(ctx, mesh, FCU_SPACE_P1_VEC3).surface_traction(fa, tq)


# ---------------------------------------------------------------------------
# fenics-solver mirror
# ---------------------------------------------------------------------------

def solve_cg(mat, b, x0=None, tol=1e-10, max_iter=1000, ctx: Context | None = None, precision=FCU_FP64):
    """solve_cg (cg.rs:40-149) -> (x, iterations, absolute residual); raises
    CgError on breakdown or non-convergence like the reference's Err."""
    ctx = ctx or default_context()
    M = mat if isinstance(mat, Matrix) else Matrix.from_csc(ctx, mat)
    try:
        x, info = M.pcg(b, x0=x0, tol=tol, max_iter=max_iter, precision=precision)
    finally:
        if M is not mat:
            M.close()
    return x, info.iterations, info.residual


def spmv(mat: CscMatrix, x, ctx: Context | None = None) -> np.ndarray:
    """spmv (cg.rs:7-23)."""
    ctx = ctx or default_context()
    M = Matrix.from_csc(ctx, mat)
    y = M.spmv(x)
    M.close()
    return y


@dataclass
class GpuSolveResult:
    """gpu.rs:24-34"""
    solution: np.ndarray
    iterations: int
    final_residual: float
    wall_ms: float
    kernel_ms: float
    gflops: float
    effective_bw_gbps: float
    devices_used: list


def solve_csr_cg_gpu(row_ptr, col_idx, vals, inv_diag, b, x0=None, rtol=1e-8, max_iter=1000,
                     device_index: int | None = None) -> GpuSolveResult:
    """solve_csr_cg_gpu (gpu.rs:1145-1442): u32 CSR, caller inverse diagonal,
    relative residual, Ok even when the iteration limit is hit."""
    import time
    t0 = time.perf_counter()
    ctx = default_context() if device_index in (None, 0) else Context(device_index)
    n = len(b)
    rp, k1 = _ptr(row_ptr, np.uint32)
    ci, k2 = _ptr(col_idx, np.uint32)
    va, k3 = _ptr(vals, np.float64)
    idg, k4 = _ptr(inv_diag, np.float64)
    bb, k5 = _ptr(b, np.float64)
    xx0, k6 = _ptr(x0, np.float64)
    x = np.empty(n)
    info = SolveInfo()
    _check(ctx, _L().fcu_solve_csr_cg(ctx.h, n, rp, ci, va, idg, bb, xx0, float(rtol), int(max_iter),
                                      x.ctypes.data, C.byref(info)))
    nnz = len(col_idx)
    secs = max(info.kernel_ms / 1e3, 1e-9)
    flops = (2.0 * nnz + 12.0 * n) * info.iterations
    return GpuSolveResult(x, info.iterations, info.rel_residual, (time.perf_counter() - t0) * 1e3,
                          info.kernel_ms, flops / secs / 1e9, info.effective_bw_gbps, [f"cuda:{ctx.device}"])


def solve_cg_gpu_or_cpu(mat: CscMatrix, b, x0=None, tol=1e-10, max_iter=1000) -> GpuSolveResult:
    """solve_cg_gpu_or_cpu (gpu.rs:1542-1602) without the CPU branch: the solve
    runs on the device or raises."""
    import time
    t0 = time.perf_counter()
    ctx = default_context()
    M = Matrix.from_csc(ctx, mat)
    x, info = M.pcg(b, x0=x0, tol=tol, max_iter=max_iter)
    M.close()
    return GpuSolveResult(x, info.iterations, info.rel_residual, (time.perf_counter() - t0) * 1e3,
                          info.kernel_ms, 0.0, info.effective_bw_gbps, [f"cuda:{ctx.device}"])


@dataclass
class PoissonSolution:
    """poisson_solver.rs:16-23"""
    u: np.ndarray
    iterations: int
    residual: float


def _device_vector(ctx: Context, n: int):
    """A device vector for the drivers: the load vector and the solution stay
    on the device from assembly to the end of the solve. It is allocated on
    the context's stream, the stream the library's kernels use it on."""
    return DeviceArray(ctx, n)


def _solve_poisson(mesh: Mesh, source, boundary_value, tol, max_iter, ctx, precision):
    ctx = ctx or default_context()
    V = FunctionSpace(ctx, mesh, FCU_SPACE_P1)
    M = Matrix(ctx, V).assemble_stiffness()
    q = V.quadrature_points()
    fq = np.broadcast_to(np.asarray(source(*[q[:, d] for d in range(mesh.dim)]), np.float64), (len(q),)).copy()
    b = V.rhs_values(fq, out=_device_vector(ctx, V.ndofs))
    bd = V.boundary_dofs()
    bv = np.broadcast_to(np.asarray(boundary_value(*[mesh.coords[bd, d] for d in range(mesh.dim)]),
                                    np.float64), (len(bd),)).copy()
    M.apply_dirichlet(b, bd, bv)
    x, info = M.pcg(b, x=_device_vector(ctx, V.ndofs), tol=tol, max_iter=max_iter, precision=precision)
    return PoissonSolution(x.numpy(), info.iterations, info.residual)


def solve_poisson_2d(mesh: Mesh, source, boundary_value, tol, max_iter, ctx=None, precision=FCU_FP64):
    """solve_poisson_2d (poisson_solver.rs:26-59), device-resident end to end."""
    return _solve_poisson(mesh, source, boundary_value, tol, max_iter, ctx, precision)


def solve_poisson_3d(mesh: Mesh, source, boundary_value, tol, max_iter, ctx=None, precision=FCU_FP64):
    """solve_poisson_3d (poisson_solver.rs:99-132)."""
    return _solve_poisson(mesh, source, boundary_value, tol, max_iter, ctx, precision)


def facets_on_plane(mesh: Mesh, axis: int, value: float, ctx: Context | None = None, eps: float = 1e-9):
    """Boundary facets (vertex triples, outward) whose vertices all lie on the
    plane x[axis] = value, from extract_boundary_facets."""
    verts, _, _ = extract_boundary_facets(mesh, ctx)
    on = np.all(np.abs(mesh.coords[verts][..., axis] - value) < eps, axis=1)
    return verts[on]


def traction_load(V, facets, traction) -> np.ndarray:
    """assemble_surface_traction_3d (boundary.rs:48-108) for a constant traction."""
    t = np.asarray(traction, np.float64)
    tq = np.broadcast_to(t, (len(facets), 3, 3)).copy()
    return V.surface_traction(np.ascontiguousarray(facets, np.int64), tq)


class ElasticityAdjoint:
    """Forward/backward pair for an objective J(u(theta)) of linear elasticity
    with per-cell modulus E_e = E0 * theta_e^3: K(theta) u = f with the clamped
    dofs eliminated. It plays the role of a torch.autograd.Function:

      forward(theta)  assembles K(theta), solves for u and returns J;
      backward(dJ)    returns dJ * dJ/dtheta, where dJ/dtheta_e =
                      -lambda_e^T (3 theta_e^2 E0 K_e^1) u_e, K lambda = dJ/du
                      solved by the same PCG on the same operator (for the
                      compliance J = f^T u, lambda = u and no second solve),
                      and the unit-modulus element matrices K_e^1 are
                      recomputed per cell by the gradient kernel.

    objective: "compliance", or a vector c for J = c^T u (e.g. a mean of
    displacement components)."""

    def __init__(self, mesh: Mesh, nu, load, clamp_dofs, objective="compliance", ctx=None, E0=1.0, tol=1e-10,
                 max_iter=100000, precision=FCU_FP64):
        self.ctx = ctx or default_context()
        self.mesh, self.nu, self.E0 = mesh, float(nu), float(E0)
        self.V = FunctionSpace(self.ctx, mesh, FCU_SPACE_P1_VEC3)
        self.M = Matrix(self.ctx, self.V)
        self.f = np.ascontiguousarray(load, np.float64)
        self.dofs = np.ascontiguousarray(clamp_dofs, np.int64)
        self.objective = objective
        self.tol, self.max_iter, self.precision = tol, max_iter, precision
        self.theta = self.u = None
        self.info = self.adjoint_info = None

    def _solve(self, rhs):
        b = rhs.copy()
        b[self.dofs] = 0.0   # the eliminated system's right-hand side (g = 0)
        x, info = self.M.pcg(b, tol=self.tol, max_iter=self.max_iter, precision=self.precision)
        return x, info

    def forward(self, theta) -> float:
        self.theta = np.ascontiguousarray(theta, np.float64)
        if self.theta.shape != (self.mesh.nc,):
            raise ValueError("one theta per cell expected")
        self.M.assemble_elasticity(self.E0, self.nu, self.E0 * self.theta ** 3)
        b = self.f.copy()
        self.M.apply_dirichlet(b, self.dofs, np.zeros(len(self.dofs)))
        self.u, self.info = self.M.pcg(b, tol=self.tol, max_iter=self.max_iter, precision=self.precision)
        c = self.f if isinstance(self.objective, str) else self.objective
        return float(np.dot(c, self.u))

    def backward(self, dJ=1.0) -> np.ndarray:
        if self.u is None:
            raise RuntimeError("forward first")
        if isinstance(self.objective, str):
            lam = self.u
        else:
            lam, self.adjoint_info = self._solve(np.ascontiguousarray(self.objective, np.float64))
        return dJ * self.V.adjoint_gradient(self.E0, self.nu, self.theta, self.u, lam)

    def close(self):
        self.M.close()
        self.V.close()


@dataclass
class BatchSolution:
    """Per-instance results of a batched solve."""
    solutions: list
    iterations: np.ndarray
    rel_residuals: np.ndarray
    statuses: np.ndarray
    info: SolveInfo
    offsets: np.ndarray


def solve_poisson_batch(meshes, kappas=None, nodal_sources=None, tol=1e-8, max_iter=100000, ctx=None,
                        precision=FCU_MIXED, raise_on_error=True) -> BatchSolution:
    """Independent P1 Poisson problems -div(kappa_e grad u) = f, u = 0 on each
    mesh's boundary, assembled as one block-diagonal system and solved by the
    batched PCG (each instance to its own relative tolerance). kappas: per-cell
    coefficients per mesh (None = 1); nodal_sources: nodal f per mesh, loaded as
    the integral of (sum_j f_j phi_j) phi_i (None = 1)."""
    ctx = ctx or default_context()
    meshes = list(meshes)
    mesh, offs = concat_meshes(meshes)
    V = FunctionSpace(ctx, mesh, FCU_SPACE_P1)
    kappa = None if kappas is None else np.concatenate([np.asarray(k, np.float64) for k in kappas])
    M = Matrix(ctx, V).assemble_stiffness(kappa)
    f = np.ones(mesh.nv) if nodal_sources is None else np.concatenate([np.asarray(v, np.float64)
                                                                      for v in nodal_sources])
    b = V.rhs_source(FCU_SRC_NODAL, nodal=f)
    bd = V.boundary_dofs()
    M.apply_dirichlet(b, bd, np.zeros(len(bd)))
    x, it, rel, st, info = M.batch_pcg(offs, b, tol=tol, max_iter=max_iter, precision=precision,
                                       raise_on_error=raise_on_error)
    M.close()
    V.close()
    return BatchSolution([x[offs[i]:offs[i + 1]] for i in range(len(meshes))], it, rel, st, info, offs)


@dataclass
class StressStates:
    """StressState of every cell (elasticity.rs:230-320), as arrays."""
    stress: np.ndarray     # [nc, 3, 3]
    strain: np.ndarray     # [nc, 3, 3]
    von_mises: np.ndarray  # [nc]
    trace: np.ndarray      # [nc]


def compute_element_stresses(mesh: Mesh, u, material: ElasticMaterial, ctx: Context | None = None) -> StressStates:
    """compute_element_stresses (elasticity.rs:230-320) on the device."""
    ctx = ctx or default_context()
    V = FunctionSpace(ctx, mesh, FCU_SPACE_P1_VEC3)
    nc = mesh.nc
    st, ep = np.empty((nc, 3, 3)), np.empty((nc, 3, 3))
    vm, tr = np.empty(nc), np.empty(nc)
    V.element_stresses(material.youngs_modulus, material.poissons_ratio, np.ascontiguousarray(u, np.float64),
                       st, ep, vm, tr)
    V.close()
    return StressStates(st, ep, vm, tr)


def compute_vertex_von_mises(mesh: Mesh, element_stresses: StressStates, ctx: Context | None = None) -> np.ndarray:
    """compute_vertex_von_mises (elasticity.rs:323-360): volume-weighted vertex
    average of the cells' von Mises stress."""
    ctx = ctx or default_context()
    V = FunctionSpace(ctx, mesh, FCU_SPACE_P1_VEC3)
    out = V.vertex_von_mises(np.ascontiguousarray(element_stresses.von_mises, np.float64))
    V.close()
    return out


def batch_costs(meshes) -> np.ndarray:
    """Estimated solve cost of each instance: (cells + vertices) * sqrt(vertices),
    i.e. work per iteration times the iteration growth of 2D Poisson."""
    return np.array([(m.nc + m.nv) * np.sqrt(max(m.nv, 1)) for m in meshes], np.float64)


def shard_instances(costs, world: int) -> list:
    """Split instances over `world` ranks, largest first onto the least loaded
    rank (ties to the lower rank). Deterministic, so every rank computes the
    same assignment without communicating. Returns one ascending index list
    per rank."""
    if world < 1:
        raise ValueError("world must be at least 1")
    costs = np.asarray(costs, np.float64)
    load = np.zeros(world)
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = int(np.argmin(load))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(sh) for sh in shards]


def solve_poisson_batch_sharded(meshes, kappas=None, nodal_sources=None, tol=1e-8, max_iter=100000, ctx=None,
                                precision=FCU_MIXED, rank=0, world=1, group=None, solve=None, all_gather=None):
    """The batch split over ranks (one GPU each): rank r solves its shard with
    the batched solver, then every rank receives every instance's result
    through one all_gather of Python objects. The solve itself exchanges
    nothing. `solve` replaces solve_poisson_batch (same arguments), e.g. for
    host-side tests. `all_gather(parts, obj)` fills `parts` (one slot per
    rank) with every rank's obj; by default torch.distributed's
    all_gather_object on `group` (the process-group plumbing, imported only
    when world > 1). Returns (solutions, iterations, rel_residuals, statuses)
    in instance order."""
    meshes = list(meshes)
    mine = shard_instances(batch_costs(meshes), world)[rank]
    solve = solve or (lambda ms, ks, fs: solve_poisson_batch(ms, ks, fs, tol=tol, max_iter=max_iter, ctx=ctx,
                                                              precision=precision, raise_on_error=False))
    local = {}
    if mine:
        res = solve([meshes[i] for i in mine], None if kappas is None else [kappas[i] for i in mine],
                    None if nodal_sources is None else [nodal_sources[i] for i in mine])
        for j, i in enumerate(mine):
            local[i] = (np.asarray(res.solutions[j]), int(res.iterations[j]), float(res.rel_residuals[j]),
                        int(res.statuses[j]))
    if world > 1:
        parts = [None] * world
        if all_gather is None:
            import torch.distributed as dist
            dist.all_gather_object(parts, local, group=group)
        else:
            all_gather(parts, local)
        merged = {}
        for part in parts:
            merged.update(part)
        local = merged
    n = len(meshes)
    return ([local[i][0] for i in range(n)], np.array([local[i][1] for i in range(n)], np.int64),
            np.array([local[i][2] for i in range(n)]), np.array([local[i][3] for i in range(n)], np.int32))


@dataclass
class ElasticitySolution:
    """elasticity_solver.rs:13-29 (displacements, iterations, residual)."""
    displacements: np.ndarray
    deformed_vertices: np.ndarray
    iterations: int
    residual: float


def solve_elasticity_3d(mesh: Mesh, material: ElasticMaterial, body_force, bc: VectorDirichletBC, tol, max_iter,
                        ctx=None, precision=FCU_FP64) -> ElasticitySolution:
    """solve_elasticity_3d (elasticity_solver.rs:31-72), assembly to solve on the device."""
    ctx = ctx or default_context()
    V = FunctionSpace(ctx, mesh, FCU_SPACE_P1_VEC3)
    M = Matrix(ctx, V).assemble_elasticity(material.youngs_modulus, material.poissons_ratio)
    f = V.body_force(body_force, out=_device_vector(ctx, V.ndofs))
    d, v = bc.arrays()
    M.apply_dirichlet(f, d, v)
    xd, info = M.pcg(f, x=_device_vector(ctx, V.ndofs), tol=tol, max_iter=max_iter, precision=precision)
    x = xd.numpy()
    return ElasticitySolution(x, mesh.coords + x.reshape(-1, 3), info.iterations, info.residual)


# ---------------------------------------------------------------------------
# mass matrices, transient heat, vibration modes (mass.rs, transient.rs,
# heat_solver.rs, eigen.rs)
# ---------------------------------------------------------------------------

def assemble_mass_2d(mesh: Mesh, ctx: Context | None = None) -> CscMatrix:
    """assemble_mass_2d (mass.rs:10-44)."""
    if mesh.dim != 2:
        raise ValueError("triangle mesh expected")
    return _assembled(FCU_SPACE_P1, mesh, ctx, lambda M: M.assemble_mass(1.0))


def assemble_mass_3d(mesh: Mesh, ctx: Context | None = None) -> CscMatrix:
    """assemble_mass_3d (mass.rs:47-81)."""
    if mesh.dim != 3:
        raise ValueError("tetrahedron mesh expected")
    return _assembled(FCU_SPACE_P1, mesh, ctx, lambda M: M.assemble_mass(1.0))


def assemble_elasticity_mass_3d(mesh: Mesh, density, ctx: Context | None = None) -> CscMatrix:
    """assemble_elasticity_mass_3d (mass.rs:84-127)."""
    if mesh.dim != 3:
        raise ValueError("tetrahedron mesh expected")
    return _assembled(FCU_SPACE_P1_VEC3, mesh, ctx, lambda M: M.assemble_mass(float(density)))


def assemble_mass_p2_3d(mesh: Mesh, density=1.0, ctx: Context | None = None) -> CscMatrix:
    """Scalar P2 mass from the exact reference products of
    assemble_elasticity_mass_p2_3d (mass.rs:137-250), on this build's P2
    numbering (vertices, then edges)."""
    return _assembled(FCU_SPACE_P2, mesh, ctx, lambda M: M.assemble_mass(float(density)))


def assemble_elasticity_mass_p2_3d(vertices, cells, density, ctx: Context | None = None) -> CscMatrix:
    """assemble_elasticity_mass_p2_3d (mass.rs:137-180): vertices = every P2
    node, cells = ten nodes per cell (4 corners, then edges 01, 12, 02, 03,
    13, 23); dof = 3 node + component."""
    ctx = ctx or default_context()
    c10 = np.ascontiguousarray(cells, dtype=np.int64).reshape(-1, 10)
    mesh = Mesh(np.ascontiguousarray(vertices, dtype=np.float64), np.ascontiguousarray(c10[:, :4]))
    V = FunctionSpace(ctx, mesh, _abi.FCU_SPACE_P2_NODES_VEC3, cells10=c10)
    M = Matrix(ctx, V).assemble_mass(float(density))
    A = M.export_csc()
    M.close()
    V.close()
    return A


def _as_matrix(ctx, mat):
    """(Matrix, owned) for a Matrix or a CscMatrix."""
    if isinstance(mat, Matrix):
        return mat, False
    return Matrix.from_csc(ctx, mat), True


def add_scaled_matrices(a, b, alpha, ctx: Context | None = None) -> CscMatrix:
    """add_scaled_matrices (transient.rs:72-97): a + alpha * b, on the union
    of the operands' patterns. Two matrices of one space combine value by
    value on the device; any other pair goes through the union build."""
    ctx = ctx or default_context()
    A, oa = _as_matrix(ctx, a)
    B, ob = _as_matrix(ctx, b)
    try:
        out = None
        if A.space is not None and A.space is B.space:
            out = A.clone()
            try:
                out.set_add_scaled(A, B, alpha)
            except FcuError as e:
                if e.code != _abi.FCU_ERR_UNSUPPORTED:
                    raise
                out.close()
                out = None   # Dirichlet or folded state: the exported operands combine below
        if out is None:
            out = Matrix.add_scaled_union(A, B, alpha)
        res = out.export_csc()
        out.close()
    finally:
        if oa:
            A.close()
        if ob:
            B.close()
    return res


def fold_dirichlet(mat, fixed_dofs, unit_diag: bool, ctx: Context | None = None) -> CscMatrix:
    """fold_dirichlet (eigen.rs:55-79): constrained rows and columns dropped,
    unit diagonal on them when unit_diag, zero entries dropped."""
    ctx = ctx or default_context()
    A, oa = _as_matrix(ctx, mat)
    try:
        F = A.clone() if not oa else A
        F.fold_dirichlet(np.asarray(fixed_dofs, dtype=np.int64), unit_diag)
        res = F.export_csc()
        if F is not A:
            F.close()
    finally:
        if oa:
            A.close()
    return res


class TimeSteppingScheme:
    """TimeSteppingScheme (transient.rs:11-18)."""
    BackwardEuler = FCU_BACKWARD_EULER
    CrankNicolson = FCU_CRANK_NICOLSON


class _Stepper:
    """A device stepper (fcu_transient) for one (mass, stiffness) pair."""

    def __init__(self, ctx: Context, M: Matrix, K: Matrix, scheme: int, dt: float):
        self.ctx = ctx
        h = C.c_void_p()
        _check(ctx, _L().fcu_transient_create(ctx.h, M.h, K.h, int(scheme), float(dt), C.byref(h)))
        self.h = h

    def set_dirichlet(self, dofs, vals):
        pd, kd = _ptr(dofs, np.int64)
        pv, kv = _ptr(vals, np.float64)
        _check(self.ctx, _L().fcu_transient_set_dirichlet(self.ctx.h, self.h, len(dofs), pd, pv))

    def step(self, u_n, f_n, f_next, u_next, tol, max_iter, precision):
        pu, ku = _ptr(u_n, np.float64)
        p0, k0 = _ptr(f_n, np.float64)
        p1, k1 = _ptr(f_next, np.float64)
        po, ko = _ptr(u_next)
        info = SolveInfo()
        rc = _L().fcu_transient_step(self.ctx.h, self.h, pu, p0, p1, po, float(tol), int(max_iter), precision,
                                     C.byref(info))
        _check(self.ctx, rc)
        return info

    def close(self):
        if getattr(self, "h", None):
            _L().fcu_transient_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TransientHeatSolver:
    """TransientHeatSolver (transient.rs:21-68). step() solves the SPD system
    (M + theta dt K) u_{n+1} = rhs with Jacobi-PCG to `tol` (relative
    residual) from u_n, where the reference factorises densely; the device
    matrices of a (mass, stiffness) pair are formed once and reused."""

    def __init__(self, scheme, dt, ctx: Context | None = None, tol=1e-12, max_iter=100000, precision=FCU_FP64):
        self.scheme, self.dt = int(scheme), float(dt)
        self.ctx = ctx or default_context()
        self.tol, self.max_iter, self.precision = tol, max_iter, precision
        self._key = None
        self._stepper = None
        self._held = []
        self.last_info = None

    def _prepare(self, mass, stiff):
        key = (id(mass), id(stiff))
        if self._key != key:
            self.close()
            M, om = _as_matrix(self.ctx, mass)
            K, ok = _as_matrix(self.ctx, stiff)
            self._stepper = _Stepper(self.ctx, M, K, self.scheme, self.dt)
            self._held = [x for x, owned in ((M, om), (K, ok)) if owned]
            self._key = key
        return self._stepper

    def step(self, mass_mat, stiff_mat, u_n, f_n, f_next):
        st = self._prepare(mass_mat, stiff_mat)
        if isinstance(u_n, DeviceArray):
            out = DeviceArray(self.ctx, len(u_n))
        elif _is_torch(u_n):
            out = u_n.new_empty(u_n.shape)
        else:
            out = np.empty(len(u_n))
        self.last_info = st.step(u_n, f_n, f_next, out, self.tol, self.max_iter, self.precision)
        return out

    def close(self):
        if self._stepper is not None:
            self._stepper.close()
        for m in self._held:
            m.close()
        self._stepper, self._held, self._key = None, [], None


@dataclass
class TransientHeatSolution:
    """heat_solver.rs:13-19"""
    time_steps: list
    temperature_history: list
    final_temperature: np.ndarray
    iterations: list = field(default_factory=list)


def solve_transient_heat_2d(mesh: Mesh, diffusivity, u_initial, bcs, dt, num_steps, scheme, heat_source=None,
                            ctx: Context | None = None, tol=1e-12, max_iter=100000, precision=FCU_FP64,
                            keep_history=True, vectorized_source=False) -> TransientHeatSolution:
    """solve_transient_heat_2d (heat_solver.rs:23-104): P1 mass and
    diffusivity-scaled stiffness on the device, Dirichlet values written into
    the state before and after every step. heat_source(t, point) is called
    per vertex like the reference's closure (or once per time with the
    (nv, 2) coordinates when vectorized_source); None means no source."""
    ctx = ctx or default_context()
    n = mesh.num_vertices()
    if len(u_initial) != n:
        raise ValueError(f"Initial temperature size {len(u_initial)} != mesh vertices {n}")
    V = FunctionSpace(ctx, mesh, FCU_SPACE_P1)
    M = Matrix(ctx, V).assemble_mass(1.0)
    K = Matrix(ctx, V).assemble_stiffness(None).scale(diffusivity)
    st = _Stepper(ctx, M, K, int(scheme), float(dt))
    dofs, vals = [], []
    for bc in bcs:
        dofs.extend(int(d) for d in bc.dofs)
        vals.extend(float(v) for v in bc.values)
    if dofs:
        st.set_dirichlet(np.asarray(dofs, np.int64), np.asarray(vals, np.float64))
    u = DeviceArray.from_numpy(ctx, u_initial, np.float64)
    un = DeviceArray(ctx, n)
    coords = mesh.coords

    def source(t):
        if heat_source is None:
            return None
        if vectorized_source:
            return np.ascontiguousarray(heat_source(t, coords), dtype=np.float64)
        return np.array([heat_source(t, coords[i]) for i in range(n)], dtype=np.float64)

    times, history, iters = [0.0], [np.asarray(u_initial, dtype=np.float64).copy()] if keep_history else [], []
    try:
        for step in range(1, num_steps + 1):
            t_curr, t_next = (step - 1) * dt, step * dt
            info = st.step(u, source(t_curr), source(t_next), un, tol, max_iter, precision)
            iters.append(int(info.iterations))
            u, un = un, u
            times.append(t_next)
            if keep_history:
                history.append(u.numpy())
        final = u.numpy()
    finally:
        st.close()
        M.close()
        K.close()
        V.close()
    if not keep_history:
        history = []
    return TransientHeatSolution(times, history, final, iters)


@dataclass
class VibrationMode:
    """VibrationMode (eigen.rs:10-19)"""
    frequency_hz: float
    omega_rad_s: float
    eigenvalue: float
    mode_shape: np.ndarray


def _vibration_modes(k, m, fixed_dofs, num_modes, max_power_iters, tol, ctx, precision, inner_tol,
                     inner_max_iter, inner):
    ctx = ctx or default_context()
    K, ok = _as_matrix(ctx, k)
    M, om = _as_matrix(ctx, m)
    n = K.n
    fixed = np.ascontiguousarray(fixed_dofs, dtype=np.int64)
    ev = np.zeros(max(num_modes, 1))
    shapes = np.zeros((max(num_modes, 1), n))
    pit = np.zeros(max(num_modes, 1), np.int64)
    info = SolveInfo()
    err = []
    cb = _abi.INNER_SOLVE()
    if inner is not None:
        L = _L()

        def trampoline(user, nn, b, x0, x):
            try:
                # b, x0 and x are device arrays; the library's stream is idle
                bh, x0h = np.empty(nn), np.empty(nn)
                _check(ctx, L.fcu_buffer_copy(ctx.h, C.c_void_p(bh.ctypes.data), C.c_void_p(b), 8 * nn))
                _check(ctx, L.fcu_buffer_copy(ctx.h, C.c_void_p(x0h.ctypes.data), C.c_void_p(x0), 8 * nn))
                res = np.ascontiguousarray(inner(bh, x0h), dtype=np.float64)
                if res.shape != (nn,):
                    raise ValueError(f"inner solve returned shape {res.shape}, expected ({nn},)")
                _check(ctx, L.fcu_buffer_copy(ctx.h, C.c_void_p(x), C.c_void_p(res.ctypes.data), 8 * nn))
                return 0
            except Exception as e:  # the reference's `?` on the closure's Err
                err.append(e)
                return _abi.FCU_ERR_NO_CONVERGENCE

        cb = _abi.INNER_SOLVE(trampoline)
    try:
        rc = _L().fcu_vibration_modes(ctx.h, K.h, M.h, len(fixed), fixed.ctypes.data if len(fixed) else None,
                                      int(num_modes), int(max_power_iters), float(tol), float(inner_tol),
                                      int(inner_max_iter), precision, cb, None, ev.ctypes.data, shapes.ctypes.data,
                                      pit.ctypes.data, C.byref(info))
        if err:
            raise err[0]
        _check(ctx, rc)
    finally:
        if ok:
            K.close()
        if om:
            M.close()
    modes = []
    for i in range(num_modes):
        lam = float(ev[i])
        omega = math.sqrt(lam)
        modes.append(VibrationMode(omega / (2.0 * math.pi), omega, lam, shapes[i].copy()))
    return modes, pit[:num_modes].copy(), info


def solve_vibration_modes(k, m, fixed_dofs, num_modes, max_power_iters, tol, ctx: Context | None = None,
                          precision=FCU_FP64, inner_tol=1e-9, inner_max_iter=1000, return_stats=False):
    """solve_vibration_modes (eigen.rs:286-300): the lowest modes of
    K u = omega^2 M u, the inner solve Jacobi-PCG on the device at
    inner_tol / inner_max_iter (reference: 1e-9, 1000). k, m: CscMatrix or
    device Matrix on one pattern."""
    modes, pit, info = _vibration_modes(k, m, fixed_dofs, num_modes, max_power_iters, tol, ctx, precision,
                                        inner_tol, inner_max_iter, None)
    return (modes, pit, info) if return_stats else modes


def solve_vibration_modes_with_inner(k, m, fixed_dofs, num_modes, max_power_iters, tol, inner,
                                     ctx: Context | None = None):
    """solve_vibration_modes_with_inner (eigen.rs:94-271): inner(b, x0) -> x
    solves the folded K x = b on host arrays; an exception from it fails the
    call like the closure's Err."""
    modes, _, _ = _vibration_modes(k, m, fixed_dofs, num_modes, max_power_iters, tol, ctx, FCU_FP64, 0.0, 0,
                                   inner)
    return modes


# ---------------------------------------------------------------------------
# 3x3 block CSR (gpu.rs:434-1141)
# ---------------------------------------------------------------------------

class GpuBsr3Context:
    """GpuBsr3Context (gpu.rs:434-658): a resident 3x3 block CSR operator with
    its inverse diagonal blocks."""

    def __init__(self, n_nodes, row_ptr, cols, vals_flat, dinv_flat, device_index: int | None = None,
                 ctx: Context | None = None):
        self.ctx = ctx or (Context(device_index) if device_index not in (None, 0) else default_context())
        self.n_nodes = int(n_nodes)
        self._nnzb = int(np.asarray(row_ptr)[-1])
        self.M = Matrix.from_bsr3(self.ctx, n_nodes, row_ptr, cols, vals_flat, dinv_flat)

    def device_name(self) -> str:
        return device_name(self.ctx.device)

    def nnz_blocks(self) -> int:
        return self._nnzb

    def spmv(self, x, y):
        """y = A x (gpu.rs:505-545); y is filled in place."""
        self.M.spmv(x, y)
        return y

    def jacobi_smooth(self, r, z, sweeps, omega, zero_initial_z):
        """`sweeps` damped block-Jacobi sweeps on z in place (gpu.rs:547-657)."""
        pr, kr = _ptr(r, np.float64)
        pz, kz = _ptr(z)
        if not _is_torch(z) and kz is not z:
            raise ValueError("z must be a contiguous float64 array (updated in place)")
        _check(self.ctx, _L().fcu_bsr3_jacobi_smooth(self.ctx.h, self.M.h, pr, pz, int(sweeps), float(omega),
                                                     1 if zero_initial_z else 0))
        return z

    def close(self):
        self.M.close()


def solve_bsr3_pcg_gpu(n_nodes, row_ptr, cols, vals_flat, dinv_flat, b, x0=None, rtol=1e-8, max_iter=1000,
                       device_index: int | None = None, ctx: Context | None = None) -> GpuSolveResult:
    """solve_bsr3_pcg_gpu (gpu.rs:775-1141): block-Jacobi PCG, Ok at the
    iteration limit, x = 0 for b = 0."""
    import time
    t0 = time.perf_counter()
    ctx = ctx or (Context(device_index) if device_index not in (None, 0) else default_context())
    n = 3 * int(n_nodes)
    x = np.empty(n)
    pr, kr = _ptr(row_ptr, np.uint32)
    pc, kc = _ptr(cols, np.uint32)
    pv, kv = _ptr(vals_flat, np.float64)
    pd, kd = _ptr(dinv_flat, np.float64)
    pb, kb = _ptr(b, np.float64)
    p0, k0 = _ptr(x0, np.float64)
    info = SolveInfo()
    _check(ctx, _L().fcu_solve_bsr3_pcg(ctx.h, int(n_nodes), pr, pc, pv, pd, pb, p0, float(rtol), int(max_iter),
                                        x.ctypes.data, C.byref(info)))
    wall = (time.perf_counter() - t0) * 1e3
    nnzb = int(np.asarray(row_ptr)[-1])
    flops = (nnzb * 18.0 + n * 16.0) * info.iterations
    return GpuSolveResult(x, int(info.iterations), float(info.rel_residual), wall, float(info.kernel_ms),
                          flops / max(info.kernel_ms * 1e-3, 1e-12) / 1e9, float(info.effective_bw_gbps),
                          [device_name(ctx.device)])


def bsr3_row_split(n_nodes, row_ptr, parts):
    """The row split of spmv_bsr3_multi_gpu (gpu.rs:662-771): contiguous
    block-row ranges of ceil(n_nodes / parts) rows. For each non-empty range
    returns (r0, r1, sub_row_ptr, b0, b1): a row pointer over all n_nodes rows
    whose rows outside [r0, r1) are empty, and the range's blocks [b0, b1)."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    n_nodes = int(n_nodes)
    chunk = (n_nodes + parts - 1) // parts
    out = []
    for slot in range(parts):
        r0, r1 = slot * chunk, min((slot + 1) * chunk, n_nodes)
        if r0 >= r1:
            continue
        sub = np.concatenate([np.full(r0 + 1, rp[r0]), rp[r0 + 1:r1 + 1], np.full(n_nodes - r1, rp[r1])]) - rp[r0]
        out.append((r0, r1, sub.astype(np.uint32), int(rp[r0]), int(rp[r1])))
    return out


def spmv_bsr3_multi_gpu(n_nodes, row_ptr, cols, vals_flat, x, max_gpus):
    """spmv_bsr3_multi_gpu (gpu.rs:662-771): the block rows split into
    g = min(max_gpus, visible devices) contiguous ranges (bsr3_row_split), each
    range's product computed on its device, concatenated on the host. Returns
    (y, device names)."""
    nd = max(1, min(int(max_gpus), device_count()))
    cols = np.asarray(cols, np.uint32)
    vals_flat = np.asarray(vals_flat, np.float64)
    y = np.zeros(3 * int(n_nodes))
    names = []
    for slot, (r0, r1, sub, b0, b1) in enumerate(bsr3_row_split(n_nodes, row_ptr, nd)):
        ctx = default_context() if slot == 0 else Context(slot)
        M = Matrix.from_bsr3(ctx, n_nodes, sub, cols[b0:b1], vals_flat[9 * b0:9 * b1])
        part = M.spmv(x)
        y[3 * r0:3 * r1] = part[3 * r0:3 * r1]
        M.close()
        names.append(device_name(ctx.device))
        if slot:
            ctx.close()
    return y, names
