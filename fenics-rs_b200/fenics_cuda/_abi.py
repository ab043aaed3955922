"""ctypes binding of libfenics_cuda.so (declarations in include/fenics_cuda.h).

The library is built in-tree by ``fenics-rs_b200/build.py``; loading fails
loudly when it is missing — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libfenics_cuda.so")

FCU_OK = 0
FCU_ERR_CUDA = 1
FCU_ERR_BAD_ARG = 2
FCU_ERR_NO_CONVERGENCE = 3
FCU_ERR_BREAKDOWN = 4
FCU_ERR_UNSUPPORTED = 5

FCU_NOALLOC_MAX_N = 131072  # row capacity of fcu_solve_csr_cg_noalloc

FCU_SPACE_P1 = 1
FCU_SPACE_P2 = 2
FCU_SPACE_P1_VEC3 = 3
FCU_SPACE_P2_NODES = 4
FCU_SPACE_P2_NODES_VEC3 = 5

FCU_FP64 = 0
FCU_MIXED = 1

FCU_SRC_CONSTANT = 0
FCU_SRC_SIN_PRODUCT = 1
FCU_SRC_NODAL = 2

FCU_BACKWARD_EULER = 0
FCU_CRANK_NICOLSON = 1


class SolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("outer_updates", C.c_int64),
        ("residual", C.c_double),
        ("rel_residual", C.c_double),
        ("kernel_ms", C.c_double),
        ("effective_bw_gbps", C.c_double),
        ("status", C.c_int),
    ]


vp = C.c_void_p
i64 = C.c_int64
dbl = C.c_double
cint = C.c_int

# fcu_inner_solve: int (*)(void* user, int64_t n, const double* b, const double* x0, double* x)
INNER_SOLVE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p)

# name -> (restype, argtypes); pointer arguments are passed as integers.
SIGNATURES = {
    "fcu_ctx_create": (cint, [cint, C.POINTER(vp)]),
    "fcu_ctx_destroy": (None, [vp]),
    "fcu_last_error": (C.c_char_p, [vp]),
    "fcu_ctx_synchronize": (cint, [vp]),
    "fcu_ctx_stream": (vp, [vp]),
    "fcu_ctx_kernel_launches": (i64, [vp]),
    "fcu_mesh_create": (cint, [vp, cint, i64, vp, i64, vp, C.POINTER(vp)]),
    "fcu_mesh_destroy": (None, [vp]),
    "fcu_mesh_num_degenerate": (cint, [vp, vp, C.POINTER(i64)]),
    "fcu_boundary_dofs": (cint, [vp, vp, vp, C.POINTER(i64)]),
    "fcu_boundary_facets": (cint, [vp, vp, vp, vp, vp, C.POINTER(i64)]),
    "fcu_space_create": (cint, [vp, vp, cint, C.POINTER(vp)]),
    "fcu_space_create_p2_nodes": (cint, [vp, vp, vp, cint, C.POINTER(vp)]),
    "fcu_space_destroy": (None, [vp]),
    "fcu_space_info": (cint, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]),
    "fcu_space_p2_dofmap": (cint, [vp, vp, vp, vp]),
    "fcu_space_boundary_dofs": (cint, [vp, vp, vp, C.POINTER(i64)]),
    "fcu_matrix_create": (cint, [vp, vp, C.POINTER(vp)]),
    "fcu_matrix_from_csc": (cint, [vp, i64, vp, vp, vp, C.POINTER(vp)]),
    "fcu_matrix_destroy": (None, [vp]),
    "fcu_matrix_info": (cint, [vp, C.POINTER(i64), C.POINTER(i64)]),
    "fcu_matrix_export_csc": (cint, [vp, vp, vp, vp, vp]),
    "fcu_assemble_stiffness": (cint, [vp, vp, vp]),
    "fcu_assemble_elasticity": (cint, [vp, vp, dbl, dbl, vp]),
    "fcu_assemble_mass": (cint, [vp, vp, dbl, vp]),
    "fcu_matrix_clone": (cint, [vp, vp, C.POINTER(vp)]),
    "fcu_matrix_add_scaled": (cint, [vp, vp, vp, vp, dbl]),
    "fcu_matrix_add_scaled_union": (cint, [vp, vp, vp, dbl, C.POINTER(vp)]),
    "fcu_matrix_scale": (cint, [vp, vp, dbl]),
    "fcu_matrix_fold_dirichlet": (cint, [vp, vp, i64, vp, cint]),
    "fcu_apply_dirichlet": (cint, [vp, vp, vp, i64, vp, vp]),
    "fcu_quadrature_points": (cint, [vp, vp, vp]),
    "fcu_assemble_rhs_values": (cint, [vp, vp, vp, vp]),
    "fcu_assemble_rhs_source": (cint, [vp, vp, cint, vp, vp, vp]),
    "fcu_assemble_body_force": (cint, [vp, vp, vp, vp]),
    "fcu_assemble_surface_traction": (cint, [vp, vp, i64, vp, vp, vp]),
    "fcu_pcg": (cint, [vp, vp, vp, vp, vp, dbl, i64, cint, C.POINTER(SolveInfo)]),
    "fcu_solve_csr_cg": (cint, [vp, i64, vp, vp, vp, vp, vp, vp, dbl, i64, vp, C.POINTER(SolveInfo)]),
    "fcu_solve_csr_cg_noalloc": (cint, [i64, vp, vp, vp, vp, vp, vp, dbl, i64, vp, C.POINTER(SolveInfo), vp]),
    "fcu_batch_pcg": (cint, [vp, vp, i64, vp, vp, vp, dbl, i64, cint, vp, vp, vp, C.POINTER(SolveInfo)]),
    "fcu_batch_config": (cint, [vp, cint, C.POINTER(cint), C.POINTER(cint), C.POINTER(cint)]),
    "fcu_element_stresses": (cint, [vp, vp, dbl, dbl, vp, vp, vp, vp, vp]),
    "fcu_vertex_von_mises": (cint, [vp, vp, vp, vp]),
    "fcu_transient_create": (cint, [vp, vp, vp, cint, dbl, C.POINTER(vp)]),
    "fcu_transient_set_dirichlet": (cint, [vp, vp, i64, vp, vp]),
    "fcu_transient_step": (cint, [vp, vp, vp, vp, vp, vp, dbl, i64, cint, C.POINTER(SolveInfo)]),
    "fcu_transient_destroy": (None, [vp]),
    "fcu_vibration_modes": (cint, [vp, vp, vp, i64, vp, i64, i64, dbl, dbl, i64, cint, INNER_SOLVE, vp, vp, vp, vp,
                                   C.POINTER(SolveInfo)]),
    "fcu_bsr3_create": (cint, [vp, i64, vp, vp, vp, vp, C.POINTER(vp)]),
    "fcu_bsr3_jacobi_smooth": (cint, [vp, vp, vp, vp, i64, dbl, cint]),
    "fcu_solve_bsr3_pcg": (cint, [vp, i64, vp, vp, vp, vp, vp, vp, dbl, i64, vp, C.POINTER(SolveInfo)]),
    "fcu_matrix_block_jacobi": (cint, [vp, vp, cint]),
    "fcu_matrix_export_bsr3": (cint, [vp, vp, vp, vp, vp, vp]),
    "fcu_spmv": (cint, [vp, vp, vp, vp]),
    "fcu_adjoint_gradient": (cint, [vp, vp, dbl, dbl, vp, vp, vp, vp]),
    "fcu_time_spmv": (cint, [vp, vp, cint, cint, C.POINTER(dbl), C.POINTER(dbl)]),
    "fcu_time_spmv_cold": (cint, [vp, vp, cint, cint, C.c_size_t, C.POINTER(dbl), C.POINTER(dbl)]),
    "fcu_time_pcg": (cint, [vp, vp, cint, C.c_int64, cint, C.c_size_t, C.POINTER(dbl), C.POINTER(dbl)]),
    "fcu_check_wait_limits": (cint, [vp, C.c_uint32, C.POINTER(cint)]),
    "fcu_buffer_alloc": (cint, [vp, C.c_size_t, C.POINTER(vp)]),
    "fcu_buffer_free": (cint, [vp, vp]),
    "fcu_buffer_copy": (cint, [vp, vp, vp, C.c_size_t]),
    "fcu_buffer_memset": (cint, [vp, vp, cint, C.c_size_t]),
    "fcu_device_count": (cint, [C.POINTER(cint)]),
    "fcu_device_name": (cint, [cint, C.c_char_p, C.c_size_t]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise ImportError(f"{SO} is missing: run `python fenics-rs_b200/build.py` (needs nvcc)")
        L = C.CDLL(SO)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
