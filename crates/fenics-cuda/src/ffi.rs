//! Raw bindings of the fenics_cuda C ABI, one item per declaration of
//! include/fenics_cuda.h (same names, same argument order and types). The
//! safe wrappers with the reference's signatures are in lib.rs.
#![allow(non_camel_case_types)]
use std::os::raw::{c_char, c_int, c_void};

pub const FCU_OK: c_int = 0;
pub const FCU_ERR_CUDA: c_int = 1;
pub const FCU_ERR_BAD_ARG: c_int = 2;
pub const FCU_ERR_NO_CONVERGENCE: c_int = 3;
pub const FCU_ERR_BREAKDOWN: c_int = 4;
pub const FCU_ERR_UNSUPPORTED: c_int = 5;

pub const FCU_SPACE_P1: c_int = 1;
pub const FCU_SPACE_P2: c_int = 2;
pub const FCU_SPACE_P1_VEC3: c_int = 3;
pub const FCU_SPACE_P2_NODES: c_int = 4;
pub const FCU_SPACE_P2_NODES_VEC3: c_int = 5;

pub const FCU_FP64: c_int = 0;
pub const FCU_MIXED: c_int = 1;

pub const FCU_SRC_CONSTANT: c_int = 0;
pub const FCU_SRC_SIN_PRODUCT: c_int = 1;
pub const FCU_SRC_NODAL: c_int = 2;

pub const FCU_BACKWARD_EULER: c_int = 0;
pub const FCU_CRANK_NICOLSON: c_int = 1;

pub const FCU_NOALLOC_MAX_N: i64 = 131072;

#[repr(C)]
pub struct fcu_ctx_s {
    _p: [u8; 0],
}
#[repr(C)]
pub struct fcu_mesh_s {
    _p: [u8; 0],
}
#[repr(C)]
pub struct fcu_space_s {
    _p: [u8; 0],
}
#[repr(C)]
pub struct fcu_matrix_s {
    _p: [u8; 0],
}
#[repr(C)]
pub struct fcu_transient_s {
    _p: [u8; 0],
}
pub type fcu_ctx = *mut fcu_ctx_s;
pub type fcu_mesh = *mut fcu_mesh_s;
pub type fcu_space = *mut fcu_space_s;
pub type fcu_matrix = *mut fcu_matrix_s;
pub type fcu_transient = *mut fcu_transient_s;

/// The inner solve of the vibration-mode iteration (the `inner` closure of
/// eigen.rs:94-102); b, x0 and x are device arrays of n doubles.
pub type fcu_inner_solve =
    Option<unsafe extern "C" fn(user: *mut c_void, n: i64, b: *const f64, x0: *const f64, x: *mut f64) -> c_int>;

/// Per-solve report: the numeric fields of GpuSolveResult (gpu.rs:24-34),
/// the status, and the absolute residual solve_cg returns.
#[repr(C)]
#[derive(Default, Clone, Copy, Debug)]
pub struct fcu_solve_info {
    pub iterations: i64,
    pub outer_updates: i64,
    pub residual: f64,
    pub rel_residual: f64,
    pub kernel_ms: f64,
    pub effective_bw_gbps: f64,
    pub status: c_int,
}

extern "C" {
    // context (CudaSession, gpu.rs:325-430)
    pub fn fcu_ctx_create(device: c_int, out: *mut fcu_ctx) -> c_int;
    pub fn fcu_ctx_destroy(ctx: fcu_ctx);
    pub fn fcu_last_error(ctx: fcu_ctx) -> *const c_char;
    pub fn fcu_ctx_synchronize(ctx: fcu_ctx) -> c_int;
    pub fn fcu_ctx_stream(ctx: fcu_ctx) -> *mut c_void;
    pub fn fcu_ctx_kernel_launches(ctx: fcu_ctx) -> i64;

    // meshes (SimplicialMesh, mesh.rs:11-20) and boundaries
    pub fn fcu_mesh_create(
        ctx: fcu_ctx,
        dim: c_int,
        nv: i64,
        coords: *const f64,
        nc: i64,
        cells: *const i64,
        out: *mut fcu_mesh,
    ) -> c_int;
    pub fn fcu_mesh_destroy(mesh: fcu_mesh);
    pub fn fcu_mesh_num_degenerate(ctx: fcu_ctx, mesh: fcu_mesh, count: *mut i64) -> c_int;
    pub fn fcu_boundary_dofs(ctx: fcu_ctx, mesh: fcu_mesh, out: *mut i64, count: *mut i64) -> c_int;
    pub fn fcu_boundary_facets(
        ctx: fcu_ctx,
        mesh: fcu_mesh,
        verts: *mut i64,
        cell: *mut i64,
        local: *mut i64,
        count: *mut i64,
    ) -> c_int;

    // function spaces
    pub fn fcu_space_create(ctx: fcu_ctx, mesh: fcu_mesh, kind: c_int, out: *mut fcu_space) -> c_int;
    pub fn fcu_space_destroy(space: fcu_space);
    pub fn fcu_space_info(space: fcu_space, ndofs: *mut i64, nnz: *mut i64, nedges: *mut i64) -> c_int;
    pub fn fcu_space_p2_dofmap(ctx: fcu_ctx, space: fcu_space, cell_dofs: *mut i64, edge_verts: *mut i64)
        -> c_int;
    pub fn fcu_space_create_p2_nodes(
        ctx: fcu_ctx,
        mesh: fcu_mesh,
        cells10: *const i64,
        vec3: c_int,
        out: *mut fcu_space,
    ) -> c_int;
    pub fn fcu_space_boundary_dofs(ctx: fcu_ctx, space: fcu_space, out: *mut i64, count: *mut i64) -> c_int;

    // matrices
    pub fn fcu_matrix_create(ctx: fcu_ctx, space: fcu_space, out: *mut fcu_matrix) -> c_int;
    pub fn fcu_matrix_from_csc(
        ctx: fcu_ctx,
        n: i64,
        colptr: *const i64,
        rowidx: *const i64,
        vals: *const f64,
        out: *mut fcu_matrix,
    ) -> c_int;
    pub fn fcu_matrix_destroy(m: fcu_matrix);
    pub fn fcu_matrix_info(m: fcu_matrix, n: *mut i64, nnz: *mut i64) -> c_int;
    pub fn fcu_matrix_export_csc(
        ctx: fcu_ctx,
        m: fcu_matrix,
        colptr: *mut i64,
        rowidx: *mut i64,
        vals: *mut f64,
    ) -> c_int;

    // assembly (poisson.rs:23,124; elasticity.rs:73; mass.rs:10-250)
    pub fn fcu_assemble_stiffness(ctx: fcu_ctx, m: fcu_matrix, cell_coef: *const f64) -> c_int;
    pub fn fcu_assemble_elasticity(ctx: fcu_ctx, m: fcu_matrix, e: f64, nu: f64, cell_e: *const f64) -> c_int;
    pub fn fcu_assemble_mass(ctx: fcu_ctx, m: fcu_matrix, rho: f64, cell_coef: *const f64) -> c_int;
    pub fn fcu_matrix_clone(ctx: fcu_ctx, src: fcu_matrix, out: *mut fcu_matrix) -> c_int;
    pub fn fcu_matrix_add_scaled(ctx: fcu_ctx, out: fcu_matrix, a: fcu_matrix, b: fcu_matrix, alpha: f64)
        -> c_int;
    pub fn fcu_matrix_add_scaled_union(
        ctx: fcu_ctx,
        a: fcu_matrix,
        b: fcu_matrix,
        alpha: f64,
        out: *mut fcu_matrix,
    ) -> c_int;
    pub fn fcu_matrix_scale(ctx: fcu_ctx, m: fcu_matrix, s: f64) -> c_int;
    pub fn fcu_matrix_fold_dirichlet(
        ctx: fcu_ctx,
        m: fcu_matrix,
        nfixed: i64,
        fixed: *const i64,
        unit_diag: c_int,
    ) -> c_int;
    pub fn fcu_apply_dirichlet(
        ctx: fcu_ctx,
        m: fcu_matrix,
        b: *mut f64,
        nbc: i64,
        dofs: *const i64,
        vals: *const f64,
    ) -> c_int;

    // right-hand sides (poisson.rs:72,168; elasticity.rs:153; boundary.rs:48)
    pub fn fcu_quadrature_points(ctx: fcu_ctx, space: fcu_space, out: *mut f64) -> c_int;
    pub fn fcu_assemble_rhs_values(ctx: fcu_ctx, space: fcu_space, fq: *const f64, b: *mut f64) -> c_int;
    pub fn fcu_assemble_rhs_source(
        ctx: fcu_ctx,
        space: fcu_space,
        source: c_int,
        params: *const f64,
        values: *const f64,
        b: *mut f64,
    ) -> c_int;
    pub fn fcu_assemble_body_force(ctx: fcu_ctx, space: fcu_space, f_body3: *const f64, b: *mut f64) -> c_int;
    pub fn fcu_assemble_surface_traction(
        ctx: fcu_ctx,
        space: fcu_space,
        nf: i64,
        facets: *const i64,
        tq: *const f64,
        b: *mut f64,
    ) -> c_int;

    // solvers (cg.rs:40; gpu.rs:1145)
    pub fn fcu_pcg(
        ctx: fcu_ctx,
        m: fcu_matrix,
        b: *const f64,
        x0: *const f64,
        x: *mut f64,
        tol: f64,
        max_iter: i64,
        precision: c_int,
        info: *mut fcu_solve_info,
    ) -> c_int;
    pub fn fcu_solve_csr_cg(
        ctx: fcu_ctx,
        n: i64,
        row_ptr: *const u32,
        col_idx: *const u32,
        vals: *const f64,
        inv_diag: *const f64,
        b: *const f64,
        x0: *const f64,
        rtol: f64,
        max_iter: i64,
        x: *mut f64,
        info: *mut fcu_solve_info,
    ) -> c_int;
    pub fn fcu_batch_pcg(
        ctx: fcu_ctx,
        m: fcu_matrix,
        nb: i64,
        offsets: *const i64,
        b: *const f64,
        x: *mut f64,
        tol: f64,
        max_iter: i64,
        precision: c_int,
        iterations: *mut i64,
        rel_residual: *mut f64,
        status: *mut c_int,
        info: *mut fcu_solve_info,
    ) -> c_int;
    pub fn fcu_batch_config(
        m: fcu_matrix,
        precision: c_int,
        lanes_per_row: *mut c_int,
        threads_per_cta: *mut c_int,
        ctas_per_cluster: *mut c_int,
    ) -> c_int;
    /// No context and no allocation: device pointers only, n <= FCU_NOALLOC_MAX_N,
    /// calls on one device must not overlap.
    pub fn fcu_solve_csr_cg_noalloc(
        n: i64,
        row_ptr: *const u32,
        col_idx: *const u32,
        vals: *const f64,
        inv_diag: *const f64,
        b: *const f64,
        x0: *const f64,
        rtol: f64,
        max_iter: i64,
        x: *mut f64,
        info: *mut fcu_solve_info,
        stream: *mut c_void,
    ) -> c_int;
    pub fn fcu_spmv(ctx: fcu_ctx, m: fcu_matrix, x: *const f64, y: *mut f64) -> c_int;

    // transient heat (transient.rs:21-68, heat_solver.rs:23-104)
    pub fn fcu_transient_create(
        ctx: fcu_ctx,
        mass: fcu_matrix,
        stiff: fcu_matrix,
        scheme: c_int,
        dt: f64,
        out: *mut fcu_transient,
    ) -> c_int;
    pub fn fcu_transient_set_dirichlet(
        ctx: fcu_ctx,
        ts: fcu_transient,
        nbc: i64,
        dofs: *const i64,
        vals: *const f64,
    ) -> c_int;
    pub fn fcu_transient_step(
        ctx: fcu_ctx,
        ts: fcu_transient,
        u_n: *const f64,
        f_n: *const f64,
        f_next: *const f64,
        u_next: *mut f64,
        tol: f64,
        max_iter: i64,
        precision: c_int,
        info: *mut fcu_solve_info,
    ) -> c_int;
    pub fn fcu_transient_destroy(ts: fcu_transient);

    // vibration modes (eigen.rs:94-300)
    pub fn fcu_vibration_modes(
        ctx: fcu_ctx,
        k: fcu_matrix,
        m: fcu_matrix,
        nfixed: i64,
        fixed: *const i64,
        num_modes: i64,
        max_power_iters: i64,
        tol: f64,
        inner_tol: f64,
        inner_max_iter: i64,
        precision: c_int,
        inner: fcu_inner_solve,
        user: *mut c_void,
        eigenvalues: *mut f64,
        mode_shapes: *mut f64,
        power_iterations: *mut i64,
        info: *mut fcu_solve_info,
    ) -> c_int;

    // 3x3 block CSR (GpuBsr3Context, solve_bsr3_pcg_gpu; gpu.rs:434-1141)
    pub fn fcu_bsr3_create(
        ctx: fcu_ctx,
        n_nodes: i64,
        row_ptr: *const u32,
        cols: *const u32,
        vals_flat: *const f64,
        dinv_flat: *const f64,
        out: *mut fcu_matrix,
    ) -> c_int;
    pub fn fcu_bsr3_jacobi_smooth(
        ctx: fcu_ctx,
        m: fcu_matrix,
        r: *const f64,
        z: *mut f64,
        sweeps: i64,
        omega: f64,
        zero_initial_z: c_int,
    ) -> c_int;
    pub fn fcu_solve_bsr3_pcg(
        ctx: fcu_ctx,
        n_nodes: i64,
        row_ptr: *const u32,
        cols: *const u32,
        vals_flat: *const f64,
        dinv_flat: *const f64,
        b: *const f64,
        x0: *const f64,
        rtol: f64,
        max_iter: i64,
        x: *mut f64,
        info: *mut fcu_solve_info,
    ) -> c_int;
    pub fn fcu_matrix_block_jacobi(ctx: fcu_ctx, m: fcu_matrix, enable: c_int) -> c_int;
    pub fn fcu_matrix_export_bsr3(
        ctx: fcu_ctx,
        m: fcu_matrix,
        row_ptr: *mut u32,
        cols: *mut u32,
        vals_flat: *mut f64,
        dinv_flat: *mut f64,
    ) -> c_int;

    // adjoint sensitivities and stress recovery (elasticity.rs:230-360)
    pub fn fcu_adjoint_gradient(
        ctx: fcu_ctx,
        space: fcu_space,
        e0: f64,
        nu: f64,
        theta: *const f64,
        u: *const f64,
        lambda: *const f64,
        grad: *mut f64,
    ) -> c_int;
    pub fn fcu_element_stresses(
        ctx: fcu_ctx,
        space: fcu_space,
        e: f64,
        nu: f64,
        u: *const f64,
        stress: *mut f64,
        strain: *mut f64,
        von_mises: *mut f64,
        trace: *mut f64,
    ) -> c_int;
    pub fn fcu_vertex_von_mises(
        ctx: fcu_ctx,
        space: fcu_space,
        cell_von_mises: *const f64,
        vertex_von_mises: *mut f64,
    ) -> c_int;

    // device buffers and devices
    pub fn fcu_buffer_alloc(ctx: fcu_ctx, bytes: usize, out: *mut *mut c_void) -> c_int;
    pub fn fcu_buffer_free(ctx: fcu_ctx, p: *mut c_void) -> c_int;
    pub fn fcu_buffer_copy(ctx: fcu_ctx, dst: *mut c_void, src: *const c_void, bytes: usize) -> c_int;
    pub fn fcu_buffer_memset(ctx: fcu_ctx, p: *mut c_void, value: c_int, bytes: usize) -> c_int;
    pub fn fcu_device_count(count: *mut c_int) -> c_int;
    pub fn fcu_device_name(device: c_int, name: *mut c_char, len: usize) -> c_int;

    // diagnostics
    pub fn fcu_time_spmv(
        ctx: fcu_ctx,
        m: fcu_matrix,
        precision: c_int,
        reps: c_int,
        ms_per_launch: *mut f64,
        bytes_per_launch: *mut f64,
    ) -> c_int;
    pub fn fcu_time_spmv_cold(
        ctx: fcu_ctx,
        m: fcu_matrix,
        precision: c_int,
        reps: c_int,
        flush_bytes: usize,
        ms_per_launch: *mut f64,
        bytes_per_launch: *mut f64,
    ) -> c_int;
    pub fn fcu_time_pcg(
        ctx: fcu_ctx,
        m: fcu_matrix,
        precision: c_int,
        iterations: i64,
        reps: c_int,
        flush_bytes: usize,
        ms_per_launch: *mut f64,
        bytes_per_launch: *mut f64,
    ) -> c_int;
    pub fn fcu_check_wait_limits(ctx: fcu_ctx, polls: u32, results: *mut c_int) -> c_int;
}
