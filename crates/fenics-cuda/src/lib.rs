//! fenics-cuda: the fenics-rs assembly + Jacobi-PCG path on a B200 (sm_100a),
//! through the fenics_cuda C ABI (`include/fenics_cuda.h`, bound in ffi.rs).
//!
//! The functions below keep the signatures of the reference's entry points
//! (crates/fenics-assembly, crates/fenics-solver), so a `cuda` feature in
//! those crates can re-export them in place of the CPU bodies. Whole-pipeline
//! callers keep the matrix on the device instead: see [`ElasticityProblem`],
//! which assembles, eliminates and solves without a CSC round trip through
//! host memory, and [`ElasticityAdjoint`], the forward/backward pair of the
//! adjoint sensitivities.
//!
//! Host slices are passed to the library directly: it stages them on the
//! device and copies results back before each call returns.

pub mod ffi;

use faer::sparse::{SparseColMat, SymbolicSparseColMat};
use fenics_assembly::{DirichletBC, ElasticMaterial, StressState, VectorDirichletBC};
use fenics_mesh::{TetrahedronMesh, TriangleMesh};
use std::ffi::CStr;
use std::os::raw::{c_int, c_void};
use std::sync::OnceLock;

// ---------------------------------------------------------------------------
// Context: the process-global session of gpu.rs:340-362, one per process,
// created on first use on device 0.
// ---------------------------------------------------------------------------

struct Ctx(ffi::fcu_ctx);
// The library orders every call of a context on its stream; callers that
// share the session from several threads are serialised by the `Mutex`-free
// contract of the C ABI ("one context per host thread, or external
// synchronisation"), which `SESSION_LOCK` provides.
unsafe impl Send for Ctx {}
unsafe impl Sync for Ctx {}
impl Drop for Ctx {
    fn drop(&mut self) {
        unsafe { ffi::fcu_ctx_destroy(self.0) }
    }
}

static SESSION_LOCK: std::sync::Mutex<()> = std::sync::Mutex::new(());

fn ctx() -> &'static Ctx {
    static CTX: OnceLock<Ctx> = OnceLock::new();
    CTX.get_or_init(|| {
        let mut h = std::ptr::null_mut();
        let rc = unsafe { ffi::fcu_ctx_create(0, &mut h) };
        assert_eq!(rc, ffi::FCU_OK, "{}", last_error(std::ptr::null_mut()));
        Ctx(h)
    })
}

fn last_error(c: ffi::fcu_ctx) -> String {
    unsafe { CStr::from_ptr(ffi::fcu_last_error(c)).to_string_lossy().into_owned() }
}

fn check(rc: c_int) -> Result<(), String> {
    if rc == ffi::FCU_OK {
        Ok(())
    } else {
        Err(last_error(ctx().0))
    }
}

// ---------------------------------------------------------------------------
// Handles (freed on drop)
// ---------------------------------------------------------------------------

struct Mesh(ffi::fcu_mesh);
impl Drop for Mesh {
    fn drop(&mut self) {
        unsafe { ffi::fcu_mesh_destroy(self.0) }
    }
}
struct Space(ffi::fcu_space);
impl Drop for Space {
    fn drop(&mut self) {
        unsafe { ffi::fcu_space_destroy(self.0) }
    }
}
struct Matrix(ffi::fcu_matrix);
impl Drop for Matrix {
    fn drop(&mut self) {
        unsafe { ffi::fcu_matrix_destroy(self.0) }
    }
}

fn device_mesh<const D: usize, const N: usize>(v: &[[f64; D]], c: &[[usize; N]]) -> Mesh {
    // [f64; D] and [usize; N] are contiguous, so the Vecs already are the AoS
    // arrays the ABI takes (usize == i64 on the 64-bit targets CUDA supports).
    let mut h = std::ptr::null_mut();
    check(unsafe {
        ffi::fcu_mesh_create(
            ctx().0,
            D as c_int,
            v.len() as i64,
            v.as_ptr() as *const f64,
            c.len() as i64,
            c.as_ptr() as *const i64,
            &mut h,
        )
    })
    .unwrap();
    Mesh(h)
}

fn space(mesh: &Mesh, kind: c_int) -> Space {
    let mut s = std::ptr::null_mut();
    check(unsafe { ffi::fcu_space_create(ctx().0, mesh.0, kind, &mut s) }).unwrap();
    Space(s)
}

fn matrix(space: &Space) -> Matrix {
    let mut m = std::ptr::null_mut();
    check(unsafe { ffi::fcu_matrix_create(ctx().0, space.0, &mut m) }).unwrap();
    Matrix(m)
}

fn ndofs(space: &Space) -> usize {
    let mut n = 0i64;
    check(unsafe { ffi::fcu_space_info(space.0, &mut n, std::ptr::null_mut(), std::ptr::null_mut()) }).unwrap();
    n as usize
}

/// The matrix as faer holds it: sorted rows per column, duplicates summed,
/// explicit zeros kept (the invariants of try_new_from_triplets).
fn export(m: &Matrix) -> SparseColMat<usize, f64> {
    let (mut n, mut nnz) = (0i64, 0i64);
    check(unsafe { ffi::fcu_matrix_info(m.0, &mut n, &mut nnz) }).unwrap();
    let mut colptr = vec![0usize; n as usize + 1];
    let mut rowidx = vec![0usize; nnz as usize];
    let mut vals = vec![0f64; nnz as usize];
    check(unsafe {
        ffi::fcu_matrix_export_csc(
            ctx().0,
            m.0,
            colptr.as_mut_ptr() as *mut i64,
            rowidx.as_mut_ptr() as *mut i64,
            vals.as_mut_ptr(),
        )
    })
    .unwrap();
    let sym = SymbolicSparseColMat::new_checked(n as usize, n as usize, colptr, None, rowidx);
    SparseColMat::new(sym, vals)
}

fn wrap_csc(a: &SparseColMat<usize, f64>) -> Matrix {
    let mut h = std::ptr::null_mut();
    check(unsafe {
        ffi::fcu_matrix_from_csc(
            ctx().0,
            a.ncols() as i64,
            a.symbolic().col_ptrs().as_ptr() as *const i64,
            a.symbolic().row_indices().as_ptr() as *const i64,
            a.values().as_ptr(),
            &mut h,
        )
    })
    .unwrap();
    Matrix(h)
}

// ---------------------------------------------------------------------------
// Assembly (crates/fenics-assembly)
// ---------------------------------------------------------------------------

/// poisson.rs:23 — same signature, GPU assembly.
pub fn assemble_stiffness_2d(mesh: &TriangleMesh) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let m = matrix(&space(&dm, ffi::FCU_SPACE_P1));
    check(unsafe { ffi::fcu_assemble_stiffness(ctx().0, m.0, std::ptr::null()) }).unwrap();
    export(&m)
}

/// poisson.rs:124 — same signature, GPU assembly.
pub fn assemble_stiffness_3d(mesh: &TetrahedronMesh) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let m = matrix(&space(&dm, ffi::FCU_SPACE_P1));
    check(unsafe { ffi::fcu_assemble_stiffness(ctx().0, m.0, std::ptr::null()) }).unwrap();
    export(&m)
}

/// elasticity.rs:73 — same signature, GPU assembly (3x3 blocks inside).
pub fn assemble_elasticity_stiffness_3d(mesh: &TetrahedronMesh, mat: &ElasticMaterial) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let m = matrix(&space(&dm, ffi::FCU_SPACE_P1_VEC3));
    check(unsafe {
        ffi::fcu_assemble_elasticity(ctx().0, m.0, mat.youngs_modulus, mat.poissons_ratio, std::ptr::null())
    })
    .unwrap();
    export(&m)
}

fn rhs_at_quadrature<const D: usize, const N: usize, F>(
    vertices: &[[f64; D]],
    cells: &[[usize; N]],
    nq: usize,
    f: F,
) -> Vec<f64>
where
    F: Fn([f64; D]) -> f64,
{
    let dm = device_mesh(vertices, cells);
    let s = space(&dm, ffi::FCU_SPACE_P1);
    let mut pts = vec![0.0; cells.len() * nq * D];
    check(unsafe { ffi::fcu_quadrature_points(ctx().0, s.0, pts.as_mut_ptr()) }).unwrap();
    // f is the caller's closure: evaluated on the host where the reference
    // evaluates it (poisson.rs:77,173), then integrated on the device.
    let fq: Vec<f64> = pts.chunks_exact(D).map(|p| f(std::array::from_fn(|d| p[d]))).collect();
    let mut b = vec![0.0; ndofs(&s)];
    check(unsafe { ffi::fcu_assemble_rhs_values(ctx().0, s.0, fq.as_ptr(), b.as_mut_ptr()) }).unwrap();
    b
}

/// poisson.rs:72 — same signature; the 3-point rule's points come from the device.
pub fn assemble_rhs_2d<F>(mesh: &TriangleMesh, f: F) -> Vec<f64>
where
    F: Fn([f64; 2]) -> f64 + Sync + Send,
{
    let _g = SESSION_LOCK.lock().unwrap();
    rhs_at_quadrature(&mesh.vertices, &mesh.cells, 3, f)
}

/// poisson.rs:168 — same signature; the 4-point Keast rule.
pub fn assemble_rhs_3d<F>(mesh: &TetrahedronMesh, f: F) -> Vec<f64>
where
    F: Fn([f64; 3]) -> f64 + Sync + Send,
{
    let _g = SESSION_LOCK.lock().unwrap();
    rhs_at_quadrature(&mesh.vertices, &mesh.cells, 4, f)
}

/// elasticity.rs:153 — same signature.
pub fn assemble_elasticity_body_force_3d(mesh: &TetrahedronMesh, f_body: [f64; 3]) -> Vec<f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let s = space(&dm, ffi::FCU_SPACE_P1_VEC3);
    let mut b = vec![0.0; ndofs(&s)];
    check(unsafe { ffi::fcu_assemble_body_force(ctx().0, s.0, f_body.as_ptr(), b.as_mut_ptr()) }).unwrap();
    b
}

fn boundary_dofs<const D: usize, const N: usize>(v: &[[f64; D]], c: &[[usize; N]]) -> Vec<usize> {
    let dm = device_mesh(v, c);
    let mut count = 0i64;
    check(unsafe { ffi::fcu_boundary_dofs(ctx().0, dm.0, std::ptr::null_mut(), &mut count) }).unwrap();
    let mut out = vec![0usize; count as usize];
    check(unsafe { ffi::fcu_boundary_dofs(ctx().0, dm.0, out.as_mut_ptr() as *mut i64, &mut count) }).unwrap();
    out
}

/// poisson.rs:266 — same signature (sorted, unique).
pub fn boundary_dofs_2d(mesh: &TriangleMesh) -> Vec<usize> {
    let _g = SESSION_LOCK.lock().unwrap();
    boundary_dofs(&mesh.vertices, &mesh.cells)
}

/// poisson.rs:278 — same signature (sorted, unique).
pub fn boundary_dofs_3d(mesh: &TetrahedronMesh) -> Vec<usize> {
    let _g = SESSION_LOCK.lock().unwrap();
    boundary_dofs(&mesh.vertices, &mesh.cells)
}

fn dirichlet(a: &SparseColMat<usize, f64>, b: &[f64], dofs: &[i64], vals: &[f64]) -> (SparseColMat<usize, f64>, Vec<f64>) {
    let m = wrap_csc(a);
    let mut b = b.to_vec();
    check(unsafe {
        ffi::fcu_apply_dirichlet(ctx().0, m.0, b.as_mut_ptr(), dofs.len() as i64, dofs.as_ptr(), vals.as_ptr())
    })
    .unwrap();
    (export(&m), b)
}

/// poisson.rs:222 — same signature.
pub fn apply_dirichlet_bc(a: &SparseColMat<usize, f64>, b: &[f64], bc: &DirichletBC) -> (SparseColMat<usize, f64>, Vec<f64>) {
    let _g = SESSION_LOCK.lock().unwrap();
    let dofs: Vec<i64> = bc.dofs.iter().map(|&d| d as i64).collect();
    dirichlet(a, b, &dofs, &bc.values)
}

/// elasticity.rs:188 — same signature.
pub fn apply_vector_dirichlet_bc(
    a: &SparseColMat<usize, f64>,
    b: &[f64],
    bc: &VectorDirichletBC,
) -> (SparseColMat<usize, f64>, Vec<f64>) {
    let _g = SESSION_LOCK.lock().unwrap();
    let dofs: Vec<i64> = bc.prescribed_dofs.iter().map(|&(d, _)| d as i64).collect();
    let vals: Vec<f64> = bc.prescribed_dofs.iter().map(|&(_, v)| v).collect();
    dirichlet(a, b, &dofs, &vals)
}

/// elasticity.rs:230 — same signature; `StressState` filled from flat arrays.
pub fn compute_element_stresses(mesh: &TetrahedronMesh, u: &[f64], mat: &ElasticMaterial) -> Vec<StressState> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let s = space(&dm, ffi::FCU_SPACE_P1_VEC3);
    let nc = mesh.cells.len();
    let (mut st, mut ep) = (vec![0.0; 9 * nc], vec![0.0; 9 * nc]);
    let (mut vm, mut tr) = (vec![0.0; nc], vec![0.0; nc]);
    check(unsafe {
        ffi::fcu_element_stresses(
            ctx().0,
            s.0,
            mat.youngs_modulus,
            mat.poissons_ratio,
            u.as_ptr(),
            st.as_mut_ptr(),
            ep.as_mut_ptr(),
            vm.as_mut_ptr(),
            tr.as_mut_ptr(),
        )
    })
    .unwrap();
    (0..nc)
        .map(|c| StressState {
            stress: std::array::from_fn(|i| std::array::from_fn(|j| st[9 * c + 3 * i + j])),
            strain: std::array::from_fn(|i| std::array::from_fn(|j| ep[9 * c + 3 * i + j])),
            von_mises: vm[c],
            trace: tr[c],
        })
        .collect()
}

/// mass.rs:10 — same signature, GPU assembly (density 1).
pub fn assemble_mass_2d(mesh: &TriangleMesh) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let m = matrix(&space(&dm, ffi::FCU_SPACE_P1));
    check(unsafe { ffi::fcu_assemble_mass(ctx().0, m.0, 1.0, std::ptr::null()) }).unwrap();
    export(&m)
}

/// mass.rs:47 — same signature, GPU assembly (density 1).
pub fn assemble_mass_3d(mesh: &TetrahedronMesh) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let m = matrix(&space(&dm, ffi::FCU_SPACE_P1));
    check(unsafe { ffi::fcu_assemble_mass(ctx().0, m.0, 1.0, std::ptr::null()) }).unwrap();
    export(&m)
}

/// mass.rs:86 — same signature: the same-component entries of the vector
/// P1 mass, exported as the reference builds them.
pub fn assemble_elasticity_mass_3d(mesh: &TetrahedronMesh, density: f64) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let dm = device_mesh(&mesh.vertices, &mesh.cells);
    let m = matrix(&space(&dm, ffi::FCU_SPACE_P1_VEC3));
    check(unsafe { ffi::fcu_assemble_mass(ctx().0, m.0, density, std::ptr::null()) }).unwrap();
    export(&m)
}

// ---------------------------------------------------------------------------
// Solvers (crates/fenics-solver)
// ---------------------------------------------------------------------------

/// transient.rs:72 — same signature: a + alpha * b on the union of the two
/// patterns, built on the device.
pub fn add_scaled_matrices(
    a: &SparseColMat<usize, f64>,
    b: &SparseColMat<usize, f64>,
    alpha: f64,
) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let (ma, mb) = (wrap_csc(a), wrap_csc(b));
    let mut h = std::ptr::null_mut();
    check(unsafe { ffi::fcu_matrix_add_scaled_union(ctx().0, ma.0, mb.0, alpha, &mut h) })
        .expect("Failed to build combined sparse matrix");
    export(&Matrix(h))
}

/// eigen.rs:51 — same signature: constrained rows and columns folded on the
/// device, a unit (or zero) diagonal on them, zero entries dropped.
pub fn fold_dirichlet(mat: &SparseColMat<usize, f64>, fixed_dofs: &[usize], unit_diag: bool) -> SparseColMat<usize, f64> {
    let _g = SESSION_LOCK.lock().unwrap();
    let m = wrap_csc(mat);
    let fixed: Vec<i64> = fixed_dofs.iter().map(|&d| d as i64).collect();
    check(unsafe {
        ffi::fcu_matrix_fold_dirichlet(ctx().0, m.0, fixed.len() as i64, fixed.as_ptr(), unit_diag as c_int)
    })
    .unwrap();
    export(&m)
}


/// cg.rs:40 — same signature and Result semantics: Err carries the
/// reference's strings ("CG failed to converge ...", "Breakdown in CG ...").
pub fn solve_cg(
    a: &SparseColMat<usize, f64>,
    b: &[f64],
    x0: Option<&[f64]>,
    tol: f64,
    max_iter: usize,
) -> Result<(Vec<f64>, usize, f64), String> {
    let _g = SESSION_LOCK.lock().unwrap();
    let m = wrap_csc(a);
    let mut x = vec![0.0; b.len()];
    let mut info = ffi::fcu_solve_info::default();
    let rc = unsafe {
        ffi::fcu_pcg(
            ctx().0,
            m.0,
            b.as_ptr(),
            x0.map_or(std::ptr::null(), |v| v.as_ptr()),
            x.as_mut_ptr(),
            tol,
            max_iter as i64,
            ffi::FCU_FP64,
            &mut info,
        )
    };
    check(rc)?;
    Ok((x, info.iterations as usize, info.residual))
}

/// The fields of fenics-solver's GpuSolveResult (gpu.rs:24-34).
#[derive(Clone, Debug)]
pub struct GpuSolveResult {
    pub solution: Vec<f64>,
    pub iterations: usize,
    pub final_residual: f64,
    pub wall_ms: f64,
    pub kernel_ms: f64,
    pub gflops: f64,
    pub effective_bw_gbps: f64,
    pub devices_used: Vec<String>,
}

/// gpu.rs:1145 — same signature. Ok at the iteration limit and Ok with a
/// zero solution for b = 0, as the reference returns.
#[allow(clippy::too_many_arguments)]
pub fn solve_csr_cg_gpu(
    row_ptr: &[u32],
    col_idx: &[u32],
    vals: &[f64],
    inv_diag: &[f64],
    b: &[f64],
    x0: Option<&[f64]>,
    rtol: f64,
    max_iter: usize,
    _device_index: Option<usize>,
) -> Result<GpuSolveResult, String> {
    let _g = SESSION_LOCK.lock().unwrap();
    let n = b.len();
    let mut x = vec![0.0; n];
    let mut info = ffi::fcu_solve_info::default();
    let t0 = std::time::Instant::now();
    check(unsafe {
        ffi::fcu_solve_csr_cg(
            ctx().0,
            n as i64,
            row_ptr.as_ptr(),
            col_idx.as_ptr(),
            vals.as_ptr(),
            inv_diag.as_ptr(),
            b.as_ptr(),
            x0.map_or(std::ptr::null(), |v| v.as_ptr()),
            rtol,
            max_iter as i64,
            x.as_mut_ptr(),
            &mut info,
        )
    })?;
    let nnz = *row_ptr.last().unwrap_or(&0) as f64;
    Ok(GpuSolveResult {
        solution: x,
        iterations: info.iterations as usize,
        final_residual: info.rel_residual,
        wall_ms: t0.elapsed().as_secs_f64() * 1e3,
        kernel_ms: info.kernel_ms,
        gflops: if info.kernel_ms > 0.0 {
            (2.0 * nnz + 10.0 * n as f64) * info.iterations as f64 / (info.kernel_ms * 1e-3) / 1e9
        } else {
            0.0
        },
        effective_bw_gbps: info.effective_bw_gbps,
        devices_used: vec![device_name(0)],
    })
}

fn device_name(device: c_int) -> String {
    let mut buf = [0 as std::os::raw::c_char; 256];
    if unsafe { ffi::fcu_device_name(device, buf.as_mut_ptr(), buf.len()) } != ffi::FCU_OK {
        return format!("cuda:{device}");
    }
    unsafe { CStr::from_ptr(buf.as_ptr()).to_string_lossy().into_owned() }
}

// ---------------------------------------------------------------------------
// Transient heat, vibration modes, 3x3 block CSR (crates/fenics-solver)
// ---------------------------------------------------------------------------

/// transient.rs:13 — the two schemes.
#[derive(Clone, Copy, Debug, PartialEq)]
pub enum TimeSteppingScheme {
    BackwardEuler,
    CrankNicolson,
}

/// transient.rs:21 — same fields; `step` runs on the device.
pub struct TransientHeatSolver {
    pub scheme: TimeSteppingScheme,
    pub dt: f64,
}

fn same_layout(a: &SparseColMat<usize, f64>, b: &SparseColMat<usize, f64>) -> bool {
    a.ncols() == b.ncols()
        && a.symbolic().col_ptrs() == b.symbolic().col_ptrs()
        && a.symbolic().row_indices() == b.symbolic().row_indices()
}

impl TransientHeatSolver {
    pub fn new(scheme: TimeSteppingScheme, dt: f64) -> Self {
        Self { scheme, dt }
    }

    /// transient.rs:32 — same signature. The left-hand system is solved by
    /// FP64 Jacobi-PCG to 1e-12 from u_n, where the reference factorises it
    /// densely. Operands of different patterns are first placed on their
    /// union (each plus 0 times the other, which keeps its values).
    pub fn step(
        &self,
        mass_mat: &SparseColMat<usize, f64>,
        stiff_mat: &SparseColMat<usize, f64>,
        u_n: &[f64],
        f_n: &[f64],
        f_next: &[f64],
    ) -> Result<Vec<f64>, String> {
        let _g = SESSION_LOCK.lock().unwrap();
        let (mut m, mut k) = (wrap_csc(mass_mat), wrap_csc(stiff_mat));
        if !same_layout(mass_mat, stiff_mat) {
            let (mut mu, mut ku) = (std::ptr::null_mut(), std::ptr::null_mut());
            check(unsafe { ffi::fcu_matrix_add_scaled_union(ctx().0, m.0, k.0, 0.0, &mut mu) })?;
            check(unsafe { ffi::fcu_matrix_add_scaled_union(ctx().0, k.0, m.0, 0.0, &mut ku) })?;
            m = Matrix(mu);
            k = Matrix(ku);
        }
        let scheme = match self.scheme {
            TimeSteppingScheme::BackwardEuler => ffi::FCU_BACKWARD_EULER,
            TimeSteppingScheme::CrankNicolson => ffi::FCU_CRANK_NICOLSON,
        };
        let mut ts = std::ptr::null_mut();
        check(unsafe { ffi::fcu_transient_create(ctx().0, m.0, k.0, scheme, self.dt, &mut ts) })?;
        let mut u = vec![0.0; u_n.len()];
        let mut info = ffi::fcu_solve_info::default();
        let rc = unsafe {
            ffi::fcu_transient_step(
                ctx().0,
                ts,
                u_n.as_ptr(),
                f_n.as_ptr(),
                f_next.as_ptr(),
                u.as_mut_ptr(),
                1e-12,
                (10 * u_n.len()).max(1000) as i64,
                ffi::FCU_FP64,
                &mut info,
            )
        };
        unsafe { ffi::fcu_transient_destroy(ts) };
        check(rc)?;
        Ok(u)
    }
}

/// eigen.rs:10 — same fields.
#[derive(Clone, Debug)]
pub struct VibrationMode {
    pub frequency_hz: f64,
    pub omega_rad_s: f64,
    pub eigenvalue: f64,
    pub mode_shape: Vec<f64>,
}

type InnerFn<'a> = &'a dyn Fn(&[f64], &[f64]) -> Result<Vec<f64>, String>;

struct InnerCall<'a> {
    f: InnerFn<'a>,
    err: Option<String>,
}

/// The C callback behind `inner`: b and x0 arrive in device memory; they are
/// copied to the host, the closure runs, and its solution is copied back.
unsafe extern "C" fn inner_trampoline(user: *mut c_void, n: i64, b: *const f64, x0: *const f64, x: *mut f64) -> c_int {
    let call = &mut *(user as *mut InnerCall);
    let n = n as usize;
    let (mut hb, mut hx0) = (vec![0.0f64; n], vec![0.0f64; n]);
    let bytes = 8 * n;
    if ffi::fcu_buffer_copy(ctx().0, hb.as_mut_ptr() as *mut c_void, b as *const c_void, bytes) != ffi::FCU_OK
        || ffi::fcu_buffer_copy(ctx().0, hx0.as_mut_ptr() as *mut c_void, x0 as *const c_void, bytes) != ffi::FCU_OK
    {
        call.err = Some("inner solve: device copy failed".to_string());
        return ffi::FCU_ERR_CUDA;
    }
    match (call.f)(&hb, &hx0) {
        Ok(v) if v.len() == n => {
            ffi::fcu_buffer_copy(ctx().0, x as *mut c_void, v.as_ptr() as *const c_void, bytes)
        }
        Ok(_) => {
            call.err = Some("inner solve returned a vector of the wrong length".to_string());
            ffi::FCU_ERR_BAD_ARG
        }
        Err(e) => {
            call.err = Some(e);
            ffi::FCU_ERR_NO_CONVERGENCE
        }
    }
}

fn vibration_modes(
    k: &SparseColMat<usize, f64>,
    m: &SparseColMat<usize, f64>,
    fixed_dofs: &[usize],
    num_modes: usize,
    max_power_iters: usize,
    tol: f64,
    inner: Option<InnerFn>,
) -> Result<Vec<VibrationMode>, String> {
    let _g = SESSION_LOCK.lock().unwrap();
    let (mk, mm) = (wrap_csc(k), wrap_csc(m));
    let n = k.nrows();
    let fixed: Vec<i64> = fixed_dofs.iter().map(|&d| d as i64).collect();
    let mut eig = vec![0.0; num_modes];
    let mut shapes = vec![0.0; num_modes * n];
    let mut info = ffi::fcu_solve_info::default();
    let mut call = inner.map(|f| InnerCall { f, err: None });
    let (cb, user): (ffi::fcu_inner_solve, *mut c_void) = match call.as_mut() {
        Some(c) => (Some(inner_trampoline), c as *mut InnerCall as *mut c_void),
        None => (None, std::ptr::null_mut()),
    };
    let rc = unsafe {
        ffi::fcu_vibration_modes(
            ctx().0,
            mk.0,
            mm.0,
            fixed.len() as i64,
            fixed.as_ptr(),
            num_modes as i64,
            max_power_iters as i64,
            tol,
            1e-9,
            1000,
            ffi::FCU_FP64,
            cb,
            user,
            eig.as_mut_ptr(),
            shapes.as_mut_ptr(),
            std::ptr::null_mut(),
            &mut info,
        )
    };
    if rc != ffi::FCU_OK {
        if let Some(e) = call.and_then(|c| c.err) {
            return Err(e);
        }
        check(rc)?;
    }
    Ok((0..num_modes)
        .map(|i| {
            let omega = eig[i].sqrt();
            VibrationMode {
                frequency_hz: omega / (2.0 * std::f64::consts::PI),
                omega_rad_s: omega,
                eigenvalue: eig[i],
                mode_shape: shapes[i * n..(i + 1) * n].to_vec(),
            }
        })
        .collect())
}

/// eigen.rs:282 — same signature: inverse power iteration on the device,
/// inner solve FP64 Jacobi-PCG at 1e-9 (the reference's default).
pub fn solve_vibration_modes(
    k: &SparseColMat<usize, f64>,
    m: &SparseColMat<usize, f64>,
    fixed_dofs: &[usize],
    num_modes: usize,
    max_power_iters: usize,
    tol: f64,
) -> Result<Vec<VibrationMode>, String> {
    vibration_modes(k, m, fixed_dofs, num_modes, max_power_iters, tol, None)
}

/// eigen.rs:94 — same signature: the caller's inner solve (K x = b from x0)
/// is called for every power iteration, on host vectors.
pub fn solve_vibration_modes_with_inner(
    k: &SparseColMat<usize, f64>,
    m: &SparseColMat<usize, f64>,
    fixed_dofs: &[usize],
    num_modes: usize,
    max_power_iters: usize,
    tol: f64,
    inner: &dyn Fn(&[f64], &[f64]) -> Result<Vec<f64>, String>,
) -> Result<Vec<VibrationMode>, String> {
    vibration_modes(k, m, fixed_dofs, num_modes, max_power_iters, tol, Some(inner))
}

/// gpu.rs:434 — a resident 3x3 block CSR matrix (its inverse diagonal blocks
/// optional).
pub struct GpuBsr3Context {
    m: Matrix,
    nnz_blocks: usize,
    device_name: String,
}

unsafe impl Send for GpuBsr3Context {}

impl GpuBsr3Context {
    /// gpu.rs:453 — same signature (an empty dinv_flat: none).
    pub fn new(
        n_nodes: usize,
        row_ptr: &[u32],
        cols: &[u32],
        vals_flat: &[f64],
        dinv_flat: &[f64],
        _device_index: Option<usize>,
    ) -> Result<Self, String> {
        let _g = SESSION_LOCK.lock().unwrap();
        let mut h = std::ptr::null_mut();
        check(unsafe {
            ffi::fcu_bsr3_create(
                ctx().0,
                n_nodes as i64,
                row_ptr.as_ptr(),
                cols.as_ptr(),
                vals_flat.as_ptr(),
                if dinv_flat.is_empty() { std::ptr::null() } else { dinv_flat.as_ptr() },
                &mut h,
            )
        })?;
        Ok(Self { m: Matrix(h), nnz_blocks: cols.len(), device_name: device_name(0) })
    }

    pub fn device_name(&self) -> &str {
        &self.device_name
    }

    pub fn nnz_blocks(&self) -> usize {
        self.nnz_blocks
    }

    /// gpu.rs:505 — y = A x.
    pub fn spmv(&self, x: &[f64], y: &mut [f64]) -> Result<(), String> {
        let _g = SESSION_LOCK.lock().unwrap();
        check(unsafe { ffi::fcu_spmv(ctx().0, self.m.0, x.as_ptr(), y.as_mut_ptr()) })
    }

    /// gpu.rs:547 — damped block-Jacobi sweeps.
    pub fn jacobi_smooth(
        &self,
        r: &[f64],
        z: &mut [f64],
        sweeps: usize,
        omega: f64,
        zero_initial_z: bool,
    ) -> Result<(), String> {
        let _g = SESSION_LOCK.lock().unwrap();
        check(unsafe {
            ffi::fcu_bsr3_jacobi_smooth(
                ctx().0,
                self.m.0,
                r.as_ptr(),
                z.as_mut_ptr(),
                sweeps as i64,
                omega,
                zero_initial_z as c_int,
            )
        })
    }
}

/// gpu.rs:775 — same signature: block-Jacobi PCG in FP64.
#[allow(clippy::too_many_arguments)]
pub fn solve_bsr3_pcg_gpu(
    n_nodes: usize,
    row_ptr: &[u32],
    cols: &[u32],
    vals_flat: &[f64],
    dinv_flat: &[f64],
    b: &[f64],
    x0: Option<&[f64]>,
    rtol: f64,
    max_iter: usize,
    _device_index: Option<usize>,
) -> Result<GpuSolveResult, String> {
    let _g = SESSION_LOCK.lock().unwrap();
    let mut x = vec![0.0; b.len()];
    let mut info = ffi::fcu_solve_info::default();
    let t0 = std::time::Instant::now();
    check(unsafe {
        ffi::fcu_solve_bsr3_pcg(
            ctx().0,
            n_nodes as i64,
            row_ptr.as_ptr(),
            cols.as_ptr(),
            vals_flat.as_ptr(),
            if dinv_flat.is_empty() { std::ptr::null() } else { dinv_flat.as_ptr() },
            b.as_ptr(),
            x0.map_or(std::ptr::null(), |v| v.as_ptr()),
            rtol,
            max_iter as i64,
            x.as_mut_ptr(),
            &mut info,
        )
    })?;
    Ok(GpuSolveResult {
        solution: x,
        iterations: info.iterations as usize,
        final_residual: info.rel_residual,
        wall_ms: t0.elapsed().as_secs_f64() * 1e3,
        kernel_ms: info.kernel_ms,
        gflops: 0.0,
        effective_bw_gbps: info.effective_bw_gbps,
        devices_used: vec![device_name(0)],
    })
}

// ---------------------------------------------------------------------------
// Device-resident pipeline (no reference counterpart)
// ---------------------------------------------------------------------------

/// Precision of a device solve.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum Precision {
    /// FP64 Jacobi-PCG, the arithmetic of cg.rs:40-149.
    Fp64,
    /// FP32 SpMV and vector updates inside FP64 residual replacement; the
    /// stopping test is the FP64 residual ||b - A x|| / ||b||.
    Mixed,
}

impl Precision {
    fn code(self) -> c_int {
        match self {
            Precision::Fp64 => ffi::FCU_FP64,
            Precision::Mixed => ffi::FCU_MIXED,
        }
    }
}

/// A vector-P1 elasticity system kept on the device: the mesh, its dof map
/// and pattern, the FP64 + FP32 stiffness and the eliminated Dirichlet dofs.
/// `solve_elasticity_3d` (elasticity_solver.rs:31-72) without the host CSC.
pub struct ElasticityProblem {
    _mesh: Mesh,
    space: Space,
    k: Matrix,
    clamp: Vec<i64>,
    ncells: usize,
}

impl ElasticityProblem {
    pub fn new(mesh: &TetrahedronMesh, clamp_dofs: &[usize]) -> Self {
        let _g = SESSION_LOCK.lock().unwrap();
        let dm = device_mesh(&mesh.vertices, &mesh.cells);
        let s = space(&dm, ffi::FCU_SPACE_P1_VEC3);
        let k = matrix(&s);
        ElasticityProblem {
            _mesh: dm,
            space: s,
            k,
            clamp: clamp_dofs.iter().map(|&d| d as i64).collect(),
            ncells: mesh.cells.len(),
        }
    }

    /// Assemble K (with per-cell moduli when `cell_e` is given), eliminate
    /// the clamped dofs from K and `load`, and solve K u = load.
    pub fn solve(
        &mut self,
        mat: &ElasticMaterial,
        cell_e: Option<&[f64]>,
        load: &[f64],
        tol: f64,
        max_iter: usize,
        precision: Precision,
    ) -> Result<(Vec<f64>, ffi::fcu_solve_info), String> {
        let _g = SESSION_LOCK.lock().unwrap();
        if let Some(e) = cell_e {
            assert_eq!(e.len(), self.ncells, "one modulus per cell");
        }
        check(unsafe {
            ffi::fcu_assemble_elasticity(
                ctx().0,
                self.k.0,
                mat.youngs_modulus,
                mat.poissons_ratio,
                cell_e.map_or(std::ptr::null(), |v| v.as_ptr()),
            )
        })?;
        let mut b = load.to_vec();
        let zeros = vec![0.0; self.clamp.len()];
        check(unsafe {
            ffi::fcu_apply_dirichlet(
                ctx().0,
                self.k.0,
                b.as_mut_ptr(),
                self.clamp.len() as i64,
                self.clamp.as_ptr(),
                zeros.as_ptr(),
            )
        })?;
        let mut u = vec![0.0; b.len()];
        let mut info = ffi::fcu_solve_info::default();
        check(unsafe {
            ffi::fcu_pcg(
                ctx().0,
                self.k.0,
                b.as_ptr(),
                std::ptr::null(),
                u.as_mut_ptr(),
                tol,
                max_iter as i64,
                precision.code(),
                &mut info,
            )
        })?;
        Ok((u, info))
    }
}

/// Objective of the adjoint pair.
pub enum Objective {
    /// J = f^T u (λ = u: no second solve).
    Compliance,
    /// J = c^T u for a fixed vector c (one adjoint solve with the same operator).
    Linear(Vec<f64>),
}

/// Forward/backward pair of the adjoint sensitivities for E_e = E0 θ_e³
/// (the role a torch.autograd.Function plays in Python): `forward(θ)` solves
/// K(θ) u = f and returns J; `backward(dJ)` returns dJ · ∂J/∂θ with
/// ∂J/∂θ_e = −λ_eᵀ (3 θ_e² E0 K_e¹) u_e, K_e¹ recomputed per cell on the device.
pub struct ElasticityAdjoint {
    problem: ElasticityProblem,
    nu: f64,
    e0: f64,
    load: Vec<f64>,
    objective: Objective,
    tol: f64,
    precision: Precision,
    theta: Vec<f64>,
    u: Vec<f64>,
}

impl ElasticityAdjoint {
    pub fn new(
        mesh: &TetrahedronMesh,
        nu: f64,
        e0: f64,
        load: Vec<f64>,
        clamp_dofs: &[usize],
        objective: Objective,
        tol: f64,
        precision: Precision,
    ) -> Self {
        ElasticityAdjoint {
            problem: ElasticityProblem::new(mesh, clamp_dofs),
            nu,
            e0,
            load,
            objective,
            tol,
            precision,
            theta: Vec::new(),
            u: Vec::new(),
        }
    }

    fn material(&self) -> ElasticMaterial {
        ElasticMaterial { youngs_modulus: self.e0, poissons_ratio: self.nu }
    }

    pub fn forward(&mut self, theta: &[f64]) -> Result<f64, String> {
        let e: Vec<f64> = theta.iter().map(|t| self.e0 * t * t * t).collect();
        let mat = self.material();
        let (u, _) = self.problem.solve(&mat, Some(&e), &self.load, self.tol, 100_000, self.precision)?;
        let c: &[f64] = match &self.objective {
            Objective::Compliance => &self.load,
            Objective::Linear(c) => c,
        };
        let j = c.iter().zip(&u).map(|(a, b)| a * b).sum();
        self.theta = theta.to_vec();
        self.u = u;
        Ok(j)
    }

    pub fn backward(&mut self, dj: f64) -> Result<Vec<f64>, String> {
        assert!(!self.u.is_empty(), "backward before forward");
        let lam = match &self.objective {
            Objective::Compliance => self.u.clone(),
            Objective::Linear(c) => {
                let e: Vec<f64> = self.theta.iter().map(|t| self.e0 * t * t * t).collect();
                let mat = self.material();
                let c = c.clone();
                self.problem.solve(&mat, Some(&e), &c, self.tol, 100_000, self.precision)?.0
            }
        };
        let _g = SESSION_LOCK.lock().unwrap();
        let mut g = vec![0.0; self.theta.len()];
        check(unsafe {
            ffi::fcu_adjoint_gradient(
                ctx().0,
                self.problem.space.0,
                self.e0,
                self.nu,
                self.theta.as_ptr(),
                self.u.as_ptr(),
                lam.as_ptr(),
                g.as_mut_ptr(),
            )
        })?;
        g.iter_mut().for_each(|v| *v *= dj);
        Ok(g)
    }
}
