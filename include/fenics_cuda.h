/*
 * fenics_cuda.h — C ABI of the B200 (sm_100a) FEM assembly + Jacobi-PCG library.
 *
 * This is the drop-in boundary for the hot path of GlassOnTin/fenics-rs:
 * the crates/fenics-assembly `assemble_*` / `apply_*dirichlet_bc` /
 * `boundary_dofs_*` functions and the crates/fenics-solver `solve_cg` /
 * `solve_csr_cg_gpu` entry points. Each declaration below names the
 * reference function it replaces (file:line inside the reference project).
 *
 * Conventions
 *  - Every call returns an int status (FCU_OK = 0); fcu_last_error(ctx)
 *    gives the message of the last failure on that context.
 *  - Array arguments may be host or device pointers (CUDA unified
 *    addressing tells them apart). Host outputs are complete when the call
 *    returns; calls whose inputs and outputs are all device memory are
 *    asynchronous on the context's stream.
 *  - Index arrays exchanged with the caller are int64 (Rust `usize`),
 *    except the u32 CSR of fcu_solve_csr_cg, which mirrors gpu.rs.
 *  - Matrices are exported in faer SparseColMat layout: column pointers,
 *    row indices sorted inside each column, explicit zeros kept.
 *  - Handles own their device memory. One context per host thread, or
 *    external synchronisation.
 */
#ifndef FENICS_CUDA_H
#define FENICS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define FCU_OK 0
#define FCU_ERR_CUDA 1           /* a CUDA runtime call failed                   */
#define FCU_ERR_BAD_ARG 2        /* invalid sizes, indices or handles            */
#define FCU_ERR_NO_CONVERGENCE 3 /* cg.rs:139-148 "CG failed to converge"       */
#define FCU_ERR_BREAKDOWN 4      /* cg.rs:102-107 "Breakdown in CG"             */
#define FCU_ERR_UNSUPPORTED 5    /* mesh outside the limits of a kernel          */

/* ---- space kinds ---------------------------------------------------------- */
#define FCU_SPACE_P1 1      /* scalar P1 on triangles (dim 2) or tetrahedra (dim 3) */
#define FCU_SPACE_P2 2      /* scalar P2 on tetrahedra: vertex dofs, then edges     */
#define FCU_SPACE_P1_VEC3 3 /* vector P1 on tetrahedra, dof = 3*vertex + component  */
/* P2 on the caller's 10-node tetrahedra (fcu_space_create_p2_nodes): dof =
 * node (scalar) or 3*node + component (vector); mass and stiffness only. */
#define FCU_SPACE_P2_NODES 4
#define FCU_SPACE_P2_NODES_VEC3 5

/* ---- solver precision ----------------------------------------------------- */
#define FCU_FP64 0  /* FP64 Jacobi-PCG (cg.rs:40-149 arithmetic)                 */
#define FCU_MIXED 1 /* FP32 SpMV/axpy, FP64 dots, FP64 residual + refinement      */

/* ---- analytic sources for fcu_assemble_rhs_source ------------------------- */
#define FCU_SRC_CONSTANT 0    /* f = p[0]                                       */
#define FCU_SRC_SIN_PRODUCT 1 /* f = p[0] * prod_d sin(p[1] * x_d)              */
#define FCU_SRC_NODAL 2       /* f = sum_j f_j phi_j, nodal values in `values`  */

/* ---- time-stepping schemes (TimeSteppingScheme, transient.rs:11-18) -------- */
#define FCU_BACKWARD_EULER 0
#define FCU_CRANK_NICOLSON 1

typedef struct fcu_ctx_s* fcu_ctx;
typedef struct fcu_mesh_s* fcu_mesh;
typedef struct fcu_space_s* fcu_space;
typedef struct fcu_matrix_s* fcu_matrix;
typedef struct fcu_transient_s* fcu_transient;

/* Per-solve report; the fields of GpuSolveResult (gpu.rs:24-34) that are
 * numbers, plus status and the absolute residual solve_cg returns. */
typedef struct {
  int64_t iterations;     /* inner PCG iterations                               */
  int64_t outer_updates;  /* FP64 residual replacements (FCU_MIXED)             */
  double residual;        /* absolute ||b - A x||_2 (cg.rs:121)                 */
  double rel_residual;    /* residual / ||b||_2 (gpu.rs:1360-1363)              */
  double kernel_ms;       /* device time of the solve (CUDA events)             */
  double effective_bw_gbps; /* algorithmic bytes / kernel_ms                    */
  int status;             /* FCU_OK, FCU_ERR_NO_CONVERGENCE or FCU_ERR_BREAKDOWN */
} fcu_solve_info;

/* ---- context (replaces CudaSession, gpu.rs:325-430) ----------------------- */
int fcu_ctx_create(int device, fcu_ctx* out);
void fcu_ctx_destroy(fcu_ctx ctx);
const char* fcu_last_error(fcu_ctx ctx);
int fcu_ctx_synchronize(fcu_ctx ctx);
void* fcu_ctx_stream(fcu_ctx ctx); /* the cudaStream_t all calls run on */
/* Number of library kernels launched on this context since creation. */
int64_t fcu_ctx_kernel_launches(fcu_ctx ctx);

/* ---- meshes (SimplicialMesh<DIM,NODES>, mesh.rs:11-20) -------------------- */
/* coords: nv*dim doubles (Vec<[f64;DIM]>); cells: nc*(dim+1) int64 (Vec<[usize;NODES]>). */
int fcu_mesh_create(fcu_ctx ctx, int dim, int64_t nv, const double* coords, int64_t nc,
                    const int64_t* cells, fcu_mesh* out);
void fcu_mesh_destroy(fcu_mesh mesh);
/* Cells with |det J| < 1e-14 (skipped by every assembler, poisson.rs:42-45). */
int fcu_mesh_num_degenerate(fcu_ctx ctx, fcu_mesh mesh, int64_t* count);

/* boundary_dofs_2d / boundary_dofs_3d (poisson.rs:266-287): sorted, unique
 * vertices of facets that belong to exactly one cell. out==NULL queries count. */
int fcu_boundary_dofs(fcu_ctx ctx, fcu_mesh mesh, int64_t* out, int64_t* count);

/* extract_boundary_facets (mesh.rs:79-113, 145-210). Facets are returned
 * sorted by their sorted vertex triple (the reference's HashMap order is
 * unspecified); 3D facets are oriented outward as in mesh.rs:166-192.
 * verts: nf*dim; cell, local: nf each (may be NULL). out==NULL queries count. */
int fcu_boundary_facets(fcu_ctx ctx, fcu_mesh mesh, int64_t* verts, int64_t* cell, int64_t* local,
                        int64_t* count);

/* ---- function spaces: dof map + sparsity pattern ----------------------- */
int fcu_space_create(fcu_ctx ctx, fcu_mesh mesh, int kind, fcu_space* out);
void fcu_space_destroy(fcu_space space);
/* ndofs, stored entries of the raw (pre-Dirichlet) matrix in reference pattern
 * terms, and P2 edge count (0 otherwise). Any pointer may be NULL. */
int fcu_space_info(fcu_space space, int64_t* ndofs, int64_t* nnz, int64_t* nedges);
/* P2: cell dof map (nc*10, P2Tetrahedron local order, lagrange.rs:286-299) and
 * edge vertex pairs (nedges*2); either may be NULL. */
int fcu_space_p2_dofmap(fcu_ctx ctx, fcu_space space, int64_t* cell_dofs, int64_t* edge_verts);
/* A P2 space on the caller's numbering (assemble_elasticity_mass_p2_3d,
 * mass.rs:137-180): `mesh` holds every P2 node as a vertex and each cell's
 * four corners as its tetrahedron; cells10 (nc*10) gives the ten nodes of
 * each cell in P2Tetrahedron order (4 corners, then edges 01, 12, 02, 03,
 * 13, 23), its first four equal to the mesh cell. vec3 != 0 gives
 * FCU_SPACE_P2_NODES_VEC3. */
int fcu_space_create_p2_nodes(fcu_ctx ctx, fcu_mesh mesh, const int64_t* cells10, int vec3, fcu_space* out);
/* Boundary dofs of the space: P1 = boundary_dofs_*; P2 = boundary vertices and
 * boundary edges, sorted. out==NULL queries count. */
int fcu_space_boundary_dofs(fcu_ctx ctx, fcu_space space, int64_t* out, int64_t* count);

/* ---- matrices -------------------------------------------------------------- */
/* Allocate a matrix on the space's pattern (values unset). */
int fcu_matrix_create(fcu_ctx ctx, fcu_space space, fcu_matrix* out);
/* Wrap a caller CSC (faer SparseColMat<usize,f64>) for fcu_pcg (cg.rs:40). */
int fcu_matrix_from_csc(fcu_ctx ctx, int64_t n, const int64_t* colptr, const int64_t* rowidx,
                        const double* vals, fcu_matrix* out);
void fcu_matrix_destroy(fcu_matrix m);
/* Order and stored entries (reference pattern: after Dirichlet if applied). */
int fcu_matrix_info(fcu_matrix m, int64_t* n, int64_t* nnz);
/* Export as faer CSC (colptr n+1, rowidx nnz, vals nnz); any may be NULL. */
int fcu_matrix_export_csc(fcu_ctx ctx, fcu_matrix m, int64_t* colptr, int64_t* rowidx, double* vals);

/* assemble_stiffness_2d / assemble_stiffness_3d (poisson.rs:23-69, 124-165)
 * for FCU_SPACE_P1; P2 stiffness for FCU_SPACE_P2 (no reference counterpart).
 * cell_coef (nc, may be NULL) multiplies each cell's contribution (kappa_e).
 * Writes the FP64 values and their FP32 copy. */
int fcu_assemble_stiffness(fcu_ctx ctx, fcu_matrix m, const double* cell_coef);
/* assemble_elasticity_stiffness_3d (elasticity.rs:73-149) for FCU_SPACE_P1_VEC3.
 * cell_E (nc, may be NULL) overrides Young's modulus per cell. ElasticMaterial::new
 * rejects nu outside (-1, 0.5) (elasticity.rs:23-26): FCU_ERR_BAD_ARG here. */
int fcu_assemble_elasticity(fcu_ctx ctx, fcu_matrix m, double E, double nu, const double* cell_E);
/* Mass matrices (mass.rs:10-250): assemble_mass_2d / assemble_mass_3d on
 * FCU_SPACE_P1 (rho = 1 gives the reference), assemble_elasticity_mass_3d on
 * FCU_SPACE_P1_VEC3 (rho = density), and for FCU_SPACE_P2 the scalar mass
 * from the exact reference-tetrahedron products of
 * assemble_elasticity_mass_p2_3d (mass.rs:137-250; one component of it).
 * cell_coef (nc, may be NULL) multiplies each cell's contribution. The
 * vector mass exports only its same-component entries, as the reference
 * builds it; it is stored in the space's 3x3 blocks (zeros elsewhere), so it
 * combines with the stiffness on that space. */
int fcu_assemble_mass(fcu_ctx ctx, fcu_matrix m, double rho, const double* cell_coef);

/* A new matrix on src's pattern with a copy of its values and Dirichlet state. */
int fcu_matrix_clone(fcu_ctx ctx, fcu_matrix src, fcu_matrix* out);
/* add_scaled_matrices (transient.rs:72-97): out = a + alpha * b entry by
 * entry (each entry a + (alpha * b), as the triplet sum rounds it). a, b and
 * out share one pattern (one space, or identical wrapped CSC layouts) and
 * carry no eliminated Dirichlet dofs, else FCU_ERR_UNSUPPORTED
 * (fcu_matrix_add_scaled_union combines any two); out may be a or b. */
int fcu_matrix_add_scaled(fcu_ctx ctx, fcu_matrix out, fcu_matrix a, fcu_matrix b, double alpha);
/* add_scaled_matrices (transient.rs:72-97) on operands of any patterns: a new
 * matrix *out holding a + alpha * b on the union of the two exported CSC
 * patterns (an entry held by both is a + (alpha * b), one held by b alone
 * alpha * b, explicit zeros kept), as the reference's triplet build gives.
 * a and b must have the same order; either may carry Dirichlet or folded
 * state (its exported matrix is the operand). *out is a wrapped CSC matrix:
 * destroy it with fcu_matrix_destroy. */
int fcu_matrix_add_scaled_union(fcu_ctx ctx, fcu_matrix a, fcu_matrix b, double alpha, fcu_matrix* out);
/* Every value times s (the diffusivity scaling of heat_solver.rs:48-57). */
int fcu_matrix_scale(fcu_ctx ctx, fcu_matrix m, double s);
/* fold_dirichlet (eigen.rs:55-79), in place: entries on a fixed row or column
 * become zero, a fixed diagonal 1 (unit_diag != 0) or 0; dofs >= n are
 * ignored. The exported pattern then omits every zero value, as the
 * reference's rebuilt matrix does. Idempotent. */
int fcu_matrix_fold_dirichlet(fcu_ctx ctx, fcu_matrix m, int64_t nfixed, const int64_t* fixed, int unit_diag);

/* apply_dirichlet_bc / apply_vector_dirichlet_bc (poisson.rs:222-263,
 * elasticity.rs:188-227), in place on m and b: b_i -= a_ik g_k for free rows,
 * Dirichlet rows/columns eliminated, unit diagonal (repeated dofs add up),
 * b_k = g_k (last occurrence wins). */
int fcu_apply_dirichlet(fcu_ctx ctx, fcu_matrix m, double* b, int64_t nbc, const int64_t* dofs,
                        const double* vals);

/* ---- right-hand sides ------------------------------------------------------ */
/* Physical quadrature points of assemble_rhs_2d/3d (poisson.rs:77,173):
 * nc*3 points (2D) or nc*4 points (3D), dim doubles each; for P2 the same
 * 4-point rule. Lets a host closure f be evaluated where the reference does. */
int fcu_quadrature_points(fcu_ctx ctx, fcu_space space, double* out);
/* assemble_rhs_2d / assemble_rhs_3d (poisson.rs:72-121, 168-218) with f given
 * at the quadrature points above (fq: nc*nq). P2: same rule, P2 basis. */
int fcu_assemble_rhs_values(fcu_ctx ctx, fcu_space space, const double* fq, double* b);
/* Same integral with f evaluated on the device (FCU_SRC_*). */
int fcu_assemble_rhs_source(fcu_ctx ctx, fcu_space space, int source, const double* params,
                            const double* values, double* b);
/* assemble_elasticity_body_force_3d (elasticity.rs:153-185). */
int fcu_assemble_body_force(fcu_ctx ctx, fcu_space space, const double* f_body3, double* b);
/* assemble_surface_traction_3d (boundary.rs:48-108): facets nf*3 vertex ids,
 * tq = traction at each facet's three edge midpoints (nf*3*3). b is overwritten. */
int fcu_assemble_surface_traction(fcu_ctx ctx, fcu_space space, int64_t nf, const int64_t* facets,
                                  const double* tq, double* b);

/* ---- solvers ---------------------------------------------------------------- */
/* solve_cg (cg.rs:40-149): Jacobi-PCG on m, x0 may be NULL (zero start), stop
 * when ||r||/||b|| < tol after the x/r update. FCU_FP64 follows the reference
 * arithmetic; FCU_MIXED runs FP32 SpMV/axpy with FP64 dot accumulation and
 * FP64 residual replacement, and stops on the FP64 residual ||b - A64 x||.
 * Returns FCU_ERR_NO_CONVERGENCE / FCU_ERR_BREAKDOWN like the reference's Err;
 * x and info are filled in every case. Small scalar systems (at most 20,000
 * rows in FP64, 32,768 in FCU_MIXED) started from x0 = NULL run as a single
 * instance of the batched solver below, in one launch. */
int fcu_pcg(fcu_ctx ctx, fcu_matrix m, const double* b, const double* x0, double* x, double tol,
            int64_t max_iter, int precision, fcu_solve_info* info);

/* solve_csr_cg_gpu (gpu.rs:1145-1442): u32 CSR, caller-supplied inverse
 * diagonal, relative tolerance. Like the reference it returns FCU_OK when the
 * iteration limit is reached (info.rel_residual tells), and FCU_OK with x = 0
 * when ||b|| = 0 (gpu.rs:1169-1180). */
int fcu_solve_csr_cg(fcu_ctx ctx, int64_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                     const double* vals, const double* inv_diag, const double* b, const double* x0,
                     double rtol, int64_t max_iter, double* x, fcu_solve_info* info);

/* Batched Jacobi-PCG over independent systems (no reference counterpart; the
 * multi-mesh batch). m is a scalar matrix that is block diagonal over the
 * row ranges [offsets[i], offsets[i+1]), i < nb (offsets: nb + 1 values,
 * offsets[0] = 0, offsets[nb] = n) - e.g. assembled on a mesh that
 * concatenates the instances' meshes. Every block is solved from x0 = 0 with
 * its own alpha, beta and stopping test ||r_i|| / ||b_i|| < tol, as
 * fcu_pcg would solve it alone (precision FCU_FP64 or FCU_MIXED), in one
 * persistent launch (captured in a CUDA graph, replayed on later calls):
 * each instance is taken by a cluster of 1-8 CTAs, largest instances first.
 * Per-instance iterations, relative residuals and statuses go to the
 * optional host arrays (nb each). Returns FCU_OK when every instance
 * converged, else the first failing status. info: max iterations, total
 * replacements, max absolute and max relative residual, device time. */
int fcu_batch_pcg(fcu_ctx ctx, fcu_matrix m, int64_t nb, const int64_t* offsets, const double* b, double* x,
                  double tol, int64_t max_iter, int precision, int64_t* iterations, double* rel_residual,
                  int* status, fcu_solve_info* info);
/* Lanes per row, threads per CTA and CTAs per instance (thread-block
 * cluster) that the batched solver's tuning chose for m and `precision`
 * (all 0 before its first solve). */
int fcu_batch_config(fcu_matrix m, int precision, int* lanes_per_row, int* threads_per_cta,
                     int* ctas_per_cluster);

/* Allocation-free variant of fcu_solve_csr_cg. No counterpart in the
 * reference: it serves callers that cannot allocate device memory when they
 * solve (an application whose pool allocator owns the device's memory, or a
 * time-stepping loop where cudaMalloc/cudaFree would synchronise the device).
 * It takes no context and allocates nothing: its work vectors and state live
 * in one fixed module-scope device array.
 *  - n <= FCU_NOALLOC_MAX_N, else FCU_ERR_BAD_ARG;
 *  - every array is device memory of the calling thread's current device
 *    (host pointers are rejected with FCU_ERR_BAD_ARG; nothing is staged);
 *    x is used as the iterate in place and may equal x0;
 *  - runs on `stream` (a cudaStream_t; NULL = legacy default stream) and
 *    synchronises it before returning;
 *  - the array is shared by every call on a device: calls that overlap in
 *    time on one device race. Callers must not overlap them;
 *  - every call looks up the array's address on the current device (no
 *    address is cached, so calls after a cudaDeviceReset stay valid); the
 *    first call on a device may load the module there, so make it before any
 *    stream capture begins;
 *  - each call resets the solver state itself (it must start at zero);
 *  - info->kernel_ms is the host wall time of the call;
 *  - errors: fcu_last_error(NULL). Results and semantics as fcu_solve_csr_cg. */
#define FCU_NOALLOC_MAX_N 131072
int fcu_solve_csr_cg_noalloc(int64_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                             const double* vals, const double* inv_diag, const double* b,
                             const double* x0, double rtol, int64_t max_iter, double* x,
                             fcu_solve_info* info, void* stream);

/* y = A x (cg.rs:7-23) with the FP64 values. */
int fcu_spmv(fcu_ctx ctx, fcu_matrix m, const double* x, double* y);

/* ---- transient heat (transient.rs:21-68, heat_solver.rs:23-104) ------------- */
/* A stepper for M du/dt + K u = F that keeps its matrices on the device:
 * lhs = M + dt K (FCU_BACKWARD_EULER) or M + (dt/2) K (FCU_CRANK_NICOLSON),
 * and the right-hand matrix M or M - (dt/2) K, all formed once by
 * add_scaled_matrices from the values mass and stiff hold at creation. */
int fcu_transient_create(fcu_ctx ctx, fcu_matrix mass, fcu_matrix stiff, int scheme, double dt,
                         fcu_transient* out);
/* Dirichlet values (heat_solver.rs:82-99) written into the state before each
 * step and into the new state after it; a repeated dof takes its last value.
 * nbc = 0 clears them. */
int fcu_transient_set_dirichlet(fcu_ctx ctx, fcu_transient ts, int64_t nbc, const int64_t* dofs,
                                const double* vals);
/* TransientHeatSolver::step (transient.rs:32-68): rhs = M u_n + dt f_next, or
 * (M - dt/2 K) u_n + (dt/2)(f_n + f_next); then lhs u_next = rhs, solved by
 * the Jacobi-PCG of fcu_pcg (precision, tol, max_iter) from x0 = u_n where
 * the reference factorises densely (direct.rs:26-53). f_n / f_next may be
 * NULL (zero load). u_next may equal u_n. Status as fcu_pcg. */
int fcu_transient_step(fcu_ctx ctx, fcu_transient ts, const double* u_n, const double* f_n,
                       const double* f_next, double* u_next, double tol, int64_t max_iter, int precision,
                       fcu_solve_info* info);
void fcu_transient_destroy(fcu_transient ts);

/* ---- vibration modes (eigen.rs:94-300) ------------------------------------- */
/* Inner solve of the inverse iteration (the `inner` closure of
 * solve_vibration_modes_with_inner, eigen.rs:94-102): solve K x = b in the
 * folded frame, x0 the previous iterate. b, x0, x are device arrays of n
 * doubles; the library's stream is idle when it is called, and x must be
 * complete when it returns. Non-zero return: the solve fails with it. */
typedef int (*fcu_inner_solve)(void* user, int64_t n, const double* b, const double* x0, double* x);
/* solve_vibration_modes / solve_vibration_modes_with_inner: the lowest
 * num_modes modes of K u = lambda M u by inverse power iteration with
 * mass-orthogonal deflation, on folded copies of k (unit diagonal) and m
 * (zero), the mass rescaled by mean|diag K| / mean|diag M|, stopping each
 * mode when the Rayleigh quotient moves less than tol relative to itself or
 * after max_power_iters. inner == NULL: Jacobi-PCG on the folded stiffness
 * at inner_tol / inner_max_iter / precision (the reference default is FP64,
 * 1e-9, 1000). k and m have one order (their patterns may differ). Outputs:
 * eigenvalues (num_modes),
 * mode_shapes (num_modes*n, mass-normalised, may be NULL), power_iterations
 * (num_modes, may be NULL); info: total inner iterations and device time.
 * A failed inner solve fails the call with its status, as the reference's
 * `?` does. */
int fcu_vibration_modes(fcu_ctx ctx, fcu_matrix k, fcu_matrix m, int64_t nfixed, const int64_t* fixed,
                        int64_t num_modes, int64_t max_power_iters, double tol, double inner_tol,
                        int64_t inner_max_iter, int precision, fcu_inner_solve inner, void* user,
                        double* eigenvalues, double* mode_shapes, int64_t* power_iterations,
                        fcu_solve_info* info);

/* ---- 3x3 block CSR (GpuBsr3Context, solve_bsr3_pcg_gpu; gpu.rs:434-1141) --- */
/* Block CSR layout of the reference: row_ptr (n_nodes + 1, u32) over block
 * rows, cols (u32) block columns, vals_flat 9 values per block row-major
 * (vals_flat[9k + 3a + b] = A(3i + a, 3 cols[k] + b)), dinv_flat the inverse
 * diagonal block of each block row (9 per row, row-major). */
/* GpuBsr3Context::new (gpu.rs:453-494): a resident block matrix; dinv_flat may
 * be NULL. fcu_spmv on it is GpuBsr3Context::spmv (gpu.rs:505-545); fcu_pcg
 * on it (FCU_FP64) preconditions with the inverse blocks when given. */
int fcu_bsr3_create(fcu_ctx ctx, int64_t n_nodes, const uint32_t* row_ptr, const uint32_t* cols,
                    const double* vals_flat, const double* dinv_flat, fcu_matrix* out);
/* GpuBsr3Context::jacobi_smooth (gpu.rs:547-657): `sweeps` damped block-Jacobi
 * sweeps z <- z + omega D^-1 (r - A z); with zero_initial_z the first sweep
 * is z = D^-1 r. sweeps = 0 leaves z untouched. */
int fcu_bsr3_jacobi_smooth(fcu_ctx ctx, fcu_matrix m, const double* r, double* z, int64_t sweeps, double omega,
                           int zero_initial_z);
/* solve_bsr3_pcg_gpu (gpu.rs:775-1141): block-Jacobi PCG in FP64 from x0 (NULL
 * = 0), stop when ||r||/||b|| < rtol after the x/r update or when
 * p.Ap <= 1e-30; FCU_OK at the iteration limit (info.rel_residual tells) and
 * x = 0 when ||b|| = 0, as the reference returns Ok. */
int fcu_solve_bsr3_pcg(fcu_ctx ctx, int64_t n_nodes, const uint32_t* row_ptr, const uint32_t* cols,
                       const double* vals_flat, const double* dinv_flat, const double* b, const double* x0,
                       double rtol, int64_t max_iter, double* x, fcu_solve_info* info);
/* Block-Jacobi preconditioning of an assembled vector matrix from its own
 * diagonal blocks (inverted at every FP64 solve), or (enable = 0) back to
 * point Jacobi. FCU_ERR_BAD_ARG if a diagonal block is singular. */
int fcu_matrix_block_jacobi(fcu_ctx ctx, fcu_matrix m, int enable);
/* The block CSR arrays of a 3x3 block matrix (assembled on FCU_SPACE_P1_VEC3
 * or created by fcu_bsr3_create), the reference's solve_bsr3_pcg_gpu inputs;
 * any output may be NULL; dinv_flat needs inverse blocks (given at creation
 * or fcu_matrix_block_jacobi). */
int fcu_matrix_export_bsr3(fcu_ctx ctx, fcu_matrix m, uint32_t* row_ptr, uint32_t* cols, double* vals_flat,
                           double* dinv_flat);

/* ---- adjoint sensitivities (no reference counterpart) ----------------------- */
/* For E_e = E0 * theta_e^3: grad_e = -lambda_e^T (3 theta_e^2 E0 K_e^1) u_e, with
 * the unit-modulus element matrix K_e^1 recomputed per cell (not stored).
 * space: FCU_SPACE_P1_VEC3; u, lambda: 3*nv; theta, grad: nc. */
int fcu_adjoint_gradient(fcu_ctx ctx, fcu_space space, double E0, double nu, const double* theta,
                         const double* u, const double* lambda, double* grad);

/* ---- stress recovery --------------------------------------------------------- */
/* compute_element_stresses (elasticity.rs:230-320) on the space's tetrahedron
 * mesh (FCU_SPACE_P1_VEC3, or FCU_SPACE_P1 in 3D): per cell the displacement
 * gradient from u (3*nv, dof = 3*vertex + component), strain = sym(grad u),
 * Cauchy stress = lambda tr(eps) I + 2 mu eps, von Mises stress and trace.
 * stress, strain: nc*9 row-major; von_mises, trace: nc; any may be NULL.
 * Degenerate cells give zeros (StressState::default()). */
int fcu_element_stresses(fcu_ctx ctx, fcu_space space, double E, double nu, const double* u,
                         double* stress, double* strain, double* von_mises, double* trace);
/* compute_vertex_von_mises (elasticity.rs:323-360): volume-weighted average of
 * the cells' von Mises stress at each vertex (nv), cells summed in ascending
 * order; vertices with no volume keep the (zero) sum. The first call on a
 * space computes its cell volumes (nc doubles) and keeps them with the space. */
int fcu_vertex_von_mises(fcu_ctx ctx, fcu_space space, const double* cell_von_mises,
                         double* vertex_von_mises);

/* ---- device buffers and devices (no reference counterpart) ------------------ */
/* For callers with no CUDA allocator of their own, such as the Python mirror
 * of the Rust API; a Rust caller may equally pass memory from its own arena.
 * Buffers come from the device's memory pool, allocated and released in
 * order on the context's stream. */
int fcu_buffer_alloc(fcu_ctx ctx, size_t bytes, void** out);
int fcu_buffer_free(fcu_ctx ctx, void* p);
/* Copy `bytes` between host and device memory, in any direction, on the
 * context's stream. Returns when the copy is complete if either side is host
 * memory; device-to-device copies are asynchronous. */
int fcu_buffer_copy(fcu_ctx ctx, void* dst, const void* src, size_t bytes);
/* Set `bytes` of device memory to the byte `value` (asynchronous). */
int fcu_buffer_memset(fcu_ctx ctx, void* p, int value, size_t bytes);
int fcu_device_count(int* count);
/* The device's name, NUL-terminated and truncated to `len` bytes. */
int fcu_device_name(int device, char* name, size_t len);

/* ---- diagnostics (no reference counterpart) -------------------------------- */
/* Average device time of one launch of the SpMV kernel the PCG of `precision`
 * runs on m (Ap = A p with the device p.Ap reduction), over `reps`
 * back-to-back launches timed with CUDA events on the context stream; and
 * the algorithmic bytes of one launch (values + column indices + row
 * pointers + one read of p + one write of Ap). */
int fcu_time_spmv(fcu_ctx ctx, fcu_matrix m, int precision, int reps, double* ms_per_launch,
                  double* bytes_per_launch);
/* As fcu_time_spmv, with the L2 cache flushed before every timed launch: a
 * read of `flush_bytes` (at least the L2 size; 0 picks 256 MiB) from a buffer
 * the call allocates (a read, so no dirty lines are written back during the
 * timed launch), then one launch bracketed by CUDA events. Returns the
 * mean of the `reps` single-launch times, so the matrix and the operand
 * vector come from HBM as they do inside a solve whose operator exceeds L2. */
int fcu_time_spmv_cold(fcu_ctx ctx, fcu_matrix m, int precision, int reps, size_t flush_bytes,
                       double* ms_per_launch, double* bytes_per_launch);
/* Device time of one launch of the persistent PCG loop (the kernel fcu_pcg
 * runs for mixed-precision solves of 3x3-block matrices with point-Jacobi
 * preconditioning; FP64 solves take it when FCU_PERSISTENT=2) doing
 * exactly `iterations` iterations from x = 0 on b = 1 (no stopping test, no
 * residual replacement, no breakdown exit), after an L2 flush as in
 * fcu_time_spmv_cold; the mean over `reps` launches, each from a fresh start,
 * and the algorithmic bytes of one launch (per iteration: the matrix once;
 * z, p_old read and Ap written by the product; x, r, D^-1, p_old, z, Ap read
 * and x, r, p, z written by the update). FCU_ERR_UNSUPPORTED for other
 * matrices. Overwrites the solver's work vectors. */
int fcu_time_pcg(fcu_ctx ctx, fcu_matrix m, int precision, int64_t iterations, int reps, size_t flush_bytes,
                 double* ms_per_launch, double* bytes_per_launch);
/* Self-check of the bounded waits (no reference counterpart): one CTA waits,
 * `polls` polls each (1 .. 2^20), at a grid barrier of the persistent PCG
 * loop whose arrival count can never be reached, then at one it reaches, and
 * on a shared-memory mbarrier of the tiled SpMV ring that nothing arrives at,
 * then on one it arrives at itself. results[4] = {1 if the unreachable grid
 * wait passed, 1 if the reachable one passed, the same for the two mbarrier
 * waits}: a correct build gives {0, 1, 0, 1}. A wait that gives up returns;
 * nothing traps, and the context stays usable. */
int fcu_check_wait_limits(fcu_ctx ctx, uint32_t polls, int* results);

#ifdef __cplusplus
}
#endif
#endif /* FENICS_CUDA_H */
