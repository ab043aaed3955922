// C ABI of the library (include/fenics_cuda.h): argument checking, host/device
// staging, handle lifetime, CSC import/export. Compute lives in the other .cu
// files; every entry point converts FcuError into a status code.

#include <climits>

#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <memory>

#include <vector>

#include "internal.cuh"

// implemented in assemble.cu / rhs.cu / solver.cu
void assemble_stiffness_impl(fcu_matrix m, const double* coef_dev);
void assemble_elasticity_impl(fcu_matrix m, double E, double nu, const double* cellE_dev);
void apply_dirichlet_impl(fcu_matrix m, double* b_dev, i64 nbc, const i64* dofs_dev, const double* vals_dev);
void adjoint_gradient_impl(fcu_space s, double E0, double nu, const double* theta, const double* u, const double* la,
                           double* grad);
void quadrature_points_impl(fcu_space s, double* out_dev);
void rhs_impl(fcu_space s, int kind, const double* fq_dev, double p0, double p1, const double* nodal_dev, double* b_dev);
void body_force_impl(fcu_space s, const double* f, double* b_dev);
void traction_impl(fcu_space s, i64 nf, const i64* facets_dev, const double* tq_dev, double* b_dev);
i64 boundary_facets_impl(fcu_mesh m, i64* verts_dev, i64* cell_dev, i64* local_dev);
i64 boundary_dofs_impl(fcu_mesh m, fcu_space s_or_null, DBuf<i64>& result);
int run_pcg(fcu_matrix m, const double* b_dev, const double* x0_dev, double* x_dev, double tol, i64 max_iter,
            int precision, bool gpu_semantics, const double* inv_diag_dev, fcu_solve_info* info);
void spmv_impl(fcu_matrix m, const double* x_dev, double* y_dev);
void time_spmv_impl(fcu_matrix m, int precision, int reps, double* ms, double* bytes);
void time_spmv_cold_impl(fcu_matrix m, int precision, int reps, size_t flush_bytes, double* ms, double* bytes);
void time_pcg_impl(fcu_matrix m, int precision, i64 iters, int reps, size_t flush_bytes, double* ms, double* bytes);
void check_wait_limits_impl(fcu_ctx ctx, unsigned limit, int* results_host);
int batch_pcg_impl(fcu_matrix m, i64 nb, const i64* offsets_host, const double* b_dev, double* x_dev, double tol,
                   i64 max_iter, int precision, i64* iters_host, double* relres_host, int* status_host,
                   fcu_solve_info* info, const int* fixed_shape = nullptr);
void batch_config(fcu_matrix m, int precision, int* vpr, int* threads, int* cluster);
void element_stresses_impl(fcu_space s, double lam, double mu, const double* u_dev, double* stress, double* strain,
                           double* vm, double* trace);
void vertex_von_mises_impl(fcu_space s, const double* cell_vm_dev, double* out_dev);
void assemble_mass_impl(fcu_matrix m, double rho, const double* coef_dev);
bool same_pattern(fcu_matrix a, fcu_matrix b);
void add_scaled_impl(fcu_matrix out, fcu_matrix a, fcu_matrix b, double alpha);
void scale_values_impl(fcu_matrix m, double s);
i64 fold_dirichlet_impl(fcu_matrix m, i64 nf, const i64* dofs_dev, bool unit_diag, DBuf<unsigned char>* fixed_out);
fcu_transient transient_create_impl(fcu_matrix mass, fcu_matrix stiff, int scheme, double dt);
void transient_destroy_impl(fcu_transient t);
fcu_ctx transient_ctx(fcu_transient t);
i64 transient_order(fcu_transient t);
void transient_set_dirichlet_impl(fcu_transient t, i64 nbc, const i64* dofs_host, const double* vals_host);
int transient_step_impl(fcu_transient t, const double* un, const double* fn, const double* fnext, double* unext,
                        double tol, i64 max_iter, int precision, fcu_solve_info* info);
int vibration_modes_impl(fcu_matrix k, fcu_matrix m, i64 nfixed, const i64* fixed_dev, i64 num_modes,
                         i64 max_power_iters, double tol, double inner_tol, i64 inner_max_iter, int precision,
                         fcu_inner_solve inner, void* user, double* eigenvalues, double* modes_dev,
                         i64* power_iters, fcu_solve_info* info, std::string* err);
fcu_matrix bsr3_create_impl(fcu_ctx ctx, i64 nn, const uint32_t* rp_dev, const uint32_t* ci_dev, i64 nnzb,
                            const double* vals_dev, const double* dinv_dev);
void bsr3_jacobi_smooth_impl(fcu_matrix m, const double* r, double* z, i64 sweeps, double omega, bool zero_init);
void matrix_block_jacobi_impl(fcu_matrix m, bool enable);
void matrix_export_bsr3_impl(fcu_matrix m, uint32_t* rp, uint32_t* ci, double* vals, double* dinv);
int run_pcg_noalloc(i64 n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* vals,
                    const double* inv_diag, const double* b, const double* x0, double rtol, i64 max_iter, double* x,
                    fcu_solve_info* info, void* stream);

namespace {

thread_local std::string g_create_err;

// Sets the allocation stream for the duration of a call.
struct AllocStreamScope {
  cudaStream_t prev;
  explicit AllocStreamScope(cudaStream_t s) : prev(fcu_alloc_stream()) { fcu_alloc_stream() = s; }
  ~AllocStreamScope() { fcu_alloc_stream() = prev; }
};

template <class F>
int guarded(fcu_ctx ctx, F&& f) {
  AllocStreamScope scope(ctx ? ctx->stream : nullptr);
  try {
    if (ctx) CUDA_CHECK(cudaSetDevice(ctx->device));
    f();
    return FCU_OK;
  } catch (const FcuError& e) {
    if (ctx) ctx->err = e.msg;
    else g_create_err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    if (ctx) ctx->err = "host allocation failed";
    return FCU_ERR_CUDA;
  }
}

void sync(fcu_ctx ctx) { CUDA_CHECK(cudaStreamSynchronize(ctx->stream)); }

__global__ void k_i64_to_i32(const i64* __restrict__ a, i64 n, i64 lim, int* __restrict__ b, int* __restrict__ bad) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
    i64 v = a[t];
    if (v < 0 || v >= lim) atomicExch(bad, 1);
    b[t] = (int)v;
  }
}

__global__ void k_u32_to_i32(const uint32_t* __restrict__ a, i64 n, i64 lim, int* __restrict__ b,
                             int* __restrict__ bad) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
    uint32_t v = a[t];
    if ((i64)v > lim) atomicExch(bad, 1);
    b[t] = (int)v;
  }
}

__global__ void k_i32_to_i64(const int* __restrict__ a, i64 n, i64* __restrict__ b) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) b[t] = a[t];
}

__global__ void k_diag_pos(const int* __restrict__ rp, const int* __restrict__ ci, i64 n, int* __restrict__ dp) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    int pos = -1;
    for (int p = rp[i]; p < rp[i + 1]; ++p)
      if (ci[p] == (int)i) { pos = p; break; }
    dp[i] = pos;
  }
}

// CSC entry k of column c -> sort key (row * n + col) for the CSR transpose.
__global__ void k_csc_keys(const i64* __restrict__ cp, const i64* __restrict__ ri, i64 n, int* __restrict__ bad,
                           unsigned long long* __restrict__ keys, unsigned* __restrict__ idx, i64 nnz) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < n; c += (i64)gridDim.x * blockDim.x) {
    i64 b = cp[c], e = cp[c + 1];
    if (b < 0 || e < b || e > nnz) { atomicExch(bad, 1); continue; }
    for (i64 k = b; k < e; ++k) {
      i64 r = ri[k];
      if (r < 0 || r >= n) { atomicExch(bad, 1); r = 0; }
      keys[k] = (unsigned long long)(r * n + c);
      idx[k] = (unsigned)k;
    }
  }
}

// Sorted keys (+ one diagonal key per row, flagged by idx = 0xffffffff) -> CSR.
__global__ void k_csr_from_sorted(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ idx,
                                  const int* __restrict__ flag, const int* __restrict__ pos, i64 ntot, i64 n,
                                  const double* __restrict__ vals, int* __restrict__ col, double* __restrict__ v,
                                  int* __restrict__ src, unsigned char* __restrict__ real, int* __restrict__ rp) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < ntot; t += (i64)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[t];
    const i64 r = (i64)(k / n);
    if (flag[t]) {
      const int s = pos[t];
      col[s] = (int)(k % n);
      if (t == 0 || keys[t - 1] / n != (unsigned long long)r) rp[r] = s;
      v[s] = 0.0;
      real[s] = 0;
      src[s] = -1;
    }
  }
}

__global__ void k_csr_fill_vals(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ idx,
                                const int* __restrict__ pos_incl, i64 ntot, const double* __restrict__ vals,
                                double* __restrict__ v, int* __restrict__ src, unsigned char* __restrict__ real) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < ntot; t += (i64)gridDim.x * blockDim.x) {
    const unsigned id = idx[t];
    if (id == 0xffffffffu) continue;
    const int s = pos_incl[t] - 1;
    atomicAdd(&v[s], vals[id]);  // duplicate (row, col) entries are summed
    src[s] = (int)id;
    real[s] = 1;
  }
}

__global__ void k_unique_keys(const unsigned long long* __restrict__ keys, i64 n, int* __restrict__ flag) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x)
    flag[t] = (t == 0 || keys[t - 1] != keys[t]) ? 1 : 0;
}

__global__ void k_diag_keys(i64 n, unsigned long long* __restrict__ keys, unsigned* __restrict__ idx) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    keys[i] = (unsigned long long)(i * n + i);
    idx[i] = 0xffffffffu;
  }
}

// --- export: space matrices (symmetric node pattern) -------------------------
// Inclusion rule of the reference pattern: a stored entry (r, c) is exported
// when its slot is structural (not an inserted diagonal) and neither r nor c
// is eliminated; an eliminated dof keeps only its diagonal. A folded matrix
// (fold_dirichlet, eigen.rs:55-79: `drop`) also omits every zero value,
// including a fixed diagonal folded to 0. `val`/`tpos` are read only then.
// A vector mass matrix (`cdiag`) holds only the same-component entries of
// each block (mass.rs:118-123).
template <int BS>
__global__ void k_export_count(const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ tpos,
                               const double* __restrict__ val, bool drop, bool cdiag,
                               const unsigned char* __restrict__ dstruct,
                               const unsigned char* __restrict__ dir, const double* __restrict__ dcount, i64 nn,
                               i64* __restrict__ cnt) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nn * BS; c += (i64)gridDim.x * blockDim.x) {
    const i64 w = c / BS;
    const int be = (int)(c - w * BS);
    const bool dc = dir ? dir[c] != 0 : false;
    i64 k = 0;
    if (dc) {
      k = (drop && dcount[c] == 0.0) ? 0 : 1;
    } else {
      for (int p = rp[w]; p < rp[w + 1]; ++p) {
        const i64 v = ci[p];
        if (v == w && !dstruct[w]) continue;
        for (int a = 0; a < BS; ++a) {
          const i64 r = v * BS + a;
          if (dir && dir[r]) continue;
          if (cdiag && a != be) continue;
          if (drop && val[(i64)tpos[p] * BS * BS + a * BS + be] == 0.0) continue;
          ++k;
        }
      }
    }
    cnt[c] = k;
  }
}

template <int BS>
__global__ void k_export_fill(const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ tpos,
                              bool drop, bool cdiag, const unsigned char* __restrict__ dstruct,
                              const unsigned char* __restrict__ dir,
                              const double* __restrict__ dcount, const double* __restrict__ val, i64 nn,
                              const i64* __restrict__ colptr, i64* __restrict__ rowidx, double* __restrict__ vals) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nn * BS; c += (i64)gridDim.x * blockDim.x) {
    const i64 w = c / BS;
    const int be = (int)(c - w * BS);
    i64 o = colptr[c];
    if (dir && dir[c]) {
      if (drop && dcount[c] == 0.0) continue;
      if (rowidx) rowidx[o] = c;
      if (vals) vals[o] = dcount[c];
      continue;
    }
    for (int p = rp[w]; p < rp[w + 1]; ++p) {
      const i64 v = ci[p];
      if (v == w && !dstruct[w]) continue;
      const i64 q = tpos[p];  // slot (v, w)
      for (int a = 0; a < BS; ++a) {
        const i64 r = v * BS + a;
        if (dir && dir[r]) continue;
        if (cdiag && a != be) continue;
        if (drop && val[q * BS * BS + a * BS + be] == 0.0) continue;
        if (rowidx) rowidx[o] = r;
        if (vals) vals[o] = val[q * BS * BS + a * BS + be];
        ++o;
      }
    }
  }
}

// --- export: wrapped CSC matrices (original CSC order) ------------------------
__global__ void k_wexport_count(const i64* __restrict__ cp, const i64* __restrict__ ri, const int* __restrict__ csr_of,
                                const double* __restrict__ val, bool drop, const unsigned char* __restrict__ dir,
                                const double* __restrict__ dcount, i64 n, i64* __restrict__ cnt) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < n; c += (i64)gridDim.x * blockDim.x) {
    if (dir && dir[c]) { cnt[c] = (drop && dcount[c] == 0.0) ? 0 : 1; continue; }
    i64 k = 0;
    for (i64 q = cp[c]; q < cp[c + 1]; ++q)
      if (!(dir && dir[ri[q]]) && !(drop && val[csr_of[q]] == 0.0)) ++k;
    cnt[c] = k;
  }
}

__global__ void k_wexport_fill(const i64* __restrict__ cp, const i64* __restrict__ ri, const int* __restrict__ csr_of,
                               bool drop, const unsigned char* __restrict__ dir, const double* __restrict__ dcount,
                               const double* __restrict__ val, i64 n, const i64* __restrict__ colptr,
                               i64* __restrict__ rowidx, double* __restrict__ vals) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < n; c += (i64)gridDim.x * blockDim.x) {
    i64 o = colptr[c];
    if (dir && dir[c]) {
      if (drop && dcount[c] == 0.0) continue;
      if (rowidx) rowidx[o] = c;
      if (vals) vals[o] = dcount[c];
      continue;
    }
    for (i64 q = cp[c]; q < cp[c + 1]; ++q) {
      if (dir && dir[ri[q]]) continue;
      if (drop && val[csr_of[q]] == 0.0) continue;
      if (rowidx) rowidx[o] = ri[q];
      if (vals) vals[o] = val[csr_of[q]];
      ++o;
    }
  }
}

__global__ void k_csr_of(const int* __restrict__ src, i64 nnz, int* __restrict__ csr_of) {
  for (i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x; s < nnz; s += (i64)gridDim.x * blockDim.x)
    if (src[s] >= 0) csr_of[src[s]] = (int)s;
}

__global__ void k_diag_struct_space(const int* __restrict__ diag_pos, const unsigned short* __restrict__ cnt, i64 nn,
                                    unsigned char* __restrict__ ds) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nn; i += (i64)gridDim.x * blockDim.x)
    ds[i] = cnt[diag_pos[i]] > 0 ? 1 : 0;
}

__global__ void k_f64_to_f32(const double* __restrict__ a, i64 n, float* __restrict__ b) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) b[t] = (float)a[t];
}

template <class T>
T read1(fcu_ctx ctx, const T* p) {
  T h;
  CUDA_CHECK(cudaMemcpyAsync(&h, p, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  sync(ctx);
  return h;
}

int cap_blocks(fcu_ctx ctx) { return ctx->num_sms * 16; }

// Assembly overwrites every value, so a re-assembled matrix starts without
// Dirichlet conditions (the mask is cleared, its storage kept).
void reset_dirichlet(fcu_matrix m) {
  if (m->bc_applied && m->dirichlet.p)
    CUDA_CHECK(cudaMemsetAsync(m->dirichlet.p, 0, m->n, m->ctx->stream));
  m->bc_applied = false;
  m->drop_zeros = false;
  m->n_dirichlet = 0;
}

void check_ctx(fcu_ctx ctx) {
  if (!ctx) fail(FCU_ERR_BAD_ARG, "null context");
}

// Spaces on the caller's P2 node numbering support mass and stiffness only.
void reject_node_space(fcu_space s) {
  if (s && (s->kind == FCU_SPACE_P2_NODES || s->kind == FCU_SPACE_P2_NODES_VEC3))
    fail(FCU_ERR_UNSUPPORTED, "a P2 space on caller nodes supports mass and stiffness assembly only");
}

__global__ void k_cells10(const i64* __restrict__ c10, const int* __restrict__ cells4, i64 nc, i64 nv,
                          int* __restrict__ out, int* __restrict__ bad) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < 10 * nc; t += (i64)gridDim.x * blockDim.x) {
    const i64 v = c10[t];
    const i64 c = t / 10;
    const int a = (int)(t - 10 * c);
    if (v < 0 || v >= nv || (a < 4 && v != cells4[4 * c + a])) atomicExch(bad, 1);
    out[t] = (int)v;
  }
}

void ctx_release(fcu_ctx c) {
  if (!c || --c->refs > 0) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->temp.release();
  for (void* p : c->pinned_pool) cudaFreeHost(p);
  cudaStreamDestroy(c->stream);
  delete c;
}

void mesh_release(fcu_mesh m) {
  if (!m || --m->refs > 0) return;
  fcu_ctx c = m->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete m;
  ctx_release(c);
}

void space_release(fcu_space s) {
  if (!s || --s->refs > 0) return;
  fcu_mesh me = s->mesh;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  delete s;
  mesh_release(me);
}

void matrix_release(fcu_matrix m) {
  if (!m || --m->refs > 0) return;
  fcu_space sp = m->space;
  fcu_ctx c = m->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete m;
  if (sp) space_release(sp);
  ctx_release(c);
}

}  // namespace

// A new matrix on src's pattern holding a copy of its values and Dirichlet
// state (one reference to it, held by the caller).
fcu_matrix matrix_clone(fcu_matrix src) {
  fcu_ctx ctx = src->ctx;
  std::unique_ptr<fcu_matrix_s> m(new fcu_matrix_s());
  m->ctx = ctx;
  m->space = src->space;
  m->n = src->n;
  m->nnodes = src->nnodes;
  m->bs = src->bs;
  m->nnzb = src->nnzb;
  m->wrapped_general = src->wrapped_general;
  auto copy = [&](auto& dst, const auto& from) {
    if (!from.p) return;
    dst.alloc(from.n);
    CUDA_CHECK(cudaMemcpyAsync(dst.p, from.p, from.bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
  };
  if (src->space) {
    m->row_ptr = src->row_ptr;
    m->col_idx = src->col_idx;
    m->diag_pos = src->diag_pos;
  } else {
    copy(m->own_row_ptr, src->own_row_ptr);
    copy(m->own_col_idx, src->own_col_idx);
    copy(m->own_diag_pos, src->own_diag_pos);
    copy(m->csc_colptr, src->csc_colptr);
    copy(m->csc_rowidx, src->csc_rowidx);
    copy(m->csr_of, src->csr_of);
    m->row_ptr = m->own_row_ptr.p;
    m->col_idx = m->own_col_idx.p;
    m->diag_pos = m->own_diag_pos.p;
  }
  copy(m->val64, src->val64);
  copy(m->val32, src->val32);
  copy(m->dirichlet, src->dirichlet);
  copy(m->diag_count, src->diag_count);
  copy(m->diag_struct, src->diag_struct);
  m->n_dirichlet = src->n_dirichlet;
  m->bc_applied = src->bc_applied;
  m->drop_zeros = src->drop_zeros;
  m->comp_diag = src->comp_diag;
  copy(m->bdinv, src->bdinv);
  m->block_jacobi = src->block_jacobi;
  m->max_row_own = src->max_row_own;
  m->missing_diag = src->missing_diag;
  m->has_values = src->has_values;
  if (m->space) m->space->refs++;
  ctx->refs++;
  return m.release();
}

void matrix_release_ref(fcu_matrix m) { matrix_release(m); }

extern "C" {

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

int fcu_ctx_create(int device, fcu_ctx* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(nullptr, [&] {
    int ndev = 0;
    CUDA_CHECK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) fail(FCU_ERR_BAD_ARG, "no such CUDA device");
    CUDA_CHECK(cudaSetDevice(device));
    int major = 0;
    CUDA_CHECK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    fcu_ctx c = new fcu_ctx_s();
    c->device = device;
    CUDA_CHECK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete c;
      fail(FCU_ERR_CUDA, cudaGetErrorString(e));
    }
    // Library buffers come from the device's default memory pool, stream
    // ordered; keep freed blocks cached in the pool rather than returning
    // them to the driver at every synchronisation.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = c;
  });
}

void fcu_ctx_destroy(fcu_ctx ctx) { ctx_release(ctx); }

const char* fcu_last_error(fcu_ctx ctx) { return ctx ? ctx->err.c_str() : g_create_err.c_str(); }

int fcu_ctx_synchronize(fcu_ctx ctx) {
  return guarded(ctx, [&] { check_ctx(ctx); sync(ctx); });
}

void* fcu_ctx_stream(fcu_ctx ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t fcu_ctx_kernel_launches(fcu_ctx ctx) { return ctx ? ctx->launches : 0; }

// ---------------------------------------------------------------------------
// device buffers and devices
// ---------------------------------------------------------------------------

int fcu_buffer_alloc(fcu_ctx ctx, size_t bytes, void** out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    check_ctx(ctx);
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes ? bytes : 1, ctx->stream);
    if (e != cudaSuccess) fail(FCU_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    *out = p;
  });
}

int fcu_buffer_free(fcu_ctx ctx, void* p) {
  return guarded(ctx, [&] {
    check_ctx(ctx);
    if (p) CUDA_CHECK(cudaFreeAsync(p, ctx->stream));
  });
}

int fcu_buffer_copy(fcu_ctx ctx, void* dst, const void* src, size_t bytes) {
  return guarded(ctx, [&] {
    check_ctx(ctx);
    if (!bytes) return;
    if (!dst || !src) fail(FCU_ERR_BAD_ARG, "null copy argument");
    CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
    if (!is_device_ptr(dst) || !is_device_ptr(src)) sync(ctx);
  });
}

int fcu_buffer_memset(fcu_ctx ctx, void* p, int value, size_t bytes) {
  return guarded(ctx, [&] {
    check_ctx(ctx);
    if (!bytes) return;
    if (!p || !is_device_ptr(p)) fail(FCU_ERR_BAD_ARG, "memset target is not device memory");
    CUDA_CHECK(cudaMemsetAsync(p, value, bytes, ctx->stream));
  });
}

int fcu_device_count(int* count) {
  if (!count) return FCU_ERR_BAD_ARG;
  *count = 0;
  return guarded(nullptr, [&] { CUDA_CHECK(cudaGetDeviceCount(count)); });
}

int fcu_device_name(int device, char* name, size_t len) {
  if (!name || !len) return FCU_ERR_BAD_ARG;
  return guarded(nullptr, [&] {
    cudaDeviceProp prop;
    CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
    std::strncpy(name, prop.name, len - 1);
    name[len - 1] = 0;
  });
}

// ---------------------------------------------------------------------------
// meshes
// ---------------------------------------------------------------------------

int fcu_mesh_create(fcu_ctx ctx, int dim, int64_t nv, const double* coords, int64_t nc, const int64_t* cells,
                    fcu_mesh* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    check_ctx(ctx);
    if (dim != 2 && dim != 3) fail(FCU_ERR_BAD_ARG, "dim must be 2 or 3");
    if (nv < 0 || nc < 0 || (nv > 0 && !coords) || (nc > 0 && !cells)) fail(FCU_ERR_BAD_ARG, "bad mesh arrays");
    if (nv >= (1ll << 31) || nc * (dim + 1) >= (1ll << 31)) fail(FCU_ERR_UNSUPPORTED, "mesh exceeds 32-bit indexing");
    std::unique_ptr<fcu_mesh_s> m(new fcu_mesh_s());
    m->ctx = ctx;
    m->dim = dim;
    m->nodes = dim + 1;
    m->nv = nv;
    m->nc = nc;
    upload(ctx, m->coords, coords, (size_t)(nv * dim));
    m->cells.alloc(nc * m->nodes);
    if (nc) {
      DevIn<i64> c64(ctx, cells, (size_t)(nc * m->nodes));
      DBuf<int> bad;
      bad.alloc(1);
      CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
      k_i64_to_i32<<<grid_for(nc * m->nodes, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(c64.p, nc * m->nodes, nv,
                                                                                         m->cells.p, bad.p);
      LAUNCH_CHECK(ctx);
      if (read1(ctx, bad.p)) fail(FCU_ERR_BAD_ARG, "cell vertex index out of range");
    }
    build_mesh_validity(m.get());
    ctx->refs++;
    *out = m.release();
  });
}

void fcu_mesh_destroy(fcu_mesh m) { mesh_release(m); }

int fcu_mesh_num_degenerate(fcu_ctx ctx, fcu_mesh mesh, int64_t* count) {
  return guarded(ctx, [&] {
    if (!mesh || !count) fail(FCU_ERR_BAD_ARG, "null argument");
    *count = mesh->n_degenerate;
  });
}

int fcu_boundary_dofs(fcu_ctx ctx, fcu_mesh mesh, int64_t* out, int64_t* count) {
  return guarded(ctx, [&] {
    if (!mesh || !count) fail(FCU_ERR_BAD_ARG, "null argument");
    DBuf<i64> res;
    i64 k = boundary_dofs_impl(mesh, nullptr, res);
    if (out) {
      if (*count < k && *count != 0) fail(FCU_ERR_BAD_ARG, "output buffer too small");
      download(ctx, out, res.p, (size_t)k);
    }
    *count = k;
    sync(ctx);
  });
}

int fcu_boundary_facets(fcu_ctx ctx, fcu_mesh mesh, int64_t* verts, int64_t* cell, int64_t* local, int64_t* count) {
  return guarded(ctx, [&] {
    if (!mesh || !count) fail(FCU_ERR_BAD_ARG, "null argument");
    i64 nf = boundary_facets_impl(mesh, nullptr, nullptr, nullptr);
    if (verts || cell || local) {
      DevOut<i64> V(verts, nf * mesh->dim), Cc(cell, nf), L(local, nf);
      boundary_facets_impl(mesh, V.p, Cc.p, L.p);
      V.finish(ctx);
      Cc.finish(ctx);
      L.finish(ctx);
    }
    *count = nf;
    sync(ctx);
  });
}

// ---------------------------------------------------------------------------
// spaces
// ---------------------------------------------------------------------------

int fcu_space_create(fcu_ctx ctx, fcu_mesh mesh, int kind, fcu_space* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    if (!mesh) fail(FCU_ERR_BAD_ARG, "null mesh");
    if (kind != FCU_SPACE_P1 && kind != FCU_SPACE_P2 && kind != FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "unknown space kind");
    if ((kind == FCU_SPACE_P2 || kind == FCU_SPACE_P1_VEC3) && mesh->dim != 3)
      fail(FCU_ERR_BAD_ARG, "P2 and vector spaces need a tetrahedral mesh");
    std::unique_ptr<fcu_space_s> s(new fcu_space_s());
    s->ctx = ctx;
    s->mesh = mesh;
    s->kind = kind;
    build_space_pattern(s.get());
    sync(ctx);
    mesh->refs++;
    *out = s.release();
  });
}

int fcu_space_create_p2_nodes(fcu_ctx ctx, fcu_mesh mesh, const int64_t* cells10, int vec3, fcu_space* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    if (!mesh || (mesh->nc > 0 && !cells10)) fail(FCU_ERR_BAD_ARG, "null argument");
    if (mesh->dim != 3) fail(FCU_ERR_BAD_ARG, "P2 spaces need a tetrahedral mesh");
    if (10 * mesh->nc >= (1ll << 31)) fail(FCU_ERR_UNSUPPORTED, "mesh exceeds 32-bit indexing");
    std::unique_ptr<fcu_space_s> s(new fcu_space_s());
    s->ctx = ctx;
    s->mesh = mesh;
    s->kind = vec3 ? FCU_SPACE_P2_NODES_VEC3 : FCU_SPACE_P2_NODES;
    s->cell_nodes.alloc(10 * mesh->nc);
    if (mesh->nc) {
      DevIn<i64> c10(ctx, cells10, 10 * mesh->nc);
      DBuf<int> bad;
      bad.alloc(1);
      CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
      k_cells10<<<grid_for(10 * mesh->nc, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(
          c10.p, mesh->cells.p, mesh->nc, mesh->nv, s->cell_nodes.p, bad.p);
      LAUNCH_CHECK(ctx);
      if (read1(ctx, bad.p)) fail(FCU_ERR_BAD_ARG, "cell node out of range or corners differ from the mesh cell");
    }
    build_space_pattern(s.get());
    sync(ctx);
    mesh->refs++;
    *out = s.release();
  });
}

void fcu_space_destroy(fcu_space s) { space_release(s); }

int fcu_space_info(fcu_space s, int64_t* ndofs, int64_t* nnz, int64_t* nedges) {
  if (!s) return FCU_ERR_BAD_ARG;
  if (ndofs) *ndofs = s->ndofs;
  if (nnz) *nnz = s->nnz_ref;
  if (nedges) *nedges = s->nedges;
  return FCU_OK;
}

int fcu_space_p2_dofmap(fcu_ctx ctx, fcu_space s, int64_t* cell_dofs, int64_t* edge_verts) {
  return guarded(ctx, [&] {
    if (!s || s->kind != FCU_SPACE_P2) fail(FCU_ERR_BAD_ARG, "not a P2 space");
    const i64 nc = s->mesh->nc;
    if (cell_dofs) {
      DevOut<i64> o(cell_dofs, 10 * nc);
      if (nc) {
        k_i32_to_i64<<<grid_for(10 * nc, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(s->cell_nodes.p, 10 * nc, o.p);
        LAUNCH_CHECK(ctx);
      }
      o.finish(ctx);
      sync(ctx);
    }
    if (edge_verts) {
      DevOut<i64> o(edge_verts, 2 * s->nedges);
      if (s->nedges) {
        k_i32_to_i64<<<grid_for(2 * s->nedges, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(s->edge_verts.p,
                                                                                           2 * s->nedges, o.p);
        LAUNCH_CHECK(ctx);
      }
      o.finish(ctx);
      sync(ctx);
    }
  });
}

int fcu_space_boundary_dofs(fcu_ctx ctx, fcu_space s, int64_t* out, int64_t* count) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || !count) fail(FCU_ERR_BAD_ARG, "null argument");
    DBuf<i64> res;
    i64 k = boundary_dofs_impl(s->mesh, s, res);
    if (out) download(ctx, out, res.p, (size_t)k);
    *count = k;
    sync(ctx);
  });
}

// ---------------------------------------------------------------------------
// matrices
// ---------------------------------------------------------------------------

int fcu_matrix_create(fcu_ctx ctx, fcu_space s, fcu_matrix* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    if (!s) fail(FCU_ERR_BAD_ARG, "null space");
    std::unique_ptr<fcu_matrix_s> m(new fcu_matrix_s());
    m->ctx = ctx;
    m->space = s;
    m->bs = s->bs;
    m->n = s->ndofs;
    m->nnodes = s->nnodes;
    m->nnzb = s->nnzb;
    m->row_ptr = s->row_ptr.p;
    m->col_idx = s->col_idx.p;
    m->diag_pos = s->diag_pos.p;
    const i64 nv = s->nnzb * s->bs * s->bs;
    m->val64.alloc(nv);
    m->val32.alloc(nv);
    m->diag_struct.alloc(s->nnodes);
    if (s->nnodes) {
      k_diag_struct_space<<<grid_for(s->nnodes, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(
          s->diag_pos.p, s->slot_cnt.p, s->nnodes, m->diag_struct.p);
      LAUNCH_CHECK(ctx);
    }
    sync(ctx);
    s->refs++;
    ctx->refs++;
    *out = m.release();
  });
}

int fcu_matrix_from_csc(fcu_ctx ctx, int64_t n, const int64_t* colptr, const int64_t* rowidx, const double* vals,
                        fcu_matrix* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    check_ctx(ctx);
    if (n <= 0 || !colptr) fail(FCU_ERR_BAD_ARG, "bad CSC arguments");
    i64 nnz = 0;
    {
      DevIn<i64> cpd(ctx, colptr, n + 1);
      nnz = read1(ctx, cpd.p + n);
    }
    if (nnz < 0 || (nnz > 0 && (!rowidx || !vals))) fail(FCU_ERR_BAD_ARG, "bad CSC arrays");
    if (nnz + n >= (1ll << 31) - 1) fail(FCU_ERR_UNSUPPORTED, "matrix exceeds 32-bit indexing");
    if ((double)n * (double)n >= 1.8e19) fail(FCU_ERR_UNSUPPORTED, "matrix order too large");
    std::unique_ptr<fcu_matrix_s> m(new fcu_matrix_s());
    m->ctx = ctx;
    m->n = n;
    m->nnodes = n;
    m->bs = 1;
    m->wrapped_general = true;
    upload(ctx, m->csc_colptr, colptr, n + 1);
    upload(ctx, m->csc_rowidx, rowidx, nnz);
    DevIn<double> vd(ctx, vals, nnz);
    const i64 ntot = nnz + n;  // + one inserted diagonal per row
    DBuf<unsigned long long> k0, k1;
    DBuf<unsigned> i0, i1;
    DBuf<int> bad, flag, pos;
    k0.alloc(ntot); k1.alloc(ntot); i0.alloc(ntot); i1.alloc(ntot); bad.alloc(1); flag.alloc(ntot); pos.alloc(ntot);
    CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
    k_csc_keys<<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(m->csc_colptr.p, m->csc_rowidx.p, n, bad.p,
                                                                          k0.p, i0.p, nnz);
    LAUNCH_CHECK(ctx);
    k_diag_keys<<<grid_for(n, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(n, k0.p + nnz, i0.p + nnz);
    LAUNCH_CHECK(ctx);
    if (read1(ctx, bad.p)) fail(FCU_ERR_BAD_ARG, "CSC index out of range");
    size_t tb = 0;
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0.p, k1.p, i0.p, i1.p, (int)ntot, 0, 64, ctx->stream));
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(ctx->temp_bytes(tb), tb, k0.p, k1.p, i0.p, i1.p, (int)ntot, 0, 64,
                                               ctx->stream));
    k_unique_keys<<<grid_for(ntot, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(k1.p, ntot, flag.p);
    LAUNCH_CHECK(ctx);
    tb = 0;
    CUDA_CHECK(cub::DeviceScan::InclusiveSum(nullptr, tb, flag.p, pos.p, (int)ntot, ctx->stream));
    CUDA_CHECK(cub::DeviceScan::InclusiveSum(ctx->temp_bytes(tb), tb, flag.p, pos.p, (int)ntot, ctx->stream));
    const i64 nslots = read1(ctx, pos.p + ntot - 1);
    m->nnzb = nslots;
    m->own_row_ptr.alloc(n + 1);
    m->own_col_idx.alloc(nslots);
    m->own_diag_pos.alloc(n);
    m->val64.alloc(nslots);
    m->val32.alloc(nslots);
    DBuf<int> src, excl;
    DBuf<unsigned char> real;
    src.alloc(nslots);
    real.alloc(nslots);
    excl.alloc(ntot);
    // exclusive positions for the slot writes
    k_unique_keys<<<grid_for(ntot, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(k1.p, ntot, flag.p);
    LAUNCH_CHECK(ctx);
    tb = 0;
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.p, excl.p, (int)ntot, ctx->stream));
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(ctx->temp_bytes(tb), tb, flag.p, excl.p, (int)ntot, ctx->stream));
    k_csr_from_sorted<<<grid_for(ntot, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(
        k1.p, i1.p, flag.p, excl.p, ntot, n, vd.p, m->own_col_idx.p, m->val64.p, src.p, real.p, m->own_row_ptr.p);
    LAUNCH_CHECK(ctx);
    k_csr_fill_vals<<<grid_for(ntot, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(k1.p, i1.p, pos.p, ntot, vd.p,
                                                                                  m->val64.p, src.p, real.p);
    LAUNCH_CHECK(ctx);
    int ns32 = (int)nslots;
    CUDA_CHECK(cudaMemcpyAsync(m->own_row_ptr.p + n, &ns32, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    k_diag_pos<<<grid_for(n, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(m->own_row_ptr.p, m->own_col_idx.p, n,
                                                                           m->own_diag_pos.p);
    LAUNCH_CHECK(ctx);
    m->csr_of.alloc(std::max<i64>(nnz, 1));
    k_csr_of<<<grid_for(nslots, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(src.p, nslots, m->csr_of.p);
    LAUNCH_CHECK(ctx);
    k_f64_to_f32<<<grid_for(nslots, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(m->val64.p, nslots, m->val32.p);
    LAUNCH_CHECK(ctx);
    m->row_ptr = m->own_row_ptr.p;
    m->col_idx = m->own_col_idx.p;
    m->diag_pos = m->own_diag_pos.p;
    m->has_values = true;
    sync(ctx);
    ctx->refs++;
    *out = m.release();
  });
}

void fcu_matrix_destroy(fcu_matrix m) { matrix_release(m); }

static i64 export_counts(fcu_matrix m, DBuf<i64>& colptr) {
  fcu_ctx ctx = m->ctx;
  if (!m->space && !m->wrapped_general)
    fail(FCU_ERR_UNSUPPORTED, "a block CSR matrix exports through fcu_matrix_export_bsr3");
  const i64 n = m->n;
  DBuf<i64> cnt;
  cnt.alloc(n + 1);
  CUDA_CHECK(cudaMemsetAsync(cnt.p + n, 0, sizeof(i64), ctx->stream));
  const unsigned char* dir = m->bc_applied ? m->dirichlet.p : nullptr;
  const bool drop = m->drop_zeros;
  if (m->wrapped_general) {
    k_wexport_count<<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(
        m->csc_colptr.p, m->csc_rowidx.p, m->csr_of.p, m->val64.p, drop, dir, m->diag_count.p, n, cnt.p);
  } else {
    const int* tpos = nullptr;
    if (drop) {
      build_transpose_positions(m->space);
      tpos = m->space->tpos.p;
    }
    if (m->bs == 3)
      k_export_count<3><<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(
          m->row_ptr, m->col_idx, tpos, m->val64.p, drop, m->comp_diag, m->diag_struct.p, dir, m->diag_count.p,
          m->nnodes, cnt.p);
    else
      k_export_count<1><<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(
          m->row_ptr, m->col_idx, tpos, m->val64.p, drop, false, m->diag_struct.p, dir, m->diag_count.p, m->nnodes,
          cnt.p);
  }
  LAUNCH_CHECK(ctx);
  colptr.alloc(n + 1);
  size_t tb = 0;
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, colptr.p, (int)(n + 1), ctx->stream));
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(ctx->temp_bytes(tb), tb, cnt.p, colptr.p, (int)(n + 1), ctx->stream));
  return read1(ctx, colptr.p + n);
}

int fcu_matrix_info(fcu_matrix m, int64_t* n, int64_t* nnz) {
  if (!m) return FCU_ERR_BAD_ARG;
  return guarded(m->ctx, [&] {
    if (n) *n = m->n;
    if (nnz) {
      if (!m->space && !m->wrapped_general) *nnz = 9 * m->nnzb;
      else if (!m->bc_applied && !m->drop_zeros && !m->comp_diag && m->space) *nnz = m->space->nnz_ref;
      else {
        DBuf<i64> cp;
        *nnz = export_counts(m, cp);
      }
    }
  });
}

// Row indices and values of the exported CSC, on the device, for the column
// pointers export_counts produced (either output may be null).
static void export_fill(fcu_matrix m, const DBuf<i64>& cp, i64* rowidx_dev, double* vals_dev) {
  fcu_ctx ctx = m->ctx;
  const i64 n = m->n;
  const unsigned char* dir = m->bc_applied ? m->dirichlet.p : nullptr;
  if (m->wrapped_general) {
    k_wexport_fill<<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(
        m->csc_colptr.p, m->csc_rowidx.p, m->csr_of.p, m->drop_zeros, dir, m->diag_count.p, m->val64.p, n, cp.p,
        rowidx_dev, vals_dev);
  } else {
    build_transpose_positions(m->space);
    if (m->bs == 3)
      k_export_fill<3><<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(
          m->row_ptr, m->col_idx, m->space->tpos.p, m->drop_zeros, m->comp_diag, m->diag_struct.p, dir,
          m->diag_count.p, m->val64.p, m->nnodes, cp.p, rowidx_dev, vals_dev);
    else
      k_export_fill<1><<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(
          m->row_ptr, m->col_idx, m->space->tpos.p, m->drop_zeros, false, m->diag_struct.p, dir, m->diag_count.p,
          m->val64.p, m->nnodes, cp.p, rowidx_dev, vals_dev);
  }
  LAUNCH_CHECK(ctx);
}

int fcu_matrix_export_csc(fcu_ctx ctx, fcu_matrix m, int64_t* colptr, int64_t* rowidx, double* vals) {
  return guarded(ctx, [&] {
    if (!m) fail(FCU_ERR_BAD_ARG, "null matrix");
    const i64 n = m->n;
    DBuf<i64> cp;
    const i64 nnz = export_counts(m, cp);
    DevOut<i64> R(rowidx, nnz);
    DevOut<double> V(vals, nnz);
    if (rowidx || vals) export_fill(m, cp, R.p, V.p);
    if (colptr) download(ctx, colptr, cp.p, (size_t)(n + 1));
    R.finish(ctx);
    V.finish(ctx);
    sync(ctx);
  });
}

int fcu_assemble_stiffness(fcu_ctx ctx, fcu_matrix m, const double* cell_coef) {
  return guarded(ctx, [&] {
    if (!m || !m->space) fail(FCU_ERR_BAD_ARG, "matrix has no function space");
    if (m->space->kind == FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "use fcu_assemble_elasticity for vector spaces");
    if (m->space->kind == FCU_SPACE_P2_NODES_VEC3) fail(FCU_ERR_UNSUPPORTED, "no vector P2 stiffness");
    DevIn<double> coef(ctx, cell_coef, (size_t)m->space->mesh->nc);
    reset_dirichlet(m);
    m->comp_diag = false;
    assemble_stiffness_impl(m, coef.p);
    m->has_values = true;
    if (coef.staged.p) sync(ctx);
  });
}

int fcu_assemble_elasticity(fcu_ctx ctx, fcu_matrix m, double E, double nu, const double* cell_E) {
  return guarded(ctx, [&] {
    if (!m || !m->space || m->space->kind != FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "needs a FCU_SPACE_P1_VEC3 matrix");
    if (!(nu > -1.0 && nu < 0.5)) fail(FCU_ERR_BAD_ARG, "Poisson's ratio must be in (-1.0, 0.5) for physical stability");
    DevIn<double> ce(ctx, cell_E, (size_t)m->space->mesh->nc);
    reset_dirichlet(m);
    m->comp_diag = false;
    assemble_elasticity_impl(m, E, nu, ce.p);
    m->has_values = true;
    if (ce.staged.p) sync(ctx);
  });
}

int fcu_assemble_mass(fcu_ctx ctx, fcu_matrix m, double rho, const double* cell_coef) {
  return guarded(ctx, [&] {
    if (!m || !m->space) fail(FCU_ERR_BAD_ARG, "matrix has no function space");
    DevIn<double> coef(ctx, cell_coef, (size_t)m->space->mesh->nc);
    reset_dirichlet(m);
    m->comp_diag = m->bs == 3;
    assemble_mass_impl(m, rho, coef.p);
    m->has_values = true;
    if (coef.staged.p) sync(ctx);
  });
}

int fcu_matrix_clone(fcu_ctx ctx, fcu_matrix src, fcu_matrix* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    if (!src) fail(FCU_ERR_BAD_ARG, "null matrix");
    fcu_matrix m = matrix_clone(src);
    sync(ctx);
    *out = m;
  });
}

int fcu_matrix_add_scaled(fcu_ctx ctx, fcu_matrix out, fcu_matrix a, fcu_matrix b, double alpha) {
  return guarded(ctx, [&] {
    if (!out || !a || !b) fail(FCU_ERR_BAD_ARG, "null matrix");
    if (!a->has_values || !b->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (a->bc_applied || b->bc_applied)
      fail(FCU_ERR_UNSUPPORTED, "add_scaled_matrices: an operand has eliminated or folded Dirichlet dofs");
    if (!same_pattern(a, b) || !same_pattern(a, out))
      fail(FCU_ERR_UNSUPPORTED, "add_scaled_matrices: operands must share one sparsity pattern");
    reset_dirichlet(out);
    out->comp_diag = a->comp_diag && b->comp_diag;
    add_scaled_impl(out, a, b, alpha);
    out->has_values = true;
    sync(ctx);
  });
}

// add_scaled_matrices on two CSC layouts (transient.rs:72-97): per column,
// the union of the two sorted row lists. The triplet build sums a duplicate
// in push order, so an entry held by both is a + (alpha * b), one held by b
// alone is alpha * b, and explicit zeros stay. One thread per column.
__global__ void k_union_count(const i64* __restrict__ acp, const i64* __restrict__ ari,
                              const i64* __restrict__ bcp, const i64* __restrict__ bri, i64 n,
                              i64* __restrict__ cnt) {
  for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < n; j += (i64)gridDim.x * blockDim.x) {
    i64 p = acp[j], q = bcp[j], c = 0;
    const i64 pe = acp[j + 1], qe = bcp[j + 1];
    while (p < pe && q < qe) {
      const i64 ra = ari[p], rb = bri[q];
      p += ra <= rb;
      q += rb <= ra;
      ++c;
    }
    cnt[j] = c + (pe - p) + (qe - q);
  }
}

__global__ void k_union_fill(const i64* __restrict__ acp, const i64* __restrict__ ari, const double* __restrict__ av,
                             const i64* __restrict__ bcp, const i64* __restrict__ bri, const double* __restrict__ bv,
                             double alpha, i64 n, const i64* __restrict__ ccp, i64* __restrict__ cri,
                             double* __restrict__ cv) {
  for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < n; j += (i64)gridDim.x * blockDim.x) {
    i64 p = acp[j], q = bcp[j], o = ccp[j];
    const i64 pe = acp[j + 1], qe = bcp[j + 1];
    while (p < pe || q < qe) {
      const i64 ra = p < pe ? ari[p] : LLONG_MAX, rb = q < qe ? bri[q] : LLONG_MAX;
      if (ra < rb) {
        cri[o] = ra;
        cv[o] = av[p++];
      } else if (rb < ra) {
        cri[o] = rb;
        cv[o] = __dmul_rn(alpha, bv[q++]);
      } else {
        cri[o] = ra;
        cv[o] = __dadd_rn(av[p++], __dmul_rn(alpha, bv[q++]));
      }
      ++o;
    }
  }
}

int fcu_matrix_add_scaled_union(fcu_ctx ctx, fcu_matrix a, fcu_matrix b, double alpha, fcu_matrix* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    if (!a || !b) fail(FCU_ERR_BAD_ARG, "null matrix");
    if (!a->has_values || !b->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (a->n != b->n) fail(FCU_ERR_BAD_ARG, "add_scaled_matrices: operands of different order");
    const i64 n = a->n;
    DBuf<i64> acp, bcp, ari, bri, ccp, cri, cnt;
    DBuf<double> av, bv, cv;
    const i64 annz = export_counts(a, acp), bnnz = export_counts(b, bcp);
    ari.alloc(std::max<i64>(annz, 1));
    av.alloc(std::max<i64>(annz, 1));
    bri.alloc(std::max<i64>(bnnz, 1));
    bv.alloc(std::max<i64>(bnnz, 1));
    export_fill(a, acp, ari.p, av.p);
    export_fill(b, bcp, bri.p, bv.p);
    cnt.alloc(n + 1);
    CUDA_CHECK(cudaMemsetAsync(cnt.p + n, 0, sizeof(i64), ctx->stream));
    k_union_count<<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(acp.p, ari.p, bcp.p, bri.p, n, cnt.p);
    LAUNCH_CHECK(ctx);
    ccp.alloc(n + 1);
    size_t tb = 0;
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, ccp.p, (int)(n + 1), ctx->stream));
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(ctx->temp_bytes(tb), tb, cnt.p, ccp.p, (int)(n + 1), ctx->stream));
    const i64 cnnz = read1(ctx, ccp.p + n);
    cri.alloc(std::max<i64>(cnnz, 1));
    cv.alloc(std::max<i64>(cnnz, 1));
    k_union_fill<<<grid_for(n, 128, cap_blocks(ctx)), 128, 0, ctx->stream>>>(acp.p, ari.p, av.p, bcp.p, bri.p, bv.p,
                                                                            alpha, n, ccp.p, cri.p, cv.p);
    LAUNCH_CHECK(ctx);
    fcu_matrix m = nullptr;
    const int rc = fcu_matrix_from_csc(ctx, n, ccp.p, cri.p, cv.p, &m);
    if (rc != FCU_OK) fail(rc, ctx->err);
    *out = m;
  });
}

int fcu_matrix_scale(fcu_ctx ctx, fcu_matrix m, double s) {
  return guarded(ctx, [&] {
    if (!m || !m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (m->bc_applied) fail(FCU_ERR_UNSUPPORTED, "scaling a matrix with eliminated Dirichlet dofs");
    scale_values_impl(m, s);
    sync(ctx);
  });
}

int fcu_matrix_fold_dirichlet(fcu_ctx ctx, fcu_matrix m, int64_t nfixed, const int64_t* fixed, int unit_diag) {
  return guarded(ctx, [&] {
    if (!m || !m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (nfixed < 0 || (nfixed > 0 && !fixed)) fail(FCU_ERR_BAD_ARG, "bad fixed dof list");
    DevIn<i64> d(ctx, fixed, nfixed);
    fold_dirichlet_impl(m, nfixed, d.p, unit_diag != 0, nullptr);
    sync(ctx);
  });
}

int fcu_apply_dirichlet(fcu_ctx ctx, fcu_matrix m, double* b, int64_t nbc, const int64_t* dofs, const double* vals) {
  return guarded(ctx, [&] {
    if (!m || !b || nbc < 0 || (nbc > 0 && (!dofs || !vals))) fail(FCU_ERR_BAD_ARG, "bad Dirichlet arguments");
    if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    DevOut<double> bo(b, m->n, b, ctx);
    DevIn<i64> d(ctx, dofs, nbc);
    DevIn<double> v(ctx, vals, nbc);
    apply_dirichlet_impl(m, bo.p, nbc, d.p, v.p);
    bo.finish(ctx);
    sync(ctx);
  });
}

// ---------------------------------------------------------------------------
// right-hand sides
// ---------------------------------------------------------------------------

static i64 num_qpoints(fcu_space s) { return s->mesh->nc * (s->mesh->dim == 2 ? 3 : 4); }

int fcu_quadrature_points(fcu_ctx ctx, fcu_space s, double* out) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || !out) fail(FCU_ERR_BAD_ARG, "null argument");
    DevOut<double> o(out, num_qpoints(s) * s->mesh->dim);
    if (s->mesh->nc) quadrature_points_impl(s, o.p);
    o.finish(ctx);
    sync(ctx);
  });
}

int fcu_assemble_rhs_values(fcu_ctx ctx, fcu_space s, const double* fq, double* b) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || !b || (!fq && s->mesh->nc)) fail(FCU_ERR_BAD_ARG, "null argument");
    if (s->kind == FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "scalar spaces only");
    DevIn<double> f(ctx, fq, num_qpoints(s));
    DevOut<double> bo(b, s->ndofs);
    rhs_impl(s, -1, f.p, 0.0, 0.0, nullptr, bo.p);
    bo.finish(ctx);
    if (bo.on_host() || f.staged.p) sync(ctx);
  });
}

int fcu_assemble_rhs_source(fcu_ctx ctx, fcu_space s, int source, const double* params, const double* values,
                            double* b) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || !b) fail(FCU_ERR_BAD_ARG, "null argument");
    if (s->kind == FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "scalar spaces only");
    double p[2] = {0.0, 0.0};
    if (source == FCU_SRC_CONSTANT || source == FCU_SRC_SIN_PRODUCT) {
      if (!params) fail(FCU_ERR_BAD_ARG, "params required");
      p[0] = params[0];
      if (source == FCU_SRC_SIN_PRODUCT) p[1] = params[1];
    } else if (source != FCU_SRC_NODAL || !values) {
      fail(FCU_ERR_BAD_ARG, "unknown source or missing nodal values");
    }
    DevIn<double> nv(ctx, values, source == FCU_SRC_NODAL ? (size_t)s->ndofs : 0);
    DevOut<double> bo(b, s->ndofs);
    rhs_impl(s, source, nullptr, p[0], p[1], nv.p, bo.p);
    bo.finish(ctx);
    if (bo.on_host() || nv.staged.p) sync(ctx);
  });
}

int fcu_assemble_body_force(fcu_ctx ctx, fcu_space s, const double* f, double* b) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || !f || !b) fail(FCU_ERR_BAD_ARG, "null argument");
    if (s->kind != FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "vector space only");
    double fh[3];
    CUDA_CHECK(cudaMemcpy(fh, f, sizeof(fh), cudaMemcpyDefault));
    DevOut<double> bo(b, s->ndofs);
    body_force_impl(s, fh, bo.p);
    bo.finish(ctx);
    if (bo.on_host()) sync(ctx);
  });
}

int fcu_assemble_surface_traction(fcu_ctx ctx, fcu_space s, int64_t nf, const int64_t* facets, const double* tq,
                                  double* b) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || !b || nf < 0 || (nf > 0 && (!facets || !tq))) fail(FCU_ERR_BAD_ARG, "bad traction arguments");
    if (s->kind != FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "vector space only");
    DevIn<i64> fd(ctx, facets, 3 * nf);
    DevIn<double> td(ctx, tq, 9 * nf);
    DevOut<double> bo(b, s->ndofs);
    traction_impl(s, nf, fd.p, td.p, bo.p);
    bo.finish(ctx);
    sync(ctx);
  });
}

// ---------------------------------------------------------------------------
// solvers
// ---------------------------------------------------------------------------

int fcu_pcg(fcu_ctx ctx, fcu_matrix m, const double* b, const double* x0, double* x, double tol, int64_t max_iter,
            int precision, fcu_solve_info* info) {
  int status = FCU_OK;
  int rc = guarded(ctx, [&] {
    if (!m || !b || !x) fail(FCU_ERR_BAD_ARG, "null argument");
    if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (precision != FCU_FP64 && precision != FCU_MIXED) fail(FCU_ERR_BAD_ARG, "unknown precision");
    if (max_iter < 0) fail(FCU_ERR_BAD_ARG, "max_iter must be >= 0");
    DevIn<double> bd(ctx, b, m->n);
    DevIn<double> xd0(ctx, x0, x0 ? m->n : 0);
    DevOut<double> xo(x, m->n);
    status = run_pcg(m, bd.p, xd0.p, xo.p, tol, max_iter, precision, false, nullptr, info);
    xo.finish(ctx);
    sync(ctx);
  });
  if (rc != FCU_OK) return rc;
  if (status == FCU_ERR_NO_CONVERGENCE)
    ctx->err = "CG failed to converge within " + std::to_string(max_iter) + " iterations";
  else if (status == FCU_ERR_BREAKDOWN)
    ctx->err = "Breakdown in CG: curvature p^T A p is near zero";
  return status;
}

int fcu_batch_pcg(fcu_ctx ctx, fcu_matrix m, int64_t nb, const int64_t* offsets, const double* b, double* x,
                  double tol, int64_t max_iter, int precision, int64_t* iterations, double* rel_residual,
                  int* status, fcu_solve_info* info) {
  int st = FCU_OK;
  int rc = guarded(ctx, [&] {
    if (!m || !offsets || !b || !x) fail(FCU_ERR_BAD_ARG, "null argument");
    if (precision != FCU_FP64 && precision != FCU_MIXED) fail(FCU_ERR_BAD_ARG, "unknown precision");
    if (nb <= 0) fail(FCU_ERR_BAD_ARG, "need at least one instance");
    std::vector<i64> offs(nb + 1);
    if (is_device_ptr(offsets)) download(ctx, offs.data(), offsets, nb + 1);
    else std::copy(offsets, offsets + nb + 1, offs.begin());
    DevIn<double> bd(ctx, b, m->n);
    DevOut<double> xo(x, m->n);
    st = batch_pcg_impl(m, nb, offs.data(), bd.p, xo.p, tol, max_iter, precision, iterations, rel_residual, status,
                        info);
    xo.finish(ctx);
    sync(ctx);
  });
  if (rc != FCU_OK) return rc;
  if (st == FCU_ERR_NO_CONVERGENCE)
    ctx->err = "CG failed to converge within " + std::to_string(max_iter) + " iterations for some instances";
  else if (st == FCU_ERR_BREAKDOWN)
    ctx->err = "Breakdown in CG: curvature p^T A p is near zero for some instances";
  return st;
}

int fcu_batch_config(fcu_matrix m, int precision, int* lanes_per_row, int* threads_per_cta, int* ctas_per_cluster) {
  if (!m || !lanes_per_row || !threads_per_cta || !ctas_per_cluster) return FCU_ERR_BAD_ARG;
  batch_config(m, precision, lanes_per_row, threads_per_cta, ctas_per_cluster);
  return FCU_OK;
}

int fcu_solve_csr_cg(fcu_ctx ctx, int64_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* vals,
                     const double* inv_diag, const double* b, const double* x0, double rtol, int64_t max_iter,
                     double* x, fcu_solve_info* info) {
  int status = FCU_OK;
  int rc = guarded(ctx, [&] {
    check_ctx(ctx);
    if (n <= 0 || !row_ptr || !inv_diag || !b || !x) fail(FCU_ERR_BAD_ARG, "bad CSR arguments");
    uint32_t nnz32 = 0;
    CUDA_CHECK(cudaMemcpy(&nnz32, row_ptr + n, sizeof(uint32_t), cudaMemcpyDefault));
    const i64 nnz = nnz32;
    if (nnz > 0 && (!col_idx || !vals)) fail(FCU_ERR_BAD_ARG, "bad CSR arrays");
    if (nnz >= (1ll << 31)) fail(FCU_ERR_UNSUPPORTED, "nnz exceeds 32-bit indexing");
    std::unique_ptr<fcu_matrix_s> m(new fcu_matrix_s());
    m->ctx = ctx;
    m->n = m->nnodes = n;
    m->bs = 1;
    m->nnzb = nnz;
    DevIn<uint32_t> rpd(ctx, row_ptr, n + 1), cid(ctx, col_idx, nnz);
    DBuf<int> bad;
    bad.alloc(1);
    CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
    m->own_row_ptr.alloc(n + 1);
    m->own_col_idx.alloc(nnz);
    m->own_diag_pos.alloc(n);
    k_u32_to_i32<<<grid_for(n + 1, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(rpd.p, n + 1, nnz, m->own_row_ptr.p, bad.p);
    LAUNCH_CHECK(ctx);
    if (nnz) {
      k_u32_to_i32<<<grid_for(nnz, 256, cap_blocks(ctx)), 256, 0, ctx->stream>>>(cid.p, nnz, n - 1, m->own_col_idx.p, bad.p);
      LAUNCH_CHECK(ctx);
    }
    if (read1(ctx, bad.p)) fail(FCU_ERR_BAD_ARG, "CSR index out of range");
    upload(ctx, m->val64, vals, nnz);
    m->val32.alloc(nnz);
    m->row_ptr = m->own_row_ptr.p;
    m->col_idx = m->own_col_idx.p;
    m->diag_pos = m->own_diag_pos.p;
    m->has_values = true;
    DevIn<double> idd(ctx, inv_diag, n), bd(ctx, b, n), x0d(ctx, x0, x0 ? n : 0);
    DevOut<double> xo(x, n);
    status = run_pcg(m.get(), bd.p, x0d.p, xo.p, rtol, max_iter, FCU_FP64, true, idd.p, info);
    xo.finish(ctx);
    sync(ctx);
  });
  return rc != FCU_OK ? rc : status;
}

// Allocation-free variant of fcu_solve_csr_cg for callers that cannot
// allocate device memory at solve time; errors go to fcu_last_error(NULL).
int fcu_solve_csr_cg_noalloc(int64_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* vals,
                             const double* inv_diag, const double* b, const double* x0, double rtol,
                             int64_t max_iter, double* x, fcu_solve_info* info, void* stream) {
  int status = FCU_OK;
  int rc = guarded(nullptr, [&] {
    status = run_pcg_noalloc(n, row_ptr, col_idx, vals, inv_diag, b, x0, rtol, max_iter, x, info, stream);
  });
  return rc != FCU_OK ? rc : status;
}

int fcu_spmv(fcu_ctx ctx, fcu_matrix m, const double* x, double* y) {
  return guarded(ctx, [&] {
    if (!m || !x || !y) fail(FCU_ERR_BAD_ARG, "null argument");
    if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    DevIn<double> xd(ctx, x, m->n);
    DevOut<double> yo(y, m->n);
    spmv_impl(m, xd.p, yo.p);
    yo.finish(ctx);
    if (yo.on_host() || xd.staged.p) sync(ctx);
  });
}

int fcu_adjoint_gradient(fcu_ctx ctx, fcu_space s, double E0, double nu, const double* theta, const double* u,
                         const double* lambda, double* grad) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || s->kind != FCU_SPACE_P1_VEC3) fail(FCU_ERR_BAD_ARG, "needs a FCU_SPACE_P1_VEC3 space");
    if (!theta || !u || !lambda || !grad) fail(FCU_ERR_BAD_ARG, "null argument");
    if (!(nu > -1.0 && nu < 0.5)) fail(FCU_ERR_BAD_ARG, "Poisson's ratio must be in (-1.0, 0.5)");
    const i64 nc = s->mesh->nc;
    DevIn<double> th(ctx, theta, nc), ud(ctx, u, s->ndofs), ld(ctx, lambda, s->ndofs);
    DevOut<double> g(grad, nc);
    if (nc) adjoint_gradient_impl(s, E0, nu, th.p, ud.p, ld.p, g.p);
    g.finish(ctx);
    if (g.on_host() || th.staged.p || ud.staged.p || ld.staged.p) sync(ctx);
  });
}

int fcu_element_stresses(fcu_ctx ctx, fcu_space s, double E, double nu, const double* u, double* stress,
                         double* strain, double* von_mises, double* trace) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || (s->kind != FCU_SPACE_P1_VEC3 && !(s->kind == FCU_SPACE_P1 && s->mesh->dim == 3)))
      fail(FCU_ERR_BAD_ARG, "needs a space on a tetrahedron mesh (P1 or vector P1)");
    if (!u) fail(FCU_ERR_BAD_ARG, "null displacement");
    if (!(nu > -1.0 && nu < 0.5)) fail(FCU_ERR_BAD_ARG, "Poisson's ratio must be in (-1.0, 0.5)");
    // ElasticMaterial::lame_lambda / lame_mu (elasticity.rs:33-47)
    const double lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    const i64 nc = s->mesh->nc;
    DevIn<double> ud(ctx, u, 3 * s->mesh->nv);
    DevOut<double> so(stress, 9 * nc), eo(strain, 9 * nc), vo(von_mises, nc), to(trace, nc);
    if (nc) element_stresses_impl(s, lam, mu, ud.p, so.p, eo.p, vo.p, to.p);
    so.finish(ctx);
    eo.finish(ctx);
    vo.finish(ctx);
    to.finish(ctx);
    sync(ctx);
  });
}

int fcu_vertex_von_mises(fcu_ctx ctx, fcu_space s, const double* cell_von_mises, double* vertex_von_mises) {
  return guarded(ctx, [&] {
    reject_node_space(s);
    if (!s || (s->kind != FCU_SPACE_P1_VEC3 && !(s->kind == FCU_SPACE_P1 && s->mesh->dim == 3)))
      fail(FCU_ERR_BAD_ARG, "needs a space on a tetrahedron mesh (P1 or vector P1)");
    if (!cell_von_mises || !vertex_von_mises) fail(FCU_ERR_BAD_ARG, "null argument");
    DevIn<double> cv(ctx, cell_von_mises, s->mesh->nc);
    DevOut<double> vo(vertex_von_mises, s->mesh->nv);
    if (s->mesh->nv) vertex_von_mises_impl(s, cv.p, vo.p);
    vo.finish(ctx);
    sync(ctx);
  });
}

// ---------------------------------------------------------------------------
// transient stepper and vibration modes
// ---------------------------------------------------------------------------

int fcu_transient_create(fcu_ctx ctx, fcu_matrix mass, fcu_matrix stiff, int scheme, double dt, fcu_transient* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    if (!mass || !stiff) fail(FCU_ERR_BAD_ARG, "null matrix");
    if (!mass->has_values || !stiff->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (scheme != FCU_BACKWARD_EULER && scheme != FCU_CRANK_NICOLSON) fail(FCU_ERR_BAD_ARG, "unknown scheme");
    if (!(dt > 0.0)) fail(FCU_ERR_BAD_ARG, "dt must be positive");
    if (mass->bc_applied || stiff->bc_applied)
      fail(FCU_ERR_UNSUPPORTED, "add_scaled_matrices: an operand has eliminated or folded Dirichlet dofs");
    if (!same_pattern(mass, stiff))
      fail(FCU_ERR_UNSUPPORTED, "add_scaled_matrices: operands must share one sparsity pattern");
    fcu_transient t = transient_create_impl(mass, stiff, scheme, dt);
    sync(ctx);
    *out = t;
  });
}

int fcu_transient_set_dirichlet(fcu_ctx ctx, fcu_transient ts, int64_t nbc, const int64_t* dofs, const double* vals) {
  return guarded(ctx, [&] {
    if (!ts || nbc < 0 || (nbc > 0 && (!dofs || !vals))) fail(FCU_ERR_BAD_ARG, "bad Dirichlet arguments");
    std::vector<i64> d(nbc);
    std::vector<double> v(nbc);
    if (nbc) {
      download(ctx, d.data(), dofs, nbc);
      download(ctx, v.data(), vals, nbc);
      sync(ctx);
    }
    transient_set_dirichlet_impl(ts, nbc, d.data(), v.data());
  });
}

int fcu_transient_step(fcu_ctx ctx, fcu_transient ts, const double* u_n, const double* f_n, const double* f_next,
                       double* u_next, double tol, int64_t max_iter, int precision, fcu_solve_info* info) {
  int status = FCU_OK;
  int rc = guarded(ctx, [&] {
    if (!ts || !u_n || !u_next) fail(FCU_ERR_BAD_ARG, "null argument");
    if (transient_ctx(ts) != ctx) fail(FCU_ERR_BAD_ARG, "stepper belongs to another context");
    if (precision != FCU_FP64 && precision != FCU_MIXED) fail(FCU_ERR_BAD_ARG, "unknown precision");
    if (max_iter < 0) fail(FCU_ERR_BAD_ARG, "max_iter must be >= 0");
    const i64 n = transient_order(ts);
    DevIn<double> u0(ctx, u_n, n);
    DevIn<double> f0(ctx, f_n, f_n ? n : 0);
    DevIn<double> f1(ctx, f_next, f_next ? n : 0);
    DevOut<double> uo(u_next, n);
    status = transient_step_impl(ts, u0.p, f0.p, f1.p, uo.p, tol, max_iter, precision, info);
    uo.finish(ctx);
    sync(ctx);
  });
  if (rc != FCU_OK) return rc;
  if (status == FCU_ERR_NO_CONVERGENCE)
    ctx->err = "CG failed to converge within " + std::to_string(max_iter) + " iterations";
  else if (status == FCU_ERR_BREAKDOWN)
    ctx->err = "Breakdown in CG: curvature p^T A p is near zero";
  return status;
}

void fcu_transient_destroy(fcu_transient ts) { transient_destroy_impl(ts); }

int fcu_vibration_modes(fcu_ctx ctx, fcu_matrix k, fcu_matrix m, int64_t nfixed, const int64_t* fixed,
                        int64_t num_modes, int64_t max_power_iters, double tol, double inner_tol,
                        int64_t inner_max_iter, int precision, fcu_inner_solve inner, void* user,
                        double* eigenvalues, double* mode_shapes, int64_t* power_iterations, fcu_solve_info* info) {
  int status = FCU_OK;
  std::string err;
  int rc = guarded(ctx, [&] {
    if (!k || !m || !eigenvalues) fail(FCU_ERR_BAD_ARG, "null argument");
    if (!k->has_values || !m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (k->n != m->n) fail(FCU_ERR_BAD_ARG, "stiffness and mass orders differ");
    if (num_modes < 0 || max_power_iters < 0 || inner_max_iter < 0 || nfixed < 0 || (nfixed > 0 && !fixed))
      fail(FCU_ERR_BAD_ARG, "bad arguments");
    if (precision != FCU_FP64 && precision != FCU_MIXED) fail(FCU_ERR_BAD_ARG, "unknown precision");
    const i64 n = k->n;
    DevIn<i64> fx(ctx, fixed, nfixed);
    DBuf<double> modes_own;
    DevOut<double> mo(mode_shapes, mode_shapes ? (size_t)(num_modes * n) : 0);
    double* modes = mo.p;
    if (!modes) {
      modes_own.alloc((size_t)std::max<i64>(num_modes, 1) * n);
      modes = modes_own.p;
    }
    std::vector<double> ev(std::max<i64>(num_modes, 1));
    std::vector<i64> pit(std::max<i64>(num_modes, 1));
    status = vibration_modes_impl(k, m, nfixed, fx.p, num_modes, max_power_iters, tol, inner_tol, inner_max_iter,
                                  precision, inner, user, ev.data(), modes, pit.data(), info, &err);
    if (status == FCU_OK) {
      std::copy(ev.begin(), ev.begin() + num_modes, eigenvalues);
      if (power_iterations) std::copy(pit.begin(), pit.begin() + num_modes, power_iterations);
      mo.finish(ctx);
    }
    sync(ctx);
  });
  if (rc != FCU_OK) return rc;
  if (status != FCU_OK) ctx->err = err;
  return status;
}

// ---------------------------------------------------------------------------
// 3x3 block CSR
// ---------------------------------------------------------------------------

static fcu_matrix bsr3_from_caller(fcu_ctx ctx, int64_t n_nodes, const uint32_t* row_ptr, const uint32_t* cols,
                                   const double* vals_flat, const double* dinv_flat) {
  if (n_nodes <= 0 || !row_ptr) fail(FCU_ERR_BAD_ARG, "bad block CSR arguments");
  i64 nnzb = 0;
  {
    DevIn<uint32_t> rp(ctx, row_ptr + n_nodes, 1);
    nnzb = read1(ctx, rp.p);
  }
  if (nnzb > 0 && (!cols || !vals_flat)) fail(FCU_ERR_BAD_ARG, "bad block CSR arrays");
  DevIn<uint32_t> rp(ctx, row_ptr, n_nodes + 1);
  DevIn<uint32_t> ci(ctx, cols, nnzb);
  DevIn<double> va(ctx, vals_flat, 9 * nnzb);
  DevIn<double> di(ctx, dinv_flat, dinv_flat ? 9 * n_nodes : 0);
  return bsr3_create_impl(ctx, n_nodes, rp.p, ci.p, nnzb, va.p, di.p);
}

int fcu_bsr3_create(fcu_ctx ctx, int64_t n_nodes, const uint32_t* row_ptr, const uint32_t* cols,
                    const double* vals_flat, const double* dinv_flat, fcu_matrix* out) {
  if (!out) return FCU_ERR_BAD_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    check_ctx(ctx);
    *out = bsr3_from_caller(ctx, n_nodes, row_ptr, cols, vals_flat, dinv_flat);
  });
}

int fcu_bsr3_jacobi_smooth(fcu_ctx ctx, fcu_matrix m, const double* r, double* z, int64_t sweeps, double omega,
                           int zero_initial_z) {
  return guarded(ctx, [&] {
    if (!m || m->bs != 3 || !r || !z || sweeps < 0) fail(FCU_ERR_BAD_ARG, "bad arguments");
    if (sweeps == 0) return;
    DevIn<double> rd(ctx, r, m->n);
    DevOut<double> zo(z, m->n, zero_initial_z ? nullptr : z, ctx);
    bsr3_jacobi_smooth_impl(m, rd.p, zo.p, sweeps, omega, zero_initial_z != 0);
    zo.finish(ctx);
    sync(ctx);
  });
}

int fcu_solve_bsr3_pcg(fcu_ctx ctx, int64_t n_nodes, const uint32_t* row_ptr, const uint32_t* cols,
                       const double* vals_flat, const double* dinv_flat, const double* b, const double* x0,
                       double rtol, int64_t max_iter, double* x, fcu_solve_info* info) {
  int status = FCU_OK;
  int rc = guarded(ctx, [&] {
    check_ctx(ctx);
    if (!b || !x || !dinv_flat) fail(FCU_ERR_BAD_ARG, "null argument");
    if (max_iter < 0) fail(FCU_ERR_BAD_ARG, "max_iter must be >= 0");
    struct Own {
      fcu_matrix p;
      ~Own() { if (p) matrix_release(p); }
    } m{bsr3_from_caller(ctx, n_nodes, row_ptr, cols, vals_flat, dinv_flat)};
    const i64 n = 3 * n_nodes;
    DevIn<double> bd(ctx, b, n);
    DevIn<double> xd0(ctx, x0, x0 ? n : 0);
    DevOut<double> xo(x, n);
    status = run_pcg(m.p, bd.p, xd0.p, xo.p, rtol, max_iter, FCU_FP64, true, nullptr, info);
    xo.finish(ctx);
    sync(ctx);
  });
  return rc != FCU_OK ? rc : status;
}

int fcu_matrix_block_jacobi(fcu_ctx ctx, fcu_matrix m, int enable) {
  return guarded(ctx, [&] {
    if (!m || m->bs != 3) fail(FCU_ERR_BAD_ARG, "needs a 3x3 block matrix");
    if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    matrix_block_jacobi_impl(m, enable != 0);
    sync(ctx);
  });
}

int fcu_matrix_export_bsr3(fcu_ctx ctx, fcu_matrix m, uint32_t* row_ptr, uint32_t* cols, double* vals_flat,
                           double* dinv_flat) {
  return guarded(ctx, [&] {
    if (!m || m->bs != 3) fail(FCU_ERR_BAD_ARG, "needs a 3x3 block matrix");
    DevOut<uint32_t> rp(row_ptr, row_ptr ? m->nnodes + 1 : 0);
    DevOut<uint32_t> ci(cols, cols ? m->nnzb : 0);
    DevOut<double> va(vals_flat, vals_flat ? 9 * m->nnzb : 0);
    DevOut<double> di(dinv_flat, dinv_flat ? 9 * m->nnodes : 0);
    matrix_export_bsr3_impl(m, rp.p, ci.p, va.p, di.p);
    rp.finish(ctx);
    ci.finish(ctx);
    va.finish(ctx);
    di.finish(ctx);
    sync(ctx);
  });
}

int fcu_time_spmv(fcu_ctx ctx, fcu_matrix m, int precision, int reps, double* ms_per_launch,
                  double* bytes_per_launch) {
  return guarded(ctx, [&] {
    if (!m || !ms_per_launch || !bytes_per_launch || reps < 0) fail(FCU_ERR_BAD_ARG, "bad arguments");
    if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (precision != FCU_FP64 && precision != FCU_MIXED) fail(FCU_ERR_BAD_ARG, "unknown precision");
    time_spmv_impl(m, precision, reps, ms_per_launch, bytes_per_launch);
  });
}

int fcu_time_spmv_cold(fcu_ctx ctx, fcu_matrix m, int precision, int reps, size_t flush_bytes,
                       double* ms_per_launch, double* bytes_per_launch) {
  return guarded(ctx, [&] {
    if (!m || !ms_per_launch || !bytes_per_launch || reps < 0) fail(FCU_ERR_BAD_ARG, "bad arguments");
    if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (precision != FCU_FP64 && precision != FCU_MIXED) fail(FCU_ERR_BAD_ARG, "unknown precision");
    time_spmv_cold_impl(m, precision, reps, flush_bytes, ms_per_launch, bytes_per_launch);
  });
}

int fcu_time_pcg(fcu_ctx ctx, fcu_matrix m, int precision, int64_t iterations, int reps, size_t flush_bytes,
                 double* ms_per_launch, double* bytes_per_launch) {
  return guarded(ctx, [&] {
    if (!m || !ms_per_launch || !bytes_per_launch || reps < 0 || iterations < 1) fail(FCU_ERR_BAD_ARG, "bad arguments");
    if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
    if (precision != FCU_FP64 && precision != FCU_MIXED) fail(FCU_ERR_BAD_ARG, "unknown precision");
    time_pcg_impl(m, precision, iterations, reps, flush_bytes, ms_per_launch, bytes_per_launch);
  });
}

int fcu_check_wait_limits(fcu_ctx ctx, uint32_t polls, int* results) {
  return guarded(ctx, [&] {
    check_ctx(ctx);
    if (!results || polls < 1 || polls > (1u << 20)) fail(FCU_ERR_BAD_ARG, "bad arguments");
    check_wait_limits_impl(ctx, polls, results);
  });
}

}  // extern "C"
