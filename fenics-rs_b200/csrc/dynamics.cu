// Consumers of the mass matrix: entry-wise matrix combinations, Dirichlet
// folding, the transient heat stepper and the vibration-mode solver
// (inverse power iteration with mass-orthogonal deflation).
//
// Data layout: every operand lives on one sparsity pattern (the space's
// node pattern, or the CSR of a wrapped CSC matrix), so combinations are
// element-wise passes over the value arrays (HBM-bound, one read per operand
// and one write). Vectors are FP64 device arrays of the matrix order.
//
// The stepper keeps its left-hand matrix (and the right-hand one for
// Crank-Nicolson) resident between steps; each step is one SpMV pass fused
// with the load terms, then the PCG of solver.cu warm-started from the
// current state. The vibration-mode solver keeps the folded stiffness, the
// folded mass and every converged mode on the device; the inner solve is the
// same PCG (or a caller's callback), and the host only sees the scalars the
// iteration branches on.

#include <cmath>
#include <memory>

#include "internal.cuh"

int run_pcg(fcu_matrix m, const double* b_dev, const double* x0_dev, double* x_dev, double tol, i64 max_iter,
            int precision, bool gpu_semantics, const double* inv_diag_dev, fcu_solve_info* info);
void spmv_impl(fcu_matrix m, const double* x_dev, double* y_dev);
fcu_matrix matrix_clone(fcu_matrix src);
void matrix_release_ref(fcu_matrix m);

namespace {

constexpr int VT = 256;

int vec_grid(fcu_ctx ctx, i64 n) { return (int)grid_for(n, VT, ctx->num_sms * 4); }

// ---------------------------------------------------------------------------
// Entry-wise value passes (val64 and its FP32 copy)
// ---------------------------------------------------------------------------

// add_scaled_matrices (transient.rs:72-97) on one pattern: the triplet list
// holds a's entry then alpha * b's, summed in that order: a + (alpha * b).
__global__ void k_add_scaled(const double* __restrict__ a, const double* __restrict__ b, double alpha, i64 n,
                             double* __restrict__ o64, float* __restrict__ o32) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const double v = __dadd_rn(a[i], __dmul_rn(alpha, b[i]));
    o64[i] = v;
    o32[i] = (float)v;
  }
}

__global__ void k_scale_values(double s, i64 n, double* __restrict__ v64, float* __restrict__ v32) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const double v = __dmul_rn(s, v64[i]);
    v64[i] = v;
    v32[i] = (float)v;
  }
}

__global__ void k_ne_i64(const i64* __restrict__ a, const i64* __restrict__ b, i64 n, int* __restrict__ diff) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    if (a[i] != b[i]) atomicExch(diff, 1);
}

// ---------------------------------------------------------------------------
// fold_dirichlet (eigen.rs:55-79): entries on a fixed row or column become 0,
// the fixed diagonal 1 (unit_diag) or 0. Out-of-range dofs are ignored.
// ---------------------------------------------------------------------------

__global__ void k_mark_fixed(const i64* __restrict__ dofs, i64 nf, i64 n, unsigned char* __restrict__ fixed,
                             int* __restrict__ bad) {
  for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < nf; j += (i64)gridDim.x * blockDim.x) {
    const i64 d = dofs[j];
    if (d < 0) atomicExch(bad, 1);
    else if (d < n) fixed[d] = 1;
  }
}

template <int BS>
__global__ void k_fold(const int* __restrict__ rp, const int* __restrict__ ci, const unsigned char* __restrict__ fixed,
                       i64 nn, bool unit_diag, double* __restrict__ v64, float* __restrict__ v32) {
  const int lane = threadIdx.x & 31;
  const i64 w0 = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
  const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
  for (i64 node = w0; node < nn; node += nw) {
    const int rs = rp[node], re = rp[node + 1];
    for (i64 q = (i64)rs * BS * BS + lane; q < (i64)re * BS * BS; q += 32) {
      const i64 p = q / (BS * BS);
      const int rem = (int)(q - p * BS * BS);
      const i64 r = node * BS + rem / BS;
      const i64 c = (i64)ci[p] * BS + rem % BS;
      if (fixed[r] || fixed[c]) {
        const double v = (r == c && unit_diag) ? 1.0 : 0.0;
        v64[q] = v;
        v32[q] = (float)v;
      }
    }
  }
}

__global__ void k_fold_flags(const unsigned char* __restrict__ fixed, i64 n, bool unit_diag,
                             unsigned char* __restrict__ dir, double* __restrict__ dcount) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    if (fixed[i]) {
      dir[i] = 1;
      dcount[i] = unit_diag ? 1.0 : 0.0;
    }
}

// ---------------------------------------------------------------------------
// Deterministic reductions: fixed grid, per-block partials in shared memory
// (fixed tree), then one block sums the partials in index order.
// ---------------------------------------------------------------------------

__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int s = VT / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] += sh[t + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(VT) k_dot_partial(const double* __restrict__ a, const double* __restrict__ b, i64 n,
                                                    double* __restrict__ part) {
  __shared__ double sh[VT];
  double acc = 0.0;
  for (i64 i = blockIdx.x * (i64)VT + threadIdx.x; i < n; i += (i64)gridDim.x * VT) acc += a[i] * b[i];
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// mean_abs_diag (eigen.rs:22-45): sum and count of the stored, non-zero
// diagonal entries (a folded matrix stores no zero entries).
template <int BS>
__global__ void __launch_bounds__(VT) k_diag_abs_partial(const int* __restrict__ diag_pos,
                                                         const double* __restrict__ v64, i64 n,
                                                         double* __restrict__ part, double* __restrict__ cpart) {
  __shared__ double sh[VT];
  double acc = 0.0, cnt = 0.0;
  for (i64 d = blockIdx.x * (i64)VT + threadIdx.x; d < n; d += (i64)gridDim.x * VT) {
    const i64 w = d / BS;
    const int a = (int)(d - w * BS);
    const int dp = diag_pos[w];
    const double v = dp >= 0 ? v64[(i64)dp * BS * BS + a * BS + a] : 0.0;
    if (v != 0.0) {
      acc += fabs(v);
      cnt += 1.0;
    }
  }
  const double s = block_sum(acc, sh);
  const double c = block_sum(cnt, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s;
    cpart[blockIdx.x] = c;
  }
}

__global__ void __launch_bounds__(VT) k_sum_partials(const double* __restrict__ part, int np, double* __restrict__ out) {
  __shared__ double sh[VT];
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += VT) acc += part[i];
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// Vector passes (explicit roundings: the reference's scalar loops)
// ---------------------------------------------------------------------------

// y -= c x (eigen.rs:160-164, 188-193)
__global__ void k_sub_scaled(double* __restrict__ y, const double* __restrict__ x, double c, i64 n) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    y[i] = __dsub_rn(y[i], __dmul_rn(c, x[i]));
}

__global__ void k_scale_vec(double* __restrict__ y, double s, i64 n) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    y[i] = __dmul_rn(y[i], s);
}

__global__ void k_div_vec(double* __restrict__ y, double s, i64 n) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    y[i] = __ddiv_rn(y[i], s);
}

__global__ void k_zero_fixed(double* __restrict__ y, const unsigned char* __restrict__ fixed, i64 n) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    if (fixed[i]) y[i] = 0.0;
}

// Deterministic start vector of a mode (eigen.rs:124-132).
__global__ void k_start_vector(double* __restrict__ v, const unsigned char* __restrict__ fixed, i64 n, i64 mode) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    if (fixed[i]) { v[i] = 0.0; continue; }
    const i64 s = ((i + 1) * 31 + (mode + 1) * 97) % 1000;
    v[i] = (double)s / 1000.0 - 0.5;
  }
}

// Right-hand side of a step (transient.rs:43-65): y = R u_n computed, then
// y + dt f_next (backward Euler) or y + (dt/2)(f_n + f_next) (Crank-Nicolson).
__global__ void k_step_rhs(double* __restrict__ y, const double* __restrict__ fn, const double* __restrict__ fnext,
                           double c, bool cn, i64 n) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    double f;
    if (cn) f = __dadd_rn(fn ? fn[i] : 0.0, fnext ? fnext[i] : 0.0);
    else f = fnext ? fnext[i] : 0.0;
    y[i] = __dadd_rn(y[i], __dmul_rn(c, f));
  }
}

__global__ void k_scatter(double* __restrict__ y, const i64* __restrict__ idx, const double* __restrict__ val, i64 k) {
  for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < k; j += (i64)gridDim.x * blockDim.x)
    y[idx[j]] = val[j];
}

// ---------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------

struct Reducer {
  fcu_ctx ctx;
  int grid;
  DBuf<double> part, cpart, out;
  explicit Reducer(fcu_ctx c, i64 n) : ctx(c) {
    grid = (int)grid_for(n, VT, c->num_sms * 2);
    part.alloc(grid);
    cpart.alloc(grid);
    out.alloc(2);
  }
  double dot(const double* a, const double* b, i64 n) {
    k_dot_partial<<<grid, VT, 0, ctx->stream>>>(a, b, n, part.p);
    LAUNCH_CHECK(ctx);
    k_sum_partials<<<1, VT, 0, ctx->stream>>>(part.p, grid, out.p);
    LAUNCH_CHECK(ctx);
    double h;
    CUDA_CHECK(cudaMemcpyAsync(&h, out.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    return h;
  }
  double mean_abs_diag(fcu_matrix m) {
    if (m->bs == 3)
      k_diag_abs_partial<3><<<grid, VT, 0, ctx->stream>>>(m->diag_pos, m->val64.p, m->n, part.p, cpart.p);
    else
      k_diag_abs_partial<1><<<grid, VT, 0, ctx->stream>>>(m->diag_pos, m->val64.p, m->n, part.p, cpart.p);
    LAUNCH_CHECK(ctx);
    k_sum_partials<<<1, VT, 0, ctx->stream>>>(part.p, grid, out.p);
    LAUNCH_CHECK(ctx);
    k_sum_partials<<<1, VT, 0, ctx->stream>>>(cpart.p, grid, out.p + 1);
    LAUNCH_CHECK(ctx);
    double h[2];
    CUDA_CHECK(cudaMemcpyAsync(h, out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    return h[1] == 0.0 ? 0.0 : h[0] / h[1];
  }
};

void launch_vec(fcu_ctx ctx) { LAUNCH_CHECK(ctx); }

}  // namespace

// ---------------------------------------------------------------------------
// Entry points (called from api.cu)
// ---------------------------------------------------------------------------

// True when a and b store the same pattern: one space, or wrapped CSC
// matrices whose column pointers and row indices are identical.
bool same_pattern(fcu_matrix a, fcu_matrix b) {
  if (a == b) return true;
  if (a->space || b->space) return a->space == b->space;
  if (a->n != b->n || a->nnzb != b->nnzb || !a->wrapped_general || !b->wrapped_general) return false;
  if (a->csc_colptr.n != b->csc_colptr.n || a->csc_rowidx.n != b->csc_rowidx.n) return false;
  fcu_ctx ctx = a->ctx;
  DBuf<int> diff;
  diff.alloc(1);
  CUDA_CHECK(cudaMemsetAsync(diff.p, 0, sizeof(int), ctx->stream));
  k_ne_i64<<<vec_grid(ctx, a->csc_colptr.n), VT, 0, ctx->stream>>>(a->csc_colptr.p, b->csc_colptr.p,
                                                                   (i64)a->csc_colptr.n, diff.p);
  LAUNCH_CHECK(ctx);
  if (a->csc_rowidx.n)
    k_ne_i64<<<vec_grid(ctx, a->csc_rowidx.n), VT, 0, ctx->stream>>>(a->csc_rowidx.p, b->csc_rowidx.p,
                                                                     (i64)a->csc_rowidx.n, diff.p);
  LAUNCH_CHECK(ctx);
  int h = 0;
  CUDA_CHECK(cudaMemcpyAsync(&h, diff.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  return h == 0;
}

void add_scaled_impl(fcu_matrix out, fcu_matrix a, fcu_matrix b, double alpha) {
  fcu_ctx ctx = out->ctx;
  const i64 nv = a->nnzb * a->bs * a->bs;
  k_add_scaled<<<vec_grid(ctx, nv), VT, 0, ctx->stream>>>(a->val64.p, b->val64.p, alpha, nv, out->val64.p,
                                                          out->val32.p);
  LAUNCH_CHECK(ctx);
}

void scale_values_impl(fcu_matrix m, double s) {
  fcu_ctx ctx = m->ctx;
  const i64 nv = m->nnzb * m->bs * m->bs;
  k_scale_values<<<vec_grid(ctx, nv), VT, 0, ctx->stream>>>(s, nv, m->val64.p, m->val32.p);
  LAUNCH_CHECK(ctx);
}

// Folds the dofs in place; returns the number of fixed dofs in range.
i64 fold_dirichlet_impl(fcu_matrix m, i64 nf, const i64* dofs_dev, bool unit_diag, DBuf<unsigned char>* fixed_out) {
  fcu_ctx ctx = m->ctx;
  const i64 n = m->n;
  DBuf<unsigned char> fixed;
  DBuf<int> bad;
  fixed.alloc(n);
  bad.alloc(1);
  CUDA_CHECK(cudaMemsetAsync(fixed.p, 0, n, ctx->stream));
  CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
  if (nf > 0) {
    k_mark_fixed<<<vec_grid(ctx, nf), VT, 0, ctx->stream>>>(dofs_dev, nf, n, fixed.p, bad.p);
    LAUNCH_CHECK(ctx);
  }
  int hbad = 0;
  CUDA_CHECK(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  if (hbad) fail(FCU_ERR_BAD_ARG, "fixed dof index is negative");
  const int cap = ctx->num_sms * 16;
  if (m->bs == 3)
    k_fold<3><<<grid_for(m->nnodes * 32, 256, cap), 256, 0, ctx->stream>>>(m->row_ptr, m->col_idx, fixed.p, m->nnodes,
                                                                          unit_diag, m->val64.p, m->val32.p);
  else
    k_fold<1><<<grid_for(m->nnodes * 32, 256, cap), 256, 0, ctx->stream>>>(m->row_ptr, m->col_idx, fixed.p, m->nnodes,
                                                                          unit_diag, m->val64.p, m->val32.p);
  LAUNCH_CHECK(ctx);
  if (!m->dirichlet.p) {
    m->dirichlet.alloc(n);
    CUDA_CHECK(cudaMemsetAsync(m->dirichlet.p, 0, n, ctx->stream));
    m->diag_count.alloc(n);
  }
  k_fold_flags<<<vec_grid(ctx, n), VT, 0, ctx->stream>>>(fixed.p, n, unit_diag, m->dirichlet.p, m->diag_count.p);
  LAUNCH_CHECK(ctx);
  std::vector<unsigned char> hm(n), hf(n);
  CUDA_CHECK(cudaMemcpyAsync(hm.data(), m->dirichlet.p, n, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaMemcpyAsync(hf.data(), fixed.p, n, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  i64 nd = 0, nfx = 0;
  for (i64 i = 0; i < n; ++i) {
    nd += hm[i];
    nfx += hf[i];
  }
  m->n_dirichlet = nd;
  m->bc_applied = true;
  m->drop_zeros = true;
  if (fixed_out) *fixed_out = std::move(fixed);
  return nfx;
}

// ---------------------------------------------------------------------------
// Transient stepper (transient.rs:21-68, heat_solver.rs:82-99)
// ---------------------------------------------------------------------------

struct fcu_transient_s {
  fcu_ctx ctx = nullptr;
  int scheme = 0;
  double dt = 0.0;
  fcu_matrix lhs = nullptr;  // M + theta dt K
  fcu_matrix rhs = nullptr;  // M (backward Euler) or M - dt/2 K (Crank-Nicolson)
  DBuf<double> u, y;         // state with the Dirichlet values, right-hand side
  DBuf<i64> bc_dofs;
  DBuf<double> bc_vals;
  ~fcu_transient_s() {
    if (lhs) matrix_release_ref(lhs);
    if (rhs) matrix_release_ref(rhs);
  }
};

fcu_transient transient_create_impl(fcu_matrix mass, fcu_matrix stiff, int scheme, double dt) {
  std::unique_ptr<fcu_transient_s> t(new fcu_transient_s());
  t->ctx = mass->ctx;
  t->scheme = scheme;
  t->dt = dt;
  t->lhs = matrix_clone(mass);
  t->lhs->comp_diag = mass->comp_diag && stiff->comp_diag;
  const double half_dt = 0.5 * dt;
  if (scheme == FCU_BACKWARD_EULER) {
    add_scaled_impl(t->lhs, mass, stiff, dt);
    t->rhs = matrix_clone(mass);
  } else {
    add_scaled_impl(t->lhs, mass, stiff, half_dt);
    t->rhs = matrix_clone(mass);
    t->rhs->comp_diag = t->lhs->comp_diag;
    add_scaled_impl(t->rhs, mass, stiff, -half_dt);
  }
  t->u.alloc(mass->n);
  t->y.alloc(mass->n);
  return t.release();
}

void transient_destroy_impl(fcu_transient t) {
  if (!t) return;
  cudaSetDevice(t->ctx->device);
  cudaStreamSynchronize(t->ctx->stream);
  delete t;
}

fcu_ctx transient_ctx(fcu_transient t) { return t->ctx; }
i64 transient_order(fcu_transient t) { return t->lhs->n; }

// Dirichlet values written into the state before and after every step, in
// list order (the last value of a repeated dof wins).
void transient_set_dirichlet_impl(fcu_transient t, i64 nbc, const i64* dofs_host, const double* vals_host) {
  const i64 n = t->lhs->n;
  std::vector<i64> last(n, -1);
  for (i64 j = 0; j < nbc; ++j) {
    if (dofs_host[j] < 0 || dofs_host[j] >= n) fail(FCU_ERR_BAD_ARG, "Dirichlet dof index out of range");
    last[dofs_host[j]] = j;
  }
  std::vector<i64> d;
  std::vector<double> v;
  for (i64 i = 0; i < n; ++i)
    if (last[i] >= 0) {
      d.push_back(i);
      v.push_back(vals_host[last[i]]);
    }
  fcu_ctx ctx = t->ctx;
  t->bc_dofs.release();
  t->bc_vals.release();
  if (!d.empty()) {
    upload(ctx, t->bc_dofs, d.data(), d.size());
    upload(ctx, t->bc_vals, v.data(), v.size());
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  }
}

int transient_step_impl(fcu_transient t, const double* un, const double* fn, const double* fnext, double* unext,
                        double tol, i64 max_iter, int precision, fcu_solve_info* info) {
  fcu_ctx ctx = t->ctx;
  const i64 n = t->lhs->n;
  const i64 nbc = (i64)t->bc_dofs.n;
  CUDA_CHECK(cudaMemcpyAsync(t->u.p, un, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (nbc) {
    k_scatter<<<vec_grid(ctx, nbc), VT, 0, ctx->stream>>>(t->u.p, t->bc_dofs.p, t->bc_vals.p, nbc);
    LAUNCH_CHECK(ctx);
  }
  spmv_impl(t->rhs, t->u.p, t->y.p);
  const bool cn = t->scheme == FCU_CRANK_NICOLSON;
  const double c = cn ? 0.5 * t->dt : t->dt;
  k_step_rhs<<<vec_grid(ctx, n), VT, 0, ctx->stream>>>(t->y.p, fn, fnext, c, cn, n);
  LAUNCH_CHECK(ctx);
  const int st = run_pcg(t->lhs, t->y.p, t->u.p, unext, tol, max_iter, precision, false, nullptr, info);
  if (nbc) {
    k_scatter<<<vec_grid(ctx, nbc), VT, 0, ctx->stream>>>(unext, t->bc_dofs.p, t->bc_vals.p, nbc);
    LAUNCH_CHECK(ctx);
  }
  return st;
}

// ---------------------------------------------------------------------------
// Vibration modes (eigen.rs:94-271)
// ---------------------------------------------------------------------------

int vibration_modes_impl(fcu_matrix k, fcu_matrix m, i64 nfixed, const i64* fixed_dev, i64 num_modes,
                         i64 max_power_iters, double tol, double inner_tol, i64 inner_max_iter, int precision,
                         fcu_inner_solve inner, void* user, double* eigenvalues, double* modes_dev,
                         i64* power_iters, fcu_solve_info* info, std::string* err) {
  fcu_ctx ctx = k->ctx;
  const i64 n = k->n;
  // Folded copies (both folds are idempotent; the caller's matrices stay).
  struct Ref {
    fcu_matrix p;
    ~Ref() { if (p) matrix_release_ref(p); }
  } kd{matrix_clone(k)}, md{matrix_clone(m)};
  DBuf<unsigned char> fixed;
  fold_dirichlet_impl(kd.p, nfixed, fixed_dev, true, &fixed);
  // a caller's block-Jacobi preconditioner follows the folded values
  if (kd.p->bdinv.p && !kd.p->block_jacobi) kd.p->bdinv.release();
  const i64 nfx = fold_dirichlet_impl(md.p, nfixed, fixed_dev, false, nullptr);
  if (n - nfx == 0) fail(FCU_ERR_BAD_ARG, "No free degrees of freedom in system");

  Reducer red(ctx, n);
  // Mass rescaling (eigen.rs:120-131): s = mean|diag K| / mean|diag M|.
  double s = 1.0;
  {
    const double kdg = red.mean_abs_diag(kd.p), mdg = red.mean_abs_diag(md.p);
    if (kdg > 0.0 && mdg > 0.0) s = kdg / mdg;
  }
  const double sqrt_s = std::sqrt(s);

  DBuf<double> v, w, mv, tmp, mprev;
  v.alloc(n);
  w.alloc(n);
  mv.alloc(n);
  tmp.alloc(n);
  mprev.alloc((size_t)std::max<i64>(num_modes, 1) * n);
  const int g = vec_grid(ctx, n);
  i64 inner_iters = 0, inner_updates = 0;
  double inner_ms = 0.0;
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  CUDA_CHECK(cudaEventRecord(e0, ctx->stream));

  auto orthogonalize = [&](double* x, i64 nprev) {
    for (i64 j = 0; j < nprev; ++j) {
      const double coeff = red.dot(x, mprev.p + j * n, n);
      k_sub_scaled<<<g, VT, 0, ctx->stream>>>(x, modes_dev + j * n, coeff, n);
      launch_vec(ctx);
    }
  };

  for (i64 mode = 0; mode < num_modes; ++mode) {
    double* vout = modes_dev + mode * n;
    k_start_vector<<<g, VT, 0, ctx->stream>>>(v.p, fixed.p, n, mode);
    launch_vec(ctx);
    // s M p for the converged modes (eigen.rs:137-142)
    if (mode > 0) {
      double* mp = mprev.p + (mode - 1) * n;
      spmv_impl(md.p, modes_dev + (mode - 1) * n, mp);
      k_scale_vec<<<g, VT, 0, ctx->stream>>>(mp, s, n);
      launch_vec(ctx);
    }
    orthogonalize(v.p, mode);
    spmv_impl(md.p, v.p, mv.p);
    k_scale_vec<<<g, VT, 0, ctx->stream>>>(mv.p, s, n);
    launch_vec(ctx);
    const double norm_m = std::sqrt(red.dot(v.p, mv.p, n));
    if (norm_m > 1e-14) {
      k_div_vec<<<g, VT, 0, ctx->stream>>>(v.p, norm_m, n);
      launch_vec(ctx);
    }
    double prev_rayleigh = 0.0;
    i64 it_done = 0;
    for (i64 it = 0; it < max_power_iters; ++it) {
      it_done = it + 1;
      spmv_impl(md.p, v.p, mv.p);
      k_scale_vec<<<g, VT, 0, ctx->stream>>>(mv.p, s, n);
      launch_vec(ctx);
      int st;
      if (inner) {
        CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        st = inner(user, n, mv.p, v.p, w.p);
        if (st != FCU_OK) {
          *err = "inner solve failed (status " + std::to_string(st) + ")";
          return st;
        }
      } else {
        fcu_solve_info ii{};
        st = run_pcg(kd.p, mv.p, v.p, w.p, inner_tol, inner_max_iter, precision, false, nullptr, &ii);
        inner_iters += ii.iterations;
        inner_updates += ii.outer_updates;
        if (st != FCU_OK) {
          *err = st == FCU_ERR_NO_CONVERGENCE
                     ? "CG failed to converge within " + std::to_string(inner_max_iter) + " iterations"
                     : std::string("Breakdown in CG: curvature p^T A p is near zero");
          return st;
        }
      }
      k_zero_fixed<<<g, VT, 0, ctx->stream>>>(w.p, fixed.p, n);
      launch_vec(ctx);
      orthogonalize(w.p, mode);
      spmv_impl(md.p, w.p, tmp.p);
      const double mw_norm = std::sqrt(red.dot(w.p, tmp.p, n)) * sqrt_s;
      if (mw_norm < 1e-15) break;
      k_div_vec<<<g, VT, 0, ctx->stream>>>(w.p, mw_norm, n);
      launch_vec(ctx);
      spmv_impl(kd.p, w.p, tmp.p);
      const double rayleigh = red.dot(w.p, tmp.p, n);
      std::swap(v, w);
      const double denom = std::max(std::fabs(rayleigh), std::fabs(prev_rayleigh));
      if (denom == 0.0 || std::fabs(rayleigh - prev_rayleigh) / denom < tol) break;
      prev_rayleigh = rayleigh;
    }
    // Final quotient on the unscaled mass (eigen.rs:247-255).
    spmv_impl(kd.p, v.p, tmp.p);
    const double vkv = red.dot(v.p, tmp.p, n);
    spmv_impl(md.p, v.p, tmp.p);
    const double vmv = red.dot(v.p, tmp.p, n);
    eigenvalues[mode] = std::max(vkv / vmv, 0.0);
    if (power_iters) power_iters[mode] = it_done;
    CUDA_CHECK(cudaMemcpyAsync(vout, v.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
  CUDA_CHECK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  inner_ms = ms;
  if (info) {
    *info = fcu_solve_info{};
    info->iterations = inner_iters;
    info->outer_updates = inner_updates;
    info->kernel_ms = inner_ms;
    info->status = FCU_OK;
  }
  return FCU_OK;
}
