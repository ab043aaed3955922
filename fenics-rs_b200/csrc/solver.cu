// Jacobi-preconditioned CG on the device: FP64 (the arithmetic of
// cg.rs:40-149) and mixed precision (FP32 SpMV and vector updates, FP64 dot
// accumulation, FP64 residual replacement b - A64 x64 and FP64 solution
// accumulation).
//
// Each iteration is three (FP64) or four (mixed) kernels:
//   spmv      Ap = A p, and p.Ap reduced on the device -> alpha
//   update    x += alpha p, r -= alpha Ap, z = D^-1 r, r.z and r.r -> beta,
//             convergence / iteration-limit decision
//   [reliable mixed only, and only when triggered: r = b - A64 (x64 + x32)]
//   direction p = D^-1 r + beta p
// Scalars never leave the device: every reduction ends in the block that
// finishes last, which sums the per-block partials in a fixed order
// (deterministic) and writes alpha/beta/flags to a small state record. The
// iteration loop is captured once per matrix as a CUDA graph of CHUNK
// iterations; kernels of a converged solve return immediately, and the host
// polls the state once per chunk.

#include <algorithm>
#include <cmath>

#include "internal.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int VBLOCK = 256;  // threads per block in solver kernels
constexpr int MAXG = 4096;   // max blocks of a reducing kernel (partials capacity)
constexpr int CHUNK = 16;    // iterations per graph launch

struct CgState {
  double rz, alpha, beta, bnorm, tol, rr, maxr, delta;
  long long iter, max_iter, updates;
  int done, status, do_update, fold;
  int gpu_semantics;  // solve_csr_cg_gpu: no breakdown test, beta guard, Ok at limit
  int pad;
  unsigned ticket[4];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Block-reduce NV doubles; the last block to finish reduces all partials in
// fixed order and returns true (tot valid in every thread of that block).
template <int NV>
__device__ bool grid_reduce(double (&v)[NV], double* __restrict__ partials, unsigned* ticket, double (&tot)[NV]) {
  __shared__ double sh[NV][VBLOCK / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double x = warp_sum(v[j]);
    if (lane == 0) sh[j][w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double s = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[j][q];
      partials[j * MAXG + blockIdx.x] = s;
    }
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += __ldcg(&partials[j * MAXG + b]);
    s = warp_sum(s);
    __syncthreads();
    if (lane == 0) sh[j][w] = s;
    __syncthreads();
    double t2 = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t2 += sh[j][q];
    tot[j] = t2;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// ---------------------------------------------------------------------------
// Row kernels. CSR: VPR lanes per row. 3x3-block CSR: 15 lanes per block
// row, lane 3j+a handles row a of blocks j, j+5, j+10, ...
// ---------------------------------------------------------------------------

template <class T>
struct XPlain {
  const T* x;
  __device__ __forceinline__ T operator()(i64 c) const { return x[c]; }
};
struct XSum {  // x64 + x32 (mixed precision residual)
  const double* a;
  const float* b;
  __device__ __forceinline__ double operator()(i64 c) const { return a[c] + (double)b[c]; }
};

template <int VPR, class T, class TA, class GX>
__device__ __forceinline__ TA csr_row(const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                                      i64 row, bool valid, int sub, const GX& gx) {
  TA s = TA(0);
  if (valid) {
    const int b = rp[row], e = rp[row + 1];
    for (int p = b + sub; p < e; p += VPR) s += (TA)val[p] * (TA)gx(ci[p]);
  }
#pragma unroll
  for (int o = VPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
  return s;
}

// Returns the partial of row-component a = sub (valid for sub < 3).
template <class T, class TA, class GX>
__device__ __forceinline__ TA bsr3_row(const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                                       i64 row, bool valid, int sub, const GX& gx) {
  TA s = TA(0);
  if (valid && sub < 15) {
    const int j = sub / 3, a = sub - 3 * j;
    const int b = rp[row], e = rp[row + 1];
    for (int kb = b + j; kb < e; kb += 5) {
      const i64 c = 3 * (i64)ci[kb];
      const T* v = val + 9 * (i64)kb + 3 * a;
      s += (TA)v[0] * (TA)gx(c) + (TA)v[1] * (TA)gx(c + 1) + (TA)v[2] * (TA)gx(c + 2);
    }
  }
  TA t;
  t = __shfl_down_sync(FULL, s, 3, 16);
  if (sub + 3 < 16) s += t;
  t = __shfl_down_sync(FULL, s, 6, 16);
  if (sub + 6 < 16) s += t;
  t = __shfl_down_sync(FULL, s, 12, 16);
  if (sub + 12 < 16) s += t;
  return s;
}

// Iterate the rows handled by this thread group; calls emit(row_scalar_index,
// value) once per output scalar row (from one lane).
template <int BS, int VPR, class T, class TA, class GX, class Emit>
__device__ __forceinline__ void spmv_rows(const int* __restrict__ rp, const int* __restrict__ ci,
                                          const T* __restrict__ val, i64 nrows, const GX& gx, Emit& emit) {
  constexpr int G = (BS == 3) ? 16 : VPR;  // lanes per node row
  const int lane = threadIdx.x & 31;
  const int sub = lane % G;
  const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
  const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
  constexpr int RPW = 32 / G;
  for (i64 base = gw * RPW; base < nrows; base += nw * RPW) {
    const i64 row = base + lane / G;
    const bool valid = row < nrows;
    if (BS == 3) {
      TA s = bsr3_row<T, TA>(rp, ci, val, row, valid, sub, gx);
      if (valid && sub < 3) emit(3 * row + sub, s);
    } else {
      TA s = csr_row<VPR, T, TA>(rp, ci, val, row, valid, sub, gx);
      if (valid && sub == 0) emit(row, s);
    }
  }
}

// --- CG step 1: Ap = A p, p.Ap -> alpha ------------------------------------
template <class T>
struct EmitAp {
  const T* p;
  T* ap;
  double dot = 0.0;
  __device__ __forceinline__ void operator()(i64 i, T s) {
    ap[i] = s;
    dot += (double)p[i] * (double)s;
  }
};

template <int BS, int VPR, class T>
__global__ void __launch_bounds__(VBLOCK) k_spmv_ap(const int* __restrict__ rp, const int* __restrict__ ci,
                                                    const T* __restrict__ val, i64 nrows, const T* __restrict__ p,
                                                    T* __restrict__ ap, CgState* st, double* partials) {
  if (st->done) return;
  EmitAp<T> em{p, ap};
  spmv_rows<BS, VPR, T, T>(rp, ci, val, nrows, XPlain<T>{p}, em);
  double v[1] = {em.dot}, tot[1];
  if (grid_reduce<1>(v, partials, &st->ticket[0], tot) && threadIdx.x == 0) {
    const double pap = tot[0];
    if (!st->gpu_semantics && fabs(pap) < 1e-30) {
      st->done = 1;
      st->status = FCU_ERR_BREAKDOWN;
      st->iter += 1;
    } else {
      st->alpha = st->rz / pap;
    }
  }
}

// --- FP64 update ------------------------------------------------------------
__device__ __forceinline__ void decide_after_update(CgState* st, double rz_new, double rr) {
  st->iter += 1;
  st->rr = rr;
  const double res = sqrt(rr);
  const double rel = st->bnorm > 0.0 ? res / st->bnorm : res;
  if (rel < st->tol) { st->done = 1; st->status = FCU_OK; return; }
  if (st->iter >= st->max_iter) {
    st->done = 1;
    st->status = st->gpu_semantics ? FCU_OK : FCU_ERR_NO_CONVERGENCE;
    return;
  }
  const double den = st->gpu_semantics ? fmax(st->rz, 1e-30) : st->rz;
  st->beta = rz_new / den;
  st->rz = rz_new;
}

__global__ void __launch_bounds__(VBLOCK) k_cg_update(i64 n, double* __restrict__ x, double* __restrict__ r,
                                                      const double* __restrict__ p, const double* __restrict__ ap,
                                                      const double* __restrict__ invd, CgState* st,
                                                      double* partials) {
  if (st->done) return;
  const double alpha = st->alpha;
  double rz = 0.0, rr = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * ap[i];
    r[i] = ri;
    const double z = ri * invd[i];
    rz += ri * z;
    rr += ri * ri;
  }
  double v[2] = {rz, rr}, tot[2];
  if (grid_reduce<2>(v, partials, &st->ticket[1], tot) && threadIdx.x == 0) decide_after_update(st, tot[0], tot[1]);
}

template <class T>
__global__ void __launch_bounds__(VBLOCK) k_cg_direction(i64 n, T* __restrict__ p, const T* __restrict__ r,
                                                         const T* __restrict__ invd, const CgState* st) {
  if (st->done) return;
  const T beta = (T)st->beta;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    p[i] = r[i] * invd[i] + beta * p[i];
}

// --- initialisation ---------------------------------------------------------
struct EmitRes {  // r = b - A x (FP64), rr, bb
  const double* b;
  double* r;
  double rr = 0.0;
  __device__ __forceinline__ void operator()(i64 i, double s) {
    const double v = b[i] - s;
    r[i] = v;
    rr += v * v;
  }
};

template <int BS, int VPR>
__global__ void __launch_bounds__(VBLOCK) k_init_residual(const int* __restrict__ rp, const int* __restrict__ ci,
                                                          const double* __restrict__ val, i64 nrows,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          double* __restrict__ r, i64 n, CgState* st,
                                                          double* partials) {
  EmitRes em{b, r};
  spmv_rows<BS, VPR, double, double>(rp, ci, val, nrows, XPlain<double>{x}, em);
  double bb = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) bb += b[i] * b[i];
  double v[2] = {em.rr, bb}, tot[2];
  if (grid_reduce<2>(v, partials, &st->ticket[2], tot) && threadIdx.x == 0) {
    st->bnorm = sqrt(tot[1]);
    st->rr = tot[0];
    const double r0 = sqrt(tot[0]);
    st->maxr = r0;
    // cg.rs:87-90
    if (!st->gpu_semantics && (r0 < st->tol || (st->bnorm > 0.0 && r0 / st->bnorm < st->tol))) {
      st->done = 1;
      st->status = FCU_OK;
    }
  }
}

// inv_diag (cg.rs:52-64): 1/a_kk when |a_kk| > 1e-15, else 1.
template <int BS>
__global__ void k_inv_diag(const int* __restrict__ diag_pos, const double* __restrict__ val, i64 nn,
                           double* __restrict__ invd, float* __restrict__ invd32) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nn * BS; t += (i64)gridDim.x * blockDim.x) {
    const i64 node = t / BS;
    const int a = (int)(t - node * BS);
    const double d = val[(i64)diag_pos[node] * BS * BS + a * BS + a];
    const double iv = fabs(d) > 1e-15 ? 1.0 / d : 1.0;
    invd[t] = iv;
    invd32[t] = (float)iv;
  }
}

// z = D^-1 r, p = z, rz (FP64) ; or the FP32 copies for the mixed path.
__global__ void __launch_bounds__(VBLOCK) k_init_direction(i64 n, const double* __restrict__ r,
                                                           const double* __restrict__ invd, double* __restrict__ p,
                                                           float* __restrict__ r32, const float* __restrict__ invd32,
                                                           float* __restrict__ p32, CgState* st, double* partials) {
  double rz = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    if (r32) {
      const float rf = (float)r[i];
      r32[i] = rf;
      const float z = rf * invd32[i];
      p32[i] = z;
      rz += (double)rf * (double)z;
    } else {
      const double z = r[i] * invd[i];
      p[i] = z;
      rz += r[i] * z;
    }
  }
  double v[1] = {rz}, tot[1];
  if (grid_reduce<1>(v, partials, &st->ticket[3], tot) && threadIdx.x == 0) st->rz = tot[0];
}

// --- mixed precision --------------------------------------------------------
__global__ void __launch_bounds__(VBLOCK) k_mx_update(i64 n, float* __restrict__ x32, float* __restrict__ r32,
                                                      const float* __restrict__ p32, const float* __restrict__ ap32,
                                                      const float* __restrict__ invd32, CgState* st,
                                                      double* partials) {
  if (st->done) return;
  const float alpha = (float)st->alpha;
  double rz = 0.0, rr = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    x32[i] += alpha * p32[i];
    const float ri = r32[i] - alpha * ap32[i];
    r32[i] = ri;
    const float z = ri * invd32[i];
    rz += (double)ri * (double)z;
    rr += (double)ri * (double)ri;
  }
  double v[2] = {rz, rr}, tot[2];
  if (grid_reduce<2>(v, partials, &st->ticket[1], tot) && threadIdx.x == 0) {
    st->iter += 1;
    st->fold = 0;
    const double res = sqrt(tot[1]);
    const double rel = st->bnorm > 0.0 ? res / st->bnorm : res;
    st->rr = tot[1];
    // Replace the recursively updated residual by the true FP64 one when it
    // has dropped by `delta` since the last replacement, or claims convergence.
    st->do_update = (rel < st->tol || res < st->delta * st->maxr) ? 1 : 0;
    if (!st->do_update) {
      if (st->iter >= st->max_iter) {
        st->done = 1;
        st->status = FCU_ERR_NO_CONVERGENCE;
        return;
      }
      st->beta = tot[0] / st->rz;
      st->rz = tot[0];
    }
  }
}

struct EmitReliable {  // r = b - A64 (x64 + x32): r32 = (float) r, rr, rz
  const double* b;
  float* r32;
  const float* invd32;
  double rr = 0.0, rz = 0.0;
  __device__ __forceinline__ void operator()(i64 i, double s) {
    const double v = b[i] - s;
    rr += v * v;
    const float rf = (float)v;
    r32[i] = rf;
    rz += (double)rf * (double)(rf * invd32[i]);
  }
};

template <int BS, int VPR>
__global__ void __launch_bounds__(VBLOCK) k_mx_reliable(const int* __restrict__ rp, const int* __restrict__ ci,
                                                        const double* __restrict__ val, i64 nrows,
                                                        const double* __restrict__ x64, const float* __restrict__ x32,
                                                        const double* __restrict__ b, float* __restrict__ r32,
                                                        const float* __restrict__ invd32, CgState* st,
                                                        double* partials) {
  if (st->done || !st->do_update) return;
  EmitReliable em{b, r32, invd32};
  spmv_rows<BS, VPR, double, double>(rp, ci, val, nrows, XSum{x64, x32}, em);
  double v[2] = {em.rz, em.rr}, tot[2];
  if (grid_reduce<2>(v, partials, &st->ticket[2], tot) && threadIdx.x == 0) {
    st->fold = 1;
    st->updates += 1;
    st->rr = tot[1];
    const double res = sqrt(tot[1]);
    const double rel = st->bnorm > 0.0 ? res / st->bnorm : res;
    if (rel < st->tol) { st->done = 1; st->status = FCU_OK; return; }
    if (st->iter >= st->max_iter) { st->done = 1; st->status = FCU_ERR_NO_CONVERGENCE; return; }
    st->maxr = res;
    st->beta = tot[0] / st->rz;
    st->rz = tot[0];
  }
}

__global__ void __launch_bounds__(VBLOCK) k_mx_direction(i64 n, float* __restrict__ p32, const float* __restrict__ r32,
                                                         const float* __restrict__ invd32, double* __restrict__ x64,
                                                         float* __restrict__ x32, const CgState* st) {
  const bool fold = st->fold != 0;
  const bool done = st->done != 0;
  if (!fold && done) return;
  const float beta = (float)st->beta;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    if (fold) {
      x64[i] += (double)x32[i];
      x32[i] = 0.0f;
    }
    if (!done) p32[i] = r32[i] * invd32[i] + beta * p32[i];
  }
}

__global__ void k_fold(i64 n, double* __restrict__ x64, float* __restrict__ x32) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    x64[i] += (double)x32[i];
    x32[i] = 0.0f;
  }
}

// --- plain SpMV (fcu_spmv) --------------------------------------------------
struct EmitStore {
  double* y;
  __device__ __forceinline__ void operator()(i64 i, double s) { y[i] = s; }
};
template <int BS, int VPR>
__global__ void k_spmv_plain(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
                             i64 nrows, const double* __restrict__ x, double* __restrict__ y) {
  EmitStore em{y};
  spmv_rows<BS, VPR, double, double>(rp, ci, val, nrows, XPlain<double>{x}, em);
}

}  // namespace

// ---------------------------------------------------------------------------
// Workspace and host driver
// ---------------------------------------------------------------------------

struct Workspace {
  i64 n = 0;
  DBuf<double> x, r, p, ap, b, invd, partials;
  DBuf<float> x32, r32, p32, ap32, invd32;
  DBuf<CgState> st;
  CgState* host_st = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int vpr = 0;  // chosen lanes per row (CSR)
  int grid = 0;
  bool invd_ready = false;
  ~Workspace() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
    if (host_st) cudaFreeHost(host_st);
  }
};

fcu_matrix_s::~fcu_matrix_s() { delete ws; }

namespace {

int solver_grid(fcu_ctx ctx, i64 n) {
  i64 want = (n + VBLOCK - 1) / VBLOCK;
  i64 cap = (i64)ctx->num_sms * 4;
  return (int)std::max<i64>(1, std::min(want, cap));
}

int pick_vpr(fcu_matrix m) {
  if (m->bs == 3) return 16;
  double avg = m->nnodes ? (double)m->nnzb / (double)m->nnodes : 1.0;
  if (avg <= 6) return 4;
  if (avg <= 14) return 8;
  if (avg <= 40) return 16;
  return 32;
}

Workspace* ensure_ws(fcu_matrix m, bool mixed) {
  fcu_ctx ctx = m->ctx;
  if (!m->ws) {
    m->ws = new Workspace();
    Workspace* w = m->ws;
    w->n = m->n;
    const i64 n = m->n;
    w->x.alloc(n); w->r.alloc(n); w->p.alloc(n); w->ap.alloc(n); w->b.alloc(n); w->invd.alloc(n);
    w->invd32.alloc(n);
    w->partials.alloc(3 * MAXG);
    w->st.alloc(1);
    CUDA_CHECK(cudaMemsetAsync(w->st.p, 0, sizeof(CgState), ctx->stream));
    CUDA_CHECK(cudaMallocHost(&w->host_st, sizeof(CgState)));
    w->vpr = pick_vpr(m);
    w->grid = solver_grid(ctx, n);
  }
  Workspace* w = m->ws;
  if (mixed && !w->x32.p) {
    const i64 n = m->n;
    w->x32.alloc(n); w->r32.alloc(n); w->p32.alloc(n); w->ap32.alloc(n);
  }
  return w;
}

// Dispatch a node-row kernel on (BS, VPR).
#define DISPATCH_ROWS(BS_, VPR_, KERNEL, GRID, ...)                                  \
  do {                                                                               \
    if ((BS_) == 3) KERNEL<3, 16><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__);    \
    else if ((VPR_) == 4) KERNEL<1, 4><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__); \
    else if ((VPR_) == 8) KERNEL<1, 8><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__); \
    else if ((VPR_) == 16) KERNEL<1, 16><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__); \
    else KERNEL<1, 32><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__);               \
    LAUNCH_CHECK(ctx);                                                               \
  } while (0)

#define DISPATCH_AP(T, BS_, VPR_, GRID, ...)                                                 \
  do {                                                                                       \
    if ((BS_) == 3) k_spmv_ap<3, 16, T><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__);      \
    else if ((VPR_) == 4) k_spmv_ap<1, 4, T><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__); \
    else if ((VPR_) == 8) k_spmv_ap<1, 8, T><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__); \
    else if ((VPR_) == 16) k_spmv_ap<1, 16, T><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__); \
    else k_spmv_ap<1, 32, T><<<GRID, VBLOCK, 0, ctx->stream>>>(__VA_ARGS__);                 \
    LAUNCH_CHECK(ctx);                                                                       \
  } while (0)

void enqueue_iteration(fcu_matrix m, Workspace* w, bool mixed) {
  fcu_ctx ctx = m->ctx;
  const int g = w->grid;
  const i64 n = m->n, nr = m->nnodes;
  if (!mixed) {
    DISPATCH_AP(double, m->bs, w->vpr, g, m->row_ptr, m->col_idx, m->val64.p, nr, w->p.p, w->ap.p, w->st.p,
                w->partials.p);
    k_cg_update<<<g, VBLOCK, 0, ctx->stream>>>(n, w->x.p, w->r.p, w->p.p, w->ap.p, w->invd.p, w->st.p, w->partials.p);
    LAUNCH_CHECK(ctx);
    k_cg_direction<double><<<g, VBLOCK, 0, ctx->stream>>>(n, w->p.p, w->r.p, w->invd.p, w->st.p);
    LAUNCH_CHECK(ctx);
  } else {
    DISPATCH_AP(float, m->bs, w->vpr, g, m->row_ptr, m->col_idx, m->val32.p, nr, w->p32.p, w->ap32.p, w->st.p,
                w->partials.p);
    k_mx_update<<<g, VBLOCK, 0, ctx->stream>>>(n, w->x32.p, w->r32.p, w->p32.p, w->ap32.p, w->invd32.p, w->st.p,
                                               w->partials.p);
    LAUNCH_CHECK(ctx);
    DISPATCH_ROWS(m->bs, w->vpr, k_mx_reliable, g, m->row_ptr, m->col_idx, m->val64.p, nr, w->x.p, w->x32.p, w->b.p,
                  w->r32.p, w->invd32.p, w->st.p, w->partials.p);
    k_mx_direction<<<g, VBLOCK, 0, ctx->stream>>>(n, w->p32.p, w->r32.p, w->invd32.p, w->x.p, w->x32.p, w->st.p);
    LAUNCH_CHECK(ctx);
  }
}

cudaGraphExec_t get_graph(fcu_matrix m, Workspace* w, bool mixed) {
  fcu_ctx ctx = m->ctx;
  cudaGraphExec_t& ge = w->graph[mixed ? 1 : 0];
  if (ge) return ge;
  cudaGraph_t g;
  CUDA_CHECK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  try {
    for (int it = 0; it < CHUNK; ++it) enqueue_iteration(m, w, mixed);
  } catch (...) {
    cudaStreamEndCapture(ctx->stream, &g);
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &g));
  CUDA_CHECK(cudaGraphInstantiate(&ge, g, 0));
  cudaGraphDestroy(g);
  // launches inside the graph are counted per replay in run_pcg
  ctx->launches -= (i64)CHUNK * (mixed ? 4 : 3);
  return ge;
}

}  // namespace

// Algorithmic bytes of one iteration (see DESIGN.md-free statement in bench):
// matrix values + indices + row pointers, x gather + y write, and 11 vector
// passes (x, p, r, Ap, D^-1 reads; x, r writes; r, D^-1, p reads + p write).
double pcg_bytes_per_iter(fcu_matrix m, bool mixed) {
  const double w = mixed ? 4.0 : 8.0;
  const double bs2 = (double)m->bs * m->bs;
  const double mat = (double)m->nnzb * (bs2 * w + 4.0) + 4.0 * (double)(m->nnodes + 1);
  return mat + 2.0 * m->n * w + 11.0 * m->n * w;
}

void ensure_inv_diag(fcu_matrix m) {
  Workspace* w = ensure_ws(m, false);
  fcu_ctx ctx = m->ctx;
  if (m->bs == 3)
    k_inv_diag<3><<<grid_for(m->n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->diag_pos, m->val64.p, m->nnodes,
                                                                                  w->invd.p, w->invd32.p);
  else
    k_inv_diag<1><<<grid_for(m->n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->diag_pos, m->val64.p, m->nnodes,
                                                                                  w->invd.p, w->invd32.p);
  LAUNCH_CHECK(ctx);
}

// Core PCG driver on device buffers: b_dev, x0_dev (nullable) -> x_dev.
// inv_diag_dev (nullable) overrides the matrix diagonal (solve_csr_cg_gpu).
int run_pcg(fcu_matrix m, const double* b_dev, const double* x0_dev, double* x_dev, double tol, i64 max_iter,
            int precision, bool gpu_semantics, const double* inv_diag_dev, fcu_solve_info* info) {
  fcu_ctx ctx = m->ctx;
  const bool mixed = precision == FCU_MIXED;
  Workspace* w = ensure_ws(m, mixed);
  const i64 n = m->n, nr = m->nnodes;
  const int g = w->grid;
  if (inv_diag_dev) {
    CUDA_CHECK(cudaMemcpyAsync(w->invd.p, inv_diag_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    // FP32 copy (mixed path) from the FP64 one
    if (mixed) fail(FCU_ERR_BAD_ARG, "caller-supplied inverse diagonal is FP64-only");
  } else {
    ensure_inv_diag(m);
  }
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  CUDA_CHECK(cudaEventRecord(e0, ctx->stream));

  CgState init{};
  init.tol = tol;
  init.max_iter = max_iter;
  init.gpu_semantics = gpu_semantics ? 1 : 0;
  init.delta = 0.1;
  CUDA_CHECK(cudaMemcpyAsync(w->st.p, &init, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_CHECK(cudaMemcpyAsync(w->b.p, b_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (x0_dev) CUDA_CHECK(cudaMemcpyAsync(w->x.p, x0_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  else CUDA_CHECK(cudaMemsetAsync(w->x.p, 0, n * sizeof(double), ctx->stream));
  if (mixed) CUDA_CHECK(cudaMemsetAsync(w->x32.p, 0, n * sizeof(float), ctx->stream));
  // r = b - A x0 ; bnorm ; initial test
  DISPATCH_ROWS(m->bs, w->vpr, k_init_residual, g, m->row_ptr, m->col_idx, m->val64.p, nr, w->x.p, w->b.p, w->r.p, n,
                w->st.p, w->partials.p);
  k_init_direction<<<g, VBLOCK, 0, ctx->stream>>>(n, w->r.p, w->invd.p, w->p.p, mixed ? w->r32.p : nullptr,
                                                  w->invd32.p, mixed ? w->p32.p : nullptr, w->st.p, w->partials.p);
  LAUNCH_CHECK(ctx);
  CUDA_CHECK(cudaMemcpyAsync(w->host_st, w->st.p, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  if (gpu_semantics && w->host_st->bnorm == 0.0) {
    // gpu.rs:1169-1180: zero right-hand side -> zero solution, Ok
    CUDA_CHECK(cudaMemsetAsync(x_dev, 0, n * sizeof(double), ctx->stream));
    w->host_st->done = 1;
    w->host_st->status = FCU_OK;
    w->host_st->iter = 0;
  } else if (!w->host_st->done && max_iter > 0) {
    cudaGraphExec_t ge = get_graph(m, w, mixed);
    const int per = mixed ? 4 : 3;
    for (i64 launched = 0; launched < max_iter + CHUNK; launched += CHUNK) {
      CUDA_CHECK(cudaGraphLaunch(ge, ctx->stream));
      ctx->launches += (i64)CHUNK * per;
      CUDA_CHECK(cudaMemcpyAsync(w->host_st, w->st.p, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      if (w->host_st->done) break;
    }
  } else if (!w->host_st->done) {
    w->host_st->status = gpu_semantics ? FCU_OK : FCU_ERR_NO_CONVERGENCE;
  }
  if (mixed) {
    k_fold<<<g, VBLOCK, 0, ctx->stream>>>(n, w->x.p, w->x32.p);
    LAUNCH_CHECK(ctx);
  }
  if (!(gpu_semantics && w->host_st->bnorm == 0.0))
    CUDA_CHECK(cudaMemcpyAsync(x_dev, w->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
  CUDA_CHECK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const CgState& hs = *w->host_st;
  if (info) {
    info->iterations = hs.iter;
    info->outer_updates = hs.updates;
    info->residual = std::sqrt(std::max(hs.rr, 0.0));
    info->rel_residual = hs.bnorm > 0.0 ? info->residual / hs.bnorm : info->residual;
    info->kernel_ms = ms;
    info->effective_bw_gbps = ms > 0 ? pcg_bytes_per_iter(m, mixed) * (double)hs.iter / (ms * 1e-3) / 1e9 : 0.0;
    info->status = hs.done ? hs.status : (gpu_semantics ? FCU_OK : FCU_ERR_NO_CONVERGENCE);
  }
  if (!hs.done) return gpu_semantics ? FCU_OK : FCU_ERR_NO_CONVERGENCE;
  return hs.status;
}

void spmv_impl(fcu_matrix m, const double* x_dev, double* y_dev) {
  fcu_ctx ctx = m->ctx;
  const int vpr = pick_vpr(m);
  const int g = solver_grid(ctx, m->n);
  DISPATCH_ROWS(m->bs, vpr, k_spmv_plain, g, m->row_ptr, m->col_idx, m->val64.p, m->nnodes, x_dev, y_dev);
}

// Average time of the PCG SpMV kernel over `reps` launches (diagnostics).
void time_spmv_impl(fcu_matrix m, int precision, int reps, double* ms, double* bytes) {
  fcu_ctx ctx = m->ctx;
  const bool mixed = precision == FCU_MIXED;
  Workspace* w = ensure_ws(m, mixed);
  const i64 nr = m->nnodes;
  const int g = w->grid;
  CgState init{};
  init.rz = 1.0;
  CUDA_CHECK(cudaMemcpyAsync(w->st.p, &init, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
  if (mixed) CUDA_CHECK(cudaMemsetAsync(w->p32.p, 0, m->n * sizeof(float), ctx->stream));
  else CUDA_CHECK(cudaMemsetAsync(w->p.p, 0, m->n * sizeof(double), ctx->stream));
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
  for (int r = 0; r < reps; ++r) {
    if (mixed)
      DISPATCH_AP(float, m->bs, w->vpr, g, m->row_ptr, m->col_idx, m->val32.p, nr, w->p32.p, w->ap32.p, w->st.p,
                  w->partials.p);
    else
      DISPATCH_AP(double, m->bs, w->vpr, g, m->row_ptr, m->col_idx, m->val64.p, nr, w->p.p, w->ap.p, w->st.p,
                  w->partials.p);
  }
  CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
  CUDA_CHECK(cudaEventSynchronize(e1));
  float t = 0.f;
  CUDA_CHECK(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = reps > 0 ? (double)t / reps : 0.0;
  const double wv = mixed ? 4.0 : 8.0;
  const double bs2 = (double)m->bs * m->bs;
  *bytes = (double)m->nnzb * (bs2 * wv + 4.0) + 4.0 * (double)(m->nnodes + 1) + 2.0 * (double)m->n * wv;
}
