// Jacobi-preconditioned CG on the device.
//
// FCU_FP64 follows the arithmetic of cg.rs:40-149 (up to the order of the
// dot-product sums). FCU_MIXED runs the inner iteration on FP32 values:
//   * the operator is applied in difference form (see bsr3_row / csr_row):
//     off-diagonal FP32 entries act on x_j - x_i and the diagonal slot holds
//     the FP64 row sum rounded to FP32, so constants (rigid translations) are
//     reproduced exactly and smooth fields lose no accuracy to cancellation;
//   * search direction p, Ap and z = D^-1 r in FP32, FP32 arithmetic in SpMV;
//   * residual r, iterate x, alpha/beta and every dot product in FP64;
//   * residual replacement r = b - A64 x with the FP64 matrix when the
//     recursive residual has dropped 10x since the last replacement or claims
//     convergence, which is then decided on the FP64 residual.
// Plain FP32 for the whole iteration (r, x or the operator rounded entry by
// entry) does not converge to 1e-8 on stiff elasticity systems: rounding
// errors act on the smooth (bending) modes with a relative size of about
// eps32 * cond(A).
//
// Each iteration is three kernels, two of them ending in a global reduction:
//   direction  p = z + beta p
//   spmv       Ap = A p, p.Ap reduced on the device -> alpha
//   update     x += alpha p, r -= alpha Ap, z = D^-1 r written, r.z and r.r ->
//              beta, convergence / iteration-limit decision
// (FCU_FUSE_DIRECTION=1 selects a two-kernel form in which the SpMV forms
// p = z + beta p_old on the fly, p double-buffered; it measured slower.) In
// mixed precision each replay of the graph starts with the replacement
// kernel, which returns at once unless an iteration of the previous replay
// asked for it. The SpMV only stores per-block p.Ap partials; every block
// of the update kernel adds them in the same fixed order and forms alpha
// itself. The update's own reduction (r.z, r.r) ends in the block that
// finishes last, which sums the per-block partials in a fixed order and
// writes beta and the flags to a small device state record. Both orders are
// fixed, so a solve repeats bit for bit. The loop is captured
// once per matrix as a CUDA graph of CHUNK iterations, launched with
// programmatic dependent launch so each kernel is scheduled while its
// predecessor drains; kernels of a finished solve return at once. The host
// reads the state once per replay while the next replay is already queued.
//
// Mixed solves on 3x3-block matrices (and FP64 ones with FCU_PERSISTENT=2)
// run instead as the persistent loop k_pcg_persistent: one cooperative launch
// per stretch between residual replacements, the tiled SpMV's CTAs resident
// throughout, two bounded grid barriers per iteration in place of kernel
// boundaries, and the direction formed from (z, p) pairs where the product
// reads them. Small scalar systems go to the batched kernel as a single
// instance (batch.cu).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <string>

#include "internal.cuh"

void refresh_block_jacobi(fcu_matrix m);  // bsr3.cu

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int VBLOCK = 256;  // threads per block in solver kernels
constexpr int MAXG = 4096;   // max blocks of a reducing kernel (partials capacity)
// Regions of the partials buffer (MAXG doubles each): 0-2 for grid_reduce,
// 3 for the SpMV's per-block p.Ap, which the update kernel reads while it
// writes its own partials into regions 0-1.
constexpr int PAP_REGION = 3;
constexpr int PARTIAL_REGIONS = 4;
constexpr int CHUNK = 16;    // iterations per graph launch (even: p double buffer)

struct CgState {
  double rz, alpha, beta, bnorm, tol, rr, maxr, delta;
  long long iter, max_iter, updates;
  int done, status, do_update;
  int pause;  // mixed: a replacement is due; the rest of the graph replay is skipped
  int gpu_semantics;  // solve_csr_cg_gpu: no breakdown test, beta guard, Ok at limit
  int fault;          // a bounded wait in a kernel gave up (reported as FCU_ERR_CUDA)
  int timing;         // SpMV timing runs: every launch computes alpha, nothing stops
  // arrival counters of the grid reductions: 32 group counters + 1 top counter
  unsigned ticket[4][33];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may be scheduled while its predecessor drains. It waits here
// until the predecessor has completed and its writes are visible, then
// allows its own successor to be scheduled (which in turn waits the same way).
__device__ __forceinline__ void grid_dep_sync() {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 900)
  cudaGridDependencySynchronize();
  cudaTriggerProgrammaticLaunchCompletion();
#endif
}

// Block-reduce NV doubles; the last block to finish reduces all partials in
// fixed order and returns true (tot valid in every thread of that block).
// Arrivals are counted in two levels (block b joins group b % 32; the last
// block of a group joins the top counter) so that at most ~gridDim/32 + 32
// same-address atomics lie on the critical path.
template <int NV>
__device__ bool grid_reduce(double (&v)[NV], double* __restrict__ partials, unsigned* ticket, double (&tot)[NV]) {
  __shared__ double sh[NV][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (int)(blockDim.x >> 5);
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
      for (int q = 0; q < nw; ++q) s += sh[j][q];
      partials[j * MAXG + blockIdx.x] = s;
    }
    const unsigned G = gridDim.x;
    const unsigned grp = blockIdx.x & 31u;
    const unsigned gsize = (G - grp + 31u) >> 5;  // blocks with this residue
    const unsigned ngroups = G < 32u ? G : 32u;
    __threadfence();
    bool is_last = false;
    if (atomicAdd(&ticket[grp], 1u) == gsize - 1) {
      ticket[grp] = 0u;
      __threadfence();
      if (atomicAdd(&ticket[32], 1u) == ngroups - 1) {
        ticket[32] = 0u;
        is_last = true;
      }
    }
    last = is_last;
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
    for (int q = 0; q < nw; ++q) t2 += sh[j][q];
    tot[j] = t2;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Row kernels. CSR: VPR lanes per row. 3x3-block CSR: a half-warp per block
// row, lane 3j+a (j < 5) handles component row a of blocks j, j+5, j+10, with
// the three blocks' loads issued together.
//
// DIFF selects the difference form used by the mixed operator: the diagonal
// (block) slot holds the row sum S_i = sum_j A_ij of the FP64 matrix, and
//   y_i = sum_{j != i} A_ij (x_j - x_i) + S_i x_i,
// which equals sum_j A_ij x_j but keeps constants exact and avoids the
// cancellation between large off-diagonal and diagonal terms, so FP32
// storage and arithmetic lose only a first-order (smooth-field) accuracy.
//
// The operand is read through a gather functor gx(i) (a plain vector, or
// the new search direction computed on the fly).
// ---------------------------------------------------------------------------

template <class T>
struct XPlain {
  const T* x;
  __device__ __forceinline__ T operator()(i64 i) const { return x[i]; }
};

// p_new(i) = z(i) + beta * p_old(i)
template <class T>
struct XDirection {
  const T* z;
  const T* pold;
  T beta;
  __device__ __forceinline__ T operator()(i64 i) const { return z[i] + beta * pold[i]; }
};

template <int VPR, bool DIFF, class T, class GX>
__device__ __forceinline__ T csr_row(const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                                     i64 row, bool valid, int sub, const GX& gx) {
  T s = T(0);
  if (valid) {
    const int b = rp[row], e = rp[row + 1];
    const T xi = DIFF ? gx(row) : T(0);
    for (int p = b + sub; p < e; p += VPR) {
      const int c = ci[p];
      if (DIFF) s += val[p] * (c == (int)row ? xi : gx(c) - xi);
      else s += val[p] * gx(c);
    }
  }
#pragma unroll
  for (int o = VPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
  return s;
}

template <bool DIFF, class T, class GX>
__device__ __forceinline__ T bsr3_block(const T* __restrict__ v, const GX& gx, int c, i64 row, T x0, T x1, T x2) {
  const i64 c3 = 3 * (i64)c;
  if (!DIFF) return v[0] * gx(c3) + v[1] * gx(c3 + 1) + v[2] * gx(c3 + 2);
  if (c == (int)row) return v[0] * x0 + v[1] * x1 + v[2] * x2;
  return v[0] * (gx(c3) - x0) + v[1] * (gx(c3 + 1) - x1) + v[2] * (gx(c3 + 2) - x2);
}

template <bool DIFF, class T, class GX>
__device__ __forceinline__ T bsr3_row(const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val,
                                      i64 row, bool valid, int sub, const GX& gx) {
  T s = T(0);
  if (valid && sub < 15) {
    const int j = sub / 3, a = sub - 3 * j;
    const int b = rp[row], e = rp[row + 1];
    T x0 = T(0), x1 = T(0), x2 = T(0);
    if (DIFF) {
      x0 = gx(3 * row);
      x1 = gx(3 * row + 1);
      x2 = gx(3 * row + 2);
    }
    for (int k0 = b + j; k0 < e; k0 += 15) {
      const int k1 = k0 + 5, k2 = k0 + 10;
      const bool h1 = k1 < e, h2 = k2 < e;
      const int c0 = ci[k0];
      const int c1 = h1 ? ci[k1] : 0;
      const int c2 = h2 ? ci[k2] : 0;
      T t = bsr3_block<DIFF>(val + 9 * (i64)k0 + 3 * a, gx, c0, row, x0, x1, x2);
      if (h1) t += bsr3_block<DIFF>(val + 9 * (i64)k1 + 3 * a, gx, c1, row, x0, x1, x2);
      if (h2) t += bsr3_block<DIFF>(val + 9 * (i64)k2 + 3 * a, gx, c2, row, x0, x1, x2);
      s += t;
    }
  }
  T t;
  t = __shfl_down_sync(FULL, s, 3, 16);
  if (sub + 3 < 16) s += t;
  t = __shfl_down_sync(FULL, s, 6, 16);
  if (sub + 6 < 16) s += t;
  t = __shfl_down_sync(FULL, s, 12, 16);
  if (sub + 12 < 16) s += t;
  return s;
}

// Iterate the rows handled by this warp; emit(node, component, value) once
// per output scalar row (from one lane).
template <int BS, int VPR, bool DIFF, class T, class GX, class Emit>
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
      T s = bsr3_row<DIFF, T>(rp, ci, val, row, valid, sub, gx);
      if (valid && sub < 3) emit(row, sub, s);
    } else {
      T s = csr_row<VPR, DIFF, T>(rp, ci, val, row, valid, sub, gx);
      if (valid && sub == 0) emit(row, 0, s);
    }
  }
}

// The SpMV's p.Ap: each block stores its sum (fixed order) in the PAP_REGION
// of the partials; no grid-wide step follows in the SpMV itself.
__device__ __forceinline__ void store_pap_partial(double dot, double* __restrict__ partials) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (int)(blockDim.x >> 5);
  const double x = warp_sum(dot);
  if (lane == 0) sh[w] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < nw; ++q) t += sh[q];
    partials[PAP_REGION * MAXG + blockIdx.x] = t;
  }
}

// alpha = r.z / p.Ap from the state record `st`, or the end of the solve:
// cg.rs:102-107 make |p.Ap| < 1e-30 a breakdown (Err); the GPU solvers
// (gpu.rs:1326-1329, 1034-1037) stop with Ok when p.Ap <= 1e-30, the
// iteration counting as done; a fault flag ends it with FCU_ERR_CUDA. The
// ending is written into `st` when `record` is set. Returns false when the
// solve ends here.
__device__ __forceinline__ bool alpha_decide(CgState* st, double pap, bool fault, bool record, double* alpha) {
  const bool brk = !st->timing && (st->gpu_semantics ? !(pap > 1e-30) : fabs(pap) < 1e-30);
  if (fault || brk) {
    if (record) {
      st->done = 1;
      if (fault) {
        st->status = FCU_ERR_CUDA;
      } else {
        st->status = st->gpu_semantics ? FCU_OK : FCU_ERR_BREAKDOWN;
        st->iter += 1;
      }
    }
    return false;
  }
  *alpha = st->rz / pap;
  return true;
}

// The update kernel's alpha = r.z / p.Ap. Every block adds the SpMV's np
// per-block partials in the same fixed order (so all blocks hold the same
// alpha, and it is the same in every run), which takes the SpMV's grid-wide
// reduction off the critical path. cg.rs:102-107: |p.Ap| < 1e-30 is a
// breakdown (Err); the GPU solvers (gpu.rs:1326-1329, 1034-1037) stop with Ok
// when p.Ap <= 1e-30, the iteration counting as done. A bulk-copy fault of the
// tiled SpMV ends the solve with FCU_ERR_CUDA. Returns false when the solve
// ends here; block 0 records it. Called by all threads of the block.
__device__ __forceinline__ bool take_alpha(CgState* st, const double* __restrict__ partials, int np,
                                           double* alpha) {
  __shared__ double sh[32];
  __shared__ double pap_s;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (int)(blockDim.x >> 5);
  double s = 0.0;
  for (int b = threadIdx.x; b < np; b += blockDim.x) s += __ldcg(&partials[PAP_REGION * MAXG + b]);
  s = warp_sum(s);
  if (lane == 0) sh[w] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < nw; ++q) t += sh[q];
    pap_s = t;
  }
  __syncthreads();
  return alpha_decide(st, pap_s, st->fault != 0, blockIdx.x == 0 && threadIdx.x == 0, alpha);
}

// Reads the stop flags once per block (block 0 of the update kernel may set
// `done` while other blocks start), so that the block's threads agree.
__device__ __forceinline__ bool block_stopped(const CgState* st) {
  __shared__ int stop;
  if (threadIdx.x == 0) stop = (st->done || st->pause) ? 1 : 0;
  __syncthreads();
  return stop != 0;
}

// --- spmv: p = z + beta p_old ; Ap = A p ; p.Ap -> alpha -----------------------
template <int BS, class T>
struct EmitAp {
  XDirection<T> dir;
  T* pnew;
  T* ap;
  double dot = 0.0;
  __device__ __forceinline__ void operator()(i64 node, int a, T s) {
    const i64 i = node * BS + a;
    const T pi = dir(i);
    pnew[i] = pi;
    ap[i] = s;
    dot += (double)pi * (double)s;
  }
};

// T = double: FP64 matrix and vectors. T = float: mixed operator (difference
// form on the FP32 values with row sums in the diagonal slots).
template <int BS, int VPR, class T>
__global__ void __launch_bounds__(VBLOCK) k_spmv_dir(const int* __restrict__ rp, const int* __restrict__ ci,
                                                     const T* __restrict__ val, i64 nrows, const T* __restrict__ z,
                                                     const T* __restrict__ pold, T* __restrict__ pnew,
                                                     T* __restrict__ ap, CgState* st, double* partials) {
  grid_dep_sync();
  if (st->done || st->pause) return;
  const XDirection<T> dir{z, pold, (T)st->beta};
  EmitAp<BS, T> em{dir, pnew, ap};
  constexpr bool DIFF = sizeof(T) == 4;
  spmv_rows<BS, VPR, DIFF, T>(rp, ci, val, nrows, dir, em);
  store_pap_partial(em.dot, partials);
}

// Unfused variant: p already updated by k_direction; Ap = A p.
template <int BS, class T>
struct EmitApPlain {
  const T* p;
  T* ap;
  double dot = 0.0;
  __device__ __forceinline__ void operator()(i64 node, int a, T s) {
    const i64 i = node * BS + a;
    ap[i] = s;
    dot += (double)p[i] * (double)s;
  }
};

template <int BS, int VPR, class T>
__global__ void __launch_bounds__(VBLOCK) k_spmv_ap(const int* __restrict__ rp, const int* __restrict__ ci,
                                                    const T* __restrict__ val, i64 nrows, const T* __restrict__ p,
                                                    T* __restrict__ ap, CgState* st, double* partials) {
  grid_dep_sync();
  if (st->done || st->pause) return;
  EmitApPlain<BS, T> em{p, ap};
  constexpr bool DIFF = sizeof(T) == 4;
  spmv_rows<BS, VPR, DIFF, T>(rp, ci, val, nrows, XPlain<T>{p}, em);
  store_pap_partial(em.dot, partials);
}

// p = z + beta p (in place), for the unfused iteration. FP32 directions go
// four floats per load when both arrays are 16-byte aligned (on the
// 421,443-dof elasticity system: 34.65 -> 34.05 us per mixed iteration; two
// doubles per load made the FP64 iteration 0.8% slower, so FP64 keeps one
// element per load); the arithmetic per element is the same either way.
__device__ __forceinline__ float4 axpy4(float4 a, float b, float4 c) {
  return make_float4(a.x + b * c.x, a.y + b * c.y, a.z + b * c.z, a.w + b * c.w);
}

template <class T>
__global__ void __launch_bounds__(VBLOCK) k_direction(i64 n, T* __restrict__ p, const T* __restrict__ z,
                                                      const CgState* st) {
  grid_dep_sync();
  if (st->done || st->pause) return;
  const T beta = (T)st->beta;
  const i64 t0 = blockIdx.x * (i64)blockDim.x + threadIdx.x, stride = (i64)gridDim.x * blockDim.x;
  i64 head = 0;
  if constexpr (sizeof(T) == 4) {
    if (((reinterpret_cast<uintptr_t>(p) | reinterpret_cast<uintptr_t>(z)) & 15) == 0) {
      const i64 nv = n / 4;
      float4* pv = reinterpret_cast<float4*>(p);
      const float4* zv = reinterpret_cast<const float4*>(z);
      for (i64 i = t0; i < nv; i += stride) pv[i] = axpy4(zv[i], beta, pv[i]);
      head = nv * 4;
    }
  }
  for (i64 i = head + t0; i < n; i += stride) p[i] = z[i] + beta * p[i];
}

// --- block and scalar SpMV with TMA-staged tiles --------------------------------
// (3x3-block CSR with tiles of TR consecutive block rows; scalar CSR, where
// each stored "block" is one entry and 1-8 lanes share a row, with tiles
// that are row ranges cut to an entry budget, listed per matrix.)
// A persistent CTA walks its tiles in turn. One thread streams
// each tile's row pointers, column indices and block values into shared memory
// with bulk asynchronous copies (cp.async.bulk, completion counted on an
// mbarrier), two stages deep, while the CTA's warps compute the previous tile
// from shared memory; only the operand gathers touch L2. Copies start and end
// on 16-byte boundaries (ranges are widened outward by at most 12 bytes on each
// side, so regions reserve 32 bytes of slack; device arrays carry 16 bytes of
// padding past their end), and every mbarrier wait is bounded: on expiry the kernel
// records a fault in the state record and stops.

// Block rows per tile: 32 (a half-warp per row) for FP64 values, 64 (8 lanes
// per row) for FP32, so that a stage carries about the same bytes in both
// precisions and the consumers' operand gathers for a tile, one L2 round
// trip, serve twice the rows in FP32. FCU_TILE64=0 keeps 32 rows for FP32.
constexpr int TILE_THREADS = 512;  // 16 consumer warps: all rows of a tile at once
constexpr unsigned WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; false when the limit expired.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned limit = WAIT_LIMIT) {
  for (unsigned i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Per-stage layout: [header 64 B][row ptrs][cols][values], regions 128-aligned.
struct TileHeader {
  int b0;        // first block of the tile
  int rows;      // rows in the tile
  int col_off;   // byte offset of ci[b0] inside the staged column region
  int val_off;   // byte offset of val[9*b0] inside the staged value region
  int r0;        // first row of the tile
  int rp_off;    // row pointers staged from rp[r0 - rp_off] (16-byte aligned copy)
};

__host__ __device__ constexpr size_t align128(size_t x) { return (x + 127) & ~(size_t)127; }

// BS x BS values per stored block: BS = 3 (3x3-block CSR) or 1 (scalar CSR,
// where a "block" is one entry).
template <class T, int TR, int BS = 3>
__host__ __device__ size_t tile_stage_bytes(int cap_blocks) {
  return align128(sizeof(TileHeader)) + align128((TR + 1) * 4 + 16) + align128((size_t)cap_blocks * 4 + 32) +
         align128((size_t)cap_blocks * BS * BS * sizeof(T) + 32);
}

// Warp-specialised pipeline: warp 0 is the producer (one elected lane issues
// the bulk copies for tiles NSTAGE ahead, waiting on per-stage "empty"
// barriers), warps 1..16 are consumers (each half-warp owns one block row of
// the tile; lane l handles blocks l, l+16, ... of it, reading the block's 9
// values and column from shared memory and the three operand entries once,
// keeping three partial sums that a 16-lane shuffle tree reduces). Consumers
// wait on per-stage "full" barriers and release a stage by arriving on its
// empty barrier.
constexpr int SPMV_CONSUMER_WARPS = 16;
constexpr int SPMV_THREADS = 32 * (SPMV_CONSUMER_WARPS + 1);
constexpr int MAX_STAGES = 4;
constexpr int TILED_CTAS_PER_SM = 2;  // resident CTAs of the tiled SpMV per SM

// Output of the tiled kernel: Ap for one scalar row, and p.Ap accumulated
// from the row's own operand value (already in registers).
template <class T, int BS = 3>
struct EmitApOwn {
  T* ap;
  double dot = 0.0;
  __device__ __forceinline__ void operator()(i64 node, int a, T s, T own) {
    ap[node * BS + a] = s;
    dot += (double)own * (double)s;
  }
};

// One tile of 3x3 block rows of the tiled SpMV, computed by the consumer
// warps from the ring stage at `base`. `tile_r0` is the first row of a fixed-size tile (BLK
// tiles carry theirs in the header). Each warp releases the stage on
// `empty_bar` as soon as it has read its operands from it.
template <bool DIFF, class T, int TR, int BS, bool BLK, class GX, class Emit>
__device__ __forceinline__ void consume_tile(const unsigned char* base, int cap_blocks, i64 tile_r0, int row_in_tile,
                                             int sub, int lane, unsigned long long* empty_bar, const GX& gx,
                                             Emit& emit) {
  constexpr int LPR = 32 * SPMV_CONSUMER_WARPS / TR;
  const TileHeader* h = reinterpret_cast<const TileHeader*>(base);
  const int* rps = reinterpret_cast<const int*>(base + align128(sizeof(TileHeader))) + (BLK ? h->rp_off : 0);
  const unsigned char* cs = base + align128(sizeof(TileHeader)) + align128((TR + 1) * 4 + 16);
  const unsigned char* vs = cs + align128((size_t)cap_blocks * 4 + 32);
  const int* cis = reinterpret_cast<const int*>(cs + h->col_off);
  const T* vls = reinterpret_cast<const T*>(vs + h->val_off);
  const int b0 = h->b0;
  const i64 row = BLK ? (i64)h->r0 + row_in_tile : tile_r0 + row_in_tile;
  const bool valid = row_in_tile < h->rows;
  static_assert(BS == 3, "scalar tiles are summed in tiled_rows");
  T a0 = T(0), a1 = T(0), a2 = T(0);
  T x0 = T(0), x1 = T(0), x2 = T(0);
  if (valid) {
    x0 = gx(3 * row);
    x1 = gx(3 * row + 1);
    x2 = gx(3 * row + 2);
    const int kb1 = rps[row_in_tile + 1] - b0;
#pragma unroll 2
    for (int kb = rps[row_in_tile] - b0 + sub; kb < kb1; kb += LPR) {
      const int c = cis[kb];
      const T* v = vls + 9 * kb;
      const i64 c3 = 3 * (i64)c;
      T y0, y1, y2;
      if (DIFF && c == (int)row) {
        y0 = x0; y1 = x1; y2 = x2;
      } else if (DIFF) {
        y0 = gx(c3) - x0; y1 = gx(c3 + 1) - x1; y2 = gx(c3 + 2) - x2;
      } else {
        y0 = gx(c3); y1 = gx(c3 + 1); y2 = gx(c3 + 2);
      }
      a0 += v[0] * y0 + v[1] * y1 + v[2] * y2;
      a1 += v[3] * y0 + v[4] * y1 + v[5] * y2;
      a2 += v[6] * y0 + v[7] * y1 + v[8] * y2;
    }
  }
  __syncwarp();
  if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(empty_bar)) : "memory");
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(FULL, a0, o);
    a1 += __shfl_xor_sync(FULL, a1, o);
    a2 += __shfl_xor_sync(FULL, a2, o);
  }
  if (valid && sub < 3)
    emit(row, sub, sub == 0 ? a0 : (sub == 1 ? a1 : a2), sub == 0 ? x0 : (sub == 1 ? x1 : x2));
}

// The matrix does not depend on the preceding kernel, so the ring's first
// stages are issued before the programmatic dependency wait and overlap the
// predecessor's tail; the producer warp's lanes fetch the row-pointer bounds
// of the CTA's next 32 tiles in one round of loads. Returns false, having
// computed nothing, when the solver state says the solve is over.
template <bool DIFF, class T, int TR, int BS, bool BLK, class GX, class Emit>
__device__ __forceinline__ bool tiled_rows(const int* __restrict__ rp, const int* __restrict__ ci,
                                           const T* __restrict__ val, i64 nrows, int cap_blocks, int nstage,
                                           const int* __restrict__ tb, i64 ntb, const GX& gx, Emit& emit,
                                           CgState* st) {
  extern __shared__ __align__(128) unsigned char tile_smem[];
  __shared__ unsigned long long full[MAX_STAGES], empty[MAX_STAGES];
  constexpr int LPR = 32 * SPMV_CONSUMER_WARPS / TR;  // consumer lanes per block row
  constexpr int VPB = BS * BS;                         // values per stored block
  static_assert(BS == 1 || BS == 3, "block size");
  static_assert(BS == 1 ? (LPR >= 1 && LPR <= 16) : (LPR == 8 || LPR == 16), "tile rows");
  const size_t stage_bytes = tile_stage_bytes<T, TR, BS>(cap_blocks);
  // tiles: TR consecutive rows each, or (BLK) the ntb row ranges
  // [tb[t], tb[t + 1]) of at most TR rows and cap_blocks entries
  const i64 ntiles = BLK ? ntb : (nrows + TR - 1) / TR;
  const i64 G = gridDim.x;
  const int mytiles = blockIdx.x < ntiles ? (int)((ntiles - blockIdx.x + G - 1) / G) : 0;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < nstage; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], SPMV_CONSUMER_WARPS);
    }
    fence_mbar_init();
  }
  __syncthreads();

  // producer (warp 0): lane j holds the row and block bounds of tile k0 + j
  int pb0 = 0, pb1 = 0, pr0 = 0, pr1 = 0;
  auto load_desc = [&](int k0) {
    const i64 t = blockIdx.x + (i64)(k0 + lane) * G;
    if (t < ntiles) {
      const i64 r0 = BLK ? (i64)tb[t] : t * TR;
      const i64 r1 = BLK ? (i64)tb[t + 1] : min(r0 + TR, nrows);
      if (BLK) {
        pr0 = (int)r0;
        pr1 = (int)r1;
      }
      pb0 = rp[r0];
      pb1 = rp[r1];
    }
  };
  auto issue = [&](int k) {
    const int b0 = __shfl_sync(FULL, pb0, k & 31), b1 = __shfl_sync(FULL, pb1, k & 31);
    int tr0 = 0, tr1 = 0;
    if constexpr (BLK) {
      tr0 = __shfl_sync(FULL, pr0, k & 31);
      tr1 = __shfl_sync(FULL, pr1, k & 31);
    }
    if (lane == 0) {
      const int s = k % nstage;
      unsigned char* base = tile_smem + s * stage_bytes;
      TileHeader* h = reinterpret_cast<TileHeader*>(base);
      unsigned char* rps = base + align128(sizeof(TileHeader));
      unsigned char* cs = rps + align128((TR + 1) * 4 + 16);
      unsigned char* vs = cs + align128((size_t)cap_blocks * 4 + 32);
      const i64 r0 = BLK ? (i64)tr0 : (blockIdx.x + (i64)k * G) * TR;
      const int rows = BLK ? tr1 - tr0 : (int)min((i64)TR, nrows - r0);
      const int rp_off = BLK ? (int)(r0 & 3) : 0;  // rp + r0 - rp_off is 16-byte aligned
      const unsigned rp_bytes = (unsigned)(((rows + 1 + rp_off) * 4 + 15) & ~15);
      const uintptr_t c_lo = reinterpret_cast<uintptr_t>(ci + b0) & ~(uintptr_t)15;
      const uintptr_t c_hi = (reinterpret_cast<uintptr_t>(ci + b1) + 15) & ~(uintptr_t)15;
      const uintptr_t v_lo = reinterpret_cast<uintptr_t>(val + VPB * (i64)b0) & ~(uintptr_t)15;
      const uintptr_t v_hi = (reinterpret_cast<uintptr_t>(val + VPB * (i64)b1) + 15) & ~(uintptr_t)15;
      h->b0 = b0;
      h->rows = rows;
      if (BLK) {
        h->r0 = (int)r0;
        h->rp_off = rp_off;
      }
      h->col_off = (int)(reinterpret_cast<uintptr_t>(ci + b0) - c_lo);
      h->val_off = (int)(reinterpret_cast<uintptr_t>(val + VPB * (i64)b0) - v_lo);
      const unsigned cb = (unsigned)(c_hi - c_lo), vb = (unsigned)(v_hi - v_lo);
      fence_proxy_async();
      mbar_arrive_expect_tx(&full[s], rp_bytes + cb + vb);
      bulk_load(rps, rp + (r0 - rp_off), rp_bytes, &full[s]);
      if (cb) bulk_load(cs, reinterpret_cast<const void*>(c_lo), cb, &full[s]);
      if (vb) bulk_load(vs, reinterpret_cast<const void*>(v_lo), vb, &full[s]);
    }
  };

  // before the dependency wait: fill the ring (no stage has been used yet)
  const int prologue = min(nstage, mytiles);
  if (warp == 0) {
    load_desc(0);
    for (int k = 0; k < prologue; ++k) issue(k);
  }
  grid_dep_sync();
  if (st->done || st->pause) {
    // the copies already issued land before the CTA exits (bounded)
    if (warp == 0 && lane == 0)
      for (int s = 0; s < prologue; ++s) mbar_wait(&full[s], 0);
    return false;
  }

  if (warp == 0) {
    bool ok = true;
    for (int k = prologue; k < mytiles; ++k) {
      if ((k & 31) == 0) load_desc(k);
      if (lane == 0) ok = mbar_wait(&empty[k % nstage], (unsigned)(((k / nstage) - 1) & 1));
      if (!__shfl_sync(FULL, ok ? 1 : 0, 0)) {
        if (lane == 0) {
          atomicExch(&st->fault, 1);
          // copies in flight land before the CTA exits (bounded waits)
          for (int q = max(0, k - nstage); q < k; ++q) mbar_wait(&full[q % nstage], (unsigned)((q / nstage) & 1));
        }
        break;
      }
      issue(k);
    }
    return true;
  }

  // consumers: LPR lanes per block row; lane `sub` handles blocks sub,
  // sub + LPR, ... of it
  const int sub = lane % LPR;
  const int row_in_tile = (warp - 1) * (32 / LPR) + lane / LPR;
  for (int k = 0; k < mytiles; ++k) {
    const int s = k % nstage;
    if (!mbar_wait(&full[s], (unsigned)((k / nstage) & 1))) {
      if (lane == 0) atomicExch(&st->fault, 1);
      break;
    }
    if constexpr (BS == 1) {
      // Scalar rows are summed here rather than through consume_tile: with
      // the loop in the helper the FP64 scalar kernel ran 28% slower on B200
      // (P2 64^3 matrix: 211 against 165 us), FP32 and 3x3 blocks unchanged.
      const unsigned char* base = tile_smem + s * stage_bytes;
      const TileHeader* h = reinterpret_cast<const TileHeader*>(base);
      const int* rps = reinterpret_cast<const int*>(base + align128(sizeof(TileHeader))) + (BLK ? h->rp_off : 0);
      const unsigned char* cs = base + align128(sizeof(TileHeader)) + align128((TR + 1) * 4 + 16);
      const unsigned char* vs = cs + align128((size_t)cap_blocks * 4 + 32);
      const int* cis = reinterpret_cast<const int*>(cs + h->col_off);
      const T* vls = reinterpret_cast<const T*>(vs + h->val_off);
      const int b0 = h->b0;
      const i64 row = BLK ? (i64)h->r0 + row_in_tile : (blockIdx.x + (i64)k * G) * TR + row_in_tile;
      const bool valid = row_in_tile < h->rows;
      T a = T(0), xo = T(0);
      if (valid) {
        xo = gx(row);
        const int kb1 = rps[row_in_tile + 1] - b0;
#pragma unroll 2
        for (int kb = rps[row_in_tile] - b0 + sub; kb < kb1; kb += LPR) {
          const int c = cis[kb];
          const T v = vls[kb];
          const T y = DIFF ? (c == (int)row ? xo : gx(c) - xo) : gx(c);
          a += v * y;
        }
      }
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[s])) : "memory");
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) a += __shfl_xor_sync(FULL, a, o);
      if (valid && sub == 0) emit(row, 0, a, xo);
    } else {
      consume_tile<DIFF, T, TR, BS, BLK>(tile_smem + s * stage_bytes, cap_blocks, (blockIdx.x + (i64)k * G) * TR,
                                         row_in_tile, sub, lane, &empty[s], gx, emit);
    }
  }
  return true;
}

template <int DIFF, class T, int TR, int BS = 3>
__global__ void __launch_bounds__(SPMV_THREADS)
    k_spmv_tiled(const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val, i64 nrows,
                 int cap_blocks, int nstage, const int* __restrict__ tb, i64 ntb, const T* __restrict__ p,
                 T* __restrict__ ap, CgState* st, double* partials) {
  EmitApOwn<T, BS> em{ap};
  if (!tiled_rows<DIFF != 0, T, TR, BS, BS == 1>(rp, ci, val, nrows, cap_blocks, nstage, tb, ntb, XPlain<T>{p}, em,
                                                 st))
    return;
  store_pap_partial(em.dot, partials);
}

// --- update -----------------------------------------------------------------
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

// Mixed precision: replace the residual when it has dropped by `delta` since
// the last replacement or claims convergence (the host runs the replacement
// next); otherwise continue.
__device__ __forceinline__ void decide_after_update_mixed(CgState* st, double rz_new, double rr) {
  st->iter += 1;
  st->rr = rr;
  const double res = sqrt(rr);
  const double rel = st->bnorm > 0.0 ? res / st->bnorm : res;
  st->do_update = (rel < st->tol || res < st->delta * st->maxr) ? 1 : 0;
  st->pause = st->do_update;
  if (!st->do_update) {
    if (st->iter >= st->max_iter) {
      st->done = 1;
      st->status = FCU_ERR_NO_CONVERGENCE;
      return;
    }
    st->beta = rz_new / st->rz;
    st->rz = rz_new;
  }
}

// x += alpha p ; r -= alpha Ap ; z = D^-1 r (stored as T) ; (r.z, r.r).
// x, r and D^-1 are FP64 in both precisions.
template <class T>
__global__ void __launch_bounds__(VBLOCK, 5) k_update(i64 n, double* __restrict__ x, double* __restrict__ r,
                                                   const T* __restrict__ p, const T* __restrict__ ap,
                                                   const double* __restrict__ invd, T* __restrict__ z, CgState* st,
                                                   double* partials, int npap) {
  // x, r, D^-1 and p are final before this kernel starts (their writers
  // completed before the SpMV it depends on began), so the first two
  // elements of each thread are fetched before the dependency wait; L2-only
  // loads keep an early start from reading a stale L1 line.
  const i64 stride = (i64)gridDim.x * blockDim.x;
  const i64 i0 = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  double xa[2], ra[2], da[2];
  T pa[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const i64 i = i0 + k * stride;
    if (i < n) {
      xa[k] = __ldcg(x + i);
      ra[k] = __ldcg(r + i);
      da[k] = __ldcg(invd + i);
      pa[k] = __ldcg(p + i);
    }
  }
  grid_dep_sync();
  // Ap of the first two elements is loaded before the p.Ap partials are
  // summed, so that the two round trips overlap
  T aa[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const i64 i = i0 + k * stride;
    if (i < n) aa[k] = __ldcg(ap + i);
  }
  if (block_stopped(st)) return;
  double alpha;
  if (!take_alpha(st, partials, npap, &alpha)) return;
  double rz = 0.0, rr = 0.0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const i64 i = i0 + k * stride;
    if (i < n) {
      x[i] = xa[k] + alpha * (double)pa[k];
      const double ri = ra[k] - alpha * (double)aa[k];
      r[i] = ri;
      const double zi = ri * da[k];
      z[i] = (T)zi;
      rz += ri * zi;
      rr += ri * ri;
    }
  }
  // the remaining elements (about six per thread at 1.5M rows): unrolled so
  // that the loads of several elements are in flight together
#pragma unroll 4
  for (i64 i = i0 + 2 * stride; i < n; i += stride) {
    x[i] += alpha * (double)p[i];
    const double ri = r[i] - alpha * (double)ap[i];
    r[i] = ri;
    const double zi = ri * invd[i];
    z[i] = (T)zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  double v[2] = {rz, rr}, tot[2];
  if (grid_reduce<2>(v, partials, st->ticket[1], tot) && threadIdx.x == 0) {
    if (sizeof(T) == 8) decide_after_update(st, tot[0], tot[1]);
    else decide_after_update_mixed(st, tot[0], tot[1]);
  }
}

// --- persistent PCG (3x3-block tiled operator, point Jacobi) -----------------
// The iteration loop in one cooperative launch. The CTAs of the tiled SpMV's
// grid stay resident, and the two grid-wide steps of an iteration (p.Ap
// before alpha; r.z and r.r before beta and the stopping test) are grid
// barriers instead of kernel boundaries. Warp 0 keeps streaming the matrix's
// tiles through the shared-memory ring across iterations (the matrix does not
// change), so the first tiles of the next product are in flight while the
// consumer warps update the vectors. No separate direction step: z and p are
// kept interleaved as pairs zp[i] = (z_i, p_i), the product forms
// p = z + beta p_old from one pair load per operand, and the update forms the
// same value for its own elements (same operands, same fused multiply-add)
// and stores the new pair. Every CTA adds the per-CTA partials in the same
// fixed order and takes the same decisions on its own copy of the state
// record; CTA 0 writes that copy back when the loop ends. The loop ends when
// the solve is over or, in mixed precision, when a residual replacement is due
// (the host runs it and launches the loop again). Every wait is bounded: a
// wait that gives up sets the fault flag, and the CTA ends the loop.
__device__ __forceinline__ float dir_fma(float beta, float pold, float z) { return __fmaf_rn(beta, pold, z); }
__device__ __forceinline__ double dir_fma(double beta, double pold, double z) { return __fma_rn(beta, pold, z); }

template <class T>
struct Pair;
template <>
struct Pair<float> {
  using type = float2;
};
template <>
struct Pair<double> {
  using type = double2;
};

// The direction operand of the persistent loop. The pairs are written by the
// same kernel (other CTAs, before the last grid barrier), so they are read
// with ordinary coherent loads, never through the read-only path.
template <class T>
struct XDirPair {
  using T2 = typename Pair<T>::type;
  const T2* zp;
  T beta;
  __device__ __forceinline__ T operator()(i64 i) const {
    const T2 v = zp[i];
    return dir_fma(beta, v.y, v.x);
  }
};

// zp[i] = (z[i], p[i]), or with p == nullptr only the z half (after a
// residual replacement, which recomputes z and keeps p).
template <class T>
__global__ void k_zp_pack(const T* __restrict__ z, const T* __restrict__ p, i64 n,
                          typename Pair<T>::type* __restrict__ zp) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    if (p) zp[i] = {z[i], p[i]};
    else zp[i].x = z[i];
  }
}

constexpr unsigned BARRIER_LIMIT = 1u << 22;  // polls of a grid barrier (~1 us each) before giving up

// Named barrier of the consumer warps (warp 0, the producer, does not join).
__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(32 * SPMV_CONSUMER_WARPS) : "memory");
}

// Grid barrier, entered by all consumer threads right after a consumer_sync
// that follows their writes: the first consumer thread of each CTA arrives
// with a release add (covering its CTA's writes, ordered before it by that
// CTA barrier), polls the arrival count with relaxed loads until `target`,
// then an acquire fence; the CTA's consumer warps pass together. False when
// the poll gave up.
__device__ __forceinline__ bool grid_barrier(unsigned long long* bar, unsigned long long target, int ctid,
                                             unsigned limit = BARRIER_LIMIT) {
  __shared__ int ok_s;
  if (ctid == 0) {
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(bar) : "memory");
    int ok = 0;
    for (unsigned i = 0; i < limit; ++i) {
      unsigned long long v;
      asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(bar) : "memory");
      if (v >= target) {
        ok = 1;
        break;
      }
      __nanosleep(32);
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    ok_s = ok;
  }
  consumer_sync();
  return ok_s != 0;
}

// Sums of the G per-CTA partials src[j * MAXG + 0 .. G) in one fixed order, the same
// in every CTA: consumer thread t loads partials t, t + NCT, ... (one each
// while G <= NCT, so the loads are one round trip), each warp adds its lanes
// in a fixed shuffle tree, and the warps' sums are added in warp order. Called
// by all consumer threads; the sums are valid in the first consumer thread.
template <int NV>
__device__ __forceinline__ void sum_partials(const double* src, int G, int ctid, double (&tot)[NV]) {
  constexpr int NCT = 32 * SPMV_CONSUMER_WARPS;
  __shared__ double ws[NV][SPMV_CONSUMER_WARPS];
  double v[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    v[j] = 0.0;
    for (int b = ctid; b < G; b += NCT) v[j] += __ldcg(src + j * MAXG + b);
    v[j] = warp_sum(v[j]);
    if ((ctid & 31) == 0) ws[j][ctid >> 5] = v[j];
  }
  consumer_sync();
  if (ctid == 0)
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double t = 0.0;
      for (int w = 0; w < SPMV_CONSUMER_WARPS; ++w) t += ws[j][w];
      tot[j] = t;
    }
}

template <bool DIFF, class T, int TR>
__global__ void __launch_bounds__(SPMV_THREADS, TILED_CTAS_PER_SM) k_pcg_persistent(
    const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ val, i64 nrows, int cap_blocks,
    int nstage, i64 n, double* x, double* r, const double* __restrict__ invd, typename Pair<T>::type* zp, T* ap,
    CgState* st, double* partials, unsigned long long* bar) {
  using T2 = typename Pair<T>::type;
  constexpr int BS = 3;
  constexpr int LPR = 32 * SPMV_CONSUMER_WARPS / TR;
  constexpr int NCT = 32 * SPMV_CONSUMER_WARPS;  // consumer threads
  extern __shared__ __align__(128) unsigned char tile_smem[];
  __shared__ unsigned long long full[MAX_STAGES], empty[MAX_STAGES];
  __shared__ CgState ls;  // this CTA's copy of the state record
  __shared__ double red[2][SPMV_CONSUMER_WARPS];
  __shared__ double alpha_s;
  __shared__ int stop_s;             // consumers: the loop has ended
  __shared__ volatile int ended_s;   // consumers -> producer: no more tiles are needed
  __shared__ volatile int pfault_s;  // producer -> consumers: a ring wait gave up
  const size_t stage_bytes = tile_stage_bytes<T, TR, BS>(cap_blocks);
  const i64 ntiles = (nrows + TR - 1) / TR;
  const i64 G = gridDim.x;
  const int mytiles = blockIdx.x < ntiles ? (int)((ntiles - blockIdx.x + G - 1) / G) : 0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < nstage; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], SPMV_CONSUMER_WARPS);
    }
    fence_mbar_init();
    ended_s = 0;
    pfault_s = 0;
  }
  static_assert(sizeof(CgState) % 4 == 0, "state record copied by words");
  for (int i = tid; i < (int)(sizeof(CgState) / 4); i += blockDim.x)
    reinterpret_cast<int*>(&ls)[i] = reinterpret_cast<const int*>(st)[i];
  __syncthreads();

  if (warp == 0) {
    // producer: tile q of the stream is tile q % mytiles of the CTA's share
    if (mytiles == 0 || ls.done || ls.pause) return;
    int pb0 = 0, pb1 = 0, desc0 = -1;
    int k = 0;            // tile of the CTA's share
    int s = 0;            // ring stage
    unsigned ph = 0;      // phase parity of the stage's current use
    int issued = 0;       // copies issued, counted up to nstage
    for (;;) {
      if ((k & 31) == 0 && desc0 != k) {
        const i64 t = blockIdx.x + (i64)(k + lane) * G;
        if (t < ntiles) {
          pb0 = rp[t * TR];
          pb1 = rp[min(t * TR + TR, nrows)];
        }
        desc0 = k;
      }
      int state = 1;  // 1: stage free, 2: loop ended, 3: wait gave up
      if (lane == 0) {
        if (issued >= nstage) {
          state = 3;
          for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
            if (mbar_try_wait(&empty[s], ph ^ 1u)) {
              state = 1;
              break;
            }
            if (ended_s) {
              state = 2;
              break;
            }
          }
        } else if (ended_s) {
          state = 2;
        }
      }
      state = __shfl_sync(FULL, state, 0);
      if (state != 1) {
        if (state == 3 && lane == 0) {
          atomicExch(&st->fault, 1);
          pfault_s = 1;
        }
        break;
      }
      const int b0 = __shfl_sync(FULL, pb0, k & 31), b1 = __shfl_sync(FULL, pb1, k & 31);
      if (lane == 0) {
        unsigned char* base = tile_smem + s * stage_bytes;
        TileHeader* h = reinterpret_cast<TileHeader*>(base);
        unsigned char* rps = base + align128(sizeof(TileHeader));
        unsigned char* cs = rps + align128((TR + 1) * 4 + 16);
        unsigned char* vs = cs + align128((size_t)cap_blocks * 4 + 32);
        const i64 r0 = (blockIdx.x + (i64)k * G) * TR;
        const int rows = (int)min((i64)TR, nrows - r0);
        const unsigned rp_bytes = (unsigned)(((rows + 1) * 4 + 15) & ~15);
        const uintptr_t c_lo = reinterpret_cast<uintptr_t>(ci + b0) & ~(uintptr_t)15;
        const uintptr_t c_hi = (reinterpret_cast<uintptr_t>(ci + b1) + 15) & ~(uintptr_t)15;
        const uintptr_t v_lo = reinterpret_cast<uintptr_t>(val + 9 * (i64)b0) & ~(uintptr_t)15;
        const uintptr_t v_hi = (reinterpret_cast<uintptr_t>(val + 9 * (i64)b1) + 15) & ~(uintptr_t)15;
        h->b0 = b0;
        h->rows = rows;
        h->col_off = (int)(reinterpret_cast<uintptr_t>(ci + b0) - c_lo);
        h->val_off = (int)(reinterpret_cast<uintptr_t>(val + 9 * (i64)b0) - v_lo);
        const unsigned cb = (unsigned)(c_hi - c_lo), vb = (unsigned)(v_hi - v_lo);
        fence_proxy_async();
        mbar_arrive_expect_tx(&full[s], rp_bytes + cb + vb);
        bulk_load(rps, rp + r0, rp_bytes, &full[s]);
        if (cb) bulk_load(cs, reinterpret_cast<const void*>(c_lo), cb, &full[s]);
        if (vb) bulk_load(vs, reinterpret_cast<const void*>(v_lo), vb, &full[s]);
      }
      if (issued < nstage) ++issued;
      if (++k == mytiles) k = 0;
      if (++s == nstage) {
        s = 0;
        ph ^= 1u;
      }
    }
    // copies still in flight (at most one per stage) land before the CTA exits
    if (lane == 0)
      for (int i = 1; i <= issued; ++i) {
        int s2 = s - i;
        unsigned p2 = ph;
        if (s2 < 0) {
          s2 += nstage;
          p2 ^= 1u;
        }
        mbar_wait(&full[s2], p2);
      }
    return;
  }

  // consumer warps
  const int ctid = tid - 32;
  const int sub = lane % LPR;
  const int row_in_tile = (warp - 1) * (32 / LPR) + lane / LPR;
  int cs = 0;                  // ring stage of the next tile
  unsigned cph = 0;            // its phase parity
  unsigned long long gen = 0;  // grid barriers passed
  const i64 step = G * NCT;
  const i64 i0 = (i64)blockIdx.x * NCT + ctid;  // the thread's first vector element
  bool run = !(ls.done || ls.pause);
  while (run) {
    const T beta = (T)ls.beta;
    // Ap = A p with p = z + beta p_old formed per operand
    XDirPair<T> gx{zp, beta};
    EmitApOwn<T, BS> em{ap};
    bool tiles_ok = true;
    for (int k = 0; k < mytiles; ++k) {
      bool got = false;
      for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try_wait(&full[cs], cph)) {
          got = true;
          break;
        }
        if (pfault_s) break;
      }
      if (!got) {
        tiles_ok = false;
        break;
      }
      consume_tile<DIFF, T, TR, BS, false>(tile_smem + cs * stage_bytes, cap_blocks, (blockIdx.x + (i64)k * G) * TR,
                                           row_in_tile, sub, lane, &empty[cs], gx, em);
      if (++cs == nstage) {
        cs = 0;
        cph ^= 1u;
      }
    }
    if (!tiles_ok && lane == 0) atomicExch(&st->fault, 1);
    double d = warp_sum(em.dot);
    if (lane == 0) red[0][warp - 1] = d;
    consumer_sync();
    if (ctid == 0) {
      double t = 0.0;
      for (int w = 0; w < SPMV_CONSUMER_WARPS; ++w) t += red[0][w];
      partials[PAP_REGION * MAXG + blockIdx.x] = t;
    }
    bool ok = grid_barrier(bar, ++gen * (unsigned long long)G, ctid);
    // alpha from the G partials, added in the same order in every CTA
    double pap[1] = {0.0};
    sum_partials<1>(partials + PAP_REGION * MAXG, ok ? (int)G : 0, ctid, pap);
    if (ctid == 0) {
      const bool fault = !ok || *reinterpret_cast<volatile int*>(&st->fault) != 0;
      if (!ok) atomicExch(&st->fault, 1);
      double a = 0.0;
      stop_s = alpha_decide(&ls, pap[0], fault, true, &a) ? 0 : 1;
      alpha_s = a;
    }
    consumer_sync();
    if (stop_s) break;
    const double alpha = alpha_s;
    // x += alpha p ; r -= alpha Ap ; z = D^-1 r ; (z, p) stored ; (r.z, r.r)
    double rz = 0.0, rr = 0.0;
    // (all loads of an element before its stores: the vectors are not
    // declared unaliased, so the compiler keeps loads behind earlier stores)
    for (i64 i = i0; i < n; i += step) {
      const T2 v = zp[i];
      const T av = __ldcg(ap + i);
      const double xv = x[i], rv = r[i], dv = invd[i];
      const T pi = dir_fma(beta, v.y, v.x);
      const double ri = rv - alpha * (double)av;
      const double zi = ri * dv;
      zp[i] = {(T)zi, pi};
      x[i] = xv + alpha * (double)pi;
      r[i] = ri;
      rz += ri * zi;
      rr += ri * ri;
    }
    rz = warp_sum(rz);
    rr = warp_sum(rr);
    if (lane == 0) {
      red[0][warp - 1] = rz;
      red[1][warp - 1] = rr;
    }
    consumer_sync();
    if (ctid == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < SPMV_CONSUMER_WARPS; ++w) {
        a += red[0][w];
        b += red[1][w];
      }
      partials[blockIdx.x] = a;
      partials[MAXG + blockIdx.x] = b;
    }
    ok = grid_barrier(bar, ++gen * (unsigned long long)G, ctid);
    double sums[2] = {0.0, 0.0};
    sum_partials<2>(partials, ok ? (int)G : 0, ctid, sums);
    if (ctid == 0) {
      if (!ok || *reinterpret_cast<volatile int*>(&st->fault) != 0) {
        if (!ok) atomicExch(&st->fault, 1);
        ls.done = 1;
        ls.status = FCU_ERR_CUDA;
      } else if (sizeof(T) == 8) {
        decide_after_update(&ls, sums[0], sums[1]);
      } else {
        decide_after_update_mixed(&ls, sums[0], sums[1]);
      }
      stop_s = (ls.done || ls.pause) ? 1 : 0;
    }
    consumer_sync();
    run = stop_s == 0;
  }
  if (ctid == 0) {
    ended_s = 1;
    if (blockIdx.x == 0) {
      st->rz = ls.rz;
      st->beta = ls.beta;
      st->rr = ls.rr;
      st->iter = ls.iter;
      st->done = ls.done;
      st->status = ls.status;
      st->do_update = ls.do_update;
      st->pause = ls.pause;
    }
  }
}

// Block-Jacobi variant (FP64). Tiles of 96 block rows (288 dofs, one thread
// per dof): x, r, p, Ap and the thread's row of the inverse block are read
// with coalesced loads, the new residual goes through shared memory, and
// each thread forms its z = sum_b Dinv[a][b] r_b (bsr3_apply_dinv). As in
// k_update, the first tile's x, r, p and inverse blocks are final before the
// kernel starts and are fetched before the dependency wait.
constexpr int UB_THREADS = 288;

__global__ void __launch_bounds__(UB_THREADS) k_update_block(i64 nn, double* __restrict__ x, double* __restrict__ r,
                                                             const double* __restrict__ p,
                                                             const double* __restrict__ ap,
                                                             const double* __restrict__ bdinv,
                                                             double* __restrict__ z, CgState* st, double* partials,
                                                             int npap) {
  __shared__ double rs[UB_THREADS];
  const i64 n = 3 * nn;
  const int t = threadIdx.x;
  const i64 tstride = (i64)gridDim.x * UB_THREADS;
  i64 i = blockIdx.x * (i64)UB_THREADS + t;
  double xa = 0.0, ra = 0.0, pa = 0.0, d0 = 0.0, d1 = 0.0, d2 = 0.0;
  if (i < n) {
    xa = __ldcg(x + i);
    ra = __ldcg(r + i);
    pa = __ldcg(p + i);
    d0 = __ldcg(bdinv + 3 * i);
    d1 = __ldcg(bdinv + 3 * i + 1);
    d2 = __ldcg(bdinv + 3 * i + 2);
  }
  grid_dep_sync();
  if (block_stopped(st)) return;
  double alpha;
  if (!take_alpha(st, partials, npap, &alpha)) return;
  double rz = 0.0, rr = 0.0;
  const i64 first = blockIdx.x * (i64)UB_THREADS;
  for (i64 tile = first; tile < n; tile += tstride, i += tstride) {
    const bool ok = i < n;
    if (ok && tile != first) {
      xa = x[i];
      ra = r[i];
      pa = p[i];
      d0 = bdinv[3 * i];
      d1 = bdinv[3 * i + 1];
      d2 = bdinv[3 * i + 2];
    }
    double rn = 0.0;
    if (ok) {
      x[i] = xa + alpha * pa;
      rn = ra - alpha * ap[i];
      r[i] = rn;
      rr += rn * rn;
    }
    rs[t] = rn;
    __syncthreads();
    if (ok) {
      const int b0 = t - t % 3;  // first dof of this block row in the tile
      const double zi = d0 * rs[b0] + d1 * rs[b0 + 1] + d2 * rs[b0 + 2];
      z[i] = zi;
      rz += rn * zi;
    }
    __syncthreads();
  }
  double v[2] = {rz, rr}, tot[2];
  if (grid_reduce<2>(v, partials, st->ticket[1], tot) && threadIdx.x == 0) decide_after_update(st, tot[0], tot[1]);
}

// After the initial residual: z = D_b^-1 r and r.z for the block-Jacobi
// preconditioner (the point-Jacobi z the residual kernel wrote is replaced).
__global__ void __launch_bounds__(VBLOCK) k_block_init(i64 nn, const double* __restrict__ r,
                                                       const double* __restrict__ bdinv, double* __restrict__ z,
                                                       CgState* st, double* partials) {
  grid_dep_sync();
  double rz = 0.0;
  for (i64 w = blockIdx.x * (i64)blockDim.x + threadIdx.x; w < nn; w += (i64)gridDim.x * blockDim.x) {
    const double* D = bdinv + 9 * w;
    const double r0 = r[3 * w], r1 = r[3 * w + 1], r2 = r[3 * w + 2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double zi = D[3 * a] * r0 + D[3 * a + 1] * r1 + D[3 * a + 2] * r2;
      z[3 * w + a] = zi;
      rz += r[3 * w + a] * zi;
    }
  }
  double v[1] = {rz}, tot[1];
  if (grid_reduce<1>(v, partials, st->ticket[3], tot) && threadIdx.x == 0) st->rz = tot[0];
}

// Point diagonal taken from the inverse blocks (read only by the residual
// kernel, whose z the block-Jacobi pass overwrites).
__global__ void k_invd_from_blocks(const double* __restrict__ bdinv, i64 n, double* __restrict__ invd) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    invd[i] = bdinv[9 * (i / 3) + 4 * (i % 3)];
}

// --- residual: r = b - A64 x, z = D^-1 r (init, and the mixed replacement) ----
template <int BS, class T>
struct EmitRes {
  const double* b;
  const double* invd;
  double* r;
  T* z;
  double rr = 0.0, rz = 0.0;
  __device__ __forceinline__ void operator()(i64 node, int a, double s) {
    const i64 i = node * BS + a;
    const double v = b[i] - s;
    r[i] = v;
    const double zi = v * invd[i];
    z[i] = (T)zi;
    rr += v * v;
    rz += v * zi;
  }
};

template <int BS, int VPR, class T>
__global__ void __launch_bounds__(VBLOCK) k_init_residual(const int* __restrict__ rp, const int* __restrict__ ci,
                                                          const double* __restrict__ val, i64 nrows,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          const double* __restrict__ invd, double* __restrict__ r,
                                                          T* __restrict__ z, T* __restrict__ pold, i64 n, CgState* st,
                                                          double* partials) {
  grid_dep_sync();
  EmitRes<BS, T> em{b, invd, r, z};
  spmv_rows<BS, VPR, false, double>(rp, ci, val, nrows, XPlain<double>{x}, em);
  double bb = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    bb += b[i] * b[i];
    pold[i] = T(0);
  }
  double v[3] = {em.rr, bb, em.rz}, tot[3];
  if (grid_reduce<3>(v, partials, st->ticket[2], tot) && threadIdx.x == 0) {
    st->bnorm = sqrt(tot[1]);
    st->rr = tot[0];
    st->rz = tot[2];
    st->beta = 0.0;  // first direction p = z
    const double r0 = sqrt(tot[0]);
    st->maxr = r0;
    // cg.rs:87-90
    if (!st->gpu_semantics && (r0 < st->tol || (st->bnorm > 0.0 && r0 / st->bnorm < st->tol))) {
      st->done = 1;
      st->status = FCU_OK;
    }
  }
}

template <int BS, int VPR>
__global__ void __launch_bounds__(VBLOCK) k_mx_replace(const int* __restrict__ rp, const int* __restrict__ ci,
                                                       const double* __restrict__ val, i64 nrows,
                                                       const double* __restrict__ x, const double* __restrict__ b,
                                                       const double* __restrict__ invd, double* __restrict__ r,
                                                       float* __restrict__ z, CgState* st, double* partials) {
  grid_dep_sync();
  if (st->done || !st->do_update) return;
  EmitRes<BS, float> em{b, invd, r, z};
  spmv_rows<BS, VPR, false, double>(rp, ci, val, nrows, XPlain<double>{x}, em);
  double v[2] = {em.rz, em.rr}, tot[2];
  if (grid_reduce<2>(v, partials, st->ticket[2], tot) && threadIdx.x == 0) {
    st->updates += 1;
    st->do_update = 0;
    st->pause = 0;
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

// inv_diag (cg.rs:52-64): 1/a_kk when |a_kk| > 1e-15, else 1.
template <int BS>
__global__ void k_inv_diag(const int* __restrict__ diag_pos, const double* __restrict__ val, i64 nn,
                           double* __restrict__ invd) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nn * BS; t += (i64)gridDim.x * blockDim.x) {
    const i64 node = t / BS;
    const int a = (int)(t - node * BS);
    const int dp = diag_pos[node];
    const double d = dp >= 0 ? val[(i64)dp * BS * BS + a * BS + a] : 0.0;
    invd[t] = fabs(d) > 1e-15 ? 1.0 / d : 1.0;
  }
}

// Mixed operator: write into each diagonal (block) slot of the FP32 values
// the row sums of the FP64 matrix, S_i[a][b] = sum_j A_ij[a][b].
template <int BS>
__global__ void k_build_rowsum32(const int* __restrict__ rp, const int* __restrict__ diag_pos,
                                 const double* __restrict__ v64, i64 nn, float* __restrict__ v32) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nn * BS * BS; t += (i64)gridDim.x * blockDim.x) {
    const i64 node = t / (BS * BS);
    const int e = (int)(t - node * BS * BS);
    double d = 0.0;
    for (int p = rp[node]; p < rp[node + 1]; ++p) d += v64[(i64)p * BS * BS + e];
    const int dp = diag_pos[node];
    if (dp >= 0) v32[(i64)dp * BS * BS + e] = (float)d;
  }
}

// --- plain SpMV (fcu_spmv) --------------------------------------------------
template <int BS>
struct EmitStore {
  double* y;
  __device__ __forceinline__ void operator()(i64 node, int a, double s) { y[node * BS + a] = s; }
};
template <int BS, int VPR>
__global__ void k_spmv_plain(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
                             i64 nrows, const double* __restrict__ x, double* __restrict__ y) {
  grid_dep_sync();
  EmitStore<BS> em{y};
  spmv_rows<BS, VPR, false, double>(rp, ci, val, nrows, XPlain<double>{x}, em);
}

// ---------------------------------------------------------------------------
// CSR-stream SpMV for scalar matrices with short rows. CTA-sized row blocks
// (at most STREAM_ROWS rows and STREAM_NNZ entries, built once per matrix)
// are taken in turn by each CTA: phase 1 reads the block's entries with
// coalesced loads (value, and the gathered operand x[col]) into shared
// memory; phase 2 gives each row to one thread, which sums its entries in
// column order (the difference form for the mixed operator, the diagonal
// found through diag_pos). A row longer than STREAM_NNZ is a block of its
// own, summed in chunks by all threads and reduced in a fixed order.
// ---------------------------------------------------------------------------

constexpr int STREAM_THREADS = 256;
constexpr int STREAM_ROWS = 256;
constexpr int STREAM_NNZ = 2048;

template <bool DIFF, class T, class Emit>
__device__ __forceinline__ void stream_rows(const int* __restrict__ rp, const int* __restrict__ ci,
                                            const T* __restrict__ val, const int* __restrict__ dpos,
                                            const int* __restrict__ rb, int nblk, const T* __restrict__ x, Emit& emit) {
  __shared__ T sv[STREAM_NNZ];
  __shared__ T sx[DIFF ? STREAM_NNZ : 1];
  __shared__ T red[STREAM_THREADS / 32];
  const int t = threadIdx.x;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const int r0 = rb[blk], r1 = rb[blk + 1];
    const int base = rp[r0], nnz = rp[r1] - base;
    if (nnz > STREAM_NNZ) {
      // one long row
      const T xi = DIFF ? x[r0] : T(0);
      const int dp = DIFF ? dpos[r0] : -1;
      T s = T(0);
      for (int q = base + t; q < base + nnz; q += STREAM_THREADS) {
        if (DIFF) s += val[q] * (q == dp ? xi : x[ci[q]] - xi);
        else s += val[q] * x[ci[q]];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
      if ((t & 31) == 0) red[t >> 5] = s;
      __syncthreads();
      if (t == 0) {
        T tot = T(0);
        for (int w = 0; w < STREAM_THREADS / 32; ++w) tot += red[w];
        emit((i64)r0, 0, tot);
      }
      __syncthreads();
      continue;
    }
    // all column and value loads of this thread first, then all gathers:
    // two dependent latencies per block instead of one per entry
    constexpr int PER = STREAM_NNZ / STREAM_THREADS;
    int cols[PER];
    T vs[PER], xs[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int q = t + k * STREAM_THREADS;
      if (q < nnz) {
        cols[k] = ci[base + q];
        vs[k] = val[base + q];
      }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int q = t + k * STREAM_THREADS;
      if (q < nnz) xs[k] = x[cols[k]];
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int q = t + k * STREAM_THREADS;
      if (q < nnz) {
        if (DIFF) {
          sv[q] = vs[k];
          sx[q] = xs[k];
        } else {
          sv[q] = vs[k] * xs[k];
        }
      }
    }
    __syncthreads();
    for (int row = r0 + t; row < r1; row += STREAM_THREADS) {
      const int b = rp[row] - base, e = rp[row + 1] - base;
      T s = T(0);
      if (DIFF) {
        const T xi = x[row];
        const int dp = dpos[row] - base;
        for (int q = b; q < e; ++q) s += sv[q] * (q == dp ? xi : sx[q] - xi);
      } else {
        for (int q = b; q < e; ++q) s += sv[q];
      }
      emit((i64)row, 0, s);
    }
    __syncthreads();
  }
}

template <class T>
__global__ void __launch_bounds__(STREAM_THREADS) k_spmv_stream(const int* __restrict__ rp, const int* __restrict__ ci,
                                                                const T* __restrict__ val,
                                                                const int* __restrict__ dpos,
                                                                const int* __restrict__ rb, int nblk,
                                                                const T* __restrict__ p, T* __restrict__ ap,
                                                                CgState* st, double* partials) {
  grid_dep_sync();
  if (st->done || st->pause) return;
  EmitApPlain<1, T> em{p, ap};
  stream_rows<sizeof(T) == 4, T>(rp, ci, val, dpos, rb, nblk, p, em);
  store_pap_partial(em.dot, partials);
}

__global__ void __launch_bounds__(STREAM_THREADS) k_spmv_stream_plain(const int* __restrict__ rp,
                                                                      const int* __restrict__ ci,
                                                                      const double* __restrict__ val,
                                                                      const int* __restrict__ rb, int nblk,
                                                                      const double* __restrict__ x,
                                                                      double* __restrict__ y) {
  grid_dep_sync();
  EmitStore<1> em{y};
  stream_rows<false, double>(rp, ci, val, nullptr, rb, nblk, x, em);
}

// Row blocks of the stream kernel: consecutive rows while at most
// STREAM_ROWS rows and STREAM_NNZ entries fit; a longer row alone.
void build_row_blocks(fcu_ctx ctx, const int* rp_dev, i64 nrows, DBuf<int>& rb, int* nblk) {
  std::vector<int> rp(nrows + 1);
  CUDA_CHECK(cudaMemcpyAsync(rp.data(), rp_dev, (nrows + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  std::vector<int> b;
  b.push_back(0);
  i64 r = 0;
  while (r < nrows) {
    i64 e = r;
    while (e < nrows && e - r < STREAM_ROWS && (i64)rp[e + 1] - rp[r] <= STREAM_NNZ) ++e;
    if (e == r) e = r + 1;  // a row longer than STREAM_NNZ
    b.push_back((int)e);
    r = e;
  }
  *nblk = (int)b.size() - 1;
  upload(ctx, rb, b.data(), b.size());
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
}

}  // namespace

// ---------------------------------------------------------------------------
// Workspace and host driver
// ---------------------------------------------------------------------------

struct Workspace {
  fcu_ctx ctx = nullptr;
  i64 n = 0;
  DBuf<double> x, r, b, invd, partials;
  DBuf<double> z64, pa64, pb64, ap64;  // FP64 path: z, p (two buffers), Ap
  DBuf<float> z32, pa32, pb32, ap32;   // mixed path
  DBuf<CgState> st;
  DBuf<unsigned long long> bar;  // arrival count of the persistent loop's grid barriers
  DBuf<float2> zp32;             // persistent loop: (z, p) pairs, mixed
  DBuf<double2> zp64;            // persistent loop: (z, p) pairs, FP64
  CgState* host_st = nullptr;  // two pinned records: [0] set-up and final state, [0]/[1] alternate between replays
  cudaEvent_t ev[2] = {nullptr, nullptr};  // a replay's state record has arrived on the host
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  bool stream[2] = {false, false};  // scalar PCG SpMV: CSR-stream kernel (FP64, FP32)
  bool tiled1[2] = {false, false};  // scalar PCG SpMV: tiled kernel (FP64, FP32), ring depth in stages[]
  int vpr = 0;    // lanes per row of the FP64 CSR kernels (tuned with the FP64 SpMV)
  int vpr32 = 0;  // lanes per row of the FP32 CSR SpMV (tuned with it)
  int stages[2] = {3, 3};  // ring depth of the tiled block SpMV: FP64, FP32
  bool tuned[2] = {false, false};
  int grid = 0;   // row kernels
  int vgrid = 0;  // element-wise vector kernels
  ~Workspace() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (host_st) {
      if (ctx) ctx->pinned_pool.push_back(host_st);
      else cudaFreeHost(host_st);
    }
  }
};

fcu_matrix_s::~fcu_matrix_s() {
  delete ws;
  destroy_batch_ws(bws);
}

namespace {

// Blocks per SM for the solver kernels (grid-stride loops); FCU_SOLVER_BPSM
// overrides the default for tuning.
int blocks_per_sm() {
  static int v = [] {
    const char* e = getenv("FCU_SOLVER_BPSM");
    int x = e ? atoi(e) : 8;
    return (x >= 1 && x <= 16) ? x : 8;
  }();
  return v;
}

int solver_grid(fcu_ctx ctx, i64 n) {
  i64 want = (n + VBLOCK - 1) / VBLOCK;
  i64 cap = (i64)ctx->num_sms * blocks_per_sm();
  return (int)std::max<i64>(1, std::min(want, cap));
}

// Blocks per SM for the element-wise vector kernels (update, direction);
// FCU_VEC_BPSM overrides the default.
int vec_blocks_per_sm() {
  static int v = [] {
    const char* e = getenv("FCU_VEC_BPSM");
    int x = e ? atoi(e) : 8;
    return (x >= 1 && x <= 16) ? x : 8;
  }();
  return v;
}

// CSR-stream SpMV for scalar rows of at most 32 entries on average
// (FCU_STREAM_SPMV=0 disables it).
bool use_stream_spmv(fcu_matrix m) {
  static int v = [] {
    const char* e = getenv("FCU_STREAM_SPMV");
    return e ? atoi(e) : 1;
  }();
  if (!v || m->bs != 1) return false;
  return m->nnodes > 0 && (double)m->nnzb <= 32.0 * (double)m->nnodes;
}

// One wave of the block-Jacobi update (its first tile is prefetched before
// the dependency wait).
int update_block_grid(fcu_ctx ctx, i64 nn) {
  static int occ = -1;
  if (occ < 0) {
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_update_block, UB_THREADS, 0));
    occ = std::max(1, std::min(occ, 8));
  }
  const i64 tiles = (3 * nn + UB_THREADS - 1) / UB_THREADS;
  return (int)std::max<i64>(1, std::min<i64>(tiles, (i64)ctx->num_sms * occ));
}

// One resident wave of the stream kernel (its CTAs loop over the row blocks).
template <class K>
int stream_grid_for(fcu_ctx ctx, int nblk, K kern) {
  static int occ = -1;
  if (occ < 0) {
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, STREAM_THREADS, 0));
    occ = std::max(1, std::min(occ, 8));
  }
  return std::max(1, std::min(nblk, ctx->num_sms * occ));
}

void ensure_row_blocks(fcu_matrix m) {
  if (!m->nrowblk) build_row_blocks(m->ctx, m->row_ptr, m->nnodes, m->rowblk, &m->nrowblk);
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
    w->x.alloc(n); w->r.alloc(n); w->b.alloc(n); w->invd.alloc(n);
    w->partials.alloc(PARTIAL_REGIONS * MAXG);
    w->st.alloc(1);
    CUDA_CHECK(cudaMemsetAsync(w->st.p, 0, sizeof(CgState), ctx->stream));
    w->ctx = ctx;
    if (!ctx->pinned_pool.empty()) {
      w->host_st = static_cast<CgState*>(ctx->pinned_pool.back());
      ctx->pinned_pool.pop_back();
    } else {
      CUDA_CHECK(cudaMallocHost(&w->host_st, 2 * sizeof(CgState)));
    }
    for (auto& e : w->ev) CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    w->vpr = pick_vpr(m);
    w->vpr32 = w->vpr;
    if (m->bs == 1 && use_stream_spmv(m)) {
      ensure_row_blocks(m);
      w->stream[0] = w->stream[1] = true;
    }
    w->grid = solver_grid(ctx, n);
    // one wave of the update kernel (its first two elements per thread are
    // fetched before the dependency wait, which only resident blocks do early)
    int occ64 = 0, occ32 = 0;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, k_update<double>, VBLOCK, 0));
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, k_update<float>, VBLOCK, 0));
    const int vbpsm = std::max(1, std::min(vec_blocks_per_sm(), std::min(occ64, occ32)));
    w->vgrid = (int)std::max<i64>(1, std::min<i64>((n + VBLOCK - 1) / VBLOCK, (i64)ctx->num_sms * vbpsm));
  }
  Workspace* w = m->ws;
  if (!mixed && !w->z64.p) {
    w->z64.alloc(m->n); w->pa64.alloc(m->n); w->pb64.alloc(m->n); w->ap64.alloc(m->n);
  }
  if (mixed && !w->z32.p) {
    w->z32.alloc(m->n); w->pa32.alloc(m->n); w->pb32.alloc(m->n); w->ap32.alloc(m->n);
  }
  return w;
}

// Launch with programmatic stream serialization: the kernel may be scheduled
// while its predecessor drains, and waits in grid_dep_sync().
template <class... KArgs, class... Args>
void launch_pdl(fcu_ctx ctx, void (*kern)(KArgs...), int grid, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(VBLOCK);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
  ctx->launches++;
}

template <class... KArgs, class... Args>
void launch_pdl_cfg(fcu_ctx ctx, void (*kern)(KArgs...), int grid, int block, size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
  ctx->launches++;
}

bool tile64_enabled() {
  static int v = [] {
    const char* e = getenv("FCU_TILE64");
    return e ? atoi(e) : 1;
  }();
  return v != 0;
}

// Block rows per tile of the tiled SpMV for FP32 (4) or FP64 (8) values.
int tile_rows(size_t value_bytes) { return (value_bytes == 4 && tile64_enabled()) ? 64 : 32; }

size_t tile_stage_bytes_rt(size_t value_bytes, int tr, int cap) {
  if (value_bytes == 4) return tr == 64 ? tile_stage_bytes<float, 64>(cap) : tile_stage_bytes<float, 32>(cap);
  return tile_stage_bytes<double, 32>(cap);
}

size_t scalar_stage_bytes(size_t value_bytes, int tr, int cap) {
  const bool f = value_bytes == 4;
  switch (tr) {
    case 512: return f ? tile_stage_bytes<float, 512, 1>(cap) : tile_stage_bytes<double, 512, 1>(cap);
    case 256: return f ? tile_stage_bytes<float, 256, 1>(cap) : tile_stage_bytes<double, 256, 1>(cap);
    case 128: return f ? tile_stage_bytes<float, 128, 1>(cap) : tile_stage_bytes<double, 128, 1>(cap);
    case 64: return f ? tile_stage_bytes<float, 64, 1>(cap) : tile_stage_bytes<double, 64, 1>(cap);
    default: return f ? tile_stage_bytes<float, 32, 1>(cap) : tile_stage_bytes<double, 32, 1>(cap);
  }
}

int max_block_row(fcu_matrix m) { return m->space ? m->space->max_row : (m->max_row_own ? m->max_row_own : 32); }

// Rows per tile of the scalar tiled SpMV (TR), or 0 when it does not fit.
// TR = 512 / lanes per row, the lanes chosen by mean row length (1 up to 16
// entries, 2 up to 32, 4 up to 64, else 8: about 7-16 entries per lane). Tiles are row ranges of at most
// TR rows and at most `cap` entries, cut greedily, with cap as large as two
// ring stages of two CTAs per SM allow: every tile then carries about as
// many bytes as the ring holds, which amortises its one round trip of
// operand gathers (a matrix whose longest row exceeds cap does not fit).
// Built once per matrix and precision, never while a graph is captured.
int scalar_tile_rows(fcu_matrix m, bool f32) {
  const int k = f32 ? 1 : 0;
  if (m->tblk_tr[k] >= 0) return m->tblk_tr[k];
  fcu_ctx ctx = m->ctx;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CUDA_CHECK(cudaStreamIsCapturing(ctx->stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) fail(FCU_ERR_CUDA, "tiles of the scalar tiled SpMV requested during capture");
  m->tblk_tr[k] = 0;
  if (m->nnodes <= 0) return 0;
  const double mean = (double)m->nnzb / (double)m->nnodes;
  const int lpr = mean <= 16.0 ? 1 : mean <= 32.0 ? 2 : mean <= 64.0 ? 4 : 8;
  const int tr = 512 / lpr;
  int optin = 0, per_sm_max = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  CUDA_CHECK(cudaDeviceGetAttribute(&per_sm_max, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
  const size_t budget = std::min((size_t)optin - 1024, (size_t)per_sm_max / TILED_CTAS_PER_SM - 2048) / 2;
  const size_t wv = f32 ? 4 : 8;
  int cap = (int)((budget - scalar_stage_bytes(wv, tr, 0)) / (4 + wv)) - 64;
  while (cap > 0 && scalar_stage_bytes(wv, tr, cap) > budget) cap -= 16;
  if (cap <= 0) return 0;
  std::vector<int> rp(m->nnodes + 1);
  CUDA_CHECK(cudaMemcpyAsync(rp.data(), m->row_ptr, (m->nnodes + 1) * sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  std::vector<int> b;
  b.push_back(0);
  for (i64 r = 0; r < m->nnodes;) {
    if (rp[r + 1] - rp[r] > cap) return 0;  // a row longer than a tile holds
    i64 e = r;
    while (e < m->nnodes && e - r < tr && (i64)rp[e + 1] - rp[r] <= cap) ++e;
    b.push_back((int)e);
    r = e;
  }
  m->ntblk[k] = (int)b.size() - 1;
  upload(ctx, m->tblk[k], b.data(), b.size());
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  m->tblk_cap[k] = cap;
  m->tblk_tr[k] = tr;
  return tr;
}

// Ring depth actually used: the requested depth, lowered until
// TILED_CTAS_PER_SM CTAs fit on an SM (at least two stages).
int fitted_stages(fcu_ctx ctx, int requested, size_t stage) {
  static int per_sm_max = 0;
  if (!per_sm_max)
    CUDA_CHECK(cudaDeviceGetAttribute(&per_sm_max, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
  int ns = requested;
  while (ns > 2 && (size_t)TILED_CTAS_PER_SM * (ns * stage + 2048) > (size_t)per_sm_max) --ns;
  return ns;
}

// Tiled 3x3-block SpMV launch: shared memory for the ring sized by the
// longest block row; grid = resident CTAs (persistent), at most one per tile.
template <int DIFF, class T, int TR, int BS = 3>
int launch_spmv_tiled_tr(fcu_matrix m, Workspace* w, const T* val, const T* p, T* ap) {
  fcu_ctx ctx = m->ctx;
  const int kp = sizeof(T) == 4 ? 1 : 0;
  const int cap = BS == 3 ? TR * max_block_row(m) : m->tblk_cap[kp];
  const int* tb = BS == 3 ? nullptr : m->tblk[kp].p;
  const i64 ntb = BS == 3 ? 0 : m->ntblk[kp];
  const size_t stage = tile_stage_bytes<T, TR, BS>(cap);
  const int nstage = fitted_stages(ctx, w->stages[sizeof(T) == 4 ? 1 : 0], stage);
  const size_t smem = nstage * stage;
  auto kern = k_spmv_tiled<DIFF, T, TR, BS>;
  static int configured_dev = -1;
  static size_t configured_smem = 0;
  if (configured_dev != ctx->device || configured_smem < smem) {
    CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured_dev = ctx->device;
    configured_smem = smem;
  }
  int per_sm = 0;
  CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SPMV_THREADS, smem));
  if (per_sm < 1) fail(FCU_ERR_UNSUPPORTED, "rows too long for the tiled SpMV");
  // The grid sets the order in which p.Ap is reduced, so it does not follow
  // the ring depth: TILED_CTAS_PER_SM CTAs per SM whenever they fit, which
  // keeps the iterates identical for every depth the tuner may pick.
  const i64 ntiles = BS == 3 ? (m->nnodes + TR - 1) / TR : ntb;
  const int grid =
      (int)std::max<i64>(1, std::min<i64>(ntiles, (i64)std::min(per_sm, TILED_CTAS_PER_SM) * ctx->num_sms));
  launch_pdl_cfg(ctx, kern, grid, SPMV_THREADS, smem, m->row_ptr, m->col_idx, val, m->nnodes, cap, nstage, tb, ntb,
                 p, ap, w->st.p, w->partials.p);
  return grid;
}

// Returns the grid (the number of p.Ap partials the update kernel adds).
template <int DIFF, class T>
int launch_spmv_tiled(fcu_matrix m, Workspace* w, const T* val, const T* p, T* ap) {
  if (tile_rows(sizeof(T)) == 64) return launch_spmv_tiled_tr<DIFF, T, 64>(m, w, val, p, ap);
  return launch_spmv_tiled_tr<DIFF, T, 32>(m, w, val, p, ap);
}

// Scalar CSR through the tiled kernel, TR rows per tile (scalar_tile_rows).
template <int DIFF, class T>
int launch_spmv_tiled_scalar(fcu_matrix m, Workspace* w, const T* val, const T* p, T* ap) {
  switch (scalar_tile_rows(m, sizeof(T) == 4)) {
    case 512: return launch_spmv_tiled_tr<DIFF, T, 512, 1>(m, w, val, p, ap);
    case 256: return launch_spmv_tiled_tr<DIFF, T, 256, 1>(m, w, val, p, ap);
    case 128: return launch_spmv_tiled_tr<DIFF, T, 128, 1>(m, w, val, p, ap);
    case 64: return launch_spmv_tiled_tr<DIFF, T, 64, 1>(m, w, val, p, ap);
    default: return launch_spmv_tiled_tr<DIFF, T, 32, 1>(m, w, val, p, ap);
  }
}

bool use_tiled_spmv() {
  static int v = [] {
    const char* e = getenv("FCU_TILED_SPMV");
    return e ? atoi(e) : 1;
  }();
  return v != 0;
}

// Dispatch a node-row kernel: KERNEL(BS, VPR) names the instantiation.
#define DISPATCH_ROWS(BS_, VPR_, GRID, KERNEL, ...)                           \
  do {                                                                        \
    if ((BS_) == 3) launch_pdl(ctx, KERNEL(3, 16), GRID, __VA_ARGS__);        \
    else if ((VPR_) == 4) launch_pdl(ctx, KERNEL(1, 4), GRID, __VA_ARGS__);   \
    else if ((VPR_) == 8) launch_pdl(ctx, KERNEL(1, 8), GRID, __VA_ARGS__);   \
    else if ((VPR_) == 16) launch_pdl(ctx, KERNEL(1, 16), GRID, __VA_ARGS__); \
    else launch_pdl(ctx, KERNEL(1, 32), GRID, __VA_ARGS__);                   \
  } while (0)

#define K_SPMV_AP64(B, V) k_spmv_ap<B, V, double>
#define K_SPMV_AP32(B, V) k_spmv_ap<B, V, float>
#define K_SPMV_DIR64(B, V) k_spmv_dir<B, V, double>
#define K_SPMV_DIR32(B, V) k_spmv_dir<B, V, float>
#define K_INIT64(B, V) k_init_residual<B, V, double>
#define K_INIT32(B, V) k_init_residual<B, V, float>
#define K_REPLACE(B, V) k_mx_replace<B, V>
#define K_PLAIN(B, V) k_spmv_plain<B, V>

// Fuse the direction update into the SpMV (1) or run it as its own kernel
// (0); FCU_FUSE_DIRECTION overrides the default.
bool fuse_direction() {
  static int v = [] {
    const char* e = getenv("FCU_FUSE_DIRECTION");
    return e ? atoi(e) : 0;
  }();
  return v != 0;
}

// One PCG iteration; `parity` selects which p buffer is old / new.
void enqueue_iteration(fcu_matrix m, Workspace* w, bool mixed, int parity) {
  fcu_ctx ctx = m->ctx;
  const int g = w->grid;
  const i64 n = m->n, nr = m->nnodes;
  if (!fuse_direction()) {
    // direction (p = z + beta p, in place on buffer a) then SpMV
    if (!mixed) {
      launch_pdl(ctx, k_direction<double>, w->vgrid, n, w->pa64.p, w->z64.p, w->st.p);
      int npap = g;
      if (m->bs == 3 && use_tiled_spmv()) {
        npap = launch_spmv_tiled<0, double>(m, w, m->val64.p, w->pa64.p, w->ap64.p);
      } else if (w->tiled1[0]) {
        npap = launch_spmv_tiled_scalar<0, double>(m, w, m->val64.p, w->pa64.p, w->ap64.p);
      } else if (w->stream[0]) {
        npap = stream_grid_for(ctx, m->nrowblk, k_spmv_stream<double>);
        launch_pdl_cfg(ctx, k_spmv_stream<double>, npap, STREAM_THREADS, 0, m->row_ptr, m->col_idx, m->val64.p,
                       m->diag_pos, m->rowblk.p, m->nrowblk, w->pa64.p, w->ap64.p, w->st.p, w->partials.p);
      } else {
        DISPATCH_ROWS(m->bs, w->vpr, g, K_SPMV_AP64, m->row_ptr, m->col_idx, m->val64.p, nr, w->pa64.p, w->ap64.p,
                      w->st.p, w->partials.p);
      }
      if (m->bdinv.p)
        launch_pdl_cfg(ctx, k_update_block, update_block_grid(ctx, m->nnodes), UB_THREADS, 0, m->nnodes, w->x.p,
                       w->r.p, w->pa64.p, w->ap64.p, m->bdinv.p, w->z64.p, w->st.p, w->partials.p, npap);
      else
        launch_pdl(ctx, k_update<double>, w->vgrid, n, w->x.p, w->r.p, w->pa64.p, w->ap64.p, w->invd.p, w->z64.p,
                   w->st.p, w->partials.p, npap);
    } else {
      launch_pdl(ctx, k_direction<float>, w->vgrid, n, w->pa32.p, w->z32.p, w->st.p);
      int npap = g;
      if (m->bs == 3 && use_tiled_spmv()) {
        npap = launch_spmv_tiled<1, float>(m, w, m->val32.p, w->pa32.p, w->ap32.p);
      } else if (w->tiled1[1]) {
        npap = launch_spmv_tiled_scalar<1, float>(m, w, m->val32.p, w->pa32.p, w->ap32.p);
      } else if (w->stream[1]) {
        npap = stream_grid_for(ctx, m->nrowblk, k_spmv_stream<float>);
        launch_pdl_cfg(ctx, k_spmv_stream<float>, npap, STREAM_THREADS, 0, m->row_ptr, m->col_idx, m->val32.p,
                       m->diag_pos, m->rowblk.p, m->nrowblk, w->pa32.p, w->ap32.p, w->st.p, w->partials.p);
      } else {
        DISPATCH_ROWS(m->bs, w->vpr32, g, K_SPMV_AP32, m->row_ptr, m->col_idx, m->val32.p, nr, w->pa32.p, w->ap32.p,
                      w->st.p, w->partials.p);
      }
      launch_pdl(ctx, k_update<float>, w->vgrid, n, w->x.p, w->r.p, w->pa32.p, w->ap32.p, w->invd.p, w->z32.p,
                 w->st.p, w->partials.p, npap);
    }
    return;
  }
  if (!mixed) {
    double* pold = parity ? w->pb64.p : w->pa64.p;
    double* pnew = parity ? w->pa64.p : w->pb64.p;
    DISPATCH_ROWS(m->bs, w->vpr, g, K_SPMV_DIR64, m->row_ptr, m->col_idx, m->val64.p, nr, w->z64.p, pold, pnew,
                  w->ap64.p, w->st.p, w->partials.p);
    launch_pdl(ctx, k_update<double>, g, n, w->x.p, w->r.p, pnew, w->ap64.p, w->invd.p, w->z64.p, w->st.p,
               w->partials.p, g);
  } else {
    float* pold = parity ? w->pb32.p : w->pa32.p;
    float* pnew = parity ? w->pa32.p : w->pb32.p;
    DISPATCH_ROWS(m->bs, w->vpr32, g, K_SPMV_DIR32, m->row_ptr, m->col_idx, m->val32.p, nr, w->z32.p, pold, pnew,
                  w->ap32.p, w->st.p, w->partials.p);
    launch_pdl(ctx, k_update<float>, g, n, w->x.p, w->r.p, pnew, w->ap32.p, w->invd.p, w->z32.p, w->st.p,
               w->partials.p, g);
  }
}

int launches_per_iteration() { return fuse_direction() ? 2 : 3; }

// The persistent loop (k_pcg_persistent) runs on 3x3-block matrices on the
// tiled SpMV with point-Jacobi preconditioning.
bool persistent_capable(fcu_matrix m) {
  return m->bs == 3 && use_tiled_spmv() && !m->bdinv.p && !fuse_direction();
}

// Which solves take the persistent loop: mixed precision by default (on B200
// at 421k and 1.57M elasticity dofs it beats the per-iteration graph by
// 3-6% per iteration); FP64 keeps the graph, whose tiled SpMV gathers one
// 8-byte operand per component instead of the loop's 16-byte (z, p) pair
// (equal at 421k dofs, 12% faster at 1.57M). FCU_PERSISTENT=0 keeps the graph
// for both, FCU_PERSISTENT=2 takes the loop for both.
bool use_persistent(fcu_matrix m, bool mixed) {
  static int v = [] {
    const char* e = getenv("FCU_PERSISTENT");
    return e ? atoi(e) : 1;
  }();
  return persistent_capable(m) && (v == 2 || (v == 1 && mixed));
}

// One cooperative launch of the persistent loop: the tiled SpMV's ring and
// CTAs (up to TILED_CTAS_PER_SM per SM, all resident); the launch fails
// rather than run when they cannot all be resident. The caller zeroes the
// barrier count (w->bar) on the stream first.
template <bool DIFF, class T, int TR>
void launch_persistent_tr(fcu_matrix m, Workspace* w, const T* val, typename Pair<T>::type* zp, T* ap) {
  fcu_ctx ctx = m->ctx;
  const int cap = TR * max_block_row(m);
  const size_t stage = tile_stage_bytes<T, TR, 3>(cap);
  const int nstage = fitted_stages(ctx, w->stages[sizeof(T) == 4 ? 1 : 0], stage);
  const size_t smem = nstage * stage;
  auto kern = k_pcg_persistent<DIFF, T, TR>;
  static int configured_dev = -1;
  static size_t configured_smem = 0;
  if (configured_dev != ctx->device || configured_smem < smem) {
    CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured_dev = ctx->device;
    configured_smem = smem;
  }
  int per_sm = 0;
  CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SPMV_THREADS, smem));
  if (per_sm < 1) fail(FCU_ERR_UNSUPPORTED, "rows too long for the tiled SpMV");
  const int grid = std::min(MAXG, std::min(per_sm, TILED_CTAS_PER_SM) * ctx->num_sms);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(SPMV_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, m->row_ptr, m->col_idx, val, m->nnodes, cap, nstage, m->n, w->x.p,
                                w->r.p, (const double*)w->invd.p, zp, ap, w->st.p, w->partials.p, w->bar.p));
  ctx->launches++;
}

// The (z, p) pairs of the persistent loop from the solver's z and p vectors;
// with_p false refreshes only the z half (after a residual replacement).
void pack_zp(fcu_matrix m, Workspace* w, bool mixed, bool with_p) {
  fcu_ctx ctx = m->ctx;
  const i64 n = m->n;
  const int g = grid_for(n, 256, ctx->num_sms * 8);
  if (mixed) {
    if (!w->zp32.p) w->zp32.alloc(n);
    k_zp_pack<float><<<g, 256, 0, ctx->stream>>>(w->z32.p, with_p ? w->pa32.p : nullptr, n, w->zp32.p);
  } else {
    if (!w->zp64.p) w->zp64.alloc(n);
    k_zp_pack<double><<<g, 256, 0, ctx->stream>>>(w->z64.p, with_p ? w->pa64.p : nullptr, n, w->zp64.p);
  }
  LAUNCH_CHECK(ctx);
}

// One launch of the persistent loop in the solve's precision, after zeroing
// its barrier count.
void launch_persistent(fcu_matrix m, Workspace* w, bool mixed) {
  fcu_ctx ctx = m->ctx;
  if (!w->bar.p) w->bar.alloc(1);
  CUDA_CHECK(cudaMemsetAsync(w->bar.p, 0, sizeof(unsigned long long), ctx->stream));
  if (mixed) {
    if (tile_rows(4) == 64) launch_persistent_tr<true, float, 64>(m, w, m->val32.p, w->zp32.p, w->ap32.p);
    else launch_persistent_tr<true, float, 32>(m, w, m->val32.p, w->zp32.p, w->ap32.p);
  } else {
    launch_persistent_tr<false, double, 32>(m, w, m->val64.p, w->zp64.p, w->ap64.p);
  }
}

// Runs the solve to its end through the persistent loop: one launch in FP64;
// in mixed precision one per stretch between residual replacements, each
// replacement run by k_mx_replace between them.
void run_persistent(fcu_matrix m, Workspace* w, bool mixed, i64 max_iter) {
  fcu_ctx ctx = m->ctx;
  CgState* hs = w->host_st;
  pack_zp(m, w, mixed, true);
  for (i64 round = 0; round <= max_iter + 1; ++round) {
    launch_persistent(m, w, mixed);
    CUDA_CHECK(cudaMemcpyAsync(hs, w->st.p, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    if (hs->done || hs->fault || !(mixed && hs->pause)) break;
    // r = b - A64 x, z = D^-1 r, and the state's replacement step
    DISPATCH_ROWS(m->bs, w->vpr, w->grid, K_REPLACE, m->row_ptr, m->col_idx, m->val64.p, m->nnodes, w->x.p, w->b.p,
                  w->invd.p, w->r.p, w->z32.p, w->st.p, w->partials.p);
    pack_zp(m, w, mixed, false);
  }
  if (hs->fault && !hs->done) {
    hs->done = 1;
    hs->status = FCU_ERR_CUDA;
  } else if (hs->fault) {
    hs->status = FCU_ERR_CUDA;
  }
}

// Kernels in one replay of the iteration graph.
int launches_per_replay(bool mixed) { return CHUNK * launches_per_iteration() + (mixed ? 1 : 0); }

cudaGraphExec_t get_graph(fcu_matrix m, Workspace* w, bool mixed) {
  fcu_ctx ctx = m->ctx;
  cudaGraphExec_t& ge = w->graph[mixed ? 1 : 0];
  if (ge) return ge;
  cudaGraph_t g;
  const i64 launches0 = ctx->launches;
  CUDA_CHECK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  try {
    // mixed: the residual replacement that an iteration of the previous
    // replay asked for (r = b - A64 x); it returns at once otherwise
    if (mixed)
      DISPATCH_ROWS(m->bs, w->vpr, w->grid, K_REPLACE, m->row_ptr, m->col_idx, m->val64.p, m->nnodes, w->x.p, w->b.p,
                    w->invd.p, w->r.p, w->z32.p, w->st.p, w->partials.p);
    for (int it = 0; it < CHUNK; ++it) enqueue_iteration(m, w, mixed, it & 1);
  } catch (...) {
    cudaStreamEndCapture(ctx->stream, &g);
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &g));
  CUDA_CHECK(cudaGraphInstantiate(&ge, g, 0));
  cudaGraphDestroy(g);
  // launches inside the graph are counted per replay in run_pcg
  ctx->launches = launches0;
  return ge;
}

}  // namespace

// Algorithmic bytes of one PCG iteration (per launch pair):
//   spmv:   matrix values + column indices + row pointers, z and p_old read
//           once, p_new and Ap written once
//   update: x, r read and written; p, Ap, D^-1 read; z written
// FP64: 8-byte values and vectors. Mixed: 4-byte values, p, Ap, z; x, r and
// D^-1 stay 8-byte.
double pcg_bytes_per_iter(fcu_matrix m, bool mixed) {
  const double bs2 = (double)m->bs * m->bs;
  const double n = (double)m->n;
  const double w = mixed ? 4.0 : 8.0;
  const double mat = (double)m->nnzb * (bs2 * w + 4.0) + 4.0 * (double)(m->nnodes + 1);
  const double spmv_vec = 4.0 * n * w;
  const double update = n * (8 + 8 + 8 + 8) + n * (w + w + 8) + n * w;
  // block-Jacobi reads 9 inverse-block values per block row instead of 3 diagonal ones
  const double block = (!mixed && m->bdinv.p) ? 2.0 * n * 8.0 : 0.0;
  return mat + spmv_vec + update + block;
}

void ensure_inv_diag(fcu_matrix m, Workspace* w) {
  fcu_ctx ctx = m->ctx;
  if (m->bs == 3)
    k_inv_diag<3><<<grid_for(m->n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->diag_pos, m->val64.p, m->nnodes,
                                                                                  w->invd.p);
  else
    k_inv_diag<1><<<grid_for(m->n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->diag_pos, m->val64.p, m->nnodes,
                                                                                  w->invd.p);
  LAUNCH_CHECK(ctx);
}

void build_rowsum32(fcu_matrix m) {
  fcu_ctx ctx = m->ctx;
  const i64 t = m->nnodes * m->bs * m->bs;
  if (m->bs == 3)
    k_build_rowsum32<3><<<grid_for(t, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->row_ptr, m->diag_pos,
                                                                                     m->val64.p, m->nnodes, m->val32.p);
  else
    k_build_rowsum32<1><<<grid_for(t, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->row_ptr, m->diag_pos,
                                                                                     m->val64.p, m->nnodes, m->val32.p);
  LAUNCH_CHECK(ctx);
}

void tune_spmv(fcu_matrix m, Workspace* w, bool mixed);

int batch_pcg_impl(fcu_matrix m, i64 nb, const i64* offsets_host, const double* b_dev, double* x_dev, double tol,
                   i64 max_iter, int precision, i64* iters_host, double* relres_host, int* status_host,
                   fcu_solve_info* info, const int* fixed_shape);

// Scalar systems of at most this many rows go through the batched kernel
// (see run_pcg): measured faster up to ~17k rows in FP64 and ~33k in mixed
// precision, slower in FP64 at 33k. FCU_SMALL_BATCHED=0 keeps them on the
// per-iteration graph.
constexpr i64 SMALL_SYSTEM_ROWS_FP64 = 20000;
constexpr i64 SMALL_SYSTEM_ROWS_MIXED = 32768;
bool small_systems_batched() {
  static int v = [] {
    const char* e = getenv("FCU_SMALL_BATCHED");
    return e ? atoi(e) : 1;
  }();
  return v != 0;
}

// Core PCG driver on device buffers: b_dev, x0_dev (nullable) -> x_dev.
// inv_diag_dev (nullable) overrides the matrix diagonal (solve_csr_cg_gpu).
int run_pcg(fcu_matrix m, const double* b_dev, const double* x0_dev, double* x_dev, double tol, i64 max_iter,
            int precision, bool gpu_semantics, const double* inv_diag_dev, fcu_solve_info* info) {
  fcu_ctx ctx = m->ctx;
  const bool mixed = precision == FCU_MIXED;
  if (mixed && !m->val32.p) fail(FCU_ERR_BAD_ARG, "matrix has no FP32 copy");
  if (mixed && m->bdinv.p) fail(FCU_ERR_UNSUPPORTED, "block-Jacobi preconditioning runs in FP64");
  if (m->block_jacobi && !inv_diag_dev) refresh_block_jacobi(m);
  if (mixed && m->missing_diag) fail(FCU_ERR_UNSUPPORTED, "the mixed operator needs every diagonal block");
  // A small scalar system solved from x0 = 0 with the point-Jacobi diagonal
  // of its own values: one launch of the batched kernel with the system as
  // its single instance (one cluster of up to 8 CTAs, reductions in
  // distributed shared memory), instead of three launches per iteration,
  // whose fixed costs dominate at this size. Same recurrence and stopping
  // rules (cg.rs:40-149); the kernel shape is fixed by rule, so the
  // iterates repeat from run to run.
  if (m->bs == 1 && !x0_dev && !gpu_semantics && !inv_diag_dev && !m->bdinv.p && max_iter > 0 &&
      m->n > 0 && m->n <= (mixed ? SMALL_SYSTEM_ROWS_MIXED : SMALL_SYSTEM_ROWS_FP64) && small_systems_batched()) {
    const double mean = (double)m->nnzb / (double)m->n;
    const int shape[3] = {mean <= 12.0 ? 1 : mean <= 40.0 ? 2 : 4, m->n <= 4096 ? 512 : 1024,
                          m->n <= 512 ? 1 : m->n <= 1024 ? 2 : m->n <= 2048 ? 4 : 8};
    const i64 offs[2] = {0, m->n};
    i64 it = 0;
    double rel = 0.0;
    int st = 0;
    return batch_pcg_impl(m, 1, offs, b_dev, x_dev, tol, max_iter, precision, &it, &rel, &st, info, shape);
  }
  Workspace* w = ensure_ws(m, mixed);
  const i64 n = m->n, nr = m->nnodes;
  const int g = w->grid;
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
  if (inv_diag_dev) {
    CUDA_CHECK(cudaMemcpyAsync(w->invd.p, inv_diag_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  } else if (m->bdinv.p) {
    k_invd_from_blocks<<<grid_for(n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->bdinv.p, n, w->invd.p);
    LAUNCH_CHECK(ctx);
  } else {
    ensure_inv_diag(m, w);
  }
  if (mixed) build_rowsum32(m);
  tune_spmv(m, w, mixed);  // first solve in this precision only

  CgState init{};
  init.tol = tol;
  init.max_iter = max_iter;
  init.gpu_semantics = gpu_semantics ? 1 : 0;
  init.delta = 0.1;
  *w->host_st = init;
  CUDA_CHECK(cudaMemcpyAsync(w->st.p, w->host_st, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_CHECK(cudaMemcpyAsync(w->b.p, b_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (x0_dev) CUDA_CHECK(cudaMemcpyAsync(w->x.p, x0_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  else CUDA_CHECK(cudaMemsetAsync(w->x.p, 0, n * sizeof(double), ctx->stream));
  // r = b - A x0 ; z = D^-1 r ; ||b|| ; r.z ; p_old = 0 ; initial test (cg.rs:79-90)
  if (mixed)
    DISPATCH_ROWS(m->bs, w->vpr, g, K_INIT32, m->row_ptr, m->col_idx, m->val64.p, nr, w->x.p, w->b.p, w->invd.p,
                  w->r.p, w->z32.p, w->pa32.p, n, w->st.p, w->partials.p);
  else
    DISPATCH_ROWS(m->bs, w->vpr, g, K_INIT64, m->row_ptr, m->col_idx, m->val64.p, nr, w->x.p, w->b.p, w->invd.p,
                  w->r.p, w->z64.p, w->pa64.p, n, w->st.p, w->partials.p);
  if (!mixed && m->bdinv.p)
    launch_pdl(ctx, k_block_init, w->vgrid, m->nnodes, w->r.p, m->bdinv.p, w->z64.p, w->st.p, w->partials.p);
  CUDA_CHECK(cudaMemcpyAsync(w->host_st, w->st.p, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  bool zero_rhs = gpu_semantics && w->host_st->bnorm == 0.0;
  if (zero_rhs) {
    // gpu.rs:1169-1180: zero right-hand side -> zero solution, Ok
    CUDA_CHECK(cudaMemsetAsync(x_dev, 0, n * sizeof(double), ctx->stream));
    w->host_st->done = 1;
    w->host_st->status = FCU_OK;
    w->host_st->iter = 0;
  } else if (!w->host_st->done && max_iter > 0 && use_persistent(m, mixed)) {
    run_persistent(m, w, mixed, max_iter);
  } else if (!w->host_st->done && max_iter > 0) {
    // Replays of CHUNK iterations, each followed by a copy of the state
    // record to the host. The host keeps one replay queued beyond the one
    // whose state it is reading, so the GPU does not wait for the host
    // between replays. In the mixed solve an iteration that flags a residual
    // replacement pauses the rest of its replay, and the next replay's first
    // kernel performs the replacement, right after that iteration. Kernels of
    // a replay queued after the solve ended return at once and change
    // nothing. Every replay but the first completes at least one iteration
    // and the iteration limit is enforced on the device, so max_iter + 2
    // replays always suffice.
    cudaGraphExec_t ge = get_graph(m, w, mixed);
    CgState* hs = w->host_st;
    auto issue = [&](int slot) {
      CUDA_CHECK(cudaGraphLaunch(ge, ctx->stream));
      ctx->launches += launches_per_replay(mixed);
      CUDA_CHECK(cudaMemcpyAsync(&hs[slot], w->st.p, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaEventRecord(w->ev[slot], ctx->stream));
    };
    const i64 max_replays = max_iter + 2;
    int slot = 0;
    issue(0);
    i64 issued = 1;
    for (;;) {
      const bool more = issued < max_replays;
      if (more) {
        issue(slot ^ 1);
        ++issued;
      }
      CUDA_CHECK(cudaEventSynchronize(w->ev[slot]));
      if (hs[slot].done || !more) break;
      slot ^= 1;
    }
    // the final state, after any replay still queued
    CUDA_CHECK(cudaMemcpyAsync(&hs[0], w->st.p, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  } else if (!w->host_st->done) {
    w->host_st->status = gpu_semantics ? FCU_OK : FCU_ERR_NO_CONVERGENCE;
  }
  if (!zero_rhs) CUDA_CHECK(cudaMemcpyAsync(x_dev, w->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
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

// Drops the captured iteration graphs (their kernels depend on the
// preconditioner the matrix carries).
void invalidate_graphs(fcu_matrix m) {
  if (!m->ws) return;
  for (auto& g : m->ws->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

void spmv_impl(fcu_matrix m, const double* x_dev, double* y_dev) {
  fcu_ctx ctx = m->ctx;
  if (use_stream_spmv(m)) {
    ensure_row_blocks(m);
    launch_pdl_cfg(ctx, k_spmv_stream_plain, stream_grid_for(ctx, m->nrowblk, k_spmv_stream_plain), STREAM_THREADS, 0, m->row_ptr, m->col_idx,
                   m->val64.p, m->rowblk.p, m->nrowblk, x_dev, y_dev);
    return;
  }
  const int vpr = pick_vpr(m);
  const int g = solver_grid(ctx, m->n);
  DISPATCH_ROWS(m->bs, vpr, g, K_PLAIN, m->row_ptr, m->col_idx, m->val64.p, m->nnodes, x_dev, y_dev);
}

// --- SpMV shape tuning --------------------------------------------------------
// The first solve of a matrix in a precision times the candidate shapes of
// its SpMV on the matrix itself and keeps the fastest: lanes per row
// {4, 8, 16, 32} for CSR, ring depth {2, 3, 4} for the tiled 3x3-block
// kernel. The choice is kept in the context by matrix shape, so a later
// matrix of the same shape takes it without timing. FCU_TUNE=0 keeps the
// defaults (CSR lanes by mean row length, three stages).

// Solver state and operand for SpMV timing: every launch does the full
// product (no convergence or breakdown exit).
void spmv_timing_state(fcu_matrix m, Workspace* w, bool mixed) {
  fcu_ctx ctx = m->ctx;
  CgState init{};
  init.rz = 1.0;
  init.beta = 0.5;
  init.gpu_semantics = 1;
  init.timing = 1;
  *w->host_st = init;
  CUDA_CHECK(cudaMemcpyAsync(w->st.p, w->host_st, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
  const i64 n = m->n;
  // any non-zero vectors (1/64 in every entry)
  if (mixed) {
    CUDA_CHECK(cudaMemsetAsync(w->z32.p, 0x3c, n * sizeof(float), ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(w->pa32.p, 0x3c, n * sizeof(float), ctx->stream));
  } else {
    CUDA_CHECK(cudaMemsetAsync(w->z64.p, 0x3f, n * sizeof(double), ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(w->pa64.p, 0x3f, n * sizeof(double), ctx->stream));
  }
}

// One launch of the PCG's SpMV (Ap = A p) with the workspace's shape.
void enqueue_spmv(fcu_matrix m, Workspace* w, bool mixed) {
  fcu_ctx ctx = m->ctx;
  const int g = w->grid;
  if (mixed) {
    if (m->bs == 3 && use_tiled_spmv()) launch_spmv_tiled<1, float>(m, w, m->val32.p, w->pa32.p, w->ap32.p);
    else if (w->tiled1[1]) launch_spmv_tiled_scalar<1, float>(m, w, m->val32.p, w->pa32.p, w->ap32.p);
    else if (w->stream[1])
      launch_pdl_cfg(ctx, k_spmv_stream<float>, stream_grid_for(ctx, m->nrowblk, k_spmv_stream<float>), STREAM_THREADS, 0, m->row_ptr,
                     m->col_idx, m->val32.p, m->diag_pos, m->rowblk.p, m->nrowblk, w->pa32.p, w->ap32.p, w->st.p,
                     w->partials.p);
    else
      DISPATCH_ROWS(m->bs, w->vpr32, g, K_SPMV_AP32, m->row_ptr, m->col_idx, m->val32.p, m->nnodes, w->pa32.p,
                    w->ap32.p, w->st.p, w->partials.p);
  } else {
    if (m->bs == 3 && use_tiled_spmv()) launch_spmv_tiled<0, double>(m, w, m->val64.p, w->pa64.p, w->ap64.p);
    else if (w->tiled1[0]) launch_spmv_tiled_scalar<0, double>(m, w, m->val64.p, w->pa64.p, w->ap64.p);
    else if (w->stream[0])
      launch_pdl_cfg(ctx, k_spmv_stream<double>, stream_grid_for(ctx, m->nrowblk, k_spmv_stream<double>), STREAM_THREADS, 0, m->row_ptr,
                     m->col_idx, m->val64.p, m->diag_pos, m->rowblk.p, m->nrowblk, w->pa64.p, w->ap64.p, w->st.p,
                     w->partials.p);
    else
      DISPATCH_ROWS(m->bs, w->vpr, g, K_SPMV_AP64, m->row_ptr, m->col_idx, m->val64.p, m->nnodes, w->pa64.p,
                    w->ap64.p, w->st.p, w->partials.p);
  }
}

// Mean device time of `reps` back-to-back SpMV launches (ms).
double time_spmv_launches(fcu_matrix m, Workspace* w, bool mixed, int reps) {
  fcu_ctx ctx = m->ctx;
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
  for (int r = 0; r < reps; ++r) enqueue_spmv(m, w, mixed);
  CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
  CUDA_CHECK(cudaEventSynchronize(e1));
  float t = 0.f;
  CUDA_CHECK(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return reps > 0 ? (double)t / reps : 0.0;
}

int scalar_tiled_mode() {
  static int v = [] {
    const char* e = getenv("FCU_SCALAR_TILED");
    return e ? atoi(e) : 1;
  }();
  return v;
}

bool tuning_enabled() {
  static int v = [] {
    const char* e = getenv("FCU_TUNE");
    return e ? atoi(e) : 1;
  }();
  return v != 0;
}

void tune_spmv(fcu_matrix m, Workspace* w, bool mixed) {
  const int k = mixed ? 1 : 0;
  if (w->tuned[k]) return;
  w->tuned[k] = true;
  if (!tuning_enabled()) return;
  fcu_ctx ctx = m->ctx;
  const std::array<i64, 5> key = {m->bs, m->n, m->nnzb, max_block_row(m), k};
  const bool tiled = m->bs == 3 && use_tiled_spmv();
  auto known = ctx->spmv_tune.find(key);
  if (known != ctx->spmv_tune.end()) {
    if (tiled) {
      w->stages[k] = known->second[0];
    } else if (known->second[1] == 2) {
      // tile sizes are measured here, never while a graph is being captured;
      // a matrix of the same shape whose tiles do not fit keeps the CSR kernels
      w->tiled1[k] = scalar_tile_rows(m, mixed) > 0;
      w->stages[k] = known->second[0];
    } else {
      (mixed ? w->vpr32 : w->vpr) = known->second[0];
      w->stream[k] = known->second[1] != 0;
    }
    return;
  }
  spmv_timing_state(m, w, mixed);
  auto trial = [&]() {
    enqueue_spmv(m, w, mixed);  // warm
    return time_spmv_launches(m, w, mixed, 8);
  };
  if (tiled) {
    int optin = 0;
    CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const size_t vb = mixed ? 4 : 8;
    const int tr = tile_rows(vb);
    const size_t stage = tile_stage_bytes_rt(vb, tr, tr * max_block_row(m));
    int best = w->stages[k];
    double best_ms = 1e30;
    int per_sm_max = 0;
    CUDA_CHECK(cudaDeviceGetAttribute(&per_sm_max, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
    for (int ns = 2; ns <= MAX_STAGES; ++ns) {
      // every candidate keeps the same grid (TILED_CTAS_PER_SM per SM)
      if (ns * stage + 1024 > (size_t)optin ||
          TILED_CTAS_PER_SM * (ns * stage + 2048) > (size_t)per_sm_max)
        continue;
      w->stages[k] = ns;
      const double ms = trial();
      if (ms < best_ms) {
        best_ms = ms;
        best = ns;
      }
    }
    w->stages[k] = best;
    ctx->spmv_tune[key] = {best, 0};
  } else {
    // The tiled kernel (TMA-staged tiles of rows) replaces the others
    // whenever its tiles fit (scalar_tile_rows): by rule, not by timing, so
    // that the choice and the iterates repeat from run to run; only its ring
    // depth is timed, which changes no result. FCU_SCALAR_TILED=0 turns it
    // off.
    if (use_tiled_spmv() && scalar_tiled_mode() != 0 && scalar_tile_rows(m, mixed) > 0) {
      w->tiled1[k] = true;
      int best_stages = 2;
      double tiled_ms = 1e30;
      for (int ns = 2; ns <= MAX_STAGES; ++ns) {
        w->stages[k] = ns;
        const double ms = trial();
        if (ms < tiled_ms) {
          tiled_ms = ms;
          best_stages = ns;
        }
      }
      w->stages[k] = best_stages;
      ctx->spmv_tune[key] = {best_stages, 2};
      return;
    }
    // Otherwise the CSR kernels. Lanes per row change the summation order
    // inside a row, so a shape replaces the default only when it is clearly
    // (10%) faster: near-ties then cannot flip the choice, and the iterates,
    // from run to run. Candidates: the CSR-stream kernel (when the rows are
    // short) and CSR vectors of 4-32 lanes per row.
    int& v = mixed ? w->vpr32 : w->vpr;
    bool& strm = w->stream[k];
    const bool dflt_stream = strm;
    const int dflt = v;
    const double dflt_ms = trial();
    bool best_stream = dflt_stream;
    int best = dflt;
    double best_ms = dflt_ms;
    strm = false;
    for (int c : {4, 8, 16, 32}) {
      if (c == dflt && !dflt_stream) continue;
      v = c;
      const double ms = trial();
      if (ms < 0.9 * dflt_ms && ms < best_ms) {
        best_ms = ms;
        best = c;
        best_stream = false;
      }
    }
    v = best;
    strm = best_stream;
    ctx->spmv_tune[key] = {best, best_stream ? 1 : 0};
  }
}

// Average time of the PCG SpMV kernel over `reps` launches (diagnostics),
// with the shape the solver uses.
void time_spmv_impl(fcu_matrix m, int precision, int reps, double* ms, double* bytes) {
  const bool mixed = precision == FCU_MIXED;
  Workspace* w = ensure_ws(m, mixed);
  if (mixed) build_rowsum32(m);
  tune_spmv(m, w, mixed);
  spmv_timing_state(m, w, mixed);
  *ms = time_spmv_launches(m, w, mixed, reps);
  const double bs2 = (double)m->bs * m->bs;
  const double wv = mixed ? 4.0 : 8.0;
  *bytes = (double)m->nnzb * (bs2 * wv + 4.0) + 4.0 * (double)(m->nnodes + 1) + 2.0 * (double)m->n * wv;
}

// Reads `n` 16-byte words and keeps one word per thread in `sink` (so the
// loads are not removed): a read-only sweep that evicts L2 without leaving
// dirty lines behind, whose write-back would otherwise land in the timed
// launch.
__global__ void k_flush_read(const uint4* __restrict__ buf, i64 n, uint4* __restrict__ sink) {
  uint4 acc = make_uint4(0u, 0u, 0u, 0u);
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const uint4 v = __ldcg(buf + i);
    acc.x ^= v.x; acc.y ^= v.y; acc.z ^= v.z; acc.w ^= v.w;
  }
  sink[blockIdx.x * (i64)blockDim.x + threadIdx.x] = acc;
}

__global__ void k_fill_value(double* __restrict__ v, i64 n, double a) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) v[i] = a;
}

// The same with L2 flushed before each launch: a read of `flush_bytes`
// evicts the matrix and p, then one SpMV is timed by events on either side.
// The sweep is queued before the first event, so the launch never waits on
// the host. Returns the mean single-launch time.
void time_spmv_cold_impl(fcu_matrix m, int precision, int reps, size_t flush_bytes, double* ms, double* bytes) {
  const bool mixed = precision == FCU_MIXED;
  Workspace* w = ensure_ws(m, mixed);
  if (mixed) build_rowsum32(m);
  tune_spmv(m, w, mixed);
  spmv_timing_state(m, w, mixed);
  fcu_ctx ctx = m->ctx;
  if (!flush_bytes) flush_bytes = 256ull << 20;
  flush_bytes = (flush_bytes + 15) / 16 * 16;
  DBuf<unsigned char> flush;
  flush.alloc(flush_bytes);
  CUDA_CHECK(cudaMemsetAsync(flush.p, 0, flush_bytes, ctx->stream));
  const int fgrid = ctx->num_sms * 8;
  DBuf<uint4> sink;
  sink.alloc((size_t)fgrid * 256);
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  double total = 0.0;
  for (int r = 0; r < reps; ++r) {
    k_flush_read<<<fgrid, 256, 0, ctx->stream>>>(reinterpret_cast<const uint4*>(flush.p), (i64)(flush_bytes / 16),
                                                 sink.p);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
    enqueue_spmv(m, w, mixed);
    CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
    CUDA_CHECK(cudaEventSynchronize(e1));
    float t = 0.f;
    CUDA_CHECK(cudaEventElapsedTime(&t, e0, e1));
    total += t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = reps > 0 ? total / reps : 0.0;
  const double bs2 = (double)m->bs * m->bs;
  const double wv = mixed ? 4.0 : 8.0;
  *bytes = (double)m->nnzb * (bs2 * wv + 4.0) + 4.0 * (double)(m->nnodes + 1) + 2.0 * (double)m->n * wv;
}

// Algorithmic bytes of one iteration of the persistent loop: the matrix
// (values, columns, row pointers) once; the product reads z and p_old and
// writes Ap; the update reads x, r, D^-1 (8-byte) and p_old, z, Ap, and
// writes x, r (8-byte) and p, z.
double persistent_bytes_per_iter(fcu_matrix m, bool mixed) {
  const double w = mixed ? 4.0 : 8.0;
  const double n = (double)m->n;
  const double mat = (double)m->nnzb * (9.0 * w + 4.0) + 4.0 * (double)(m->nnodes + 1);
  return mat + n * 3.0 * w + n * (24.0 + 3.0 * w) + n * (16.0 + 2.0 * w);
}

// Device time of one launch of the persistent loop running exactly `iters`
// iterations (no stopping test, no residual replacement, no breakdown exit)
// from x = 0 on b = 1, after a read sweep of `flush_bytes` that evicts L2;
// the mean over `reps` launches, each from a fresh start.
// Self-check of the bounded waits the persistent loop and the tiled SpMV
// rely on, with `limit` polls each. One CTA of the tiled kernels' shape:
// its consumer threads wait at a grid barrier whose count can never be
// reached (target 2 with one CTA arriving) and then at the same target,
// which their second arrival reaches; warp 0 waits on an mbarrier nothing arrives at and then
// on one whose single arrival it makes. out = {first grid wait passed,
// second grid wait passed, first mbarrier wait passed, second mbarrier wait
// passed}; a correct build gives {0, 1, 0, 1}.
__global__ void __launch_bounds__(SPMV_THREADS) k_wait_limits(unsigned long long* bar, unsigned limit,
                                                              int* __restrict__ out) {
  __shared__ unsigned long long mb[2];
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&mb[0], 1);
    mbar_init(&mb[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid >= 32) {
    const int ctid = tid - 32;
    const bool a = grid_barrier(bar, 2, ctid, limit);
    const bool b = grid_barrier(bar, 2, ctid, limit);  // the count is now 2
    if (ctid == 0) {
      out[0] = a ? 1 : 0;
      out[1] = b ? 1 : 0;
    }
  } else if (tid == 0) {
    out[2] = mbar_wait(&mb[0], 0, limit) ? 1 : 0;
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&mb[1])) : "memory");
    out[3] = mbar_wait(&mb[1], 0, limit) ? 1 : 0;
  }
}

void check_wait_limits_impl(fcu_ctx ctx, unsigned limit, int* results_host) {
  DBuf<unsigned long long> bar;
  DBuf<int> out;
  bar.alloc(1);
  out.alloc(4);
  CUDA_CHECK(cudaMemsetAsync(bar.p, 0, sizeof(unsigned long long), ctx->stream));
  CUDA_CHECK(cudaMemsetAsync(out.p, 0xff, 4 * sizeof(int), ctx->stream));
  k_wait_limits<<<1, SPMV_THREADS, 0, ctx->stream>>>(bar.p, limit, out.p);
  LAUNCH_CHECK(ctx);
  CUDA_CHECK(cudaMemcpyAsync(results_host, out.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  ctx->launches++;
}

void time_pcg_impl(fcu_matrix m, int precision, i64 iters, int reps, size_t flush_bytes, double* ms,
                   double* bytes) {
  if (!persistent_capable(m)) fail(FCU_ERR_UNSUPPORTED, "the persistent loop runs on 3x3-block point-Jacobi systems");
  const bool mixed = precision == FCU_MIXED;
  if (mixed && !m->val32.p) fail(FCU_ERR_BAD_ARG, "matrix has no FP32 copy");
  if (mixed && m->missing_diag) fail(FCU_ERR_UNSUPPORTED, "the mixed operator needs every diagonal block");
  fcu_ctx ctx = m->ctx;
  Workspace* w = ensure_ws(m, mixed);
  if (!w->bar.p) w->bar.alloc(1);
  ensure_inv_diag(m, w);
  if (mixed) build_rowsum32(m);
  tune_spmv(m, w, mixed);
  const i64 n = m->n;
  k_fill_value<<<grid_for(n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(w->b.p, n, 1.0);
  LAUNCH_CHECK(ctx);
  if (!flush_bytes) flush_bytes = 256ull << 20;
  flush_bytes = (flush_bytes + 15) / 16 * 16;
  DBuf<unsigned char> flush;
  flush.alloc(flush_bytes);
  CUDA_CHECK(cudaMemsetAsync(flush.p, 0, flush_bytes, ctx->stream));
  const int fgrid = ctx->num_sms * 8;
  DBuf<uint4> sink;
  sink.alloc((size_t)fgrid * 256);
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  double total = 0.0;
  for (int rep = 0; rep < reps; ++rep) {
    CgState init{};
    init.tol = 0.0;
    init.max_iter = iters;
    init.delta = 0.0;
    init.timing = 1;
    *w->host_st = init;
    CUDA_CHECK(cudaMemcpyAsync(w->st.p, w->host_st, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(w->x.p, 0, n * sizeof(double), ctx->stream));
    if (mixed)
      DISPATCH_ROWS(m->bs, w->vpr, w->grid, K_INIT32, m->row_ptr, m->col_idx, m->val64.p, m->nnodes, w->x.p, w->b.p,
                    w->invd.p, w->r.p, w->z32.p, w->pa32.p, n, w->st.p, w->partials.p);
    else
      DISPATCH_ROWS(m->bs, w->vpr, w->grid, K_INIT64, m->row_ptr, m->col_idx, m->val64.p, m->nnodes, w->x.p, w->b.p,
                    w->invd.p, w->r.p, w->z64.p, w->pa64.p, n, w->st.p, w->partials.p);
    pack_zp(m, w, mixed, true);
    k_flush_read<<<fgrid, 256, 0, ctx->stream>>>(reinterpret_cast<const uint4*>(flush.p), (i64)(flush_bytes / 16),
                                                 sink.p);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaMemsetAsync(w->bar.p, 0, sizeof(unsigned long long), ctx->stream));
    CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
    if (mixed) {
      if (tile_rows(4) == 64) launch_persistent_tr<true, float, 64>(m, w, m->val32.p, w->zp32.p, w->ap32.p);
      else launch_persistent_tr<true, float, 32>(m, w, m->val32.p, w->zp32.p, w->ap32.p);
    } else {
      launch_persistent_tr<false, double, 32>(m, w, m->val64.p, w->zp64.p, w->ap64.p);
    }
    CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
    CUDA_CHECK(cudaEventSynchronize(e1));
    float t = 0.f;
    CUDA_CHECK(cudaEventElapsedTime(&t, e0, e1));
    total += t;
    CUDA_CHECK(cudaMemcpy(w->host_st, w->st.p, sizeof(CgState), cudaMemcpyDeviceToHost));
    if (w->host_st->fault) fail(FCU_ERR_CUDA, "a bounded wait of the persistent loop gave up");
    if (w->host_st->iter != iters) fail(FCU_ERR_CUDA, "the persistent loop stopped before its iteration count");
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = reps > 0 ? total / reps : 0.0;
  *bytes = persistent_bytes_per_iter(m, mixed) * (double)iters;
}

// ---------------------------------------------------------------------------
// Allocation-free CSR PCG (fcu_solve_csr_cg_noalloc).
//
// Some callers cannot allocate device memory when they solve. One example is
// an application whose own pool allocator reserves the device's memory up
// front and leaves nothing for a library to cudaMalloc. Another is a
// time-stepping loop that solves many small systems: cudaMalloc and cudaFree
// synchronise the whole device, which would stall that application's other
// streams every step. For them this variant runs the same kernels as
// fcu_solve_csr_cg (FP64, gpu.rs semantics) but keeps all its work vectors,
// reduction partials and solver state in one fixed module-scope device
// array. A call allocates no device memory: no cudaMalloc, cudaMallocHost or
// cudaFree, no graph instantiation, no library routine that allocates.
//
// Limits and rules:
//  - at most NOALLOC_MAX_N rows (the array holds four vectors of that
//    length, about 4 MiB in all);
//  - every array argument is device memory of the current device (nothing
//    is staged, since staging would allocate);
//  - the array is shared by all calls on a device, so calls that overlap in
//    time on one device (from several host threads) race and corrupt each
//    other's results. Callers must not overlap them;
//  - every call looks up the array's device address on the current device
//    with cudaGetSymbolAddress (no address is cached, so a call made after a
//    cudaDeviceReset, which may reload the module at another address, still
//    gets the right one). The first call on a device may load this module
//    onto that device: make that first call before any stream capture
//    begins on the device;
//  - the solver state (grid-reduction arrival counters included) must start
//    at zero. Each call writes a fresh state block over the array's header
//    on the caller's stream before its first kernel. The vectors need no
//    initial value: the initial residual kernel writes r, z and p before
//    anything reads them.
// ---------------------------------------------------------------------------
namespace {

constexpr i64 NOALLOC_MAX_N = 131072;

struct NoAllocHeader {
  CgState st;
  int bad;  // set by the index check
};
static_assert(sizeof(NoAllocHeader) <= 1024, "header region");

constexpr size_t NA_HEADER_WORDS = 1024 / sizeof(double);
constexpr size_t NA_PARTIAL_WORDS = PARTIAL_REGIONS * MAXG;
constexpr size_t NA_VEC_WORDS = (size_t)NOALLOC_MAX_N;
constexpr size_t NA_WORDS = NA_HEADER_WORDS + NA_PARTIAL_WORDS + 4 * NA_VEC_WORDS;

}  // namespace

// The scratch array. On the host this name only stands for the symbol; its
// device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_scratch[NA_WORDS];

namespace {

// Device address of the scratch array on the current device, looked up on
// every call: cheap once the module is loaded, allocates nothing, and never
// stale (a cached address would outlive a cudaDeviceReset).
double* noalloc_scratch() {
  void* a = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
  if (e != cudaSuccess) fail(FCU_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  if (!a) fail(FCU_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
  return static_cast<double*>(a);
}

// Same acceptance rule as the u32 -> i32 conversion of fcu_solve_csr_cg:
// row pointers at most nnz, column indices below n.
__global__ void k_noalloc_check(const uint32_t* __restrict__ rp, i64 n, const uint32_t* __restrict__ ci, i64 nnz,
                                int* __restrict__ bad) {
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t <= n; t += stride)
    if ((i64)rp[t] > nnz) atomicExch(bad, 1);
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nnz; t += stride)
    if ((i64)ci[t] >= n) atomicExch(bad, 1);
}

void require_device_ptr(const void* p, int dev, const char* what) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    fail(FCU_ERR_BAD_ARG, std::string(what) + ": not a device pointer (the no-alloc solver stages nothing)");
  }
  const bool dev_mem = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
  if (!dev_mem) fail(FCU_ERR_BAD_ARG, std::string(what) + ": not a device pointer (the no-alloc solver stages nothing)");
  if (a.type == cudaMemoryTypeDevice && a.device != dev)
    fail(FCU_ERR_BAD_ARG, std::string(what) + ": memory of another device");
}

template <int VPR>
void noalloc_chunk(cudaStream_t s, int g, int vg, const int* rp, const int* ci, const double* val, i64 n, double* x,
                   double* r, double* z, double* p, double* ap, const double* invd, CgState* st, double* partials) {
  for (int it = 0; it < CHUNK; ++it) {
    k_direction<double><<<vg, VBLOCK, 0, s>>>(n, p, z, st);
    k_spmv_ap<1, VPR, double><<<g, VBLOCK, 0, s>>>(rp, ci, val, n, p, ap, st, partials);
    k_update<double><<<vg, VBLOCK, 0, s>>>(n, x, r, p, ap, invd, z, st, partials, g);
  }
  CUDA_CHECK(cudaGetLastError());
}

template <int VPR>
void noalloc_init(cudaStream_t s, int g, const int* rp, const int* ci, const double* val, i64 n, const double* x,
                  const double* b, const double* invd, double* r, double* z, double* p, CgState* st,
                  double* partials) {
  k_init_residual<1, VPR, double><<<g, VBLOCK, 0, s>>>(rp, ci, val, n, x, b, invd, r, z, p, n, st, partials);
  CUDA_CHECK(cudaGetLastError());
}

}  // namespace

int run_pcg_noalloc(i64 n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* vals,
                    const double* inv_diag, const double* b, const double* x0, double rtol, i64 max_iter, double* x,
                    fcu_solve_info* info, void* stream) {
  const auto t0 = std::chrono::steady_clock::now();
  if (n <= 0) fail(FCU_ERR_BAD_ARG, "n must be positive");
  if (n > NOALLOC_MAX_N)
    fail(FCU_ERR_BAD_ARG, "n = " + std::to_string(n) + " exceeds the no-alloc solver's capacity of " +
                              std::to_string(NOALLOC_MAX_N) + " rows");
  if (max_iter < 0) fail(FCU_ERR_BAD_ARG, "max_iter must be non-negative");
  if (!row_ptr || !inv_diag || !b || !x) fail(FCU_ERR_BAD_ARG, "null CSR argument");
  int dev = 0;
  CUDA_CHECK(cudaGetDevice(&dev));
  require_device_ptr(row_ptr, dev, "row_ptr");
  require_device_ptr(inv_diag, dev, "inv_diag");
  require_device_ptr(b, dev, "b");
  require_device_ptr(x, dev, "x");
  if (x0) require_device_ptr(x0, dev, "x0");
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  uint32_t nnz32 = 0;
  CUDA_CHECK(cudaMemcpyAsync(&nnz32, row_ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CUDA_CHECK(cudaStreamSynchronize(s));
  const i64 nnz = nnz32;
  if (nnz >= (1ll << 31)) fail(FCU_ERR_UNSUPPORTED, "nnz exceeds 32-bit indexing");
  if (nnz > 0) {
    if (!col_idx || !vals) fail(FCU_ERR_BAD_ARG, "null CSR arrays");
    require_device_ptr(col_idx, dev, "col_idx");
    require_device_ptr(vals, dev, "vals");
  }

  double* base = noalloc_scratch();
  NoAllocHeader* hdr = reinterpret_cast<NoAllocHeader*>(base);
  double* partials = base + NA_HEADER_WORDS;
  double* r = partials + NA_PARTIAL_WORDS;
  double* z = r + NA_VEC_WORDS;
  double* p = z + NA_VEC_WORDS;
  double* ap = p + NA_VEC_WORDS;

  NoAllocHeader init{};
  init.st.tol = rtol;
  init.st.max_iter = max_iter;
  init.st.gpu_semantics = 1;
  init.st.delta = 0.1;
  CUDA_CHECK(cudaMemcpyAsync(hdr, &init, sizeof(init), cudaMemcpyHostToDevice, s));

  int num_sms = 0;
  CUDA_CHECK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  const i64 want = (n + VBLOCK - 1) / VBLOCK;
  const int g = (int)std::max<i64>(1, std::min<i64>(want, (i64)num_sms * blocks_per_sm()));
  const int vg = (int)std::max<i64>(1, std::min<i64>(want, (i64)num_sms * vec_blocks_per_sm()));
  if (g > MAXG || vg > MAXG) fail(FCU_ERR_UNSUPPORTED, "grid exceeds the reduction capacity");

  const int check_grid = (int)std::max<i64>(1, std::min<i64>((std::max(n + 1, nnz) + 255) / 256, (i64)num_sms * 8));
  k_noalloc_check<<<check_grid, 256, 0, s>>>(row_ptr, n, col_idx, nnz, &hdr->bad);
  CUDA_CHECK(cudaGetLastError());
  int bad = 0;
  CUDA_CHECK(cudaMemcpyAsync(&bad, &hdr->bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_CHECK(cudaStreamSynchronize(s));
  if (bad) fail(FCU_ERR_BAD_ARG, "CSR index out of range");
  // Every index is now known to be below 2^31, so the u32 arrays read as i32.
  const int* rp = reinterpret_cast<const int*>(row_ptr);
  const int* ci = reinterpret_cast<const int*>(col_idx);

  // CSR lanes per row by average row length (as for library matrices).
  const double avg = (double)nnz / (double)n;
  const int vpr = avg <= 6 ? 4 : avg <= 14 ? 8 : avg <= 40 ? 16 : 32;

  if (x0 && x0 != x) CUDA_CHECK(cudaMemcpyAsync(x, x0, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  else if (!x0) CUDA_CHECK(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  CgState* st = &hdr->st;
  switch (vpr) {
    case 4: noalloc_init<4>(s, g, rp, ci, vals, n, x, b, inv_diag, r, z, p, st, partials); break;
    case 8: noalloc_init<8>(s, g, rp, ci, vals, n, x, b, inv_diag, r, z, p, st, partials); break;
    case 16: noalloc_init<16>(s, g, rp, ci, vals, n, x, b, inv_diag, r, z, p, st, partials); break;
    default: noalloc_init<32>(s, g, rp, ci, vals, n, x, b, inv_diag, r, z, p, st, partials); break;
  }
  CgState hs{};
  CUDA_CHECK(cudaMemcpyAsync(&hs, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  CUDA_CHECK(cudaStreamSynchronize(s));
  const bool zero_rhs = hs.bnorm == 0.0;
  if (zero_rhs) {
    // gpu.rs:1169-1180: zero right-hand side -> zero solution, Ok
    CUDA_CHECK(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    hs.done = 1;
    hs.status = FCU_OK;
    hs.iter = 0;
  } else if (!hs.done && max_iter > 0) {
    for (i64 launched = 0; launched < max_iter + CHUNK; launched += CHUNK) {
      switch (vpr) {
        case 4: noalloc_chunk<4>(s, g, vg, rp, ci, vals, n, x, r, z, p, ap, inv_diag, st, partials); break;
        case 8: noalloc_chunk<8>(s, g, vg, rp, ci, vals, n, x, r, z, p, ap, inv_diag, st, partials); break;
        case 16: noalloc_chunk<16>(s, g, vg, rp, ci, vals, n, x, r, z, p, ap, inv_diag, st, partials); break;
        default: noalloc_chunk<32>(s, g, vg, rp, ci, vals, n, x, r, z, p, ap, inv_diag, st, partials); break;
      }
      CUDA_CHECK(cudaMemcpyAsync(&hs, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
      CUDA_CHECK(cudaStreamSynchronize(s));
      if (hs.done) break;
    }
  } else if (!hs.done) {
    hs.status = FCU_OK;  // zero iterations allowed: Ok at the limit (gpu.rs semantics)
  }
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (info) {
    info->iterations = hs.iter;
    info->outer_updates = hs.updates;
    info->residual = std::sqrt(std::max(hs.rr, 0.0));
    info->rel_residual = hs.bnorm > 0.0 ? info->residual / hs.bnorm : info->residual;
    info->kernel_ms = ms;
    // same algorithmic count as the library solver: matrix + SpMV vectors + update vectors
    const double bytes_iter = (double)nnz * 12.0 + 4.0 * (double)(n + 1) + 4.0 * n * 8.0 + 64.0 * n;
    info->effective_bw_gbps = ms > 0 ? bytes_iter * (double)hs.iter / (ms * 1e-3) / 1e9 : 0.0;
    info->status = hs.done ? hs.status : FCU_OK;
  }
  return hs.done ? hs.status : FCU_OK;
}
