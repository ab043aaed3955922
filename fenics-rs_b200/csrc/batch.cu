// Batched Jacobi-PCG over many independent systems (no reference
// counterpart; the batch of the scope table's multi-mesh case).
//
// The systems are the diagonal blocks of one block-diagonal matrix: meshes
// of uneven sizes are concatenated into one mesh (vertex ranges disjoint), so
// the library's pattern, assembly, load-vector and Dirichlet kernels build
// the whole batch in one pass each, and block i is rows [off[i], off[i+1]).
//
// One persistent launch solves the batch. Each thread-block cluster (1 to 8
// CTAs) takes the next instance from a queue ordered by estimated cost
// (largest first) and runs that instance's whole PCG: the cluster's CTAs own
// contiguous shares of its rows, phases are separated by cluster barriers,
// and every reduction sums the CTAs' partials through distributed shared
// memory in rank order, so instances converge, stop and report independently
// and no grid-wide synchronisation exists. The arithmetic per instance is
// that of the library's single-system PCG (cg.rs:40-149 for FP64; for mixed,
// FP32 difference-form operator with FP64 r, x and dots and FP64 residual
// replacement). The launch is captured in a CUDA graph together with the
// queue reset, and the graph is replayed on later solves. Lanes per row,
// threads per CTA and CTAs per cluster are picked by timing the candidates on
// the batch itself (first solve of a matrix and precision), unless
// FCU_BATCH_VPR / FCU_BATCH_THREADS / FCU_BATCH_CLUSTER fix them; a single
// system (the small-system path of the PCG) takes a shape fixed by rule.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include <cooperative_groups.h>

#include "internal.cuh"

namespace cg = cooperative_groups;

void build_rowsum32(fcu_matrix m);

namespace {

constexpr unsigned BFULL = 0xffffffffu;

__device__ __forceinline__ double bwarp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(BFULL, v, o);
  return v;
}

// Sum NV doubles over the cluster that owns the instance; every thread of
// every CTA of the cluster gets the totals. Each CTA reduces its threads in a
// fixed order and publishes its sum in a shared-memory slot; after the
// cluster barrier (release/acquire at cluster scope, so it also orders the
// CTAs' global-memory writes) every thread adds the slots in rank order. The
// slots alternate between two buffers: a CTA rewrites a buffer only after the
// next barrier, which every CTA reaches after reading it.
template <int NV, int BT>
__device__ __forceinline__ void cluster_sum(double (&v)[NV], double (*slots)[4], int& parity,
                                            cg::cluster_group& cl) {
  __shared__ double sh[NV][BT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    const double x = bwarp_sum(v[j]);
    if (lane == 0) sh[j][w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double t = 0.0;
      for (int q = 0; q < BT / 32; ++q) t += sh[j][q];
      slots[parity][j] = t;
    }
  }
  cl.sync();
  const unsigned nr = cl.num_blocks();
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = 0.0;
  for (unsigned k = 0; k < nr; ++k) {
    const double* rs = cl.map_shared_rank(&slots[parity][0], k);
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] += rs[j];
  }
  parity ^= 1;
}

// One CSR row with VPR >= 2 lanes (all lanes of the warp call it). DIFF: the
// mixed operator y_i = sum_{j != i} a_ij (x_j - x_i) + S_i x_i, with S_i in
// the diagonal slot; otherwise y_i = sum_j a_ij x_j.
template <int VPR, bool DIFF, class T, class GV>
__device__ __forceinline__ T batch_row(const int* __restrict__ rp, const int* __restrict__ ci,
                                       const T* __restrict__ val, i64 row, bool valid, int sub, const GV& xv) {
  T s = T(0);
  if (valid) {
    const int b = rp[row], e = rp[row + 1];
    const T xi = DIFF ? xv(row) : T(0);
    for (int q = b + sub; q < e; q += VPR) {
      const int c = ci[q];
      if (DIFF) s += val[q] * (c == (int)row ? xi : xv(c) - xi);
      else s += val[q] * xv(c);
    }
  }
#pragma unroll
  for (int o = VPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(BFULL, s, o);
  return s;
}

// One CSR row per thread (VPR = 1): a block of entries (eight for FP32,
// four for FP64, to stay within the register budget) is loaded, values and
// columns, then all its operand entries, before the arithmetic. Entries are
// summed in CSR order; unused slots read row 0's operand with weight 0.
template <bool DIFF, class T, class GV>
__device__ __forceinline__ T batch_row1(int a0, int a1, const int* __restrict__ ci, const T* __restrict__ val, i64 row,
                                        const GV& xv) {
  constexpr int E = sizeof(T) == 4 ? 8 : 4;
  const T xa = DIFF ? xv(row) : T(0);
  T s = T(0);
  for (int k0 = a0; k0 < a1; k0 += E) {
    const int na = a1 - k0;
    int c[E];
    T wv[E], g[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const bool h = k < na;
      c[k] = h ? ci[k0 + k] : 0;
      wv[k] = h ? val[k0 + k] : T(0);
    }
#pragma unroll
    for (int k = 0; k < E; ++k) g[k] = xv(c[k]);
#pragma unroll
    for (int k = 0; k < E; ++k) {
      if (DIFF) s += wv[k] * (c[k] == (int)row ? xa : g[k] - xa);
      else s += wv[k] * g[k];
    }
  }
  return s;
}

struct BatchArgs {
  const int* rp;
  const int* ci;
  const double* val64;
  const float* val32;
  const i64* off;    // nb + 1 row offsets
  const int* order;  // instances, largest first
  int nb;
  const double* b;
  double* x;
  double* r;
  const double* invd;
  void* z;   // T
  void* p;   // T
  void* ap;  // T
  void* p2;  // T: the second direction buffer (p alternates between p and p2)
  double tol;
  i64 max_iter;
  double delta;
  unsigned* counter;  // queue head (zeroed before every launch)
  i64* iters;
  i64* updates;
  double* relres;
  double* resid;  // absolute residual ||r|| per instance
  int* status;
};

// Operator rows [c0, c1) of this CTA: y = A v; emit(row, y) once per row.
template <int VPR, int BT, bool DIFF, class T, class GV, class Emit>
__device__ __forceinline__ void batch_spmv(const int* __restrict__ rp, const int* __restrict__ ci,
                                           const T* __restrict__ val, i64 c0, i64 c1, const GV& v, Emit emit) {
  const int tid = threadIdx.x;
  if (VPR == 1) {
    // the next row's bounds are fetched while this row is summed
    i64 row = c0 + tid;
    int a0 = 0, a1 = 0;
    if (row < c1) {
      a0 = rp[row];
      a1 = rp[row + 1];
    }
    for (; row < c1; row += BT) {
      const i64 nxt = row + BT;
      int n0 = 0, n1 = 0;
      if (nxt < c1) {
        n0 = rp[nxt];
        n1 = rp[nxt + 1];
      }
      emit(row, batch_row1<DIFF, T>(a0, a1, ci, val, row, v));
      a0 = n0;
      a1 = n1;
    }
  } else {
    constexpr int G = BT / VPR;
    const int g = tid / VPR, sub = tid % VPR;
    for (i64 base = c0; base < c1; base += G) {
      const i64 row = base + g;
      const bool valid = row < c1;
      const T s = batch_row<VPR, DIFF, T>(rp, ci, val, row, valid, sub, v);
      if (valid && sub == 0) emit(row, s);
    }
  }
}

// Operand gathers of the batched SpMV: a plain vector, or the new direction
// p = z + beta p_old formed on the fly from the previous iteration's z and
// p_old (one fused multiply-add, as the direction update rounds it), so no
// cluster barrier is needed between forming p and reading it.
template <class T>
struct BatchPlain {
  const T* v;
  __device__ __forceinline__ T operator()(i64 i) const { return v[i]; }
};
template <class T>
struct BatchDirection {
  const T* z;
  const T* pold;
  T beta;
  __device__ __forceinline__ T operator()(i64 i) const { return fma(beta, pold[i], z[i]); }
};

// A cluster of CTAs (1 to 8; the launch's cluster size) solves one instance
// at a time: CTA rank k owns rows [r0 + k len / CL, r0 + (k + 1) len / CL)
// for every phase, and the phases are separated by cluster barriers.
// FD: the direction p = z + beta p_old is formed where the SpMV reads it,
// with p alternating between two buffers (no direction phase and no cluster
// barrier before the SpMV, at the cost of gathering z and p_old); otherwise
// a direction phase writes p in place and a cluster barrier follows it. Both
// round p with one fused multiply-add, so the iterates are the same.
template <int VPR, int BT, class T, bool FD>
__global__ void __launch_bounds__(BT, 1024 / BT) k_batch_pcg(BatchArgs a) {
  constexpr bool MIXED = sizeof(T) == 4;
  __shared__ int s_q;
  __shared__ double slots[2][4];
  cg::cluster_group cl = cg::this_cluster();
  const unsigned ncl = cl.num_blocks(), rank = cl.block_rank();
  int parity = 0;
  // the parameter block's address is never taken (no local copy of it)
  T* const z = static_cast<T*>(a.z);
  T* const pa = static_cast<T*>(a.p);
  T* const pb = static_cast<T*>(a.p2);
  T* const ap = static_cast<T*>(a.ap);
  const int tid = threadIdx.x;

  for (;;) {
    if (rank == 0 && tid == 0) s_q = (int)atomicAdd(a.counter, 1u);
    cl.sync();
    const int q = *cl.map_shared_rank(&s_q, 0);
    cl.sync();
    if (q >= a.nb) break;
    const int inst = a.order[q];
    const i64 r0 = a.off[inst], r1 = a.off[inst + 1];
    // rank k owns len / ncl rows, one more for the first len % ncl ranks
    // (32-bit arithmetic: rows are int32-indexed)
    const unsigned len = (unsigned)(r1 - r0);
    const unsigned share = len / ncl, extra = len % ncl;
    const i64 c0 = r0 + (i64)(share * rank + min(rank, extra));
    const i64 c1 = c0 + (i64)(share + (rank < extra ? 1u : 0u));

    // x0 = 0: r = b, z = D^-1 r, p = 0; r.z, r.r, b.b (cg.rs:79-90)
    double v3[3] = {0.0, 0.0, 0.0};
    for (i64 i = c0 + tid; i < c1; i += BT) {
      a.x[i] = 0.0;
      const double ri = a.b[i];
      a.r[i] = ri;
      const double zi = ri * a.invd[i];
      z[i] = (T)zi;
      pa[i] = T(0);
      v3[0] += ri * zi;
      v3[1] += ri * ri;
    }
    v3[2] = v3[1];
    cluster_sum<3, BT>(v3, slots, parity, cl);
    double rz = v3[0], rr = v3[1];
    const double bnorm = sqrt(v3[2]);
    double maxr = sqrt(rr);
    double beta = 0.0;
    i64 iter = 0, updates = 0;
    int status = FCU_ERR_NO_CONVERGENCE;
    [[maybe_unused]] int flip = 0;  // FD: p_old is pa when 0, pb when 1
    {
      const double r0n = sqrt(rr);
      if (r0n < a.tol || (bnorm > 0.0 && r0n / bnorm < a.tol)) status = FCU_OK;
    }
    while (status != FCU_OK && iter < a.max_iter) {
      const T* const vals = MIXED ? reinterpret_cast<const T*>(a.val32) : reinterpret_cast<const T*>(a.val64);
      double v1[1] = {0.0};
      T* p;
      if constexpr (FD) {
        // Ap and p.Ap with p = z + beta p_old formed where it is read; each
        // row's p is stored for the update and the next iteration
        const BatchDirection<T> dir{z, flip ? pb : pa, (T)beta};
        p = flip ? pa : pb;
        flip ^= 1;
        batch_spmv<VPR, BT, MIXED, T>(a.rp, a.ci, vals, c0, c1, dir, [&v1, ap, p, &dir](i64 row, T s) {
          const T pr = dir(row);
          p[row] = pr;
          ap[row] = s;
          v1[0] += (double)pr * (double)s;
        });
      } else {
        // direction, then Ap and p.Ap
        p = pa;
        const T bt = (T)beta;
        for (i64 i = c0 + tid; i < c1; i += 4 * BT) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const i64 k = i + u * BT;
            if (k < c1) p[k] = fma(bt, p[k], z[k]);
          }
        }
        cl.sync();
        batch_spmv<VPR, BT, MIXED, T>(a.rp, a.ci, vals, c0, c1, BatchPlain<T>{p}, [&v1, ap, p](i64 row, T s) {
          ap[row] = s;
          v1[0] += (double)p[row] * (double)s;
        });
      }
      cluster_sum<1, BT>(v1, slots, parity, cl);
      if (fabs(v1[0]) < 1e-30) {  // cg.rs:102-107
        iter += 1;
        status = FCU_ERR_BREAKDOWN;
        break;
      }
      const double alpha = rz / v1[0];
      // x += alpha p, r -= alpha Ap, z = D^-1 r
      double v2[2] = {0.0, 0.0};
      for (i64 i = c0 + tid; i < c1; i += 2 * BT) {
        double xi[2], ri[2], di[2];
        T pi[2], api[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const i64 k = i + u * BT;
          if (k < c1) {
            xi[u] = a.x[k];
            ri[u] = a.r[k];
            di[u] = a.invd[k];
            pi[u] = p[k];
            api[u] = ap[k];
          }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const i64 k = i + u * BT;
          if (k < c1) {
            a.x[k] = xi[u] + alpha * (double)pi[u];
            const double rn = ri[u] - alpha * (double)api[u];
            a.r[k] = rn;
            const double zi = rn * di[u];
            z[k] = (T)zi;
            v2[0] += rn * zi;
            v2[1] += rn * rn;
          }
        }
      }
      cluster_sum<2, BT>(v2, slots, parity, cl);
      iter += 1;
      rr = v2[1];
      const double res = sqrt(v2[1]);
      const double rel = bnorm > 0.0 ? res / bnorm : res;
      if (!MIXED) {
        if (rel < a.tol) {
          status = FCU_OK;
          break;
        }
        beta = v2[0] / rz;
        rz = v2[0];
        continue;
      }
      if (!(rel < a.tol || res < a.delta * maxr)) {
        beta = v2[0] / rz;
        rz = v2[0];
        continue;
      }
      // residual replacement with the FP64 matrix: r = b - A64 x, z = D^-1 r
      // (x of the whole instance is complete since the cluster sum above)
      double v4[2] = {0.0, 0.0};
      batch_spmv<VPR, BT, false, double>(a.rp, a.ci, a.val64, c0, c1, BatchPlain<double>{a.x},
                                         [&v4, z, rv = a.r, bv = a.b, dv = a.invd](i64 row, double s) {
                                           const double rn = bv[row] - s;
                                           rv[row] = rn;
                                           const double zi = rn * dv[row];
                                           z[row] = (T)zi;
                                           v4[0] += rn * zi;
                                           v4[1] += rn * rn;
                                         });
      cluster_sum<2, BT>(v4, slots, parity, cl);
      updates += 1;
      rr = v4[1];
      const double res2 = sqrt(v4[1]);
      const double rel2 = bnorm > 0.0 ? res2 / bnorm : res2;
      if (rel2 < a.tol) {
        status = FCU_OK;
        break;
      }
      maxr = res2;
      beta = v4[0] / rz;
      rz = v4[0];
    }
    if (rank == 0 && tid == 0) {
      a.iters[inst] = iter;
      a.updates[inst] = updates;
      a.relres[inst] = bnorm > 0.0 ? sqrt(rr) / bnorm : sqrt(rr);
      a.resid[inst] = sqrt(rr);
      a.status[inst] = status;
    }
  }
}

// D^-1 from the diagonal slots (cg.rs:52-64: 1 when |a_kk| <= 1e-15).
__global__ void k_batch_invd(const int* __restrict__ diag_pos, const double* __restrict__ val, i64 n,
                             double* __restrict__ invd) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const int dp = diag_pos[i];
    const double d = dp >= 0 ? val[dp] : 0.0;
    invd[i] = fabs(d) > 1e-15 ? 1.0 / d : 1.0;
  }
}

// Every row of block i must only reference columns of block i.
__global__ void k_batch_check(const int* __restrict__ rp, const int* __restrict__ ci, const i64* __restrict__ off,
                              int nb, int* __restrict__ bad) {
  const int inst = blockIdx.x;
  if (inst >= nb) return;
  const i64 r0 = off[inst], r1 = off[inst + 1];
  for (i64 row = r0 + threadIdx.x; row < r1; row += blockDim.x)
    for (int q = rp[row]; q < rp[row + 1]; ++q)
      if (ci[q] < r0 || ci[q] >= r1) atomicExch(bad, 1);
}

struct BatchConfig {
  int vpr = 1;
  int threads = 1024;
  int cluster = 1;
};

using BatchKernel = void (*)(BatchArgs);

template <class T>
BatchKernel batch_kernel(int vpr, int threads, bool fd) {
#define FCU_BATCH_CASE(V, B) \
  if (vpr == V && threads == B) return fd ? k_batch_pcg<V, B, T, true> : k_batch_pcg<V, B, T, false>;
  FCU_BATCH_CASE(1, 512) FCU_BATCH_CASE(1, 1024)
  FCU_BATCH_CASE(2, 512) FCU_BATCH_CASE(2, 1024)
  FCU_BATCH_CASE(4, 512) FCU_BATCH_CASE(4, 1024)
#undef FCU_BATCH_CASE
  return nullptr;
}

}  // namespace

// Per-matrix state of the batched solver: the instance layout, work buffers,
// the tuned configuration and the instantiated graph, per precision.
struct BatchWorkspace {
  int nb = 0;
  std::vector<i64> off;  // host copy of the offsets
  DBuf<i64> off_d;
  DBuf<int> order;
  DBuf<double> b, x, r, invd;
  DBuf<double> z64, p64, q64, ap64;  // q: the second direction buffer
  DBuf<float> z32, p32, q32, ap32;
  DBuf<unsigned> counter;
  DBuf<i64> iters, updates;
  DBuf<double> relres, resid;
  DBuf<int> status;
  BatchConfig cfg[2];
  bool tuned[2] = {false, false};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_key[2] = {-1, -1};  // configuration of the captured launch
  double tol_g[2] = {0.0, 0.0};
  i64 iters_g[2] = {0, 0};
  ~BatchWorkspace() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
  }
};

void destroy_batch_ws(BatchWorkspace* w) { delete w; }

namespace {

int env_int(const char* name, int dflt) {
  const char* e = getenv(name);
  return e ? atoi(e) : dflt;
}

BatchArgs make_args(fcu_matrix m, BatchWorkspace* w, bool mixed, double tol, i64 max_iter) {
  BatchArgs a;
  a.rp = m->row_ptr;
  a.ci = m->col_idx;
  a.val64 = m->val64.p;
  a.val32 = m->val32.p;
  a.off = w->off_d.p;
  a.order = w->order.p;
  a.nb = w->nb;
  a.b = w->b.p;
  a.x = w->x.p;
  a.r = w->r.p;
  a.invd = w->invd.p;
  a.z = mixed ? (void*)w->z32.p : (void*)w->z64.p;
  a.p = mixed ? (void*)w->p32.p : (void*)w->p64.p;
  a.p2 = mixed ? (void*)w->q32.p : (void*)w->q64.p;
  a.ap = mixed ? (void*)w->ap32.p : (void*)w->ap64.p;
  a.tol = tol;
  a.max_iter = max_iter;
  a.delta = 0.1;
  a.counter = w->counter.p;
  a.iters = w->iters.p;
  a.updates = w->updates.p;
  a.relres = w->relres.p;
  a.resid = w->resid.p;
  a.status = w->status.p;
  return a;
}

// Directions formed in the SpMV (FD) for FP64 and for single-instance
// launches (the small-system path), where the saved cluster barrier pays;
// mixed batches keep the direction phase (on the 256-problem batch the extra
// gathers cost more than the barrier: 108.9 against 106.7 ms, while FP64 went
// from 144.7 to 138.6 ms and single systems of 4k-16k rows gained 9-14%).
bool fused_direction(bool mixed, int nb) { return !mixed || nb == 1; }

BatchKernel pick_kernel(bool mixed, const BatchConfig& c, int nb) {
  const bool fd = fused_direction(mixed, nb);
  return mixed ? batch_kernel<float>(c.vpr, c.threads, fd) : batch_kernel<double>(c.vpr, c.threads, fd);
}

// Persistent grid: as many clusters as fit on the device at once (at most
// one per instance). 0 when the configuration cannot be placed.
int batch_grid(fcu_ctx ctx, BatchKernel k, const BatchConfig& c, int nb) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(c.cluster * std::max(1, std::min(nb, ctx->num_sms))));
  cfg.blockDim = dim3((unsigned)c.threads);
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)c.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nclusters = 0;
  if (cudaOccupancyMaxActiveClusters(&nclusters, k, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c.cluster * std::min(nb, nclusters);
}

void launch_batch(fcu_ctx ctx, BatchWorkspace* w, BatchKernel k, const BatchConfig& c, int grid,
                  const BatchArgs& a) {
  CUDA_CHECK(cudaMemsetAsync(w->counter.p, 0, sizeof(unsigned), ctx->stream));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)c.threads);
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)c.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, k, a));
}

// Time each candidate (lanes per row x threads per CTA x CTAs per cluster) on
// the batch itself with a short iteration cap and keep the fastest.
BatchConfig autotune(fcu_matrix m, BatchWorkspace* w, bool mixed, double tol) {
  BatchConfig fixed;
  fixed.vpr = env_int("FCU_BATCH_VPR", 0);
  fixed.threads = env_int("FCU_BATCH_THREADS", 0);
  fixed.cluster = env_int("FCU_BATCH_CLUSTER", 0);
  if (fixed.vpr && fixed.threads && fixed.cluster && pick_kernel(mixed, fixed, w->nb) &&
      batch_grid(m->ctx, pick_kernel(mixed, fixed, w->nb), fixed, w->nb) > 0)
    return fixed;
  fcu_ctx ctx = m->ctx;
  const int vprs[3] = {1, 2, 4};
  const int thr[2] = {512, 1024};
  const int cls[4] = {1, 2, 4, 8};
  BatchConfig best;
  float best_ms = 1e30f;
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  const BatchArgs a = make_args(m, w, mixed, tol, 24);
  for (int v : vprs)
    for (int t : thr)
      for (int cs : cls) {
        BatchConfig c;
        c.vpr = v;
        c.threads = t;
        c.cluster = cs;
        BatchKernel k = pick_kernel(mixed, c, w->nb);
        if (!k) continue;
        const int grid = batch_grid(ctx, k, c, w->nb);
        if (grid <= 0) continue;
        launch_batch(ctx, w, k, c, grid, a);  // warm
        CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
        launch_batch(ctx, w, k, c, grid, a);
        CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
        CUDA_CHECK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
          best_ms = ms;
          best = c;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_ms >= 1e30f) fail(FCU_ERR_UNSUPPORTED, "no batched PCG configuration fits this device");
  return best;
}

}  // namespace

// Batched PCG driver; b, x and the per-instance outputs are device or host
// buffers handled by the caller (api.cu) through staging.
int batch_pcg_impl(fcu_matrix m, i64 nb, const i64* offsets_host, const double* b_dev, double* x_dev, double tol,
                   i64 max_iter, int precision, i64* iters_host, double* relres_host, int* status_host,
                   fcu_solve_info* info, const int* fixed_shape) {
  fcu_ctx ctx = m->ctx;
  const bool mixed = precision == FCU_MIXED;
  if (m->bs != 1) fail(FCU_ERR_UNSUPPORTED, "batched PCG takes scalar (CSR) matrices");
  if (!m->has_values) fail(FCU_ERR_BAD_ARG, "matrix has no values");
  if (mixed && !m->val32.p) fail(FCU_ERR_BAD_ARG, "matrix has no FP32 copy");
  if (nb <= 0 || nb > (1 << 30)) fail(FCU_ERR_BAD_ARG, "bad instance count");
  if (offsets_host[0] != 0 || offsets_host[nb] != m->n) fail(FCU_ERR_BAD_ARG, "offsets must span the matrix rows");
  for (i64 i = 0; i < nb; ++i)
    if (offsets_host[i + 1] < offsets_host[i]) fail(FCU_ERR_BAD_ARG, "offsets must not decrease");
  if (max_iter < 0) fail(FCU_ERR_BAD_ARG, "max_iter must be non-negative");

  BatchWorkspace*& w = m->bws;
  const bool same = w && w->nb == nb && std::equal(w->off.begin(), w->off.end(), offsets_host);
  if (!same) {
    delete w;
    w = new BatchWorkspace();
    w->nb = (int)nb;
    w->off.assign(offsets_host, offsets_host + nb + 1);
    upload(ctx, w->off_d, w->off.data(), nb + 1);
    DBuf<int> bad;
    bad.alloc(1);
    CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
    k_batch_check<<<(unsigned)nb, 256, 0, ctx->stream>>>(m->row_ptr, m->col_idx, w->off_d.p, (int)nb, bad.p);
    LAUNCH_CHECK(ctx);
    int hbad = 0;
    download(ctx, &hbad, bad.p, 1);
    if (hbad) fail(FCU_ERR_BAD_ARG, "matrix is not block diagonal over the given offsets");
    // queue order: estimated cost (stored entries x sqrt(rows), the 2D
    // iteration growth), largest first
    std::vector<int> hrp(nb + 1);
    std::vector<int> rpv(m->n + 1);
    download(ctx, rpv.data(), m->row_ptr, m->n + 1);
    std::vector<double> cost(nb);
    for (i64 i = 0; i < nb; ++i) {
      const double rows = (double)(offsets_host[i + 1] - offsets_host[i]);
      const double nnz = (double)(rpv[offsets_host[i + 1]] - rpv[offsets_host[i]]);
      cost[i] = (nnz + rows) * std::sqrt(std::max(rows, 1.0));
    }
    std::vector<int> ord(nb);
    for (i64 i = 0; i < nb; ++i) ord[i] = (int)i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    upload(ctx, w->order, ord.data(), nb);
    const i64 n = m->n;
    w->b.alloc(n);
    w->x.alloc(n);
    w->r.alloc(n);
    w->invd.alloc(n);
    w->counter.alloc(1);
    w->iters.alloc(nb);
    w->updates.alloc(nb);
    w->relres.alloc(nb);
    w->resid.alloc(nb);
    w->status.alloc(nb);
  }
  const i64 n = m->n;
  if (mixed && !w->z32.p) {
    w->z32.alloc(n);
    w->p32.alloc(n);
    w->q32.alloc(n);
    w->ap32.alloc(n);
  }
  if (!mixed && !w->z64.p) {
    w->z64.alloc(n);
    w->p64.alloc(n);
    w->q64.alloc(n);
    w->ap64.alloc(n);
  }
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
  k_batch_invd<<<grid_for(n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(m->diag_pos, m->val64.p, n, w->invd.p);
  LAUNCH_CHECK(ctx);
  if (mixed) build_rowsum32(m);
  CUDA_CHECK(cudaMemcpyAsync(w->b.p, b_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  const int k = mixed ? 1 : 0;
  if (!w->tuned[k]) {
    if (fixed_shape) {
      w->cfg[k].vpr = fixed_shape[0];
      w->cfg[k].threads = fixed_shape[1];
      w->cfg[k].cluster = fixed_shape[2];
      if (!pick_kernel(mixed, w->cfg[k], w->nb)) fail(FCU_ERR_BAD_ARG, "no batched PCG kernel of that shape");
    } else {
      w->cfg[k] = autotune(m, w, mixed, tol);
    }
    w->tuned[k] = true;
  }
  const BatchConfig c = w->cfg[k];
  BatchKernel kern = pick_kernel(mixed, c, w->nb);
  const int key = (c.vpr * 4096 + c.threads) * 16 + c.cluster;
  if (!w->graph[k] || w->graph_key[k] != key || w->tol_g[k] != tol || w->iters_g[k] != max_iter) {
    if (w->graph[k]) {
      cudaGraphExecDestroy(w->graph[k]);
      w->graph[k] = nullptr;
    }
    const BatchArgs a = make_args(m, w, mixed, tol, max_iter);
    cudaGraph_t g;
    CUDA_CHECK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int grid = batch_grid(ctx, kern, c, w->nb);
    if (grid <= 0) fail(FCU_ERR_UNSUPPORTED, "batched PCG configuration does not fit this device");
    try {
      launch_batch(ctx, w, kern, c, grid, a);
    } catch (...) {
      cudaStreamEndCapture(ctx->stream, &g);
      throw;
    }
    CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &g));
    CUDA_CHECK(cudaGraphInstantiate(&w->graph[k], g, 0));
    cudaGraphDestroy(g);
    w->graph_key[k] = key;
    w->tol_g[k] = tol;
    w->iters_g[k] = max_iter;
  }
  CUDA_CHECK(cudaGraphLaunch(w->graph[k], ctx->stream));
  ctx->launches += 1;
  CUDA_CHECK(cudaMemcpyAsync(x_dev, w->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
  CUDA_CHECK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::vector<i64> it(nb), up(nb);
  std::vector<double> rel(nb), res(nb);
  std::vector<int> st(nb);
  download(ctx, it.data(), w->iters.p, nb);
  download(ctx, up.data(), w->updates.p, nb);
  download(ctx, rel.data(), w->relres.p, nb);
  download(ctx, res.data(), w->resid.p, nb);
  download(ctx, st.data(), w->status.p, nb);
  if (iters_host) std::copy(it.begin(), it.end(), iters_host);
  if (relres_host) std::copy(rel.begin(), rel.end(), relres_host);
  if (status_host) std::copy(st.begin(), st.end(), status_host);
  int worst = FCU_OK;
  i64 max_it = 0, sum_it = 0, sum_up = 0;
  double max_rel = 0.0, max_res = 0.0;
  double bytes = 0.0;
  const double w8 = mixed ? 4.0 : 8.0;
  for (i64 i = 0; i < nb; ++i) {
    if (st[i] != FCU_OK && worst == FCU_OK) worst = st[i];
    max_it = std::max(max_it, it[i]);
    sum_it += it[i];
    sum_up += up[i];
    max_rel = std::max(max_rel, rel[i]);
    max_res = std::max(max_res, res[i]);
    // per iteration: values + columns + row pointers, then the vector passes
    // (direction 3w, SpMV p and Ap 2w, update 40 + 3w bytes per row)
    const double rows = (double)(offsets_host[i + 1] - offsets_host[i]);
    bytes += (double)it[i] * (rows * (8.0 * w8 + 44.0));
  }
  if (info) {
    info->iterations = max_it;
    info->outer_updates = sum_up;
    info->residual = max_res;
    info->rel_residual = max_rel;
    info->kernel_ms = ms;
    info->effective_bw_gbps = ms > 0 ? bytes / (ms * 1e-3) / 1e9 : 0.0;
    info->status = worst;
  }
  (void)sum_it;
  return worst;
}

void batch_config(fcu_matrix m, int precision, int* vpr, int* threads, int* cluster) {
  const int k = precision == FCU_MIXED ? 1 : 0;
  if (!m->bws || !m->bws->tuned[k]) {
    *vpr = *threads = *cluster = 0;
    return;
  }
  *vpr = m->bws->cfg[k].vpr;
  *threads = m->bws->cfg[k].threads;
  *cluster = m->bws->cfg[k].cluster;
}
