// Internal types of the fenics_cuda library: handles, device buffers, error
// plumbing and small device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "../../include/fenics_cuda.h"

typedef int64_t i64;

// ---------------------------------------------------------------------------
// Errors: every internal routine throws FcuError; the C ABI layer converts it
// into a status code and the context's last-error string.
// ---------------------------------------------------------------------------

struct FcuError {
  int code;
  std::string msg;
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw FcuError{code, msg}; }

#define CUDA_CHECK(expr)                                                                        \
  do {                                                                                          \
    cudaError_t e_ = (expr);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      fail(FCU_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_) + " at " __FILE__); \
  } while (0)

// ---------------------------------------------------------------------------
// Device buffer (RAII, stream-ordered allocation on the context stream)
// ---------------------------------------------------------------------------

// The stream library allocations are ordered on: the calling context's
// stream for the duration of a C-ABI call (set by the call wrapper).
inline cudaStream_t& fcu_alloc_stream() {
  static thread_local cudaStream_t s = nullptr;
  return s;
}

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;  // stream the allocation and its release are ordered on
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    if (count) {
      s = fcu_alloc_stream();
      // 16 extra bytes so vector loads that round a range outward stay inside.
      cudaError_t e = cudaMallocAsync((void**)&p, count * sizeof(T) + 16, s);
      if (e != cudaSuccess) {
        p = nullptr;
        fail(FCU_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
      }
    }
    n = count;
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------------------
// Handles
// ---------------------------------------------------------------------------

struct Workspace;       // solver state, defined in solver.cu
struct BatchWorkspace;  // batched solver state, defined in batch.cu
void destroy_batch_ws(BatchWorkspace* w);

// Handles are reference counted: a mesh holds its context, a space its mesh,
// a matrix its space and context. fcu_*_destroy drops the caller's reference,
// so handles may be destroyed in any order.
struct fcu_ctx_s {
  int refs = 1;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  i64 launches = 0;          // kernels launched by this library on this context
  DBuf<unsigned char> temp;  // reusable scratch (CUB temporary storage)
  int num_sms = 148;
  // SpMV shapes the PCG tuner picked, by matrix shape (block size, rows,
  // stored blocks, longest row, precision): a later matrix of the same shape
  // (a new solve on the same mesh) takes them without timing candidates.
  std::map<std::array<i64, 5>, std::array<int, 2>> spmv_tune;
  // Pinned solver state records of released matrices, reused by later ones
  // (pinned allocation and release are slow and synchronising), freed with
  // the context.
  std::vector<void*> pinned_pool;
  unsigned char* temp_bytes(size_t b) {
    if (temp.n < b) temp.alloc(b);
    return temp.p;
  }
};

struct fcu_mesh_s {
  int refs = 1;
  fcu_ctx ctx = nullptr;
  int dim = 0, nodes = 0;
  i64 nv = 0, nc = 0;
  DBuf<double> coords;    // nv*dim, AoS as the reference stores Vec<[f64;DIM]>
  DBuf<int> cells;        // nc*nodes, int32
  DBuf<unsigned char> valid;  // 1 if |det J| >= 1e-14
  i64 n_degenerate = -1;
};

// Sparsity pattern at node level (node = dof for scalar spaces, vertex for
// the vector space whose 3x3 blocks are stored contiguously) plus the
// row-gather structures the assembly kernels read.
struct fcu_space_s {
  int refs = 1;
  fcu_ctx ctx = nullptr;
  fcu_mesh mesh = nullptr;
  int kind = 0;
  int k = 0;        // nodes per cell (3, 4, 10)
  int bs = 1;       // dofs per node (1 or 3)
  i64 nnodes = 0;   // rows of the node pattern
  i64 ndofs = 0;
  i64 nedges = 0;   // P2 only
  i64 nnzb = 0;     // stored node-pattern entries (diagonals always present)
  i64 nnz_ref = 0;  // entries of the raw reference pattern (scalar)
  int max_row = 0;  // longest node row
  int max_contrib = 0;
  DBuf<int> cell_nodes;    // nc*k  (P1: the mesh cells; P2: vertex + edge dofs)
  DBuf<int> edge_verts;    // P2: nedges*2
  DBuf<int> row_ptr;       // nnodes+1
  DBuf<int> col_idx;       // nnzb
  DBuf<int> diag_pos;      // nnodes: position of (i,i)
  DBuf<int> contrib_ptr;   // nnodes+1
  DBuf<int> contrib;       // (cell << 4) | local, sorted by cell within a row
  DBuf<unsigned short> slot_cnt;   // nnzb: contributions to each slot
  DBuf<unsigned short> slot_ent;   // k*ncontrib: (t_local << 4) | b, per slot in cell order
  DBuf<int> tpos;          // nnzb: position of the transposed entry (built on demand)
  DBuf<double> cell_vol;   // nc: |det J| / 6 per tet (built by the first vertex average)
  // Vector P1: the upper off-diagonal blocks (i, j), j > i, as a flat list.
  // Block u sits at slot up_slot[u], its transpose at up_tslot[u]; the cells
  // that couple i and j are up_ent[up_ptr[u] .. up_ptr[u+1]), each packed as
  // (cell << 4) | (a << 2) | b with a, b the local indices of i and j, in
  // ascending cell order.
  i64 nup = 0;
  DBuf<int> up_ptr, up_slot, up_tslot;
  DBuf<unsigned> up_ent;
  DBuf<double> cell_rec;   // vector P1: per-cell gradient records (16 doubles each)
  // Vector P1: for every stored off-diagonal block (i, j) in CSR order, the
  // cells that couple i and j, packed as up_ent is, at sl_ent[sl_ptr[p] ..
  // sl_ptr[p+1]) (diagonal slots have empty lists).
  DBuf<int> sl_ptr;
  DBuf<unsigned> sl_ent;
  // P2 scalar: for contribution t of a row (position in `contrib_a`) and local
  // column b, the slot of dof cell_nodes[cell][b] within the row, as an
  // offset from the row's first slot (rows of at most 255 slots; empty when
  // a longer row exists).
  DBuf<unsigned char> cmap;
  // P2 scalar: the row's contributions ordered by (local index, cell); cmap
  // follows this order when contrib_a is present.
  DBuf<int> contrib_a;
};

struct fcu_matrix_s {
  int refs = 1;
  fcu_ctx ctx = nullptr;
  fcu_space space = nullptr;   // nullptr for a wrapped CSC/CSR
  i64 n = 0;                   // scalar order
  i64 nnodes = 0;              // block rows (== n when bs == 1)
  int bs = 1;
  i64 nnzb = 0;
  // Pattern (owned copies for wrapped matrices, else the space's arrays).
  const int* row_ptr = nullptr;
  const int* col_idx = nullptr;
  const int* diag_pos = nullptr;
  DBuf<int> own_row_ptr, own_col_idx, own_diag_pos;
  bool wrapped_general = false;  // wrapped CSC (export needs the stored layout)
  DBuf<double> val64;   // nnzb*bs*bs
  DBuf<float> val32;
  DBuf<unsigned char> dirichlet;  // n: 1 if eliminated (empty when no BC applied)
  i64 n_dirichlet = 0;
  DBuf<double> diag_count;        // n: diagonal value for eliminated dofs
  bool bc_applied = false;
  bool drop_zeros = false;  // folded (eigen.rs:55-79): export omits zero-valued entries
  bool comp_diag = false;   // vector mass (mass.rs:118-123): only same-component entries are in the pattern
  bool has_values = false;
  DBuf<unsigned char> diag_struct;  // node rows whose diagonal is in the raw pattern
  DBuf<i64> csc_colptr, csc_rowidx; // wrapped CSC: the caller's layout, for export
  DBuf<int> csr_of;                 // wrapped CSC: CSC position -> CSR slot
  // 3x3 block-Jacobi preconditioner (inverse diagonal blocks, row-major, one
  // per block row): when present, the FP64 PCG applies it instead of the
  // point Jacobi diagonal (bsr3_apply_dinv of solve_bsr3_pcg_gpu).
  DBuf<double> bdinv;
  bool block_jacobi = false;  // bdinv derived from the values at every solve
  int max_row_own = 0;  // longest block row of a wrapped block CSR matrix
  bool missing_diag = false;  // a wrapped block row without a diagonal block
  DBuf<int> rowblk;     // row blocks of the CSR-stream SpMV (scalar, built on first use)
  int nrowblk = 0;
  // scalar tiled SpMV, per precision (FP64, FP32): tile row bounds, their
  // count, the most rows (TR) and entries (cap) a tile may hold; TR = -1 not
  // yet built, 0 = the tiled kernel does not fit this matrix
  DBuf<int> tblk[2];
  int ntblk[2] = {0, 0};
  int tblk_tr[2] = {-1, -1};
  int tblk_cap[2] = {0, 0};
  Workspace* ws = nullptr;
  BatchWorkspace* bws = nullptr;
  ~fcu_matrix_s();
};

// ---------------------------------------------------------------------------
// Host <-> device helpers
// ---------------------------------------------------------------------------

inline bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Copy `count` elements from a host or device pointer into a device buffer.
template <class T>
inline void upload(fcu_ctx ctx, DBuf<T>& dst, const T* src, size_t count) {
  dst.alloc(count);
  if (count) CUDA_CHECK(cudaMemcpyAsync(dst.p, src, count * sizeof(T), cudaMemcpyDefault, ctx->stream));
}

template <class T>
inline void download(fcu_ctx ctx, T* dst, const T* src_dev, size_t count) {
  if (count) CUDA_CHECK(cudaMemcpyAsync(dst, src_dev, count * sizeof(T), cudaMemcpyDefault, ctx->stream));
}

// A read-only view of a caller array on the device: the caller's pointer when
// it is device memory, else a staged copy.
template <class T>
struct DevIn {
  const T* p = nullptr;
  DBuf<T> staged;
  DevIn(fcu_ctx ctx, const T* src, size_t count) {
    if (!src || !count) { p = nullptr; return; }
    if (is_device_ptr(src)) { p = src; return; }
    upload(ctx, staged, src, count);
    p = staged.p;
  }
};

// A writable device view of a caller output: writes land directly in device
// memory, or in a staging buffer copied back by finish().
template <class T>
struct DevOut {
  T* p = nullptr;
  T* host = nullptr;
  size_t count = 0;
  DBuf<T> staged;
  DevOut(T* dst, size_t n, const T* init_from = nullptr, fcu_ctx ctx = nullptr) : count(n) {
    if (!dst || !n) return;
    if (is_device_ptr(dst)) { p = dst; }
    else {
      host = dst;
      staged.alloc(n);
      p = staged.p;
    }
    if (init_from && ctx && init_from != p)
      CUDA_CHECK(cudaMemcpyAsync(p, init_from, n * sizeof(T), cudaMemcpyDefault, ctx->stream));
  }
  void finish(fcu_ctx ctx) {
    if (host) download(ctx, host, p, count);
  }
  bool on_host() const { return host != nullptr; }
};

// Launch bookkeeping: count and check every kernel launch.
#define LAUNCH_CHECK(ctx)                 \
  do {                                    \
    (ctx)->launches++;                    \
    CUDA_CHECK(cudaGetLastError());       \
  } while (0)

inline unsigned grid_for(i64 work, int block, int cap_blocks) {
  i64 g = (work + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap_blocks) g = cap_blocks;
  return (unsigned)g;
}

// ---------------------------------------------------------------------------
// Device geometry shared by assembly, RHS and adjoint kernels.
// ---------------------------------------------------------------------------

// AffineSimplexMap (jacobian.rs:18-41, 60-85): J columns v_i - v0, det by
// cofactor expansion along the first row, J^{-T} from the adjugate.
struct Geo3 {
  double G[3][3];  // J^{-T}
  double det;
  bool ok;
};

__device__ __forceinline__ Geo3 tet_geometry(const double* __restrict__ X, const int* v) {
  Geo3 g;
  double a[3][3];
  const double* p0 = X + 3 * (i64)v[0];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double* pc = X + 3 * (i64)v[c + 1];
#pragma unroll
    for (int r = 0; r < 3; ++r) a[r][c] = pc[r] - p0[r];
  }
  double m1 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
  double m2 = a[1][0] * a[2][2] - a[2][0] * a[1][2];
  double m3 = a[1][0] * a[2][1] - a[2][0] * a[1][1];
  double d = a[0][0] * m1 - a[0][1] * m2 + a[0][2] * m3;
  g.det = d;
  g.ok = fabs(d) >= 1e-14;
  double id = 1.0 / d;
  // inverse (row-major) then transposed into G
  double inv[3][3];
  inv[0][0] = m1 * id;
  inv[0][1] = (a[0][2] * a[2][1] - a[2][2] * a[0][1]) * id;
  inv[0][2] = (a[0][1] * a[1][2] - a[1][1] * a[0][2]) * id;
  inv[1][0] = -m2 * id;
  inv[1][1] = (a[0][0] * a[2][2] - a[2][0] * a[0][2]) * id;
  inv[1][2] = (a[1][0] * a[0][2] - a[0][0] * a[1][2]) * id;
  inv[2][0] = m3 * id;
  inv[2][1] = (a[2][0] * a[0][1] - a[0][0] * a[2][1]) * id;
  inv[2][2] = (a[0][0] * a[1][1] - a[1][0] * a[0][1]) * id;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) g.G[r][c] = inv[c][r];
  return g;
}

struct Geo2 {
  double G[2][2];
  double det;
  bool ok;
};

__device__ __forceinline__ Geo2 tri_geometry(const double* __restrict__ X, const int* v) {
  Geo2 g;
  const double* p0 = X + 2 * (i64)v[0];
  const double* p1 = X + 2 * (i64)v[1];
  const double* p2 = X + 2 * (i64)v[2];
  double a00 = p1[0] - p0[0], a10 = p1[1] - p0[1];
  double a01 = p2[0] - p0[0], a11 = p2[1] - p0[1];
  double d = a00 * a11 - a10 * a01;
  g.det = d;
  g.ok = fabs(d) >= 1e-14;
  double id = 1.0 / d;
  // inv = [a11, -a01; -a10, a00] / d ; G = inv^T
  g.G[0][0] = a11 * id;
  g.G[0][1] = -a10 * id;
  g.G[1][0] = -a01 * id;
  g.G[1][1] = a00 * id;
  return g;
}

// Kernels implemented in the .cu files and used across them.
void build_mesh_validity(fcu_mesh m);
void build_space_pattern(fcu_space s);
void build_transpose_positions(fcu_space s);
