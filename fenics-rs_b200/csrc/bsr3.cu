// 3x3 block CSR operators (GpuBsr3Context and solve_bsr3_pcg_gpu,
// gpu.rs:434-658, 775-1141): import of the reference's u32 block CSR with its
// inverse diagonal blocks, block-Jacobi smoothing sweeps, the inverse
// diagonal blocks of an assembled vector matrix, and export of a vector
// matrix in the same block layout.
//
// Layout in HBM: one block row per vertex (node); block k of row i holds
// vals[9k + 3a + b] = A(3i + a, 3 cols[k] + b) (row-major blocks, the order the
// assembly kernels write), inverse diagonal blocks row-major in the same way.
// A wrapped block matrix is an fcu_matrix with bs = 3 and no space, so the
// PCG of solver.cu (tiled block SpMV, graph-captured iterations) runs on it
// unchanged; its preconditioner is the caller's inverse blocks.

#include <memory>

#include "internal.cuh"

void spmv_impl(fcu_matrix m, const double* x_dev, double* y_dev);
void invalidate_graphs(fcu_matrix m);

namespace {

constexpr int T = 256;

int grid(fcu_ctx ctx, i64 n) { return (int)grid_for(n, T, ctx->num_sms * 8); }

__global__ void k_bsr3_import(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci, i64 nn, i64 nnzb,
                              int* __restrict__ rp32, int* __restrict__ ci32, int* __restrict__ dpos,
                              int* __restrict__ maxrow, int* __restrict__ bad) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nn; i += (i64)gridDim.x * blockDim.x) {
    const uint32_t a = rp[i], b = rp[i + 1];
    rp32[i] = (int)a;
    if (i == nn - 1) rp32[nn] = (int)b;
    if (b < a || (i64)b > nnzb) { atomicExch(bad, 1); dpos[i] = -1; continue; }
    atomicMax(maxrow, (int)(b - a));
    int d = -1;
    for (uint32_t k = a; k < b; ++k) {
      const uint32_t c = ci[k];
      if ((i64)c >= nn) atomicExch(bad, 2);
      ci32[k] = (int)c;
      if ((i64)c == i && d < 0) d = (int)k;
    }
    dpos[i] = d;
    if (d < 0) atomicAdd(maxrow + 2, 1);
  }
}

__global__ void k_to_f32(const double* __restrict__ a, i64 n, float* __restrict__ b) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

__device__ __forceinline__ void apply3(const double* D, const double* r, double* z) {
#pragma unroll
  for (int a = 0; a < 3; ++a) z[a] = D[3 * a] * r[0] + D[3 * a + 1] * r[1] + D[3 * a + 2] * r[2];
}

// bsr3_apply_dinv: z = D^-1 r per block row.
__global__ void k_apply_dinv(const double* __restrict__ dinv, const double* __restrict__ r, i64 nn,
                             double* __restrict__ z) {
  for (i64 w = blockIdx.x * (i64)blockDim.x + threadIdx.x; w < nn; w += (i64)gridDim.x * blockDim.x) {
    double rr[3] = {r[3 * w], r[3 * w + 1], r[3 * w + 2]}, zz[3];
    apply3(dinv + 9 * w, rr, zz);
    z[3 * w] = zz[0];
    z[3 * w + 1] = zz[1];
    z[3 * w + 2] = zz[2];
  }
}

// bsr3_jacobi_step: z += omega D^-1 (r - y), y = A z of the previous sweep.
__global__ void k_jacobi_step(const double* __restrict__ dinv, const double* __restrict__ r,
                              const double* __restrict__ y, double omega, i64 nn, double* __restrict__ z) {
  for (i64 w = blockIdx.x * (i64)blockDim.x + threadIdx.x; w < nn; w += (i64)gridDim.x * blockDim.x) {
    double d[3] = {r[3 * w] - y[3 * w], r[3 * w + 1] - y[3 * w + 1], r[3 * w + 2] - y[3 * w + 2]}, c[3];
    apply3(dinv + 9 * w, d, c);
#pragma unroll
    for (int a = 0; a < 3; ++a) z[3 * w + a] += omega * c[a];
  }
}

// Inverse of each diagonal block by the adjugate over the determinant
// (cofactor expansion along the first row). A singular block is flagged.
__global__ void k_block_inverse(const int* __restrict__ dpos, const double* __restrict__ val, i64 nn,
                                double* __restrict__ dinv, int* __restrict__ bad) {
  for (i64 w = blockIdx.x * (i64)blockDim.x + threadIdx.x; w < nn; w += (i64)gridDim.x * blockDim.x) {
    double* o = dinv + 9 * w;
    if (dpos[w] < 0) {
      atomicExch(bad, 1);
      for (int q = 0; q < 9; ++q) o[q] = 0.0;
      continue;
    }
    const double* A = val + 9 * (i64)dpos[w];
    const double c00 = A[4] * A[8] - A[5] * A[7];
    const double c01 = A[5] * A[6] - A[3] * A[8];
    const double c02 = A[3] * A[7] - A[4] * A[6];
    const double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
    if (det == 0.0 || !isfinite(det)) {
      atomicExch(bad, 1);
      for (int q = 0; q < 9; ++q) o[q] = 0.0;
      continue;
    }
    const double id = 1.0 / det;
    o[0] = c00 * id;
    o[1] = (A[2] * A[7] - A[1] * A[8]) * id;
    o[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    o[3] = c01 * id;
    o[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    o[5] = (A[2] * A[3] - A[0] * A[5]) * id;
    o[6] = c02 * id;
    o[7] = (A[1] * A[6] - A[0] * A[7]) * id;
    o[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  }
}

__global__ void k_to_u32(const int* __restrict__ a, i64 n, uint32_t* __restrict__ b) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

int read_int(fcu_ctx ctx, const int* p) {
  int h = 0;
  CUDA_CHECK(cudaMemcpyAsync(&h, p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  return h;
}

}  // namespace

// GpuBsr3Context::new (gpu.rs:453-494): the reference's block CSR (u32 row
// pointers over n_nodes block rows, u32 block columns, 9 values per block)
// and inverse diagonal blocks (9 per block row; NULL = none).
fcu_matrix bsr3_create_impl(fcu_ctx ctx, i64 nn, const uint32_t* rp_dev, const uint32_t* ci_dev, i64 nnzb,
                            const double* vals_dev, const double* dinv_dev) {
  if (nnzb + nn >= (1ll << 31) - 1 || 9 * nnzb >= (1ll << 62)) fail(FCU_ERR_UNSUPPORTED, "matrix exceeds 32-bit indexing");
  std::unique_ptr<fcu_matrix_s> m(new fcu_matrix_s());
  m->ctx = ctx;
  m->n = 3 * nn;
  m->nnodes = nn;
  m->bs = 3;
  m->nnzb = nnzb;
  m->own_row_ptr.alloc(nn + 1);
  m->own_col_idx.alloc(std::max<i64>(nnzb, 1));
  m->own_diag_pos.alloc(nn);
  DBuf<int> flags;  // longest row, bad input, rows without a diagonal block
  flags.alloc(3);
  CUDA_CHECK(cudaMemsetAsync(flags.p, 0, 3 * sizeof(int), ctx->stream));
  k_bsr3_import<<<grid(ctx, nn), T, 0, ctx->stream>>>(rp_dev, ci_dev, nn, nnzb, m->own_row_ptr.p, m->own_col_idx.p,
                                                       m->own_diag_pos.p, flags.p, flags.p + 1);
  LAUNCH_CHECK(ctx);
  const int bad = read_int(ctx, flags.p + 1);
  if (bad == 1) fail(FCU_ERR_BAD_ARG, "row_ptr is not non-decreasing or exceeds the block count");
  if (bad == 2) fail(FCU_ERR_BAD_ARG, "block column index out of range");
  m->max_row_own = std::max(1, read_int(ctx, flags.p));
  m->missing_diag = read_int(ctx, flags.p + 2) > 0;
  m->val64.alloc(9 * std::max<i64>(nnzb, 1));
  m->val32.alloc(9 * std::max<i64>(nnzb, 1));
  if (nnzb) {
    CUDA_CHECK(cudaMemcpyAsync(m->val64.p, vals_dev, 9 * nnzb * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    k_to_f32<<<grid(ctx, 9 * nnzb), T, 0, ctx->stream>>>(m->val64.p, 9 * nnzb, m->val32.p);
    LAUNCH_CHECK(ctx);
  }
  if (dinv_dev) {
    m->bdinv.alloc(9 * nn);
    CUDA_CHECK(cudaMemcpyAsync(m->bdinv.p, dinv_dev, 9 * nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  m->row_ptr = m->own_row_ptr.p;
  m->col_idx = m->own_col_idx.p;
  m->diag_pos = m->own_diag_pos.p;
  m->has_values = true;
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  ctx->refs++;
  return m.release();
}

// GpuBsr3Context::jacobi_smooth (gpu.rs:547-657): `sweeps` damped block-Jacobi
// sweeps z <- z + omega D^-1 (r - A z); with zero_initial_z the first sweep is
// z = D^-1 r (one SpMV saved). z is read (unless zero_initial_z) and written.
void bsr3_jacobi_smooth_impl(fcu_matrix m, const double* r, double* z, i64 sweeps, double omega, bool zero_init) {
  fcu_ctx ctx = m->ctx;
  if (sweeps <= 0) return;
  if (!m->bdinv.p) fail(FCU_ERR_BAD_ARG, "matrix has no inverse diagonal blocks");
  const i64 nn = m->nnodes;
  DBuf<double> y;
  y.alloc(m->n);
  i64 start = 0;
  if (zero_init) {
    k_apply_dinv<<<grid(ctx, nn), T, 0, ctx->stream>>>(m->bdinv.p, r, nn, z);
    LAUNCH_CHECK(ctx);
    start = 1;
  }
  for (i64 s = start; s < sweeps; ++s) {
    spmv_impl(m, z, y.p);
    k_jacobi_step<<<grid(ctx, nn), T, 0, ctx->stream>>>(m->bdinv.p, r, y.p, omega, nn, z);
    LAUNCH_CHECK(ctx);
  }
}

// The inverse diagonal blocks of the matrix's current values.
void refresh_block_jacobi(fcu_matrix m) {
  fcu_ctx ctx = m->ctx;
  m->bdinv.alloc(9 * m->nnodes);
  DBuf<int> bad;
  bad.alloc(1);
  CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
  k_block_inverse<<<grid(ctx, m->nnodes), T, 0, ctx->stream>>>(m->diag_pos, m->val64.p, m->nnodes, m->bdinv.p,
                                                               bad.p);
  LAUNCH_CHECK(ctx);
  if (read_int(ctx, bad.p)) fail(FCU_ERR_BAD_ARG, "a diagonal block is missing or singular");
}

// Block-Jacobi preconditioning of a vector matrix from its own diagonal
// blocks, recomputed at every solve (enable), or back to point Jacobi.
void matrix_block_jacobi_impl(fcu_matrix m, bool enable) {
  invalidate_graphs(m);
  m->block_jacobi = false;
  m->bdinv.release();
  if (!enable) return;
  refresh_block_jacobi(m);
  m->block_jacobi = true;
}

// Block CSR arrays of a vector matrix (any output may be NULL); dinv needs
// the block-Jacobi preconditioner (fcu_matrix_block_jacobi).
void matrix_export_bsr3_impl(fcu_matrix m, uint32_t* rp, uint32_t* ci, double* vals, double* dinv) {
  fcu_ctx ctx = m->ctx;
  if (rp) {
    k_to_u32<<<grid(ctx, m->nnodes + 1), T, 0, ctx->stream>>>(m->row_ptr, m->nnodes + 1, rp);
    LAUNCH_CHECK(ctx);
  }
  if (ci && m->nnzb) {
    k_to_u32<<<grid(ctx, m->nnzb), T, 0, ctx->stream>>>(m->col_idx, m->nnzb, ci);
    LAUNCH_CHECK(ctx);
  }
  if (vals && m->nnzb)
    CUDA_CHECK(cudaMemcpyAsync(vals, m->val64.p, 9 * m->nnzb * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (dinv) {
    if (m->block_jacobi) refresh_block_jacobi(m);
    if (!m->bdinv.p) fail(FCU_ERR_BAD_ARG, "matrix has no inverse diagonal blocks");
    CUDA_CHECK(cudaMemcpyAsync(dinv, m->bdinv.p, 9 * m->nnodes * sizeof(double), cudaMemcpyDeviceToDevice,
                               ctx->stream));
  }
}
