// Matrix assembly kernels (scalar P1/P2 Poisson stiffness, vector-P1
// elasticity), Dirichlet elimination, and the adjoint gradient kernel.
//
// Layout in HBM
//   scalar spaces: CSR over dofs, val[p] for slot p of row i (p in row_ptr[i]..)
//   vector space : CSR over vertices with 3x3 blocks, val[9p + 3*alpha + beta]
//                  is the (3i+alpha, 3j+beta) entry of block slot p = (i, j)
// Both FP64 and FP32 values are written by the same pass.
//
// Work decomposition: rows are owned, never scattered into, so every value
// is written exactly once, with no atomics and no zero-fill pass, and every
// sum runs in a fixed order (the results repeat bit for bit).
//   * scalar P1 (and the row-gather forms kept for comparison): one warp per
//     row evaluates each of the row's cells' element rows into shared memory
//     (the row's "contributions", ascending cell id), then each lane sums the
//     entries of its slot in ascending cell order;
//   * P2: per-cell metric records, then three rows per warp, a lane per local
//     column, adding each contribution's entry into the row's shared-memory
//     accumulators (k_assemble_p2_rows);
//   * vector-P1 elasticity and mass: per-cell records (gradients and scale,
//     or the scale alone), then one lane per off-diagonal 3x3 block summing
//     the block's cell list, the diagonal block from the row (k_elast_rows,
//     k_mass_rows_vec).
// Rows are written with coalesced stores in every form.

#include "internal.cuh"

namespace {

constexpr int WARPS = 8;   // warps per block, scalar assembly
constexpr int EWARPS = 6;  // warps per block, elasticity assembly (shared-memory bound)
// Staging rows use odd strides (in doubles) so that lanes writing "their" row
// hit distinct banks.
__host__ __device__ constexpr int odd_stride(int k) { return (k % 2) ? k : k + 1; }
constexpr unsigned FULL = 0xffffffffu;

// Sum over the warp by an xor butterfly: every lane ends with the same bits
// (each step adds the same two operands in every lane of a pair).
__device__ __forceinline__ double warp_sum_xor(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// The diagonal slot of a row receives one entry from every cell around the
// row's node (about 24 on a tetrahedral mesh) while the other slots receive
// a handful, so a lane summing it alone holds the warp back. The warp sums
// it instead, chunk by chunk in contribution order, by a fixed butterfly
// over the contributions staged in the chunk (P1 stiffness, elasticity and
// mass; P2 stiffness rows are dominated by staging ten-entry rows, and the
// tree measured no faster there).

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  *total = __shfl_sync(FULL, x, 31);
  return x - v;
}

// ---------------------------------------------------------------------------
// Scalar stiffness: P1 triangle (k=3), P1 tetrahedron (k=4), P2 tet (k=10).
// Element row a of cell c is staged as stage[t][b] = K_e[a][b].
// ---------------------------------------------------------------------------

// Symmetrised reference tensors of the P2 tetrahedron for the degree-2 Keast
// rule: R[m][a][b] with m over the metric entries (00,11,22,01,02,12); the
// off-diagonal ones hold R^{de}+R^{ed}. Filled from the host at first use.
__constant__ double c_p2_R[6][10][10];

template <int K, int DIM>
__device__ __forceinline__ void p1_element_row(const double* __restrict__ X, const int* __restrict__ cn, int c, int a,
                                               double coef, double* out) {
  int v[K];
#pragma unroll
  for (int i = 0; i < K; ++i) v[i] = cn[(i64)c * K + i];
  if (DIM == 3) {
    Geo3 g = tet_geometry(X, v);
    // gradients of the P1 basis: g_0 = -(G e0 + G e1 + G e2), g_i = G e_{i-1}
    double gr[4][3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      gr[1][r] = g.G[r][0];
      gr[2][r] = g.G[r][1];
      gr[3][r] = g.G[r][2];
      gr[0][r] = -g.G[r][0] - g.G[r][1] - g.G[r][2];
    }
    double s = (1.0 / 6.0) * fabs(g.det) * coef;
    // row a selected with compile-time indices (a runtime index would put gr in local memory)
    double ga[3] = {gr[0][0], gr[0][1], gr[0][2]};
#pragma unroll
    for (int i = 1; i < 4; ++i)
      if (a == i) ga[0] = gr[i][0], ga[1] = gr[i][1], ga[2] = gr[i][2];
#pragma unroll
    for (int b = 0; b < 4; ++b) out[b] = (ga[0] * gr[b][0] + ga[1] * gr[b][1] + ga[2] * gr[b][2]) * s;
  } else {
    Geo2 g = tri_geometry(X, v);
    double gr[3][2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      gr[1][r] = g.G[r][0];
      gr[2][r] = g.G[r][1];
      gr[0][r] = -g.G[r][0] - g.G[r][1];
    }
    double s = 0.5 * fabs(g.det) * coef;
    double ga[2] = {gr[0][0], gr[0][1]};
#pragma unroll
    for (int i = 1; i < 3; ++i)
      if (a == i) ga[0] = gr[i][0], ga[1] = gr[i][1];
#pragma unroll
    for (int b = 0; b < 3; ++b) out[b] = (ga[0] * gr[b][0] + ga[1] * gr[b][1]) * s;
  }
}

// Metric S = G^T G scaled by kappa*|det J| (6 entries, off-diagonals doubled
// are folded into the tensors instead).
__device__ __forceinline__ void p2_metric(const double* __restrict__ X, const int* __restrict__ cn, int c, double coef,
                                          double* S) {
  int v[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = cn[(i64)c * 10 + i];
  Geo3 g = tet_geometry(X, v);
  double s = fabs(g.det) * coef;
  // (G^T G)_{de} = sum_r G[r][d] G[r][e]
  const int D[6] = {0, 1, 2, 0, 0, 1}, E[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int m = 0; m < 6; ++m)
    S[m] = (g.G[0][D[m]] * g.G[0][E[m]] + g.G[1][D[m]] * g.G[1][E[m]] + g.G[2][D[m]] * g.G[2][E[m]]) * s;
}

// P2 metric records. A P2 cell feeds ten rows of the row-gather assembly,
// so its scaled metric (p2_metric) is computed once per assembly call by a
// cell-parallel pass, and the row kernel reads one 64-byte record per
// contribution instead of recomputing the geometry from the connectivity and
// coordinates (three dependent gathers). The record holds exactly the values
// p2_metric computes: S[0..5], then two pad entries (16-byte aligned, read
// with 128-bit loads).
constexpr int P2_GEO = 8;

__global__ void k_p2_metric_records(const int* __restrict__ cn, const double* __restrict__ X,
                                    const double* __restrict__ coef, i64 nc, double* __restrict__ geo) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    double S[P2_GEO];
    p2_metric(X, cn, (int)c, coef ? coef[c] : 1.0, S);
    S[6] = S[7] = 0.0;
    double2* o = reinterpret_cast<double2*>(geo + c * P2_GEO);
#pragma unroll
    for (int q = 0; q < P2_GEO / 2; ++q) o[q] = make_double2(S[2 * q], S[2 * q + 1]);
  }
}

// P2 stiffness, three rows per warp (the kernel fcu_assemble_stiffness runs on
// P2 spaces whose rows have at most 255 slots). Lanes 10g .. 10g+9 own row g
// of the warp's three consecutive rows, lane 10g+b local column b. At each
// step every group takes its row's next contribution (cell c with the row's
// dof at local index a; contributions ordered by (a, c)), forms the element
// entry K_e[a][b] = sum_m S_c[m] R[m][a][b] from the cell's metric record,
// and adds it to the row's accumulator of slot cmap[t][b] in shared memory.
// The ten columns of one cell are ten distinct dofs, so the ten lanes of a
// group update ten distinct slots: no atomics, and every slot sums its
// contributions in one fixed order (the values repeat bit for bit; they agree
// with the triplet assembly's ascending-cell sums to round-off). The three
// rows' slots are contiguous in the pattern, so the warp writes them with
// coalesced stores. One element entry costs one metric record read (shared by
// the group), six FMAs and one shared-memory add; no per-entry summation
// lists are read.
constexpr int P2W = 8;  // warps per block

__device__ __forceinline__ void p2_record(const double* __restrict__ p2geo, int cc, double2& s01, double2& s23,
                                          double2& s45) {
  const double2* rec = reinterpret_cast<const double2*>(p2geo + (i64)(cc >> 4) * P2_GEO);
  s01 = __ldg(rec);
  s23 = __ldg(rec + 1);
  s45 = __ldg(rec + 2);
}

// Each row's contributions come ordered by (local index a of the row's dof,
// cell), so a lane keeps its six reference-tensor entries R[m][a][b] in
// registers and reloads them from shared memory only when a changes (at most
// four times on a vertex row, six on an edge row) instead of at every step.
__global__ void __launch_bounds__(P2W * 32) k_assemble_p2_rows(
    const int* __restrict__ row_ptr, const int* __restrict__ contrib_ptr, const int* __restrict__ contrib_a,
    const unsigned char* __restrict__ cmap, const double* __restrict__ p2geo, i64 nrows, int stride,
    double* __restrict__ v64, float* __restrict__ v32) {
  extern __shared__ double p2sh[];
  double* R = p2sh;  // 6 x 10 x 10
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  for (int q = threadIdx.x; q < 600; q += blockDim.x) R[q] = (&c_p2_R[0][0][0])[q];
  __syncthreads();
  const int g = lane / 10, b = lane - 10 * g;  // g == 3 on lanes 30 and 31
  double* acc = p2sh + 600 + (i64)wib * 3 * stride;
  double* my = acc + (g < 3 ? g : 0) * stride;
  const i64 nwarps = (i64)gridDim.x * P2W;
  for (i64 r0 = ((i64)blockIdx.x * P2W + wib) * 3; r0 < nrows; r0 += nwarps * 3) {
    const i64 row = r0 + g;
    int L = 0, cs = 0, nct = 0;
    if (g < 3 && row < nrows) {
      L = row_ptr[row + 1] - row_ptr[row];
      cs = contrib_ptr[row];
      nct = contrib_ptr[row + 1] - cs;
    }
    for (int q = b; q < L; q += 10) my[q] = 0.0;
    const int steps = __reduce_max_sync(FULL, nct);
    __syncwarp();
    int a_cur = -1;
    double r0v = 0.0, r1v = 0.0, r2v = 0.0, r3v = 0.0, r4v = 0.0, r5v = 0.0;
    for (int t = 0; t < steps; ++t) {
      if (t < nct) {
        const i64 ci = (i64)cs + t;
        const int cc = contrib_a[ci];
        double2 s01, s23, s45;
        p2_record(p2geo, cc, s01, s23, s45);
        const int sl = cmap[ci * 10 + b];
        const int a = cc & 15;
        if (a != a_cur) {
          const double* Rab = R + a * 10 + b;
          r0v = Rab[0];
          r1v = Rab[100];
          r2v = Rab[200];
          r3v = Rab[300];
          r4v = Rab[400];
          r5v = Rab[500];
          a_cur = a;
        }
        double v = s01.x * r0v;
        v += s01.y * r1v;
        v += s23.x * r2v;
        v += s23.y * r3v;
        v += s45.x * r4v;
        v += s45.y * r5v;
        my[sl] += v;
      }
      __syncwarp();
    }
    const i64 rend = r0 + 3 < nrows ? r0 + 3 : nrows;
    const int base = row_ptr[r0];
    const int tot = row_ptr[rend] - base;
    const int off1 = row_ptr[r0 + 1 < rend ? r0 + 1 : rend] - base;
    const int off2 = row_ptr[r0 + 2 < rend ? r0 + 2 : rend] - base;
    for (int q = lane; q < tot; q += 32) {
      const int gg = q >= off2 ? 2 : (q >= off1 ? 1 : 0);
      const double v = acc[gg * stride + q - (gg == 2 ? off2 : gg == 1 ? off1 : 0)];
      v64[base + q] = v;
      v32[base + q] = (float)v;
    }
    __syncwarp();
  }
}

// Header of a row-gather row, spread over the warp: lane k < 5 holds
// row_ptr[row], row_ptr[row + 1], contrib_ptr[row], contrib_ptr[row + 1],
// diag_pos[row] (read back with shuffles). The kernels fetch the next row's
// header while they sum the current row.
__device__ __forceinline__ int row_header(const int* __restrict__ row_ptr, const int* __restrict__ contrib_ptr,
                                          const int* __restrict__ diag_pos, i64 row, i64 nrows, int lane) {
  if (row >= nrows || lane >= 5) return 0;
  const int* src = lane < 2 ? row_ptr : lane < 4 ? contrib_ptr : diag_pos;
  return src[row + (lane == 1 || lane == 3 ? 1 : 0)];
}

template <int K, int DIM, bool IS_P2>
__global__ void __launch_bounds__(WARPS * 32) k_assemble_scalar(
    const int* __restrict__ row_ptr, const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
    const unsigned short* __restrict__ slot_cnt, const unsigned short* __restrict__ slot_ent,
    const int* __restrict__ cn, const double* __restrict__ X, const double* __restrict__ coef,
    const double* __restrict__ p2geo, const int* __restrict__ diag_pos, i64 nrows,
    double* __restrict__ v64, float* __restrict__ v32) {
  constexpr int KS = odd_stride(K);
  __shared__ double stage_all[WARPS][32][KS];
  __shared__ unsigned short ent_all[WARPS][32 * K];
  __shared__ double metric_all[IS_P2 ? WARPS : 1][32][7];
  __shared__ int sa_all[IS_P2 ? WARPS : 1][32];
  __shared__ double R[IS_P2 ? 6 * 100 : 1];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (IS_P2) {
    for (int t = threadIdx.x; t < 600; t += blockDim.x) R[t] = (&c_p2_R[0][0][0])[t];
    __syncthreads();
  }
  double(*stage)[KS] = stage_all[wib];
  const i64 nwarps = (i64)gridDim.x * WARPS;
  const i64 row0 = (i64)blockIdx.x * WARPS + wib;
  int hdr = row_header(row_ptr, contrib_ptr, diag_pos, row0, nrows, lane);
  for (i64 row = row0; row < nrows; row += nwarps) {
    const int rs = __shfl_sync(FULL, hdr, 0), L = __shfl_sync(FULL, hdr, 1) - rs;
    const int cs = __shfl_sync(FULL, hdr, 2), nct = __shfl_sync(FULL, hdr, 3) - cs;
    const int dl = __shfl_sync(FULL, hdr, 4) - rs;  // slot of the diagonal
    hdr = row_header(row_ptr, contrib_ptr, diag_pos, row + nwarps, nrows, lane);
    const i64 ebase = (i64)K * cs;
    // the first group's slot counts and the first chunk's contributions are
    // fetched together with the entry list
    const int cnt_first = lane < L ? (int)slot_cnt[rs + lane] : 0;
    const int cc_first = lane < nct ? contrib[cs + lane] : 0;
    // The row's (contribution, column) entry list, staged once per row with a
    // coalesced copy when it fits (at most 32 contributions).
    const bool staged = nct <= 32;
    if (staged)
      for (int q = lane; q < K * nct; q += 32) ent_all[wib][q] = slot_ent[ebase + q];
    __syncwarp();
    int run = 0;  // entries consumed by earlier slot groups
    for (int g0 = 0; g0 < L; g0 += 32) {
      const int s = g0 + lane;
      const int cnt = g0 == 0 ? cnt_first : (s < L) ? (int)slot_cnt[rs + s] : 0;
      int tot;
      const int off = warp_excl_scan(cnt, lane, &tot);
      i64 e = ebase + run + off;
      const i64 e1 = e + cnt;
      run += tot;
      const bool has_diag = !IS_P2 && dl >= g0 && dl < g0 + 32;  // uniform over the warp
      if (has_diag && s == dl) e = e1;
      double acc = 0.0;
      for (int ch = 0; ch < nct; ch += 32) {
        // stage element rows of contributions ch .. ch+31
        const int t = ch + lane;
        int a_own = 0;
        // P2 rows of more than 32 slots (vertex rows) with at most 32
        // contributions reuse the element rows staged by the first slot group
        const bool restage = !(IS_P2 && g0 > 0 && nct <= 32);
        if (IS_P2) {
          if (restage && t < nct) {
            const int cc = ch == 0 ? cc_first : contrib[cs + t];
            const double2* g = reinterpret_cast<const double2*>(p2geo + (i64)(cc >> 4) * P2_GEO);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              const double2 v = g[q];
              metric_all[wib][lane][2 * q] = v.x;
              metric_all[wib][lane][2 * q + 1] = v.y;
            }
            sa_all[wib][lane] = cc & 15;
          }
          __syncwarp();
          const int nt = restage ? min(32, nct - ch) : 0;
          for (int q = lane; q < nt * K; q += 32) {
            const int tt = q / K, b = q - tt * K;
            const int a = sa_all[wib][tt];
            const double* S = metric_all[wib][tt];
            double v = 0.0;
#pragma unroll
            for (int m = 0; m < 6; ++m) v += S[m] * R[m * 100 + a * 10 + b];
            stage[tt][b] = v;
          }
        } else {
          if (t < nct) {
            const int cc = ch == 0 ? cc_first : contrib[cs + t];
            a_own = cc & 15;
            p1_element_row<K, DIM>(X, cn, cc >> 4, cc & 15, coef ? coef[cc >> 4] : 1.0, stage[lane]);
          }
        }
        __syncwarp();
        if (has_diag) {
          double d = 0.0;
          if (t < nct) d = stage[lane][a_own];
          d = warp_sum_xor(d);
          if (s == dl) acc += d;
        }
        while (e < e1) {
          const unsigned ent = staged ? ent_all[wib][e - ebase] : slot_ent[e];
          const int tl = (int)(ent >> 4);
          if (tl >= ch + 32) break;
          acc += stage[tl - ch][ent & 15];
          ++e;
        }
        __syncwarp();
      }
      if (s < L) {
        v64[rs + s] = acc;
        v32[rs + s] = (float)acc;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Vector-P1 elasticity (elasticity.rs:73-149). For block (i, j) of a cell:
//   K_{i a, j b} = vol (lam g_j[b] g_i[a] + mu (g_i.g_j) d_ab + mu g_j[a] g_i[b])
// = (lam M + mu M^T + mu tr(M) I)[a][b] with M = vol g_i g_j^T. The kernel sums
// M over the cells of each block (per-cell moduli folded into vol), then forms
// the block once. Staged per contribution: h = s_e g_i (3) and g_0..g_3 (12).
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(EWARPS * 32, 4) k_assemble_elasticity(
    const int* __restrict__ row_ptr, const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
    const unsigned short* __restrict__ slot_cnt, const unsigned short* __restrict__ slot_ent,
    const int* __restrict__ cn, const double* __restrict__ X, const double* __restrict__ cellE, double lam,
    double mu, const int* __restrict__ diag_pos, i64 nrows, double* __restrict__ v64,
    float* __restrict__ v32) {
  __shared__ double st_all[EWARPS][32][17];
  __shared__ double out_all[EWARPS][32 * 9];
  __shared__ unsigned short ent_all[EWARPS][32 * 4];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double(*st)[17] = st_all[wib];
  double* out = out_all[wib];
  const i64 nwarps = (i64)gridDim.x * EWARPS;
  const i64 row0 = (i64)blockIdx.x * EWARPS + wib;
  int hdr = row_header(row_ptr, contrib_ptr, diag_pos, row0, nrows, lane);
  for (i64 row = row0; row < nrows; row += nwarps) {
    const int rs = __shfl_sync(FULL, hdr, 0), L = __shfl_sync(FULL, hdr, 1) - rs;
    const int cs = __shfl_sync(FULL, hdr, 2), nct = __shfl_sync(FULL, hdr, 3) - cs;
    const int dl = __shfl_sync(FULL, hdr, 4) - rs;
    hdr = row_header(row_ptr, contrib_ptr, diag_pos, row + nwarps, nrows, lane);
    const i64 ebase = 4 * (i64)cs;
    const int cnt_first = lane < L ? (int)slot_cnt[rs + lane] : 0;
    const int cc_first = lane < nct ? contrib[cs + lane] : 0;
    const bool staged = nct <= 32;
    if (staged)
      for (int q = lane; q < 4 * nct; q += 32) ent_all[wib][q] = slot_ent[ebase + q];
    __syncwarp();
    int run = 0;
    for (int g0 = 0; g0 < L; g0 += 32) {
      const int s = g0 + lane;
      const int cnt = g0 == 0 ? cnt_first : (s < L) ? (int)slot_cnt[rs + s] : 0;
      int tot;
      const int off = warp_excl_scan(cnt, lane, &tot);
      i64 e = ebase + run + off;
      const i64 e1 = e + cnt;
      run += tot;
      const bool has_diag = dl >= g0 && dl < g0 + 32;  // uniform over the warp
      if (has_diag && s == dl) e = e1;
      double M[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) M[q] = 0.0;
      for (int ch = 0; ch < nct; ch += 32) {
        const int t = ch + lane;
        int a_own = 0;
        if (t < nct) {
          const int cc = ch == 0 ? cc_first : contrib[cs + t];
          const int c = cc >> 4, a = cc & 15;
          a_own = a;
          int v[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) v[i] = cn[4 * (i64)c + i];
          Geo3 g = tet_geometry(X, v);
          double sc = (1.0 / 6.0) * fabs(g.det);
          if (cellE) sc *= cellE[c];
          double* w = st[lane];
#pragma unroll
          for (int r = 0; r < 3; ++r) {
            w[3 + r] = -g.G[r][0] - g.G[r][1] - g.G[r][2];
            w[6 + r] = g.G[r][0];
            w[9 + r] = g.G[r][1];
            w[12 + r] = g.G[r][2];
          }
#pragma unroll
          for (int r = 0; r < 3; ++r) w[r] = sc * w[3 + 3 * a + r];
        }
        __syncwarp();
        if (has_diag) {
          // a contribution's diagonal block is (sc g)(g^T) with g the gradient of its own
          // basis function: symmetric, so six sums cover it
          const double* w = st[lane];
          const double* g = w + 3 + 3 * a_own;
          const bool live = t < nct;
          const double d00 = warp_sum_xor(live ? w[0] * g[0] : 0.0);
          const double d11 = warp_sum_xor(live ? w[1] * g[1] : 0.0);
          const double d22 = warp_sum_xor(live ? w[2] * g[2] : 0.0);
          const double d01 = warp_sum_xor(live ? w[0] * g[1] : 0.0);
          const double d02 = warp_sum_xor(live ? w[0] * g[2] : 0.0);
          const double d12 = warp_sum_xor(live ? w[1] * g[2] : 0.0);
          if (s == dl) {
            M[0] += d00; M[4] += d11; M[8] += d22;
            M[1] += d01; M[3] += d01;
            M[2] += d02; M[6] += d02;
            M[5] += d12; M[7] += d12;
          }
        }
        while (e < e1) {
          const unsigned ent = staged ? ent_all[wib][e - ebase] : slot_ent[e];
          const int tl = (int)(ent >> 4);
          if (tl >= ch + 32) break;
          const double* w = st[tl - ch];
          const int b = ent & 15;
          const double h0 = w[0], h1 = w[1], h2 = w[2];
          const double q0 = w[3 + 3 * b], q1 = w[4 + 3 * b], q2 = w[5 + 3 * b];
          M[0] += h0 * q0; M[1] += h0 * q1; M[2] += h0 * q2;
          M[3] += h1 * q0; M[4] += h1 * q1; M[5] += h1 * q2;
          M[6] += h2 * q0; M[7] += h2 * q1; M[8] += h2 * q2;
          ++e;
        }
        __syncwarp();
      }
      const double tr = mu * (M[0] + M[4] + M[8]);
      if (s < L) {
        double* o = out + 9 * lane;
#pragma unroll
        for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
          for (int b2 = 0; b2 < 3; ++b2)
            o[3 * a2 + b2] = lam * M[3 * a2 + b2] + mu * M[3 * b2 + a2] + (a2 == b2 ? tr : 0.0);
      }
      __syncwarp();
      const int nb = min(32, L - g0);
      const i64 base = 9 * ((i64)rs + g0);
      for (int q = lane; q < 9 * nb; q += 32) {
        const double v = out[q];
        v64[base + q] = v;
        v32[base + q] = (float)v;
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// Vector-P1 elasticity, block-parallel form (the kernels fcu_assemble_elasticity
// runs). Two passes:
//
//  1. k_elast_records, one thread per cell: the cell's four basis gradients
//     g_b = J^{-T} grad(phi_b) and its scale s_c = |det J| / 6 (times E_c),
//     stored as four 32-byte groups {g_b.x, g_b.y, g_b.z, s_c}. Each cell's
//     geometry is computed once (the row-gather kernel above computes it once
//     per vertex, four times).
//  2. k_elast_blocks, one thread per block: for an upper off-diagonal block
//     (i, j), j > i, the thread sums M = sum_c s_c g_a g_b^T over the cells
//     that hold the edge (ascending cell order, a and b the local indices of
//     i and j), forms K_ij = lam M + mu M^T + mu tr(M) I, and writes K_ij
//     and its transpose K_ji; for a diagonal block (i, i) it sums the
//     symmetric D = sum_c s_c g_a g_a^T over the cells around i and writes
//     (lam + mu) D + mu tr(D) I. Every value is written once, with no atomics,
//     and the assembled matrix is exactly symmetric.
//
// Both passes read and write with plain coalesced or 32-byte vector accesses;
// the records of the cells around a window of rows stay in L2 between the
// threads that share them.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_elast_records(const int* __restrict__ cn, const double* __restrict__ X,
                                                       const unsigned char* __restrict__ valid,
                                                       const double* __restrict__ cellE, i64 nc,
                                                       double* __restrict__ rec) {
  // Each warp computes 32 consecutive cells' records, stages them in shared
  // memory (rows of 18 doubles, so 16-byte accesses by 8 lanes hit distinct
  // banks) and writes the 4 KB with contiguous 16-byte stores.
  constexpr int RS = 18;
  __shared__ double2 st_all[8][32 * RS / 2];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double2* st = st_all[wib];
  const i64 nwarps = (i64)gridDim.x * (blockDim.x >> 5);
  for (i64 c0 = ((i64)blockIdx.x * (blockDim.x >> 5) + wib) * 32; c0 < nc; c0 += nwarps * 32) {
    const i64 c = c0 + lane;
    double2* o = st + lane * (RS / 2);
    if (c < nc && valid[c]) {
      const int4 q = reinterpret_cast<const int4*>(cn)[c];
      const int v[4] = {q.x, q.y, q.z, q.w};
      const Geo3 g = tet_geometry(X, v);
      double sc = (1.0 / 6.0) * fabs(g.det);
      if (cellE) sc *= cellE[c];
      o[0] = make_double2(-g.G[0][0] - g.G[0][1] - g.G[0][2], -g.G[1][0] - g.G[1][1] - g.G[1][2]);
      o[1] = make_double2(-g.G[2][0] - g.G[2][1] - g.G[2][2], sc);
#pragma unroll
      for (int b = 1; b < 4; ++b) {
        o[2 * b] = make_double2(g.G[0][b - 1], g.G[1][b - 1]);
        o[2 * b + 1] = make_double2(g.G[2][b - 1], sc);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) o[k] = make_double2(0.0, 0.0);
    }
    __syncwarp();
    const i64 ncell = nc - c0 < 32 ? nc - c0 : 32;
    double2* dst = reinterpret_cast<double2*>(rec + 16 * c0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int f = lane + 32 * k;  // 16-byte word f of the warp's 32 records
      if (f < 8 * ncell) dst[f] = st[(f >> 3) * (RS / 2) + (f & 7)];
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void load_rec(const double* __restrict__ rec, unsigned c, unsigned a, double& x, double& y,
                                         double& z, double& s) {
  const double2* r = reinterpret_cast<const double2*>(rec + 16 * (i64)c + 4 * a);
  const double2 p = __ldg(r), q = __ldg(r + 1);
  x = p.x;
  y = p.y;
  z = q.x;
  s = q.y;
}

__global__ void __launch_bounds__(256) k_elast_blocks(i64 nup, const int* __restrict__ up_ptr,
                                                      const unsigned* __restrict__ up_ent,
                                                      const int* __restrict__ up_slot,
                                                      const int* __restrict__ up_tslot, i64 nn,
                                                      const int* __restrict__ contrib_ptr,
                                                      const int* __restrict__ contrib,
                                                      const int* __restrict__ diag_pos,
                                                      const double* __restrict__ rec, double lam, double mu,
                                                      double* __restrict__ v64, float* __restrict__ v32) {
  const i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (t < nup) {
    double M[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) M[k] = 0.0;
    const int e1 = up_ptr[t + 1];
    for (int e = up_ptr[t]; e < e1; ++e) {
      const unsigned ent = up_ent[e];
      const unsigned c = ent >> 4, a = (ent >> 2) & 3u, b = ent & 3u;
      double hx, hy, hz, s, gx, gy, gz, s2;
      load_rec(rec, c, a, hx, hy, hz, s);
      load_rec(rec, c, b, gx, gy, gz, s2);
      hx *= s;
      hy *= s;
      hz *= s;
      M[0] += hx * gx; M[1] += hx * gy; M[2] += hx * gz;
      M[3] += hy * gx; M[4] += hy * gy; M[5] += hy * gz;
      M[6] += hz * gx; M[7] += hz * gy; M[8] += hz * gz;
    }
    const double tr = mu * (M[0] + M[4] + M[8]);
    double K[9];
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
      for (int b2 = 0; b2 < 3; ++b2)
        K[3 * a2 + b2] = lam * M[3 * a2 + b2] + mu * M[3 * b2 + a2] + (a2 == b2 ? tr : 0.0);
    const i64 p = up_slot[t], q = up_tslot[t];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      v64[9 * p + k] = K[k];
      v32[9 * p + k] = (float)K[k];
    }
    if (q < 0) return;  // the pattern is symmetric, so this does not happen
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
      for (int b2 = 0; b2 < 3; ++b2) {
        v64[9 * q + 3 * b2 + a2] = K[3 * a2 + b2];
        v32[9 * q + 3 * b2 + a2] = (float)K[3 * a2 + b2];
      }
  } else if (t - nup < nn) {
    const i64 i = t - nup;
    double d00 = 0.0, d11 = 0.0, d22 = 0.0, d01 = 0.0, d02 = 0.0, d12 = 0.0;
    const int c1 = contrib_ptr[i + 1];
    for (int k = contrib_ptr[i]; k < c1; ++k) {
      const unsigned cc = (unsigned)contrib[k];
      double gx, gy, gz, s;
      load_rec(rec, cc >> 4, cc & 15u, gx, gy, gz, s);
      const double hx = s * gx, hy = s * gy, hz = s * gz;
      d00 += hx * gx; d11 += hy * gy; d22 += hz * gz;
      d01 += hx * gy; d02 += hx * gz; d12 += hy * gz;
    }
    const double tr = mu * (d00 + d11 + d22);
    const double lm = lam + mu;
    const double K[9] = {lm * d00 + tr, lm * d01, lm * d02, lm * d01, lm * d11 + tr, lm * d12,
                         lm * d02, lm * d12, lm * d22 + tr};
    const i64 p = diag_pos[i];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      v64[9 * p + k] = K[k];
      v32[9 * p + k] = (float)K[k];
    }
  }
}

// Vector-P1 elasticity, row form over the gradient records: LPR lanes per
// block row (16 when every row has at most 16 blocks, as on the Kuhn box
// meshes, else 32), one off-diagonal block per lane. A lane sums
// M = sum_c s_c (g_a g_b^T) over the block's cell list (sl_ent, ascending
// cell order) reading two 32-byte gradient records per cell, two cells per
// round so that four record loads are in flight, forms
// K = lam M + mu M^T + mu tr(M) I, and stages it in shared memory; each chunk
// of LPR blocks is then written with contiguous stores. Each product
// g_a[i] g_b[j] is rounded before it is scaled by s_c, so block (j, i) comes
// out as the exact transpose of block (i, j): the assembled matrix, and its
// FP32 copy, are exactly symmetric. The diagonal block comes from the
// row-sum identity: every cell's gradients sum to zero, so
// sum_j M_ij = 0 and M_ii = -sum_{j != i} M_ij; K is linear in M, so
// K_ii = -sum_{j != i} K_ij (symmetrised), summed by nine lanes over the
// blocks staged for the row's stores; relative to the summed-per-cell
// diagonal this moves it by a few ulps of the row's largest block.
// One 32-byte gradient record {g.x, g.y, g.z, s} with a single 256-bit load
// (read-only path): one L1 request per record instead of two 16-byte ones.
__device__ __forceinline__ void ld_rec4(const double* p, double2& a, double2& b) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p));
}

__device__ __forceinline__ void elast_accumulate(double (&M)[9], double s, double2 a01, double2 a2s, double2 b01,
                                                 double2 b2s) {
  const double ga[3] = {a01.x, a01.y, a2s.x}, gb[3] = {b01.x, b01.y, b2s.x};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) M[3 * i + j] = fma(s, ga[i] * gb[j], M[3 * i + j]);
}

template <int LPR>
__global__ void __launch_bounds__(256, 4) k_elast_rows(const int* __restrict__ row_ptr,
                                                       const int* __restrict__ diag_pos,
                                                       const int* __restrict__ sl_ptr,
                                                       const unsigned* __restrict__ sl_ent,
                                                       const double* __restrict__ rec, i64 nrows, double lam,
                                                       double mu, double* __restrict__ v64, float* __restrict__ v32) {
  constexpr int RPW = 32 / LPR;
  constexpr int W = 8;
  __shared__ double out_all[W][32 * 9];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int sub = lane % LPR, seg = lane / LPR;
  double* out = out_all[wib];
  const i64 nwarps = (i64)gridDim.x * W;
  for (i64 r0 = ((i64)blockIdx.x * W + wib) * RPW; r0 < nrows; r0 += nwarps * RPW) {
    const i64 row = r0 + seg;
    const bool valid = row < nrows;
    int rs = 0, L = 0, dl = -1;
    if (valid) {
      rs = row_ptr[row];
      L = row_ptr[row + 1] - rs;
      dl = diag_pos[row] - rs;
    }
    double t = 0.0;  // lanes sub < 9: entry sub of the row's sum of off-diagonal K blocks
    const int nch = __reduce_max_sync(FULL, (L + LPR - 1) / LPR);
    for (int ch = 0; ch < nch; ++ch) {
      const int q = ch * LPR + sub;
      if (q < L && q != dl) {
        double M[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) M[k] = 0.0;
        int e = sl_ptr[rs + q];
        const int e1 = sl_ptr[rs + q + 1];
        // the next pair's list entries are fetched while this pair is summed
        unsigned n0 = e < e1 ? sl_ent[e] : 0u, n1 = e + 1 < e1 ? sl_ent[e + 1] : 0u;
        for (; e + 1 < e1; e += 2) {
          const unsigned u0 = n0, u1 = n1;
          n0 = e + 2 < e1 ? sl_ent[e + 2] : 0u;
          n1 = e + 3 < e1 ? sl_ent[e + 3] : 0u;
          double2 a01, a2s, b01, b2s, c01, c2s, d01, d2s;
          ld_rec4(rec + 16 * (i64)(u0 >> 4) + 4 * ((u0 >> 2) & 3u), a01, a2s);
          ld_rec4(rec + 16 * (i64)(u0 >> 4) + 4 * (u0 & 3u), b01, b2s);
          ld_rec4(rec + 16 * (i64)(u1 >> 4) + 4 * ((u1 >> 2) & 3u), c01, c2s);
          ld_rec4(rec + 16 * (i64)(u1 >> 4) + 4 * (u1 & 3u), d01, d2s);
          elast_accumulate(M, a2s.y, a01, a2s, b01, b2s);
          elast_accumulate(M, c2s.y, c01, c2s, d01, d2s);
        }
        if (e < e1) {
          const unsigned u0 = n0;
          double2 a01, a2s, b01, b2s;
          ld_rec4(rec + 16 * (i64)(u0 >> 4) + 4 * ((u0 >> 2) & 3u), a01, a2s);
          ld_rec4(rec + 16 * (i64)(u0 >> 4) + 4 * (u0 & 3u), b01, b2s);
          elast_accumulate(M, a2s.y, a01, a2s, b01, b2s);
        }
        const double tr = mu * (M[0] + M[4] + M[8]);
        double* o = out + 9 * lane;
#pragma unroll
        for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
          for (int b2 = 0; b2 < 3; ++b2)
            o[3 * a2 + b2] = lam * M[3 * a2 + b2] + mu * M[3 * b2 + a2] + (a2 == b2 ? tr : 0.0);
      }
      __syncwarp();
      const int n = L - ch * LPR < LPR ? L - ch * LPR : LPR;
      if (sub < 9)
        for (int l = 0; l < n; ++l)
          if (ch * LPR + l != dl) t += out[9 * (seg * LPR + l) + sub];
      const i64 base = 9 * ((i64)rs + ch * LPR);
      for (int idx = sub; idx < 9 * n; idx += LPR) {
        const int blk = idx / 9;
        if (ch * LPR + blk == dl) continue;
        const double v = out[9 * seg * LPR + idx];
        v64[base + idx] = v;
        v32[base + idx] = (float)v;
      }
      __syncwarp();
    }
    // diagonal block: K_ii = -sum_{j != i} K_ij (K is linear in M and
    // M_ii = -sum_{j != i} M_ij), symmetrised
    __syncwarp();
    if (sub < 9) out[9 * seg * LPR + sub] = t;
    __syncwarp();
    if (valid && sub < 9 && dl >= 0) {
      const double* S = out + 9 * seg * LPR;
      const int a2 = sub / 3, b2 = sub - 3 * (sub / 3);
      const double v = -0.5 * (S[3 * a2 + b2] + S[3 * b2 + a2]);
      v64[9 * ((i64)rs + dl) + sub] = v;
      v32[9 * ((i64)rs + dl) + sub] = (float)v;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Mass matrices (mass.rs:10-250). Entry (a, b) of cell c is s_c F[a][b]:
// s_c = rho * measure (area |det|/2, volume |det|/6; the P2 products already
// carry the reference volume, so there the measure is |det|), times the
// per-cell coefficient when one is given; F = 1/6, 1/12 (triangle), 1/10,
// 1/20 (tetrahedron) or the exact P2 reference products. Each product is
// rounded before it is summed, in ascending cell order, as the triplet
// assembly sums it. The vector space stores s F I_3 per block (the same
// scalar on each displacement component, mass.rs:118-123).
// ---------------------------------------------------------------------------

struct MassTable {
  double F[100];  // F[a * K + b]
};

template <int K, int DIM, int BS>
__global__ void __launch_bounds__(WARPS * 32) k_assemble_mass(
    const int* __restrict__ row_ptr, const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
    const unsigned short* __restrict__ slot_cnt, const unsigned short* __restrict__ slot_ent,
    const int* __restrict__ cn, const double* __restrict__ X, const double* __restrict__ coef, double rho,
    const MassTable tab, const int* __restrict__ diag_pos, i64 nrows, double* __restrict__ v64,
    float* __restrict__ v32) {
  __shared__ double s_all[WARPS][32];
  __shared__ int a_all[WARPS][32];
  __shared__ unsigned short ent_all[WARPS][32 * K];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const i64 nwarps = (i64)gridDim.x * WARPS;
  const i64 row0 = (i64)blockIdx.x * WARPS + wib;
  int hdr = row_header(row_ptr, contrib_ptr, diag_pos, row0, nrows, lane);
  for (i64 row = row0; row < nrows; row += nwarps) {
    const int rs = __shfl_sync(FULL, hdr, 0), L = __shfl_sync(FULL, hdr, 1) - rs;
    const int cs = __shfl_sync(FULL, hdr, 2), nct = __shfl_sync(FULL, hdr, 3) - cs;
    const int dl = __shfl_sync(FULL, hdr, 4) - rs;
    hdr = row_header(row_ptr, contrib_ptr, diag_pos, row + nwarps, nrows, lane);
    const i64 ebase = (i64)K * cs;
    const int cnt_first = lane < L ? (int)slot_cnt[rs + lane] : 0;
    const int cc_first = lane < nct ? contrib[cs + lane] : 0;
    const bool staged = nct <= 32;
    if (staged)
      for (int q = lane; q < K * nct; q += 32) ent_all[wib][q] = slot_ent[ebase + q];
    __syncwarp();
    int run = 0;
    for (int g0 = 0; g0 < L; g0 += 32) {
      const int s = g0 + lane;
      const int cnt = g0 == 0 ? cnt_first : (s < L) ? (int)slot_cnt[rs + s] : 0;
      int tot;
      const int off = warp_excl_scan(cnt, lane, &tot);
      i64 e = ebase + run + off;
      const i64 e1 = e + cnt;
      run += tot;
      const bool has_diag = dl >= g0 && dl < g0 + 32;  // uniform over the warp
      if (has_diag && s == dl) e = e1;
      double acc = 0.0;
      for (int ch = 0; ch < nct; ch += 32) {
        const int t = ch + lane;
        if (t < nct) {
          const int cc = ch == 0 ? cc_first : contrib[cs + t];
          const int c = cc >> 4;
          int v[DIM + 1];
#pragma unroll
          for (int i = 0; i <= DIM; ++i) v[i] = cn[(i64)c * K + i];
          const double det = (DIM == 3) ? tet_geometry(X, v).det : tri_geometry(X, v).det;
          const double meas = (K == 10) ? fabs(det) : (DIM == 3 ? (1.0 / 6.0) * fabs(det) : 0.5 * fabs(det));
          double sc = __dmul_rn(rho, meas);
          if (coef) sc = __dmul_rn(sc, coef[c]);
          s_all[wib][lane] = sc;
          a_all[wib][lane] = cc & 15;
        }
        __syncwarp();
        if (has_diag) {
          const int a = a_all[wib][lane];
          const double d = warp_sum_xor(t < nct ? __dmul_rn(s_all[wib][lane], tab.F[a * K + a]) : 0.0);
          if (s == dl) acc = __dadd_rn(acc, d);
        }
        while (e < e1) {
          const unsigned ent = staged ? ent_all[wib][e - ebase] : slot_ent[e];
          const int tl = (int)(ent >> 4);
          if (tl >= ch + 32) break;
          acc = __dadd_rn(acc, __dmul_rn(s_all[wib][tl - ch], tab.F[a_all[wib][tl - ch] * K + (ent & 15)]));
          ++e;
        }
        __syncwarp();
      }
      if (s < L) {
        if (BS == 1) {
          v64[rs + s] = acc;
          v32[rs + s] = (float)acc;
        } else {
          const i64 o = 9 * ((i64)rs + s);
#pragma unroll
          for (int q = 0; q < 9; ++q) {
            const double v = (q % 4 == 0) ? acc : 0.0;
            v64[o + q] = v;
            v32[o + q] = (float)v;
          }
        }
      }
    }
  }
}

// Exact products of the P2 basis on the reference tetrahedron
// (mass.rs:195-250): every basis function is a sum of barycentric monomials
// (corner i: 2 l_i^2 - l_i; edge (i, j): 4 l_i l_j), and
// int l0^m0 l1^m1 l2^m2 l3^m3 = m0! m1! m2! m3! / (m0+m1+m2+m3+3)!.
// Node order: corners 0-3, then edges 01, 12, 02, 03, 13, 23.
void p2_mass_products(double out[100]) {
  const double fact[12] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0, 362880.0, 3628800.0, 39916800.0};
  struct Term { int m[4]; double c; };
  std::vector<std::vector<Term>> basis(10);
  for (int i = 0; i < 4; ++i) {
    Term sq{{0, 0, 0, 0}, 2.0}, lin{{0, 0, 0, 0}, -1.0};
    sq.m[i] = 2;
    lin.m[i] = 1;
    basis[i] = {sq, lin};
  }
  const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  for (int e = 0; e < 6; ++e) {
    Term t{{0, 0, 0, 0}, 4.0};
    t.m[edges[e][0]] = 1;
    t.m[edges[e][1]] = 1;
    basis[4 + e] = {t};
  }
  for (int a = 0; a < 10; ++a)
    for (int b = 0; b < 10; ++b) {
      double acc = 0.0;
      for (const Term& ta : basis[a])
        for (const Term& tb : basis[b]) {
          int m[4], deg = 0;
          for (int q = 0; q < 4; ++q) { m[q] = ta.m[q] + tb.m[q]; deg += m[q]; }
          acc += ta.c * tb.c * fact[m[0]] * fact[m[1]] * fact[m[2]] * fact[m[3]] / fact[deg + 3];
        }
      out[a * 10 + b] = acc;
    }
}

// Vector-P1 mass, row form over the per-block cell lists of the elasticity
// pattern (sl_ptr / sl_ent, ascending cell order). k_mass_scales computes
// each cell's s_c = rho * |det J| / 6 (* coefficient) once, with the
// arithmetic of k_assemble_mass; k_mass_rows_vec gives each off-diagonal
// block one lane, which adds s_c F[a][b] (each product rounded) over the
// block's cells in ascending order, exactly as k_assemble_mass sums that
// entry, and the diagonal block's entry is summed over the row's
// contributions by the row's lanes (a fixed butterfly). A block is m I_3;
// the row's blocks are written with contiguous stores, the lane that holds
// a block's m handing it to the lanes that store it. One 8-byte load per
// (block, cell) instead of one geometry per contribution.
__global__ void __launch_bounds__(256) k_mass_scales(const int* __restrict__ cn, const double* __restrict__ X,
                                                     const double* __restrict__ coef, double rho, i64 nc,
                                                     double* __restrict__ sc) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    const int4 q = reinterpret_cast<const int4*>(cn)[c];
    const int v[4] = {q.x, q.y, q.z, q.w};
    const double meas = (1.0 / 6.0) * fabs(tet_geometry(X, v).det);
    double s = __dmul_rn(rho, meas);
    if (coef) s = __dmul_rn(s, coef[c]);
    sc[c] = s;
  }
}

template <int LPR>
__global__ void __launch_bounds__(256) k_mass_rows_vec(const int* __restrict__ row_ptr,
                                                       const int* __restrict__ diag_pos,
                                                       const int* __restrict__ sl_ptr,
                                                       const unsigned* __restrict__ sl_ent,
                                                       const int* __restrict__ contrib_ptr,
                                                       const int* __restrict__ contrib,
                                                       const double* __restrict__ sc, const MassTable tab,
                                                       i64 nrows, double* __restrict__ v64, float* __restrict__ v32) {
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % LPR, seg = lane / LPR;
  const i64 nwarps = (i64)gridDim.x * (blockDim.x >> 5);
  for (i64 r0 = ((i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * RPW; r0 < nrows; r0 += nwarps * RPW) {
    const i64 row = r0 + seg;
    const bool valid = row < nrows;
    int rs = 0, L = 0, dl = -1, c0 = 0, c1 = 0;
    if (valid) {
      rs = row_ptr[row];
      L = row_ptr[row + 1] - rs;
      dl = diag_pos[row] - rs;
      c0 = contrib_ptr[row];
      c1 = contrib_ptr[row + 1];
    }
    // diagonal: sum of s_c F[a][a] over the row's contributions
    double dsum = 0.0;
    for (int k0 = c0 + sub; k0 < c1; k0 += 2 * LPR) {
      const int k1 = k0 + LPR;
      const int cc0 = contrib[k0], cc1 = k1 < c1 ? contrib[k1] : 0;
      const double f0 = sc[cc0 >> 4], f1 = k1 < c1 ? sc[cc1 >> 4] : 0.0;
      dsum = __dadd_rn(dsum, __dmul_rn(f0, tab.F[(cc0 & 15) * 5]));
      if (k1 < c1) dsum = __dadd_rn(dsum, __dmul_rn(f1, tab.F[(cc1 & 15) * 5]));
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) dsum = __dadd_rn(dsum, __shfl_xor_sync(FULL, dsum, o));
    const int nch = __reduce_max_sync(FULL, (L + LPR - 1) / LPR);
    for (int ch = 0; ch < nch; ++ch) {
      const int q = ch * LPR + sub;
      double m = 0.0;
      if (q < L) {
        if (q == dl) {
          m = dsum;
        } else {
          // four list entries and their scales in flight at a time, added in list order
          const int e1 = sl_ptr[rs + q + 1];
          for (int e0 = sl_ptr[rs + q]; e0 < e1; e0 += 4) {
            unsigned u[4];
            double f[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) u[j] = e0 + j < e1 ? sl_ent[e0 + j] : 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) f[j] = e0 + j < e1 ? sc[u[j] >> 4] : 0.0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (e0 + j < e1) m = __dadd_rn(m, __dmul_rn(f[j], tab.F[((u[j] >> 2) & 3u) * 4 + (u[j] & 3u)]));
          }
        }
      }
      // the chunk's 9 * n values: value idx of the chunk is entry idx % 9 of block idx / 9
      const int left = L - ch * LPR;
      const int n = left < LPR ? left : LPR;
      const i64 base = 9 * ((i64)rs + ch * LPR);
#pragma unroll
      for (int it = 0; it < 9; ++it) {
        const int idx = sub + it * LPR;
        const int blk = idx / 9;
        const double mb = __shfl_sync(FULL, m, seg * LPR + (blk < LPR ? blk : LPR - 1));
        if (idx < 9 * n) {
          const double v = (idx - 9 * blk) % 4 == 0 ? mb : 0.0;
          v64[base + idx] = v;
          v32[base + idx] = (float)v;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Dirichlet elimination (poisson.rs:222-263, elasticity.rs:188-227)
// ---------------------------------------------------------------------------

__global__ void k_bc_mark(const i64* __restrict__ dofs, i64 nbc, i64 n, int* __restrict__ count, int* __restrict__ last,
                          int* __restrict__ bad) {
  for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < nbc; j += (i64)gridDim.x * blockDim.x) {
    i64 d = dofs[j];
    if (d < 0 || d >= n) { atomicExch(bad, 1); continue; }
    atomicAdd(&count[d], 1);
    atomicMax(&last[d], (int)j);
  }
}

__global__ void k_bc_flags(const int* __restrict__ count, const int* __restrict__ last, const double* __restrict__ vals,
                           i64 n, unsigned char* __restrict__ dir, double* __restrict__ g, double* __restrict__ dcount) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    int c = count[i];
    if (c > 0) {
      dir[i] = 1;
      g[i] = vals[last[i]];
      dcount[i] = (double)c;
    } else {
      g[i] = 0.0;
    }
  }
}

// Lifting: b_r -= a_rc g_c over eliminated-now columns c in ascending order,
// for rows r not eliminated now (uses values before elimination).
template <int BS>
__global__ void k_bc_lift(const int* __restrict__ row_ptr, const int* __restrict__ col_idx,
                          const double* __restrict__ v64, const int* __restrict__ count, const double* __restrict__ g,
                          i64 nn, double* __restrict__ b) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nn * BS; t += (i64)gridDim.x * blockDim.x) {
    const i64 node = t / BS;
    const int al = (int)(t - node * BS);
    if (count[t] > 0) continue;
    double acc = b[t];
    for (int p = row_ptr[node]; p < row_ptr[node + 1]; ++p) {
      const i64 j = col_idx[p];
#pragma unroll
      for (int be = 0; be < BS; ++be) {
        const i64 c = j * BS + be;
        // explicit roundings: no FMA contraction, same arithmetic as the
        // reference's `new_b[row] -= val * dirichlet_val[col]`
        if (count[c] > 0) acc = __dsub_rn(acc, __dmul_rn(v64[(i64)p * BS * BS + al * BS + be], g[c]));
      }
    }
    b[t] = acc;
  }
}

template <int BS>
__global__ void k_bc_eliminate(const int* __restrict__ row_ptr, const int* __restrict__ col_idx,
                               const int* __restrict__ count, const double* __restrict__ dcount, i64 nn,
                               double* __restrict__ v64, float* __restrict__ v32) {
  const int lane = threadIdx.x & 31;
  const i64 w0 = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
  const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
  for (i64 node = w0; node < nn; node += nw) {
    const int rs = row_ptr[node], re = row_ptr[node + 1];
    for (i64 q = (i64)rs * BS * BS + lane; q < (i64)re * BS * BS; q += 32) {
      const i64 p = q / (BS * BS);
      const int rem = (int)(q - p * BS * BS);
      const i64 r = node * BS + rem / BS;
      const i64 c = (i64)col_idx[p] * BS + rem % BS;
      if (count[r] > 0 || count[c] > 0) {
        const double v = (r == c && count[r] > 0) ? dcount[r] : 0.0;
        v64[q] = v;
        v32[q] = (float)v;
      }
    }
  }
}

__global__ void k_bc_rhs(const int* __restrict__ count, const double* __restrict__ g, i64 n, double* __restrict__ b) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    if (count[i] > 0) b[i] = g[i];
}

__global__ void k_or_mask(const unsigned char* __restrict__ add, i64 n, unsigned char* __restrict__ m) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    if (add[i]) m[i] = 1;
}

// ---------------------------------------------------------------------------
// Adjoint gradient: grad_e = -(3 theta_e^2 E0) lam_e^T K_e^1 u_e with
// lam^T K^1 u = vol (l1 tr(Dl) tr(Du) + m1 (Dl:Du + Dl:Du^T)), D = nodal
// gradient of the field (D[a][b] = sum_i f_{i a} g_i[b]); l1, m1 the Lame
// constants at E = 1.
// ---------------------------------------------------------------------------

__global__ void k_adjoint_grad(const double* __restrict__ X, const int* __restrict__ cells,
                               const unsigned char* __restrict__ valid, i64 nc, double l1, double m1, double E0,
                               const double* __restrict__ theta, const double* __restrict__ u,
                               const double* __restrict__ la, double* __restrict__ grad) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    if (!valid[c]) { grad[c] = 0.0; continue; }
    const int4 q = __ldg(reinterpret_cast<const int4*>(cells) + c);
    const int v[4] = {q.x, q.y, q.z, q.w};
    Geo3 g = tet_geometry(X, v);
    double gr[4][3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      gr[1][r] = g.G[r][0];
      gr[2][r] = g.G[r][1];
      gr[3][r] = g.G[r][2];
      gr[0][r] = -g.G[r][0] - g.G[r][1] - g.G[r][2];
    }
    double Du[3][3] = {{0}}, Dl[3][3] = {{0}};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double* ui = u + 3 * (i64)v[i];
      const double* li = la + 3 * (i64)v[i];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          Du[a][b] += ui[a] * gr[i][b];
          Dl[a][b] += li[a] * gr[i][b];
        }
    }
    double trU = Du[0][0] + Du[1][1] + Du[2][2], trL = Dl[0][0] + Dl[1][1] + Dl[2][2];
    double dd = 0.0, dt = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        dd += Dl[a][b] * Du[a][b];
        dt += Dl[a][b] * Du[b][a];
      }
    const double vol = (1.0 / 6.0) * fabs(g.det);
    const double s = vol * (l1 * trL * trU + m1 * (dd + dt));
    const double th = theta[c];
    grad[c] = -(3.0 * th * th * E0) * s;
  }
}

bool g_p2_tables_ready[64] = {false};

void ensure_p2_tables(fcu_ctx ctx) {
  if (g_p2_tables_ready[ctx->device & 63]) return;
  // Degree-2 Keast rule (quadrature.rs:157-183) and P2 gradients
  // (lagrange.rs:324-346): R^{de}_{ab} = sum_q w_q d_d phi_a(xi_q) d_e phi_b(xi_q).
  const double s5 = std::sqrt(5.0);
  const double A = (5.0 - s5) / 20.0, B = (5.0 + 3.0 * s5) / 20.0, W = 1.0 / 24.0;
  const double P[4][3] = {{A, A, A}, {B, A, A}, {A, B, A}, {A, A, B}};
  double Rde[3][3][10][10] = {};
  for (int q = 0; q < 4; ++q) {
    double x = P[q][0], y = P[q][1], z = P[q][2];
    double l0 = 1.0 - x - y - z, l1 = x, l2 = y, l3 = z;
    double G[10][3] = {{-(4 * l0 - 1), -(4 * l0 - 1), -(4 * l0 - 1)},
                       {4 * l1 - 1, 0, 0},
                       {0, 4 * l2 - 1, 0},
                       {0, 0, 4 * l3 - 1},
                       {4 * (l0 - l1), -4 * l1, -4 * l1},
                       {4 * l2, 4 * l1, 0},
                       {-4 * l2, 4 * (l0 - l2), -4 * l2},
                       {-4 * l3, -4 * l3, 4 * (l0 - l3)},
                       {4 * l3, 0, 4 * l1},
                       {0, 4 * l3, 4 * l2}};
    for (int d = 0; d < 3; ++d)
      for (int e = 0; e < 3; ++e)
        for (int a = 0; a < 10; ++a)
          for (int b = 0; b < 10; ++b) Rde[d][e][a][b] += W * G[a][d] * G[b][e];
  }
  double R[6][10][10];
  const int D[6] = {0, 1, 2, 0, 0, 1}, E[6] = {0, 1, 2, 1, 2, 2};
  for (int m = 0; m < 6; ++m)
    for (int a = 0; a < 10; ++a)
      for (int b = 0; b < 10; ++b)
        R[m][a][b] = (m < 3) ? Rde[D[m]][E[m]][a][b] : Rde[D[m]][E[m]][a][b] + Rde[E[m]][D[m]][a][b];
  CUDA_CHECK(cudaMemcpyToSymbol(c_p2_R, R, sizeof(R)));
  g_p2_tables_ready[ctx->device & 63] = true;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host entry points (called from api.cu)
// ---------------------------------------------------------------------------

// FCU_P2_ROWGATHER=1 selects the slot-list P2 kernel (kept as the comparison).
bool p2_row_gather() {
  static const bool v = [] {
    const char* e = getenv("FCU_P2_ROWGATHER");
    return e && atoi(e) != 0;
  }();
  return v;
}

// FCU_ELAST_KERNEL selects the elasticity kernel: 0 = row form over the
// gradient records (default), 1 = block-parallel form, 2 = row-gather with
// per-contribution geometry (kept as comparisons).
int elasticity_kernel() {
  static const int v = [] {
    const char* e = getenv("FCU_ELAST_KERNEL");
    return e ? atoi(e) : 0;
  }();
  return v;
}

int assembly_blocks(fcu_ctx ctx, i64 rows, int warps = WARPS) {
  i64 need = (rows + warps - 1) / warps;
  i64 cap = (i64)ctx->num_sms * 8;
  return (int)std::max<i64>(1, std::min(need, cap));
}

void assemble_stiffness_impl(fcu_matrix m, const double* coef_dev) {
  fcu_space s = m->space;
  fcu_ctx ctx = m->ctx;
  fcu_mesh me = s->mesh;
  const int nb = assembly_blocks(ctx, s->nnodes);
  if (s->kind == FCU_SPACE_P2 || s->kind == FCU_SPACE_P2_NODES) {
    ensure_p2_tables(ctx);
    DBuf<double> geo;
    geo.alloc((size_t)me->nc * P2_GEO);
    k_p2_metric_records<<<grid_for(me->nc, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(
        s->cell_nodes.p, me->coords.p, coef_dev, me->nc, geo.p);
    LAUNCH_CHECK(ctx);
    if (s->cmap.p && s->contrib_a.p && !p2_row_gather()) {
      const int stride = s->max_row | 1;  // odd, so the three rows' accumulators start in different banks
      const size_t smem = (600 + (size_t)P2W * 3 * stride) * sizeof(double);
      static bool attr_set[64] = {};
      if (smem > 48 * 1024 && !attr_set[ctx->device & 63]) {
        CUDA_CHECK(cudaFuncSetAttribute(k_assemble_p2_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        attr_set[ctx->device & 63] = true;
      }
      const i64 groups = (s->nnodes + 3 * P2W - 1) / (3 * P2W);
      const int nbp = (int)std::max<i64>(1, std::min<i64>(groups, (i64)ctx->num_sms * 8));
      k_assemble_p2_rows<<<nbp, P2W * 32, smem, ctx->stream>>>(s->row_ptr.p, s->contrib_ptr.p, s->contrib_a.p,
                                                                s->cmap.p, geo.p, s->nnodes, stride, m->val64.p,
                                                                m->val32.p);
      LAUNCH_CHECK(ctx);
      return;
    }
    k_assemble_scalar<10, 3, true><<<nb, WARPS * 32, 0, ctx->stream>>>(
        s->row_ptr.p, s->contrib_ptr.p, s->contrib.p, s->slot_cnt.p, s->slot_ent.p, s->cell_nodes.p, me->coords.p,
        coef_dev, geo.p, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  } else if (me->dim == 3) {
    k_assemble_scalar<4, 3, false><<<nb, WARPS * 32, 0, ctx->stream>>>(
        s->row_ptr.p, s->contrib_ptr.p, s->contrib.p, s->slot_cnt.p, s->slot_ent.p, s->cell_nodes.p, me->coords.p,
        coef_dev, nullptr, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  } else {
    k_assemble_scalar<3, 2, false><<<nb, WARPS * 32, 0, ctx->stream>>>(
        s->row_ptr.p, s->contrib_ptr.p, s->contrib.p, s->slot_cnt.p, s->slot_ent.p, s->cell_nodes.p, me->coords.p,
        coef_dev, nullptr, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  }
  LAUNCH_CHECK(ctx);
}

void assemble_elasticity_impl(fcu_matrix m, double E, double nu, const double* cellE_dev) {
  fcu_space s = m->space;
  fcu_ctx ctx = m->ctx;
  // ElasticMaterial::lame_lambda / lame_mu (elasticity.rs:33-47)
  const double Eref = cellE_dev ? 1.0 : E;
  const double lam = (Eref * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double mu = Eref / (2.0 * (1.0 + nu));
  const int mode = elasticity_kernel();
  if (mode == 2) {
    const int nb = assembly_blocks(ctx, s->nnodes, EWARPS);
    k_assemble_elasticity<<<nb, EWARPS * 32, 0, ctx->stream>>>(s->row_ptr.p, s->contrib_ptr.p, s->contrib.p,
                                                              s->slot_cnt.p, s->slot_ent.p, s->cell_nodes.p,
                                                              s->mesh->coords.p, cellE_dev, lam, mu, s->diag_pos.p,
                                                              s->nnodes, m->val64.p, m->val32.p);
    LAUNCH_CHECK(ctx);
    return;
  }
  fcu_mesh me = s->mesh;
  if (!s->cell_rec.p) s->cell_rec.alloc((size_t)me->nc * 16);
  if (me->nc) {
    k_elast_records<<<grid_for((me->nc + 31) / 32 * 32, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
        s->cell_nodes.p, me->coords.p, me->valid.p, cellE_dev, me->nc, s->cell_rec.p);
    LAUNCH_CHECK(ctx);
  }
  if (mode == 0) {
    const i64 rows_per_block = 8 * (s->max_row <= 16 ? 2 : 1);
    const i64 need = (s->nnodes + rows_per_block - 1) / rows_per_block;
    const int nbr = (int)std::max<i64>(1, std::min<i64>(need, (i64)ctx->num_sms * 8));
    if (s->max_row <= 16)
      k_elast_rows<16><<<nbr, 256, 0, ctx->stream>>>(s->row_ptr.p, s->diag_pos.p, s->sl_ptr.p, s->sl_ent.p,
                                                      s->cell_rec.p, s->nnodes, lam, mu, m->val64.p, m->val32.p);
    else
      k_elast_rows<32><<<nbr, 256, 0, ctx->stream>>>(s->row_ptr.p, s->diag_pos.p, s->sl_ptr.p, s->sl_ent.p,
                                                      s->cell_rec.p, s->nnodes, lam, mu, m->val64.p, m->val32.p);
    LAUNCH_CHECK(ctx);
    return;
  }
  const i64 work = s->nup + s->nnodes;
  if (work) {
    k_elast_blocks<<<(unsigned)((work + 255) / 256), 256, 0, ctx->stream>>>(
        s->nup, s->up_ptr.p, s->up_ent.p, s->up_slot.p, s->up_tslot.p, s->nnodes, s->contrib_ptr.p, s->contrib.p,
        s->diag_pos.p, s->cell_rec.p, lam, mu, m->val64.p, m->val32.p);
    LAUNCH_CHECK(ctx);
  }
}

// FCU_MASS_ROWGATHER=1 keeps the row-gather mass kernel on vector P1 spaces
// (for comparison).
bool mass_row_gather() {
  static const bool v = [] {
    const char* e = getenv("FCU_MASS_ROWGATHER");
    return e && atoi(e) != 0;
  }();
  return v;
}

void assemble_mass_impl(fcu_matrix m, double rho, const double* coef_dev) {
  fcu_space s = m->space;
  fcu_ctx ctx = m->ctx;
  fcu_mesh me = s->mesh;
  MassTable tab{};
  const bool p2 = s->kind == FCU_SPACE_P2 || s->kind == FCU_SPACE_P2_NODES || s->kind == FCU_SPACE_P2_NODES_VEC3;
  if (p2) {
    p2_mass_products(tab.F);
  } else {
    const int K = s->k;
    const double dg = (K == 3) ? 1.0 / 6.0 : 1.0 / 10.0, od = (K == 3) ? 1.0 / 12.0 : 1.0 / 20.0;
    for (int a = 0; a < K; ++a)
      for (int b = 0; b < K; ++b) tab.F[a * K + b] = (a == b) ? dg : od;
  }
  const int nb = assembly_blocks(ctx, s->nnodes);
  const int* cn = s->cell_nodes.p;
  const double* X = me->coords.p;
  if (s->kind == FCU_SPACE_P2_NODES_VEC3) {
    k_assemble_mass<10, 3, 3><<<nb, WARPS * 32, 0, ctx->stream>>>(s->row_ptr.p, s->contrib_ptr.p, s->contrib.p,
                                                                   s->slot_cnt.p, s->slot_ent.p, cn, X, coef_dev, rho,
                                                                   tab, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  } else if (p2) {
    k_assemble_mass<10, 3, 1><<<nb, WARPS * 32, 0, ctx->stream>>>(s->row_ptr.p, s->contrib_ptr.p, s->contrib.p,
                                                                   s->slot_cnt.p, s->slot_ent.p, cn, X, coef_dev, rho,
                                                                   tab, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  } else if (s->kind == FCU_SPACE_P1_VEC3 && s->sl_ptr.p && !mass_row_gather()) {
    DBuf<double> scales;
    scales.alloc(std::max<i64>(me->nc, 1));
    if (me->nc) {
      k_mass_scales<<<grid_for(me->nc, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(cn, X, coef_dev, rho, me->nc,
                                                                                     scales.p);
      LAUNCH_CHECK(ctx);
    }
    const int lpr = s->max_row <= 16 ? 16 : 32;
    const i64 need = (s->nnodes + 8 * (32 / lpr) - 1) / (8 * (32 / lpr));
    const int nbr = (int)std::max<i64>(1, std::min<i64>(need, (i64)ctx->num_sms * 8));
    if (lpr == 16)
      k_mass_rows_vec<16><<<nbr, 256, 0, ctx->stream>>>(s->row_ptr.p, s->diag_pos.p, s->sl_ptr.p, s->sl_ent.p,
                                                         s->contrib_ptr.p, s->contrib.p, scales.p, tab, s->nnodes,
                                                         m->val64.p, m->val32.p);
    else
      k_mass_rows_vec<32><<<nbr, 256, 0, ctx->stream>>>(s->row_ptr.p, s->diag_pos.p, s->sl_ptr.p, s->sl_ent.p,
                                                         s->contrib_ptr.p, s->contrib.p, scales.p, tab, s->nnodes,
                                                         m->val64.p, m->val32.p);
  } else if (s->kind == FCU_SPACE_P1_VEC3) {
    k_assemble_mass<4, 3, 3><<<nb, WARPS * 32, 0, ctx->stream>>>(s->row_ptr.p, s->contrib_ptr.p, s->contrib.p,
                                                                  s->slot_cnt.p, s->slot_ent.p, cn, X, coef_dev, rho,
                                                                  tab, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  } else if (me->dim == 3) {
    k_assemble_mass<4, 3, 1><<<nb, WARPS * 32, 0, ctx->stream>>>(s->row_ptr.p, s->contrib_ptr.p, s->contrib.p,
                                                                  s->slot_cnt.p, s->slot_ent.p, cn, X, coef_dev, rho,
                                                                  tab, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  } else {
    k_assemble_mass<3, 2, 1><<<nb, WARPS * 32, 0, ctx->stream>>>(s->row_ptr.p, s->contrib_ptr.p, s->contrib.p,
                                                                  s->slot_cnt.p, s->slot_ent.p, cn, X, coef_dev, rho,
                                                                  tab, s->diag_pos.p, s->nnodes, m->val64.p, m->val32.p);
  }
  LAUNCH_CHECK(ctx);
}

void apply_dirichlet_impl(fcu_matrix m, double* b_dev, i64 nbc, const i64* dofs_dev, const double* vals_dev) {
  fcu_ctx ctx = m->ctx;
  const i64 n = m->n, nn = m->nnodes;
  const int cap = ctx->num_sms * 16;
  DBuf<int> count, last, bad;
  DBuf<double> g;
  DBuf<unsigned char> dnow;
  count.alloc(n); last.alloc(n); bad.alloc(1); g.alloc(n); dnow.alloc(n);
  if (!m->dirichlet.p) {
    m->dirichlet.alloc(n);
    CUDA_CHECK(cudaMemsetAsync(m->dirichlet.p, 0, n, ctx->stream));
    m->diag_count.alloc(n);
  }
  CUDA_CHECK(cudaMemsetAsync(count.p, 0, n * sizeof(int), ctx->stream));
  CUDA_CHECK(cudaMemsetAsync(last.p, 0xff, n * sizeof(int), ctx->stream));
  CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
  CUDA_CHECK(cudaMemsetAsync(dnow.p, 0, n, ctx->stream));
  if (nbc > 0) {
    k_bc_mark<<<grid_for(nbc, 256, cap), 256, 0, ctx->stream>>>(dofs_dev, nbc, n, count.p, last.p, bad.p);
    LAUNCH_CHECK(ctx);
  }
  int hbad = 0;
  CUDA_CHECK(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  if (hbad) fail(FCU_ERR_BAD_ARG, "Dirichlet dof index out of range");
  k_bc_flags<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(count.p, last.p, vals_dev, n, dnow.p, g.p,
                                                             m->diag_count.p);
  LAUNCH_CHECK(ctx);
  if (m->bs == 3) {
    k_bc_lift<3><<<grid_for(n, 128, cap), 128, 0, ctx->stream>>>(m->row_ptr, m->col_idx, m->val64.p, count.p, g.p, nn, b_dev);
    LAUNCH_CHECK(ctx);
    k_bc_eliminate<3><<<grid_for(nn * 32, 256, cap), 256, 0, ctx->stream>>>(m->row_ptr, m->col_idx, count.p,
                                                                             m->diag_count.p, nn, m->val64.p, m->val32.p);
  } else {
    k_bc_lift<1><<<grid_for(n, 128, cap), 128, 0, ctx->stream>>>(m->row_ptr, m->col_idx, m->val64.p, count.p, g.p, nn, b_dev);
    LAUNCH_CHECK(ctx);
    k_bc_eliminate<1><<<grid_for(nn * 32, 256, cap), 256, 0, ctx->stream>>>(m->row_ptr, m->col_idx, count.p,
                                                                             m->diag_count.p, nn, m->val64.p, m->val32.p);
  }
  LAUNCH_CHECK(ctx);
  k_bc_rhs<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(count.p, g.p, n, b_dev);
  LAUNCH_CHECK(ctx);
  k_or_mask<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(dnow.p, n, m->dirichlet.p);
  LAUNCH_CHECK(ctx);
  std::vector<unsigned char> hm(n);
  CUDA_CHECK(cudaMemcpyAsync(hm.data(), m->dirichlet.p, n, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  i64 nd = 0;
  for (unsigned char v : hm) nd += v;
  m->n_dirichlet = nd;
  m->bc_applied = true;
}

void adjoint_gradient_impl(fcu_space s, double E0, double nu, const double* theta, const double* u, const double* la,
                           double* grad) {
  fcu_ctx ctx = s->ctx;
  fcu_mesh me = s->mesh;
  const double l1 = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double m1 = 1.0 / (2.0 * (1.0 + nu));
  k_adjoint_grad<<<grid_for(me->nc, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(
      me->coords.p, me->cells.p, me->valid.p, me->nc, l1, m1, E0, theta, u, la, grad);
  LAUNCH_CHECK(ctx);
}
