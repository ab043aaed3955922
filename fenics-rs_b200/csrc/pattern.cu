// Setup kernels: cell validity, P2 edge numbering, the node-level sparsity
// pattern and the row-gather maps used by the assembly kernels.
//
// The pattern reproduces faer's triplet -> CSC result for the reference
// assemblers (poisson.rs:68, elasticity.rs:148): it is the union of the
// (row, col) pairs of every non-degenerate cell, with explicit zeros kept.
// Diagonal slots are always stored (needed for Dirichlet rows); a diagonal
// that no cell produced is marked by slot_cnt == 0 and left out of exports.
//
// Instead of a cell -> nnz scatter map, each row stores the list of its
// contributing (cell, local node) pairs in ascending cell order, and each slot
// the (contribution, local column) pairs that sum into it, also in cell order.
// The assembly kernels then reduce every row in on-chip memory and write each
// value once, with no atomics.

#include <cub/cub.cuh>

#include "internal.cuh"

namespace {

__global__ void k_validity_tet(const double* __restrict__ X, const int* __restrict__ cells, i64 nc,
                               unsigned char* __restrict__ valid) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    int v[4] = {cells[4 * c], cells[4 * c + 1], cells[4 * c + 2], cells[4 * c + 3]};
    valid[c] = tet_geometry(X, v).ok ? 1 : 0;
  }
}

__global__ void k_validity_tri(const double* __restrict__ X, const int* __restrict__ cells, i64 nc,
                               unsigned char* __restrict__ valid) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    int v[3] = {cells[3 * c], cells[3 * c + 1], cells[3 * c + 2]};
    valid[c] = tri_geometry(X, v).ok ? 1 : 0;
  }
}

// P2 local edges in P2Tetrahedron order: 01, 12, 02, 03, 13, 23.
__constant__ int c_p2_edge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};

__global__ void k_edge_keys(const int* __restrict__ cells, i64 nc, i64 nv, unsigned long long* __restrict__ keys) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < 6 * nc; t += (i64)gridDim.x * blockDim.x) {
    i64 c = t / 6;
    int e = (int)(t % 6);
    i64 a = cells[4 * c + c_p2_edge[e][0]], b = cells[4 * c + c_p2_edge[e][1]];
    i64 lo = a < b ? a : b, hi = a < b ? b : a;
    keys[t] = (unsigned long long)(lo * nv + hi);
  }
}

__global__ void k_unique_flags(const unsigned long long* __restrict__ keys, i64 n, unsigned long long sentinel,
                               int* __restrict__ flags) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
    unsigned long long k = keys[t];
    flags[t] = (k != sentinel && (t == 0 || keys[t - 1] != k)) ? 1 : 0;
  }
}

__global__ void k_scatter_unique(const unsigned long long* __restrict__ keys, const int* __restrict__ flags,
                                 const int* __restrict__ pos, i64 n, unsigned long long* __restrict__ out) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x)
    if (flags[t]) out[pos[t]] = keys[t];
}

__device__ __forceinline__ i64 lower_bound_u64(const unsigned long long* a, i64 n, unsigned long long key) {
  i64 lo = 0, hi = n;
  while (lo < hi) {
    i64 mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void k_p2_cell_dofs(const int* __restrict__ cells, i64 nc, i64 nv, const unsigned long long* __restrict__ edges,
                               i64 ne, int* __restrict__ cd) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    int v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) { v[i] = cells[4 * c + i]; cd[10 * c + i] = v[i]; }
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      i64 a = v[c_p2_edge[e][0]], b = v[c_p2_edge[e][1]];
      i64 lo = a < b ? a : b, hi = a < b ? b : a;
      cd[10 * c + 4 + e] = (int)(nv + lower_bound_u64(edges, ne, (unsigned long long)(lo * nv + hi)));
    }
  }
}

__global__ void k_edge_verts(const unsigned long long* __restrict__ edges, i64 ne, i64 nv, int* __restrict__ ev) {
  for (i64 e = blockIdx.x * (i64)blockDim.x + threadIdx.x; e < ne; e += (i64)gridDim.x * blockDim.x) {
    ev[2 * e] = (int)(edges[e] / nv);
    ev[2 * e + 1] = (int)(edges[e] % nv);
  }
}

// One entry per (valid cell, a, b) plus one marker per diagonal.
// value = emission index (cell*k*k + a*k + b) or 0xFFFFFFFF for markers.
__global__ void k_emit_pairs(const int* __restrict__ cn, const unsigned char* __restrict__ valid, i64 nc, int k,
                             i64 nn, unsigned long long sentinel, unsigned long long* __restrict__ keys,
                             unsigned* __restrict__ vals) {
  const i64 kk = (i64)k * k;
  const i64 total = nc * kk + nn;
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total; t += (i64)gridDim.x * blockDim.x) {
    if (t < nc * kk) {
      i64 c = t / kk;
      int a = (int)((t / k) % k), b = (int)(t % k);
      if (valid[c]) {
        i64 i = cn[c * k + a], j = cn[c * k + b];
        keys[t] = (unsigned long long)(i * nn + j);
      } else {
        keys[t] = sentinel;
      }
      vals[t] = (unsigned)t;
    } else {
      i64 i = t - nc * kk;
      keys[t] = (unsigned long long)(i * nn + i);
      vals[t] = 0xFFFFFFFFu;
    }
  }
}

// For sorted entries: slot index (inclusive scan of flags - 1), real-entry
// flags for compaction, slot first entry, column, row starts, slot counts.
__global__ void k_pattern_fill(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ vals,
                               const int* __restrict__ flags, const int* __restrict__ slot_incl, i64 nE, i64 nn,
                               unsigned long long sentinel, int* __restrict__ col_idx, int* __restrict__ row_ptr,
                               int* __restrict__ slot_first, unsigned* __restrict__ cnt32,
                               int* __restrict__ diag_pos, int* __restrict__ real) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nE; t += (i64)gridDim.x * blockDim.x) {
    unsigned long long key = keys[t];
    if (key == sentinel) { real[t] = 0; continue; }
    int s = slot_incl[t] - 1;
    i64 i = (i64)(key / nn), j = (i64)(key % nn);
    bool is_marker = vals[t] == 0xFFFFFFFFu;
    real[t] = is_marker ? 0 : 1;
    if (flags[t]) {
      col_idx[s] = (int)j;
      slot_first[s] = (int)t;
      if (i == j) diag_pos[i] = s;
      // first slot of row i: previous slot belongs to a smaller row
      bool row_start = (t == 0) || (keys[t - 1] / nn != (unsigned long long)i);
      if (row_start) row_ptr[i] = s;
    }
    if (!is_marker) atomicAdd(&cnt32[s], 1u);
  }
}

__global__ void k_contrib_counts(const unsigned* __restrict__ cnt32, const int* __restrict__ diag_pos, i64 nn,
                                 int* __restrict__ ccount) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nn; i += (i64)gridDim.x * blockDim.x)
    ccount[i] = (int)cnt32[diag_pos[i]];
}

__global__ void k_contrib_fill(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ vals,
                               const int* __restrict__ slot_incl, const int* __restrict__ slot_first, i64 nE, i64 nn,
                               int k, unsigned long long sentinel, const int* __restrict__ contrib_ptr,
                               int* __restrict__ contrib) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nE; t += (i64)gridDim.x * blockDim.x) {
    unsigned long long key = keys[t];
    if (key == sentinel) continue;
    unsigned v = vals[t];
    if (v == 0xFFFFFFFFu) continue;
    i64 i = (i64)(key / nn), j = (i64)(key % nn);
    if (i != j) continue;
    i64 kk = (i64)k * k;
    i64 c = v / kk;
    int a = (int)((v / k) % k);
    int b = (int)(v % k);
    if (a != b) continue;  // a repeated vertex would add a second (i,i) pair
    int s = slot_incl[t] - 1;
    contrib[contrib_ptr[i] + (t - slot_first[s])] = (int)((c << 4) | a);
  }
}

__global__ void k_slot_entries(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ vals,
                               const int* __restrict__ real_excl, i64 nE, i64 nn, int k, unsigned long long sentinel,
                               const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
                               unsigned short* __restrict__ ent, int* __restrict__ overflow) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nE; t += (i64)gridDim.x * blockDim.x) {
    unsigned long long key = keys[t];
    if (key == sentinel) continue;
    unsigned v = vals[t];
    if (v == 0xFFFFFFFFu) continue;
    i64 i = (i64)(key / nn);
    i64 kk = (i64)k * k;
    int c = (int)(v / kk);
    int b = (int)(v % k);
    int lo = contrib_ptr[i], hi = contrib_ptr[i + 1];
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if ((contrib[mid] >> 4) < c) lo = mid + 1;
      else hi = mid;
    }
    int tl = lo - contrib_ptr[i];
    if (tl >= 4096) atomicExch(overflow, 1);
    ent[real_excl[t]] = (unsigned short)((tl << 4) | b);
  }
}

// Upper off-diagonal block lists (vector P1). On the sorted (row, col)
// pairs: one flag per cell entry with col > row; on the slots: one flag per
// slot with col > row.
__global__ void k_up_entry_flags(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ vals,
                                 i64 nE, i64 nn, unsigned long long sentinel, int* __restrict__ f) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nE; t += (i64)gridDim.x * blockDim.x) {
    const unsigned long long key = keys[t];
    f[t] = (key != sentinel && vals[t] != 0xFFFFFFFFu && key % nn > key / nn) ? 1 : 0;
  }
}

__global__ void k_off_entry_flags(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ vals,
                                  i64 nE, i64 nn, unsigned long long sentinel, int* __restrict__ f) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nE; t += (i64)gridDim.x * blockDim.x) {
    const unsigned long long key = keys[t];
    f[t] = (key != sentinel && vals[t] != 0xFFFFFFFFu && key % nn != key / nn) ? 1 : 0;
  }
}

__global__ void k_slot_list_ptr(const int* __restrict__ slot_first, const int* __restrict__ epos, i64 nnzb,
                                int* __restrict__ sl_ptr) {
  for (i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x; s < nnzb; s += (i64)gridDim.x * blockDim.x)
    sl_ptr[s] = epos[slot_first[s]];
}

__global__ void k_up_slot_flags(const unsigned long long* __restrict__ keys, const int* __restrict__ slot_first,
                                i64 nnzb, i64 nn, int* __restrict__ f) {
  for (i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x; s < nnzb; s += (i64)gridDim.x * blockDim.x) {
    const unsigned long long key = keys[slot_first[s]];
    f[s] = key % nn > key / nn ? 1 : 0;
  }
}

__global__ void k_up_fill_slots(const int* __restrict__ sflag, const int* __restrict__ sid,
                                const int* __restrict__ slot_first, const int* __restrict__ epos, i64 nnzb,
                                int* __restrict__ up_slot, int* __restrict__ up_ptr) {
  for (i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x; s < nnzb; s += (i64)gridDim.x * blockDim.x) {
    if (!sflag[s]) continue;
    const int u = sid[s];
    up_slot[u] = (int)s;
    up_ptr[u] = epos[slot_first[s]];
  }
}

__global__ void k_up_fill_entries(const unsigned* __restrict__ vals, const int* __restrict__ eflag,
                                  const int* __restrict__ epos, i64 nE, unsigned* __restrict__ ent) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nE; t += (i64)gridDim.x * blockDim.x) {
    if (!eflag[t]) continue;
    ent[epos[t]] = vals[t];  // the emission index cell*16 + a*4 + b (k = 4) is the packed entry
  }
}

// Position of the transposed block of each upper block (binary search in row j).
__global__ void k_up_tslot(const int* __restrict__ row_ptr, const int* __restrict__ col_idx,
                           const int* __restrict__ up_slot, const unsigned long long* __restrict__ keys,
                           const int* __restrict__ slot_first, i64 nup, i64 nn, int* __restrict__ up_tslot) {
  for (i64 u = blockIdx.x * (i64)blockDim.x + threadIdx.x; u < nup; u += (i64)gridDim.x * blockDim.x) {
    const int p = up_slot[u];
    const unsigned long long key = keys[slot_first[p]];
    const int i = (int)(key / nn), j = (int)(key % nn);
    int lo = row_ptr[j], hi = row_ptr[j + 1];
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (col_idx[mid] < i) lo = mid + 1;
      else hi = mid;
    }
    up_tslot[u] = (lo < row_ptr[j + 1] && col_idx[lo] == i) ? lo : -1;
  }
}

// Per-contribution slot map (P2 scalar): entry (i, j) of cell c with local
// indices (a, b) is column b of contribution (c, a) of row i.
__global__ void k_contrib_slot_map(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ vals,
                                   const int* __restrict__ slot_incl, i64 nE, i64 nn, int k,
                                   unsigned long long sentinel, const int* __restrict__ row_ptr,
                                   const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
                                   unsigned char* __restrict__ cmap) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nE; t += (i64)gridDim.x * blockDim.x) {
    const unsigned long long key = keys[t];
    if (key == sentinel) continue;
    const unsigned v = vals[t];
    if (v == 0xFFFFFFFFu) continue;
    const i64 i = (i64)(key / nn);
    const i64 kk = (i64)k * k;
    const int c = (int)(v / kk);
    const int b = (int)(v % k);
    int lo = contrib_ptr[i], hi = contrib_ptr[i + 1];
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((contrib[mid] >> 4) < c) lo = mid + 1;
      else hi = mid;
    }
    cmap[(i64)lo * k + b] = (unsigned char)(slot_incl[t] - 1 - row_ptr[i]);
  }
}

// P2 contributions reordered by (row, local index of the row's dof, cell),
// so that the assembly kernel can keep one reference-tensor row in
// registers across the contributions that share it.
__global__ void k_contrib_sort_keys(const int* __restrict__ contrib_ptr, const int* __restrict__ contrib, i64 nn,
                                    unsigned long long* __restrict__ keys, int* __restrict__ idx) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nn; i += (i64)gridDim.x * blockDim.x)
    for (int t = contrib_ptr[i]; t < contrib_ptr[i + 1]; ++t) {
      const unsigned cc = (unsigned)contrib[t];
      keys[t] = ((unsigned long long)i << 32) | ((unsigned long long)(cc & 15u) << 28) | (cc >> 4);
      idx[t] = t;
    }
}

__global__ void k_contrib_permute(const int* __restrict__ order, const int* __restrict__ contrib,
                                  const unsigned char* __restrict__ cmap, i64 nct, int k,
                                  int* __restrict__ contrib_a, unsigned char* __restrict__ cmap_a) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nct; t += (i64)gridDim.x * blockDim.x) {
    const int src = order[t];
    contrib_a[t] = contrib[src];
    for (int b = 0; b < k; ++b) cmap_a[t * k + b] = cmap[(i64)src * k + b];
  }
}

__global__ void k_u32_to_u16(const unsigned* __restrict__ a, i64 n, unsigned short* __restrict__ b,
                             int* __restrict__ overflow) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
    unsigned v = a[t];
    if (v > 65535u) atomicExch(overflow, 1);
    b[t] = (unsigned short)v;
  }
}

__global__ void k_tpos(const int* __restrict__ row_ptr, const int* __restrict__ col_idx, i64 nn, int* __restrict__ tpos) {
  // one thread per row, walks its slots; binary search in the transposed row
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nn; i += (i64)gridDim.x * blockDim.x) {
    for (int p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
      int j = col_idx[p];
      int lo = row_ptr[j], hi = row_ptr[j + 1];
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (col_idx[mid] < i) lo = mid + 1;
        else hi = mid;
      }
      tpos[p] = (lo < row_ptr[j + 1] && col_idx[lo] == (int)i) ? lo : -1;
    }
  }
}

int bit_length(unsigned long long v) {
  int b = 0;
  while (v) { ++b; v >>= 1; }
  return b;
}

}  // namespace

void build_mesh_validity(fcu_mesh m) {
  fcu_ctx ctx = m->ctx;
  m->valid.alloc(m->nc);
  if (m->nc == 0) { m->n_degenerate = 0; return; }
  unsigned g = grid_for(m->nc, 256, 148 * 16);
  if (m->dim == 3) k_validity_tet<<<g, 256, 0, ctx->stream>>>(m->coords.p, m->cells.p, m->nc, m->valid.p);
  else k_validity_tri<<<g, 256, 0, ctx->stream>>>(m->coords.p, m->cells.p, m->nc, m->valid.p);
  LAUNCH_CHECK(ctx);
  std::vector<unsigned char> hv(m->nc);
  CUDA_CHECK(cudaMemcpyAsync(hv.data(), m->valid.p, m->nc, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  i64 bad = 0;
  for (unsigned char v : hv) bad += (v == 0);
  m->n_degenerate = bad;
}

template <class T>
static void exclusive_scan(fcu_ctx ctx, const T* in, T* out, i64 n) {
  size_t tb = 0;
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, ctx->stream));
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(ctx->temp_bytes(tb), tb, in, out, (int)n, ctx->stream));
}
template <class T>
static void inclusive_scan(fcu_ctx ctx, const T* in, T* out, i64 n) {
  size_t tb = 0;
  CUDA_CHECK(cub::DeviceScan::InclusiveSum(nullptr, tb, in, out, (int)n, ctx->stream));
  CUDA_CHECK(cub::DeviceScan::InclusiveSum(ctx->temp_bytes(tb), tb, in, out, (int)n, ctx->stream));
}

template <class T>
static T read_scalar(fcu_ctx ctx, const T* dev) {
  T h;
  CUDA_CHECK(cudaMemcpyAsync(&h, dev, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  return h;
}

void build_space_pattern(fcu_space s) {
  fcu_ctx ctx = s->ctx;
  fcu_mesh m = s->mesh;
  const int cap = ctx->num_sms * 16;
  if (m->n_degenerate < 0) build_mesh_validity(m);
  const i64 nc = m->nc, nv = m->nv;

  // --- cell -> node map -----------------------------------------------------
  if (s->kind == FCU_SPACE_P2_NODES || s->kind == FCU_SPACE_P2_NODES_VEC3) {
    // the caller's ten nodes per cell are already in cell_nodes
    s->k = 10;
    s->nnodes = nv;
    s->bs = s->kind == FCU_SPACE_P2_NODES_VEC3 ? 3 : 1;
  } else if (s->kind == FCU_SPACE_P2) {
    s->k = 10;
    i64 ne6 = 6 * nc;
    DBuf<unsigned long long> ek, eks;
    ek.alloc(ne6);
    eks.alloc(ne6);
    k_edge_keys<<<grid_for(ne6, 256, cap), 256, 0, ctx->stream>>>(m->cells.p, nc, nv, ek.p);
    LAUNCH_CHECK(ctx);
    size_t tb = 0;
    int ebits = bit_length((unsigned long long)(nv * nv));
    CUDA_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, tb, ek.p, eks.p, (int)ne6, 0, ebits, ctx->stream));
    CUDA_CHECK(cub::DeviceRadixSort::SortKeys(ctx->temp_bytes(tb), tb, ek.p, eks.p, (int)ne6, 0, ebits, ctx->stream));
    DBuf<int> fl, pos;
    fl.alloc(ne6);
    pos.alloc(ne6);
    k_unique_flags<<<grid_for(ne6, 256, cap), 256, 0, ctx->stream>>>(eks.p, ne6, ~0ull, fl.p);
    LAUNCH_CHECK(ctx);
    exclusive_scan(ctx, fl.p, pos.p, ne6);
    i64 ne = ne6 ? (i64)read_scalar(ctx, pos.p + ne6 - 1) + read_scalar(ctx, fl.p + ne6 - 1) : 0;
    k_scatter_unique<<<grid_for(ne6, 256, cap), 256, 0, ctx->stream>>>(eks.p, fl.p, pos.p, ne6, ek.p);
    LAUNCH_CHECK(ctx);
    s->nedges = ne;
    s->edge_verts.alloc(2 * ne);
    if (ne) {
      k_edge_verts<<<grid_for(ne, 256, cap), 256, 0, ctx->stream>>>(ek.p, ne, nv, s->edge_verts.p);
      LAUNCH_CHECK(ctx);
    }
    s->cell_nodes.alloc(10 * nc);
    if (nc) {
      k_p2_cell_dofs<<<grid_for(nc, 256, cap), 256, 0, ctx->stream>>>(m->cells.p, nc, nv, ek.p, ne, s->cell_nodes.p);
      LAUNCH_CHECK(ctx);
    }
    s->nnodes = nv + ne;
    s->bs = 1;
  } else {
    s->k = m->nodes;
    s->cell_nodes.alloc(nc * s->k);
    if (nc) CUDA_CHECK(cudaMemcpyAsync(s->cell_nodes.p, m->cells.p, nc * s->k * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
    s->nnodes = nv;
    s->bs = (s->kind == FCU_SPACE_P1_VEC3) ? 3 : 1;
  }
  s->ndofs = s->nnodes * s->bs;
  const i64 nn = s->nnodes;
  const int k = s->k;

  // --- (row, col) pairs -------------------------------------------------------
  const i64 nE = nc * k * k + nn;
  if (nE >= (i64)0xFFFFFFFFll) fail(FCU_ERR_UNSUPPORTED, "mesh too large for 32-bit pattern indices");
  const unsigned long long sentinel = (unsigned long long)(nn * nn);
  const int kbits = bit_length(sentinel);
  DBuf<unsigned long long> keys, keys_s;
  DBuf<unsigned> vals, vals_s;
  keys.alloc(nE); keys_s.alloc(nE); vals.alloc(nE); vals_s.alloc(nE);
  k_emit_pairs<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(s->cell_nodes.p, m->valid.p, nc, k, nn, sentinel,
                                                                keys.p, vals.p);
  LAUNCH_CHECK(ctx);
  {
    size_t tb = 0;
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, keys_s.p, vals.p, vals_s.p, (int)nE, 0, kbits, ctx->stream));
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(ctx->temp_bytes(tb), tb, keys.p, keys_s.p, vals.p, vals_s.p, (int)nE, 0,
                                               kbits, ctx->stream));
  }
  keys.release();
  vals.release();
  DBuf<int> flags, slot_incl;
  flags.alloc(nE);
  slot_incl.alloc(nE);
  k_unique_flags<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, nE, sentinel, flags.p);
  LAUNCH_CHECK(ctx);
  inclusive_scan(ctx, flags.p, slot_incl.p, nE);
  const i64 nnzb = read_scalar(ctx, slot_incl.p + nE - 1);
  s->nnzb = nnzb;
  s->col_idx.alloc(nnzb);
  s->row_ptr.alloc(nn + 1);
  s->diag_pos.alloc(nn);
  DBuf<int> slot_first, real, real_excl;
  DBuf<unsigned> cnt32;
  slot_first.alloc(nnzb);
  cnt32.alloc(nnzb);
  real.alloc(nE);
  real_excl.alloc(nE);
  CUDA_CHECK(cudaMemsetAsync(cnt32.p, 0, nnzb * sizeof(unsigned), ctx->stream));
  k_pattern_fill<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, vals_s.p, flags.p, slot_incl.p, nE, nn,
                                                                  sentinel, s->col_idx.p, s->row_ptr.p, slot_first.p,
                                                                  cnt32.p, s->diag_pos.p, real.p);
  LAUNCH_CHECK(ctx);
  CUDA_CHECK(cudaMemcpyAsync(s->row_ptr.p + nn, &s->nnzb, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  {
    int nnzb32 = (int)nnzb;
    CUDA_CHECK(cudaMemcpyAsync(s->row_ptr.p + nn, &nnzb32, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  }
  DBuf<int> overflow;
  overflow.alloc(1);
  CUDA_CHECK(cudaMemsetAsync(overflow.p, 0, sizeof(int), ctx->stream));
  s->slot_cnt.alloc(nnzb);
  k_u32_to_u16<<<grid_for(nnzb, 256, cap), 256, 0, ctx->stream>>>(cnt32.p, nnzb, s->slot_cnt.p, overflow.p);
  LAUNCH_CHECK(ctx);

  // --- contributions per row --------------------------------------------------
  DBuf<int> ccount;
  ccount.alloc(nn + 1);
  CUDA_CHECK(cudaMemsetAsync(ccount.p + nn, 0, sizeof(int), ctx->stream));
  k_contrib_counts<<<grid_for(nn, 256, cap), 256, 0, ctx->stream>>>(cnt32.p, s->diag_pos.p, nn, ccount.p);
  LAUNCH_CHECK(ctx);
  s->contrib_ptr.alloc(nn + 1);
  exclusive_scan(ctx, ccount.p, s->contrib_ptr.p, nn + 1);
  const i64 ncontrib = read_scalar(ctx, s->contrib_ptr.p + nn);
  s->contrib.alloc(ncontrib);
  k_contrib_fill<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, vals_s.p, slot_incl.p, slot_first.p, nE, nn,
                                                                  k, sentinel, s->contrib_ptr.p, s->contrib.p);
  LAUNCH_CHECK(ctx);
  exclusive_scan(ctx, real.p, real_excl.p, nE);
  s->slot_ent.alloc((i64)k * ncontrib);
  k_slot_entries<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, vals_s.p, real_excl.p, nE, nn, k, sentinel,
                                                                  s->contrib_ptr.p, s->contrib.p, s->slot_ent.p,
                                                                  overflow.p);
  LAUNCH_CHECK(ctx);
  if (read_scalar(ctx, overflow.p))
    fail(FCU_ERR_UNSUPPORTED, "a node has more than 4095 incident cells or a slot more than 65535 contributions");

  // --- upper off-diagonal block lists (vector P1 stiffness) -------------------
  if (s->kind == FCU_SPACE_P1_VEC3) {
    if (nc >= (1ll << 28)) fail(FCU_ERR_UNSUPPORTED, "mesh too large for the packed block lists");
    DBuf<int> ef, epos, sf, sid;
    ef.alloc(nE);
    epos.alloc(nE);
    sf.alloc(nnzb);
    sid.alloc(nnzb);
    k_up_entry_flags<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, vals_s.p, nE, nn, sentinel, ef.p);
    LAUNCH_CHECK(ctx);
    exclusive_scan(ctx, ef.p, epos.p, nE);
    const i64 nent = (i64)read_scalar(ctx, epos.p + nE - 1) + read_scalar(ctx, ef.p + nE - 1);
    k_up_slot_flags<<<grid_for(nnzb, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, slot_first.p, nnzb, nn, sf.p);
    LAUNCH_CHECK(ctx);
    exclusive_scan(ctx, sf.p, sid.p, nnzb);
    const i64 nup = (i64)read_scalar(ctx, sid.p + nnzb - 1) + read_scalar(ctx, sf.p + nnzb - 1);
    s->nup = nup;
    s->up_slot.alloc(nup);
    s->up_tslot.alloc(nup);
    s->up_ptr.alloc(nup + 1);
    s->up_ent.alloc(nent);
    const int nent32 = (int)nent;
    CUDA_CHECK(cudaMemcpyAsync(s->up_ptr.p + nup, &nent32, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    if (nup) {
      k_up_fill_slots<<<grid_for(nnzb, 256, cap), 256, 0, ctx->stream>>>(sf.p, sid.p, slot_first.p, epos.p, nnzb,
                                                                          s->up_slot.p, s->up_ptr.p);
      LAUNCH_CHECK(ctx);
      k_up_fill_entries<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(vals_s.p, ef.p, epos.p, nE, s->up_ent.p);
      LAUNCH_CHECK(ctx);
      k_up_tslot<<<grid_for(nup, 256, cap), 256, 0, ctx->stream>>>(s->row_ptr.p, s->col_idx.p, s->up_slot.p,
                                                                   keys_s.p, slot_first.p, nup, nn, s->up_tslot.p);
      LAUNCH_CHECK(ctx);
    }
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));  // nent32 is a host temporary

    // lists of every off-diagonal block, in CSR order
    k_off_entry_flags<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, vals_s.p, nE, nn, sentinel, ef.p);
    LAUNCH_CHECK(ctx);
    exclusive_scan(ctx, ef.p, epos.p, nE);
    const i64 noff = (i64)read_scalar(ctx, epos.p + nE - 1) + read_scalar(ctx, ef.p + nE - 1);
    s->sl_ptr.alloc(nnzb + 1);
    s->sl_ent.alloc(noff);
    const int noff32 = (int)noff;
    CUDA_CHECK(cudaMemcpyAsync(s->sl_ptr.p + nnzb, &noff32, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    k_slot_list_ptr<<<grid_for(nnzb, 256, cap), 256, 0, ctx->stream>>>(slot_first.p, epos.p, nnzb, s->sl_ptr.p);
    LAUNCH_CHECK(ctx);
    k_up_fill_entries<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(vals_s.p, ef.p, epos.p, nE, s->sl_ent.p);
    LAUNCH_CHECK(ctx);
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));  // noff32 is a host temporary
  }

  // --- host-side statistics -----------------------------------------------
  std::vector<int> rp(nn + 1), cp(nn + 1);
  CUDA_CHECK(cudaMemcpyAsync(rp.data(), s->row_ptr.p, (nn + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaMemcpyAsync(cp.data(), s->contrib_ptr.p, (nn + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  int mr = 0, mc = 0;
  i64 empty_rows = 0;
  for (i64 i = 0; i < nn; ++i) {
    mr = std::max(mr, rp[i + 1] - rp[i]);
    int cc = cp[i + 1] - cp[i];
    mc = std::max(mc, cc);
    empty_rows += (cc == 0);
  }
  s->max_row = mr;
  s->max_contrib = mc;
  s->nnz_ref = (nnzb - empty_rows) * (i64)s->bs * s->bs;

  // --- per-contribution slot map (P2 stiffness) --------------------------------
  if ((s->kind == FCU_SPACE_P2 || s->kind == FCU_SPACE_P2_NODES) && mr <= 255 && ncontrib > 0) {
    s->cmap.alloc((i64)k * ncontrib);
    k_contrib_slot_map<<<grid_for(nE, 256, cap), 256, 0, ctx->stream>>>(keys_s.p, vals_s.p, slot_incl.p, nE, nn, k,
                                                                        sentinel, s->row_ptr.p, s->contrib_ptr.p,
                                                                        s->contrib.p, s->cmap.p);
    LAUNCH_CHECK(ctx);
    if (nc < (1ll << 28)) {
      // reorder each row's contributions by (local index, cell), map along
      DBuf<unsigned long long> ck, cks;
      DBuf<int> ci, cis;
      ck.alloc(ncontrib); cks.alloc(ncontrib); ci.alloc(ncontrib); cis.alloc(ncontrib);
      k_contrib_sort_keys<<<grid_for(nn, 256, cap), 256, 0, ctx->stream>>>(s->contrib_ptr.p, s->contrib.p, nn, ck.p,
                                                                            ci.p);
      LAUNCH_CHECK(ctx);
      const int kb = 32 + bit_length((unsigned long long)nn);
      size_t tb = 0;
      CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, ck.p, cks.p, ci.p, cis.p, (int)ncontrib, 0, kb,
                                                 ctx->stream));
      CUDA_CHECK(cub::DeviceRadixSort::SortPairs(ctx->temp_bytes(tb), tb, ck.p, cks.p, ci.p, cis.p, (int)ncontrib, 0,
                                                 kb, ctx->stream));
      s->contrib_a.alloc(ncontrib);
      DBuf<unsigned char> cm;
      cm.alloc((i64)k * ncontrib);
      k_contrib_permute<<<grid_for(ncontrib, 256, cap), 256, 0, ctx->stream>>>(cis.p, s->contrib.p, s->cmap.p,
                                                                               ncontrib, k, s->contrib_a.p, cm.p);
      LAUNCH_CHECK(ctx);
      s->cmap = std::move(cm);
    }
  }
}

void build_transpose_positions(fcu_space s) {
  if (s->tpos.p) return;
  fcu_ctx ctx = s->ctx;
  s->tpos.alloc(s->nnzb);
  k_tpos<<<grid_for(s->nnodes, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(s->row_ptr.p, s->col_idx.p, s->nnodes,
                                                                               s->tpos.p);
  LAUNCH_CHECK(ctx);
}
