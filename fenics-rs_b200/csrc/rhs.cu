// Load vectors, quadrature points and boundary extraction.
//
// This file is compiled with --fmad=false: every load-vector entry is
// accumulated per dof over its cells in ascending cell order, with the same
// operation order as the reference's serial scatter loops
// (poisson.rs:116-120, elasticity.rs:171-182, boundary.rs:90-104), so given
// the same inputs the results reproduce a sequential CPU evaluation of those
// loops bit for bit.

#include <cub/cub.cuh>

#include "internal.cuh"

namespace {

__device__ __constant__ double c_tri_q2[3][2] = {{0.5, 0.0}, {0.5, 0.5}, {0.0, 0.5}};

__device__ __forceinline__ void keast_point(int q, double* xi) {
  // tetrahedron_quadrature(2) (quadrature.rs:157-183)
  const double s5 = sqrt(5.0);
  const double a = (5.0 - s5) / 20.0, b = (5.0 + 3.0 * s5) / 20.0;
  xi[0] = a; xi[1] = a; xi[2] = a;
  if (q > 0) xi[q - 1] = b;
}

__device__ __forceinline__ void p2_basis(const double* xi, double* phi) {
  double l0 = 1.0 - xi[0] - xi[1] - xi[2], l1 = xi[0], l2 = xi[1], l3 = xi[2];
  phi[0] = l0 * (2.0 * l0 - 1.0);
  phi[1] = l1 * (2.0 * l1 - 1.0);
  phi[2] = l2 * (2.0 * l2 - 1.0);
  phi[3] = l3 * (2.0 * l3 - 1.0);
  phi[4] = 4.0 * l0 * l1;
  phi[5] = 4.0 * l1 * l2;
  phi[6] = 4.0 * l0 * l2;
  phi[7] = 4.0 * l0 * l3;
  phi[8] = 4.0 * l1 * l3;
  phi[9] = 4.0 * l2 * l3;
}

// Physical point x = v0 + J xi (jacobian.rs:44-48, 88-92).
__device__ __forceinline__ void phys_point(const double* __restrict__ X, const int* v, int dim, const double* xi,
                                           double* x) {
  const double* p0 = X + dim * (i64)v[0];
  for (int r = 0; r < dim; ++r) {
    double s = 0.0;
    for (int c = 0; c < dim; ++c) {
      double jrc = X[dim * (i64)v[c + 1] + r] - p0[r];
      s = (c == 0) ? jrc * xi[0] : s + jrc * xi[c];
    }
    x[r] = p0[r] + s;
  }
}

__global__ void k_quad_points(const double* __restrict__ X, const int* __restrict__ cells,
                              const unsigned char* __restrict__ valid, i64 nc, int dim, double* __restrict__ out) {
  const int nq = dim == 2 ? 3 : 4;
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nc * nq; t += (i64)gridDim.x * blockDim.x) {
    const i64 c = t / nq;
    const int q = (int)(t - c * nq);
    int v[4];
    for (int i = 0; i <= dim; ++i) v[i] = cells[(dim + 1) * c + i];
    double xi[3];
    if (dim == 2) { xi[0] = c_tri_q2[q][0]; xi[1] = c_tri_q2[q][1]; }
    else keast_point(q, xi);
    double x[3];
    if (valid[c]) phys_point(X, v, dim, xi, x);
    else x[0] = x[1] = x[2] = nan("");
    for (int r = 0; r < dim; ++r) out[t * dim + r] = x[r];
  }
}

// f at a quadrature point: from caller values, or an analytic source.
struct SourceEval {
  int kind;          // -1: values array; FCU_SRC_*
  const double* fq;  // nc*nq values (kind -1)
  double p0, p1;
  const double* nodal;  // FCU_SRC_NODAL: values per node
  __device__ double operator()(i64 c, int q, const double* x, int dim, const int* nodes, const double* phi, int k) const {
    if (kind < 0) return fq[c * (dim == 2 ? 3 : 4) + q];
    if (kind == FCU_SRC_CONSTANT) return p0;
    if (kind == FCU_SRC_SIN_PRODUCT) {
      double s = p0;
      for (int d = 0; d < dim; ++d) s = s * sin(p1 * x[d]);
      return s;
    }
    // FCU_SRC_NODAL: interpolate sum_j f_j phi_j(xi_q)
    double s = 0.0;
    for (int j = 0; j < k; ++j) s = (j == 0) ? nodal[nodes[j]] * phi[j] : s + nodal[nodes[j]] * phi[j];
    return s;
  }
};

// assemble_rhs_2d/3d and the P2 load: one thread per dof, summing its cells'
// local loads in ascending cell order.
template <int DIM, int K>
__global__ void k_rhs_gather(const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
                             const int* __restrict__ cn, const int* __restrict__ cells, const double* __restrict__ X,
                             SourceEval f, i64 nn, double* __restrict__ b) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nn; i += (i64)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int t = contrib_ptr[i]; t < contrib_ptr[i + 1]; ++t) {
      const int cc = contrib[t];
      const i64 c = cc >> 4;
      const int a = cc & 15;
      int v[4];
      for (int j = 0; j <= DIM; ++j) v[j] = cells[(DIM + 1) * c + j];
      double detj;
      if (DIM == 3) detj = fabs(tet_geometry(X, v).det);
      else detj = fabs(tri_geometry(X, v).det);
      int nodes[K];
      for (int j = 0; j < K; ++j) nodes[j] = cn[K * c + j];
      double lb = 0.0;
      const int nq = DIM == 2 ? 3 : 4;
      for (int q = 0; q < nq; ++q) {
        double xi[3], phi[K];
        if (DIM == 2) { xi[0] = c_tri_q2[q][0]; xi[1] = c_tri_q2[q][1]; }
        else keast_point(q, xi);
        if (K == 10) p2_basis(xi, phi);
        else if (DIM == 2) { phi[0] = 1.0 - xi[0] - xi[1]; phi[1] = xi[0]; phi[2] = xi[1]; }
        else { phi[0] = 1.0 - xi[0] - xi[1] - xi[2]; phi[1] = xi[0]; phi[2] = xi[1]; phi[3] = xi[2]; }
        double x[3] = {0.0, 0.0, 0.0};
        if (f.kind == FCU_SRC_SIN_PRODUCT) phys_point(X, v, DIM, xi, x);
        const double fv = f(c, q, x, DIM, nodes, phi, K);
        const double w = DIM == 2 ? 1.0 / 6.0 : 1.0 / 24.0;
        lb += w * detj * fv * phi[a];
      }
      acc += lb;
    }
    b[i] = acc;
  }
}

// assemble_elasticity_body_force_3d (elasticity.rs:153-185)
__global__ void k_body_force(const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
                             const int* __restrict__ cells, const double* __restrict__ X, double f0, double f1,
                             double f2, i64 nv, double* __restrict__ b) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nv; i += (i64)gridDim.x * blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int t = contrib_ptr[i]; t < contrib_ptr[i + 1]; ++t) {
      const i64 c = contrib[t] >> 4;
      int v[4] = {cells[4 * c], cells[4 * c + 1], cells[4 * c + 2], cells[4 * c + 3]};
      const double vol = (1.0 / 6.0) * fabs(tet_geometry(X, v).det);
      a0 += f0 * (vol * 0.25);
      a1 += f1 * (vol * 0.25);
      a2 += f2 * (vol * 0.25);
    }
    b[3 * i] = a0;
    b[3 * i + 1] = a1;
    b[3 * i + 2] = a2;
  }
}

// Traction: one (vertex, facet) pair per facet corner, sorted by vertex then
// facet index, so each vertex sums its facets in the caller's facet order.
__global__ void k_traction_pairs(const i64* __restrict__ facets, i64 nf, i64 nv, unsigned long long* __restrict__ keys,
                                 int* __restrict__ bad) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < 3 * nf; t += (i64)gridDim.x * blockDim.x) {
    const i64 v = facets[t];
    if (v < 0 || v >= nv) { atomicExch(bad, 1); keys[t] = ~0ull; continue; }
    keys[t] = ((unsigned long long)v << 32) | (unsigned long long)(t / 3);
  }
}

__global__ void k_traction_gather(const unsigned long long* __restrict__ keys, i64 npairs, const i64* __restrict__ facets,
                                  const double* __restrict__ X, const double* __restrict__ tq, i64 nv,
                                  double* __restrict__ b) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < npairs; t += (i64)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[t];
    if (k == ~0ull) continue;
    const i64 v = (i64)(k >> 32);
    if (t > 0 && (keys[t - 1] >> 32) == (unsigned long long)v) continue;  // not the first pair of v
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (i64 u = t; u < npairs && (keys[u] >> 32) == (unsigned long long)v; ++u) {
      const i64 f = (i64)(keys[u] & 0xffffffffull);
      const double* p0 = X + 3 * facets[3 * f];
      const double* p1 = X + 3 * facets[3 * f + 1];
      const double* p2 = X + 3 * facets[3 * f + 2];
      double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
      double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
      double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      const double w = area / 3.0;
      for (int q = 0; q < 3; ++q) {
        const double* tv = tq + (3 * f + q) * 3;
        a0 += (w / 3.0) * tv[0];
        a1 += (w / 3.0) * tv[1];
        a2 += (w / 3.0) * tv[2];
      }
    }
    b[3 * v] = a0;
    b[3 * v + 1] = a1;
    b[3 * v + 2] = a2;
  }
}

// ---------------------------------------------------------------------------
// Boundary facets (mesh.rs:79-113, 145-210)
// ---------------------------------------------------------------------------

__global__ void k_facet_keys(const int* __restrict__ cells, i64 nc, int dim, i64 nv, unsigned long long* __restrict__ keys,
                             unsigned* __restrict__ vals) {
  const int nfc = dim + 1;
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nc * nfc; t += (i64)gridDim.x * blockDim.x) {
    const i64 c = t / nfc;
    const int l = (int)(t - c * nfc);
    const int* cv = cells + nfc * c;
    unsigned long long key;
    if (dim == 2) {
      // local edge l: (1,2), (2,0), (0,1)
      i64 a = cv[(l + 1) % 3], b = cv[(l + 2) % 3];
      i64 lo = a < b ? a : b, hi = a < b ? b : a;
      key = (unsigned long long)(lo * nv + hi);
    } else {
      // local face l omits vertex l
      i64 f[3];
      int q = 0;
      for (int i = 0; i < 4; ++i)
        if (i != l) f[q++] = cv[i];
      if (f[0] > f[1]) { i64 s = f[0]; f[0] = f[1]; f[1] = s; }
      if (f[1] > f[2]) { i64 s = f[1]; f[1] = f[2]; f[2] = s; }
      if (f[0] > f[1]) { i64 s = f[0]; f[0] = f[1]; f[1] = s; }
      key = ((unsigned long long)f[0] * nv + f[1]) * nv + f[2];
    }
    keys[t] = key;
    vals[t] = (unsigned)t;
  }
}

__global__ void k_facet_single(const unsigned long long* __restrict__ keys, i64 n, int* __restrict__ flag) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
    bool first = (t == 0) || keys[t - 1] != keys[t];
    bool last = (t == n - 1) || keys[t + 1] != keys[t];
    flag[t] = (first && last) ? 1 : 0;
  }
}

__global__ void k_facet_emit(const unsigned* __restrict__ vals, const int* __restrict__ flag, const int* __restrict__ pos,
                             i64 n, const int* __restrict__ cells, const double* __restrict__ X, int dim,
                             i64* __restrict__ verts, i64* __restrict__ cell_out, i64* __restrict__ local_out) {
  const int nfc = dim + 1;
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
    if (!flag[t]) continue;
    const i64 f = pos[t];
    const unsigned e = vals[t];
    const i64 c = e / nfc;
    const int l = (int)(e - c * nfc);
    const int* cv = cells + nfc * c;
    if (cell_out) cell_out[f] = c;
    if (local_out) local_out[f] = l;
    if (!verts) continue;
    if (dim == 2) {
      i64 a = cv[(l + 1) % 3], b = cv[(l + 2) % 3];
      verts[2 * f] = a < b ? a : b;
      verts[2 * f + 1] = a < b ? b : a;
    } else {
      i64 fc[3];
      int q = 0;
      for (int i = 0; i < 4; ++i)
        if (i != l) fc[q++] = cv[i];
      const i64 opp = cv[l];
      const double* va = X + 3 * fc[0];
      const double* vb = X + 3 * fc[1];
      const double* vc = X + 3 * fc[2];
      const double* vo = X + 3 * opp;
      double ab[3] = {vb[0] - va[0], vb[1] - va[1], vb[2] - va[2]};
      double ac[3] = {vc[0] - va[0], vc[1] - va[1], vc[2] - va[2]};
      double nrm[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
      double tf[3] = {va[0] - vo[0], va[1] - vo[1], va[2] - vo[2]};
      double dot = nrm[0] * tf[0] + nrm[1] * tf[1] + nrm[2] * tf[2];
      verts[3 * f] = fc[0];
      verts[3 * f + 1] = dot >= 0.0 ? fc[1] : fc[2];
      verts[3 * f + 2] = dot >= 0.0 ? fc[2] : fc[1];
    }
  }
}

// P2 boundary edges: each boundary facet adds its vertices and edge dofs.
__global__ void k_p2_bnd_dofs(const i64* __restrict__ fv, i64 nf, const int* __restrict__ edge_verts, i64 ne, i64 nv,
                              i64* __restrict__ out) {
  for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < nf; f += (i64)gridDim.x * blockDim.x) {
    const i64 v[3] = {fv[3 * f], fv[3 * f + 1], fv[3 * f + 2]};
    for (int i = 0; i < 3; ++i) out[6 * f + i] = v[i];
    const int pr[3][2] = {{0, 1}, {1, 2}, {0, 2}};
    for (int e = 0; e < 3; ++e) {
      i64 a = v[pr[e][0]], b = v[pr[e][1]];
      i64 lo = a < b ? a : b, hi = a < b ? b : a;
      unsigned long long key = (unsigned long long)(lo * nv + hi);
      i64 L = 0, H = ne;
      while (L < H) {
        i64 M = (L + H) >> 1;
        unsigned long long km = (unsigned long long)((i64)edge_verts[2 * M] * nv + edge_verts[2 * M + 1]);
        if (km < key) L = M + 1;
        else H = M;
      }
      out[6 * f + 3 + e] = nv + L;
    }
  }
}

__global__ void k_flag_unique_i64(const i64* __restrict__ a, i64 n, int* __restrict__ flag) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x)
    flag[t] = (t == 0 || a[t - 1] != a[t]) ? 1 : 0;
}

__global__ void k_scatter_i64(const i64* __restrict__ a, const int* __restrict__ flag, const int* __restrict__ pos, i64 n,
                              i64* __restrict__ out) {
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x)
    if (flag[t]) out[pos[t]] = a[t];
}

template <class T>
T read1(fcu_ctx ctx, const T* p) {
  T h;
  CUDA_CHECK(cudaMemcpyAsync(&h, p, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  return h;
}

}  // namespace

// ---------------------------------------------------------------------------

void quadrature_points_impl(fcu_space s, double* out_dev) {
  fcu_ctx ctx = s->ctx;
  fcu_mesh m = s->mesh;
  const int nq = m->dim == 2 ? 3 : 4;
  k_quad_points<<<grid_for(m->nc * nq, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(m->coords.p, m->cells.p,
                                                                                     m->valid.p, m->nc, m->dim, out_dev);
  LAUNCH_CHECK(ctx);
}

void rhs_impl(fcu_space s, int kind, const double* fq_dev, double p0, double p1, const double* nodal_dev, double* b_dev) {
  fcu_ctx ctx = s->ctx;
  fcu_mesh m = s->mesh;
  SourceEval f{kind, fq_dev, p0, p1, nodal_dev};
  const unsigned g = grid_for(s->nnodes, 128, ctx->num_sms * 16);
  if (s->kind == FCU_SPACE_P2)
    k_rhs_gather<3, 10><<<g, 128, 0, ctx->stream>>>(s->contrib_ptr.p, s->contrib.p, s->cell_nodes.p, m->cells.p,
                                                    m->coords.p, f, s->nnodes, b_dev);
  else if (m->dim == 3)
    k_rhs_gather<3, 4><<<g, 128, 0, ctx->stream>>>(s->contrib_ptr.p, s->contrib.p, s->cell_nodes.p, m->cells.p,
                                                   m->coords.p, f, s->nnodes, b_dev);
  else
    k_rhs_gather<2, 3><<<g, 128, 0, ctx->stream>>>(s->contrib_ptr.p, s->contrib.p, s->cell_nodes.p, m->cells.p,
                                                   m->coords.p, f, s->nnodes, b_dev);
  LAUNCH_CHECK(ctx);
}

void body_force_impl(fcu_space s, const double* f, double* b_dev) {
  fcu_ctx ctx = s->ctx;
  fcu_mesh m = s->mesh;
  k_body_force<<<grid_for(m->nv, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(
      s->contrib_ptr.p, s->contrib.p, m->cells.p, m->coords.p, f[0], f[1], f[2], m->nv, b_dev);
  LAUNCH_CHECK(ctx);
}

void traction_impl(fcu_space s, i64 nf, const i64* facets_dev, const double* tq_dev, double* b_dev) {
  fcu_ctx ctx = s->ctx;
  fcu_mesh m = s->mesh;
  const int cap = ctx->num_sms * 16;
  CUDA_CHECK(cudaMemsetAsync(b_dev, 0, 3 * m->nv * sizeof(double), ctx->stream));
  if (nf == 0) return;
  if (nf >= (1ll << 31)) fail(FCU_ERR_UNSUPPORTED, "too many traction facets");
  const i64 np = 3 * nf;
  DBuf<unsigned long long> keys, keys_s;
  DBuf<int> bad;
  keys.alloc(np); keys_s.alloc(np); bad.alloc(1);
  CUDA_CHECK(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
  k_traction_pairs<<<grid_for(np, 256, cap), 256, 0, ctx->stream>>>(facets_dev, nf, m->nv, keys.p, bad.p);
  LAUNCH_CHECK(ctx);
  if (read1(ctx, bad.p)) fail(FCU_ERR_BAD_ARG, "traction facet vertex out of range");
  size_t tb = 0;
  CUDA_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.p, keys_s.p, (int)np, 0, 64, ctx->stream));
  CUDA_CHECK(cub::DeviceRadixSort::SortKeys(ctx->temp_bytes(tb), tb, keys.p, keys_s.p, (int)np, 0, 64, ctx->stream));
  k_traction_gather<<<grid_for(np, 128, cap), 128, 0, ctx->stream>>>(keys_s.p, np, facets_dev, m->coords.p, tq_dev,
                                                                    m->nv, b_dev);
  LAUNCH_CHECK(ctx);
}

// Returns the facet count; writes outputs (device pointers) when non-null.
i64 boundary_facets_impl(fcu_mesh m, i64* verts_dev, i64* cell_dev, i64* local_dev) {
  fcu_ctx ctx = m->ctx;
  const int cap = ctx->num_sms * 16;
  const int nfc = m->dim + 1;
  const i64 n = m->nc * nfc;
  if (n == 0) return 0;
  if (m->dim == 3 && (double)m->nv * m->nv * m->nv >= 1.8e19)
    fail(FCU_ERR_UNSUPPORTED, "boundary extraction supports fewer than 2.6M vertices");
  if (n >= (1ll << 31)) fail(FCU_ERR_UNSUPPORTED, "too many facets");
  DBuf<unsigned long long> k0, k1;
  DBuf<unsigned> v0, v1;
  DBuf<int> flag, pos;
  k0.alloc(n); k1.alloc(n); v0.alloc(n); v1.alloc(n); flag.alloc(n); pos.alloc(n);
  k_facet_keys<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(m->cells.p, m->nc, m->dim, m->nv, k0.p, v0.p);
  LAUNCH_CHECK(ctx);
  size_t tb = 0;
  CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0.p, k1.p, v0.p, v1.p, (int)n, 0, 64, ctx->stream));
  CUDA_CHECK(cub::DeviceRadixSort::SortPairs(ctx->temp_bytes(tb), tb, k0.p, k1.p, v0.p, v1.p, (int)n, 0, 64, ctx->stream));
  k_facet_single<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(k1.p, n, flag.p);
  LAUNCH_CHECK(ctx);
  tb = 0;
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.p, pos.p, (int)n, ctx->stream));
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(ctx->temp_bytes(tb), tb, flag.p, pos.p, (int)n, ctx->stream));
  const i64 nf = (i64)read1(ctx, pos.p + n - 1) + read1(ctx, flag.p + n - 1);
  if (verts_dev || cell_dev || local_dev) {
    k_facet_emit<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(v1.p, flag.p, pos.p, n, m->cells.p, m->coords.p,
                                                                 m->dim, verts_dev, cell_dev, local_dev);
    LAUNCH_CHECK(ctx);
  }
  return nf;
}

// Sorted unique entries of a device array (in place into out_dev); returns count.
static i64 sort_unique(fcu_ctx ctx, i64* a_dev, i64 n, i64* out_dev) {
  if (n == 0) return 0;
  const int cap = ctx->num_sms * 16;
  DBuf<i64> s;
  DBuf<int> flag, pos;
  s.alloc(n); flag.alloc(n); pos.alloc(n);
  size_t tb = 0;
  CUDA_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, tb, a_dev, s.p, (int)n, 0, 64, ctx->stream));
  CUDA_CHECK(cub::DeviceRadixSort::SortKeys(ctx->temp_bytes(tb), tb, a_dev, s.p, (int)n, 0, 64, ctx->stream));
  k_flag_unique_i64<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(s.p, n, flag.p);
  LAUNCH_CHECK(ctx);
  tb = 0;
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.p, pos.p, (int)n, ctx->stream));
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(ctx->temp_bytes(tb), tb, flag.p, pos.p, (int)n, ctx->stream));
  const i64 cnt = (i64)read1(ctx, pos.p + n - 1) + read1(ctx, flag.p + n - 1);
  if (out_dev) {
    k_scatter_i64<<<grid_for(n, 256, cap), 256, 0, ctx->stream>>>(s.p, flag.p, pos.p, n, out_dev);
    LAUNCH_CHECK(ctx);
  }
  return cnt;
}

// Boundary dofs: returns the count and fills `result` (device) with the sorted list.
i64 boundary_dofs_impl(fcu_mesh m, fcu_space s_or_null, DBuf<i64>& result) {
  fcu_ctx ctx = m->ctx;
  const i64 nf = boundary_facets_impl(m, nullptr, nullptr, nullptr);
  const int fvn = m->dim;  // vertices per facet
  DBuf<i64> fv;
  fv.alloc(nf * fvn);
  if (nf) boundary_facets_impl(m, fv.p, nullptr, nullptr);
  DBuf<i64> all;
  i64 nall;
  if (s_or_null && s_or_null->kind == FCU_SPACE_P2) {
    nall = 6 * nf;
    all.alloc(nall);
    if (nf) {
      k_p2_bnd_dofs<<<grid_for(nf, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(
          fv.p, nf, s_or_null->edge_verts.p, s_or_null->nedges, m->nv, all.p);
      LAUNCH_CHECK(ctx);
    }
  } else {
    nall = nf * fvn;
    all = std::move(fv);
  }
  result.alloc(nall);
  return sort_unique(ctx, all.p, nall, result.p);
}

// ---------------------------------------------------------------------------
// Stress recovery (elasticity.rs:230-360): per-cell displacement gradient,
// strain, Cauchy stress and von Mises stress, and the volume-weighted vertex
// average of the von Mises stress. Compiled without FMA contraction, with the
// reference's order of summation.
// ---------------------------------------------------------------------------
namespace {

// One thread per cell; any output may be null. Degenerate cells give zeros
// (StressState::default()).
__global__ void k_element_stresses(const double* __restrict__ X, const int* __restrict__ cells,
                                   const unsigned char* __restrict__ valid, i64 nc, const double* __restrict__ u,
                                   double lam, double mu, double* __restrict__ stress, double* __restrict__ strain,
                                   double* __restrict__ vm, double* __restrict__ trace) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    double s[3][3] = {{0.0}}, e[3][3] = {{0.0}};
    double v = 0.0, t = 0.0;
    if (valid[c]) {
      const int4 q = __ldg(reinterpret_cast<const int4*>(cells) + c);
      const int vv[4] = {q.x, q.y, q.z, q.w};
      const Geo3 g3 = tet_geometry(X, vv);
      // P1 gradients: g_0 = J^-T (-1,-1,-1), g_k = J^-T e_{k-1}
      double gr[4][3];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        gr[0][r] = -g3.G[r][0] - g3.G[r][1] - g3.G[r][2];
        gr[1][r] = g3.G[r][0];
        gr[2][r] = g3.G[r][1];
        gr[3][r] = g3.G[r][2];
      }
      double un[4][3];
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i) un[k][i] = u[3 * (i64)vv[k] + i];
      double gu[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          double a = 0.0;
#pragma unroll
          for (int k = 0; k < 4; ++k) a += un[k][i] * gr[k][j];
          gu[i][j] = a;
        }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) e[i][j] = 0.5 * (gu[i][j] + gu[j][i]);
      const double tr = e[0][0] + e[1][1] + e[2][2];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) s[i][j] = lam * tr * (i == j ? 1.0 : 0.0) + 2.0 * mu * e[i][j];
      const double d01 = s[0][0] - s[1][1], d12 = s[1][1] - s[2][2], d20 = s[2][2] - s[0][0];
      const double vm2 =
          0.5 * (d01 * d01 + d12 * d12 + d20 * d20 + 6.0 * (s[0][1] * s[0][1] + s[1][2] * s[1][2] + s[2][0] * s[2][0]));
      v = sqrt(fmax(vm2, 0.0));
      t = s[0][0] + s[1][1] + s[2][2];
    }
    if (stress)
#pragma unroll
      for (int q = 0; q < 9; ++q) stress[9 * c + q] = s[q / 3][q % 3];
    if (strain)
#pragma unroll
      for (int q = 0; q < 9; ++q) strain[9 * c + q] = e[q / 3][q % 3];
    if (vm) vm[c] = v;
    if (trace) trace[c] = t;
  }
}

// |det J| / 6 of every tet: the weights of the vertex average, computed on a
// space's first vertex average and kept with the space (its mesh does not
// change), with the expression the average used per cell before.
__global__ void k_cell_volumes(const double* __restrict__ X, const int* __restrict__ cells, i64 nc,
                               double* __restrict__ vol) {
  for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c < nc; c += (i64)gridDim.x * blockDim.x) {
    int vv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) vv[i] = cells[4 * c + i];
    vol[c] = (1.0 / 6.0) * fabs(tet_geometry(X, vv).det);
  }
}

// One thread per vertex: sum over its cells in ascending order (the row's
// contribution list) of vm * vol and vol, then the quotient (kept as the sum
// when the volume is ~0, as the reference leaves it).
__global__ void k_vertex_von_mises(const int* __restrict__ contrib_ptr, const int* __restrict__ contrib,
                                   const double* __restrict__ cell_vol, const double* __restrict__ cell_vm, i64 nv,
                                   double* __restrict__ out) {
  for (i64 v = blockIdx.x * (i64)blockDim.x + threadIdx.x; v < nv; v += (i64)gridDim.x * blockDim.x) {
    double sv = 0.0, sw = 0.0;
    const int q1 = contrib_ptr[v + 1];
#pragma unroll 4
    for (int q = contrib_ptr[v]; q < q1; ++q) {
      const int c = contrib[q] >> 4;
      const double vol = cell_vol[c];
      sv += cell_vm[c] * vol;
      sw += vol;
    }
    out[v] = sw > 1e-15 ? sv / sw : sv;
  }
}

}  // namespace

void element_stresses_impl(fcu_space s, double lam, double mu, const double* u_dev, double* stress, double* strain,
                           double* vm, double* trace) {
  fcu_mesh m = s->mesh;
  fcu_ctx ctx = m->ctx;
  k_element_stresses<<<grid_for(m->nc, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(
      m->coords.p, m->cells.p, m->valid.p, m->nc, u_dev, lam, mu, stress, strain, vm, trace);
  LAUNCH_CHECK(ctx);
}

void vertex_von_mises_impl(fcu_space s, const double* cell_vm_dev, double* out_dev) {
  fcu_mesh m = s->mesh;
  fcu_ctx ctx = m->ctx;
  if (!s->cell_vol.p) {
    s->cell_vol.alloc(m->nc);
    k_cell_volumes<<<grid_for(m->nc, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(m->coords.p, m->cells.p, m->nc,
                                                                                     s->cell_vol.p);
    LAUNCH_CHECK(ctx);
  }
  k_vertex_von_mises<<<grid_for(m->nv, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(
      s->contrib_ptr.p, s->contrib.p, s->cell_vol.p, cell_vm_dev, m->nv, out_dev);
  LAUNCH_CHECK(ctx);
}
