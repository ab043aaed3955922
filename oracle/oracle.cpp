// ORACLE — test infrastructure only.
//
// A CPU FP64 restatement of the GlassOnTin/fenics-rs assembly + Jacobi-PCG path,
// used as the checker for the CUDA library and as the timed CPU baseline. The
// product never links, loads or calls this file: only tests/, the smoke check
// and bench.py's CPU baseline leg do.
//
// The reference is a Rust workspace; it cannot be compiled in this image (no
// cargo/rustc, and crates/fenics-solver/src/gpu.rs:116 include_str!s a PTX file
// that is absent). Every function below restates the reference's arithmetic in
// the same operation order and cites the file:line it follows. Third-party
// pieces the reference relies on are restated from their published algorithms:
//   * nalgebra 0.33.3 (Cargo.lock): 2x2/3x3 determinant by cofactor expansion
//     along the first row, inverse by adjugate / determinant.
//   * faer 0.20.2 (Cargo.lock): SparseColMat::try_new_from_triplets — rows
//     sorted inside each column, duplicate (row, col) pairs summed in triplet
//     order, explicit zeros kept.
//   * rayon 1.12.0: par_iter().flat_map().collect() keeps cell order, so the
//     triplet list is in cell order; restated with OpenMP writing each cell's
//     triplets to its own fixed slot.
// Extensions the reference does not have (P2 global numbering and stiffness,
// per-cell coefficients, adjoint gradient, batched solves, mixed precision)
// are defined here the same way the CUDA library defines them; their parity is
// restatement-pinned, not reference-pinned.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

typedef int64_t i64;

namespace {

// ---------------------------------------------------------------------------
// nalgebra-style small dense algebra (jacobian.rs:18-41, 60-85)
// ---------------------------------------------------------------------------

struct Map2 {
  double J[2][2];     // J[row][col], columns are v1-v0, v2-v0
  double invT[2][2];  // (J^{-1})^T
  double det;
};

struct Map3 {
  double J[3][3];
  double invT[3][3];
  double det;
};

// AffineSimplexMap::from_triangle_vertices (jacobian.rs:18-41). Returns false
// for |det| < 1e-14 (the reference returns Err and the caller skips the cell).
bool map_triangle(const double* v0, const double* v1, const double* v2, Map2& m) {
  for (int r = 0; r < 2; ++r) {
    m.J[r][0] = v1[r] - v0[r];
    m.J[r][1] = v2[r] - v0[r];
  }
  // nalgebra 2x2 determinant: m11*m22 - m21*m12
  m.det = m.J[0][0] * m.J[1][1] - m.J[1][0] * m.J[0][1];
  if (std::fabs(m.det) < 1e-14) return false;
  double d = m.J[0][0] * m.J[1][1] - m.J[1][0] * m.J[0][1];
  if (d == 0.0) return false;
  double inv[2][2];
  inv[0][0] = m.J[1][1] / d;
  inv[0][1] = -m.J[0][1] / d;
  inv[1][0] = -m.J[1][0] / d;
  inv[1][1] = m.J[0][0] / d;
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 2; ++c) m.invT[r][c] = inv[c][r];
  return true;
}

double det3(const double a[3][3]) {
  double m1 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
  double m2 = a[1][0] * a[2][2] - a[2][0] * a[1][2];
  double m3 = a[1][0] * a[2][1] - a[2][0] * a[1][1];
  return a[0][0] * m1 - a[0][1] * m2 + a[0][2] * m3;
}

// AffineSimplexMap::from_tetrahedron_vertices (jacobian.rs:60-85).
bool map_tet(const double* v0, const double* v1, const double* v2, const double* v3, Map3& m) {
  for (int r = 0; r < 3; ++r) {
    m.J[r][0] = v1[r] - v0[r];
    m.J[r][1] = v2[r] - v0[r];
    m.J[r][2] = v3[r] - v0[r];
  }
  m.det = det3(m.J);
  if (std::fabs(m.det) < 1e-14) return false;
  const double(*a)[3] = m.J;
  double m1 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
  double m2 = a[1][0] * a[2][2] - a[2][0] * a[1][2];
  double m3 = a[1][0] * a[2][1] - a[2][0] * a[1][1];
  double d = a[0][0] * m1 - a[0][1] * m2 + a[0][2] * m3;
  if (d == 0.0) return false;
  double inv[3][3];
  inv[0][0] = m1 / d;
  inv[0][1] = (a[0][2] * a[2][1] - a[2][2] * a[0][1]) / d;
  inv[0][2] = (a[0][1] * a[1][2] - a[1][1] * a[0][2]) / d;
  inv[1][0] = -m2 / d;
  inv[1][1] = (a[0][0] * a[2][2] - a[2][0] * a[0][2]) / d;
  inv[1][2] = (a[1][0] * a[0][2] - a[0][0] * a[1][2]) / d;
  inv[2][0] = m3 / d;
  inv[2][1] = (a[2][0] * a[0][1] - a[0][0] * a[2][1]) / d;
  inv[2][2] = (a[0][0] * a[1][1] - a[1][0] * a[0][1]) / d;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m.invT[r][c] = inv[c][r];
  return true;
}

// transform_gradient (jacobian.rs:51-55, 95-99): g = J^{-T} g_ref
inline void tgrad2(const Map2& m, const double* gr, double* g) {
  for (int r = 0; r < 2; ++r) g[r] = m.invT[r][0] * gr[0] + m.invT[r][1] * gr[1];
}
inline void tgrad3(const Map3& m, const double* gr, double* g) {
  for (int r = 0; r < 3; ++r)
    g[r] = m.invT[r][0] * gr[0] + m.invT[r][1] * gr[1] + m.invT[r][2] * gr[2];
}

// map_to_physical (jacobian.rs:44-48, 88-92): x = v0 + J xi
inline void phys2(const Map2& m, const double* v0, const double* xi, double* x) {
  for (int r = 0; r < 2; ++r) x[r] = v0[r] + (m.J[r][0] * xi[0] + m.J[r][1] * xi[1]);
}
inline void phys3(const Map3& m, const double* v0, const double* xi, double* x) {
  for (int r = 0; r < 3; ++r)
    x[r] = v0[r] + (m.J[r][0] * xi[0] + m.J[r][1] * xi[1] + m.J[r][2] * xi[2]);
}

// P1 reference gradients (lagrange.rs:71-73, 106-113)
const double P1TRI_G[3][2] = {{-1.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}};
const double P1TET_G[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};

// triangle_quadrature(2): edge midpoints, w = 1/6 (quadrature.rs:95-114)
const double TRI_Q2[3][2] = {{0.5, 0.0}, {0.5, 0.5}, {0.0, 0.5}};
const double TRI_Q2_W = 1.0 / 6.0;
// triangle_quadrature(3): 4-point rule (quadrature.rs:116-142)
const double TRI_Q3[4][2] = {{1.0 / 3.0, 1.0 / 3.0}, {0.6, 0.2}, {0.2, 0.6}, {0.2, 0.2}};
const double TRI_Q3_W[4] = {-27.0 / 96.0, 25.0 / 96.0, 25.0 / 96.0, 25.0 / 96.0};

// tetrahedron_quadrature(2): Keast 4-point (quadrature.rs:157-183)
void tet_q2(double pts[4][3], double* w) {
  const double s5 = std::sqrt(5.0);
  const double a = (5.0 - s5) / 20.0;
  const double b = (5.0 + 3.0 * s5) / 20.0;
  const double P[4][3] = {{a, a, a}, {b, a, a}, {a, b, a}, {a, a, b}};
  std::memcpy(pts, P, sizeof(P));
  *w = 1.0 / 24.0;
}
// tetrahedron_quadrature(3): 5-point (quadrature.rs:185-218)
const double TET_Q3[5][3] = {{0.25, 0.25, 0.25},
                             {0.5, 1.0 / 6.0, 1.0 / 6.0},
                             {1.0 / 6.0, 0.5, 1.0 / 6.0},
                             {1.0 / 6.0, 1.0 / 6.0, 0.5},
                             {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0}};
const double TET_Q3_W[5] = {-2.0 / 15.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0};

// P2Tetrahedron basis and gradients (lagrange.rs:301-346); node order:
// 4 corners, then edges 01, 12, 02, 03, 13, 23 (lagrange.rs:286-299).
void p2_basis(const double* xi, double* phi) {
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
void p2_grads(const double* xi, double g[10][3]) {
  double l0 = 1.0 - xi[0] - xi[1] - xi[2], l1 = xi[0], l2 = xi[1], l3 = xi[2];
  const double G[10][3] = {{-(4.0 * l0 - 1.0), -(4.0 * l0 - 1.0), -(4.0 * l0 - 1.0)},
                           {4.0 * l1 - 1.0, 0.0, 0.0},
                           {0.0, 4.0 * l2 - 1.0, 0.0},
                           {0.0, 0.0, 4.0 * l3 - 1.0},
                           {4.0 * (l0 - l1), -4.0 * l1, -4.0 * l1},
                           {4.0 * l2, 4.0 * l1, 0.0},
                           {-4.0 * l2, 4.0 * (l0 - l2), -4.0 * l2},
                           {-4.0 * l3, -4.0 * l3, 4.0 * (l0 - l3)},
                           {4.0 * l3, 0.0, 4.0 * l1},
                           {0.0, 4.0 * l3, 4.0 * l2}};
  std::memcpy(g, G, sizeof(G));
}
// Local edge -> local corner pairs of the P2 node order above.
const int P2_EDGE[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};

int nthreads_or_default(int t) {
#ifdef _OPENMP
  return t > 0 ? t : omp_get_max_threads();
#else
  (void)t;
  return 1;
#endif
}

}  // namespace

// ---------------------------------------------------------------------------
// CSC with faer try_new_from_triplets semantics
// ---------------------------------------------------------------------------

struct orc_csc {
  i64 n;
  std::vector<i64> colptr, rowidx;
  std::vector<double> vals;
};

static orc_csc* build_csc(i64 n, i64 nt, const i64* rows, const i64* cols, const double* vals) {
  orc_csc* m = new orc_csc;
  m->n = n;
  // Stable counting sort by column, then stable sort by row inside each
  // column; equal (row, col) pairs are summed in triplet order.
  std::vector<i64> cnt(n + 1, 0);
  for (i64 t = 0; t < nt; ++t) cnt[cols[t] + 1]++;
  for (i64 c = 0; c < n; ++c) cnt[c + 1] += cnt[c];
  std::vector<i64> order(nt);
  {
    std::vector<i64> cur(cnt.begin(), cnt.end() - 1);
    for (i64 t = 0; t < nt; ++t) order[cur[cols[t]]++] = t;
  }
  m->colptr.assign(n + 1, 0);
  m->rowidx.reserve(nt);
  m->vals.reserve(nt);
  for (i64 c = 0; c < n; ++c) {
    i64 b = cnt[c], e = cnt[c + 1];
    std::stable_sort(order.begin() + b, order.begin() + e,
                     [&](i64 x, i64 y) { return rows[x] < rows[y]; });
    i64 t = b;
    while (t < e) {
      i64 r = rows[order[t]];
      double s = vals[order[t]];
      ++t;
      while (t < e && rows[order[t]] == r) {
        s += vals[order[t]];
        ++t;
      }
      m->rowidx.push_back(r);
      m->vals.push_back(s);
    }
    m->colptr[c + 1] = (i64)m->rowidx.size();
  }
  return m;
}

extern "C" {

void* orc_csc_from_triplets(i64 n, i64 nt, const i64* rows, const i64* cols, const double* vals) {
  return build_csc(n, nt, rows, cols, vals);
}

void* orc_csc_from_arrays(i64 n, const i64* colptr, const i64* rowidx, const double* vals) {
  orc_csc* m = new orc_csc;
  m->n = n;
  m->colptr.assign(colptr, colptr + n + 1);
  i64 nnz = colptr[n];
  m->rowidx.assign(rowidx, rowidx + nnz);
  m->vals.assign(vals, vals + nnz);
  return m;
}

i64 orc_csc_n(void* h) { return ((orc_csc*)h)->n; }
i64 orc_csc_nnz(void* h) { return (i64)((orc_csc*)h)->rowidx.size(); }
void orc_csc_export(void* h, i64* colptr, i64* rowidx, double* vals) {
  orc_csc* m = (orc_csc*)h;
  if (colptr) std::copy(m->colptr.begin(), m->colptr.end(), colptr);
  if (rowidx) std::copy(m->rowidx.begin(), m->rowidx.end(), rowidx);
  if (vals) std::copy(m->vals.begin(), m->vals.end(), vals);
}
void orc_csc_free(void* h) { delete (orc_csc*)h; }

// ---------------------------------------------------------------------------
// Mesh generators (generators.rs:24-55, 58-111)
// ---------------------------------------------------------------------------

void orc_unit_square(i64 nx, i64 ny, double* coords, i64* cells) {
  i64 k = 0;
  for (i64 j = 0; j <= ny; ++j) {
    double y = (double)j / (double)ny;
    for (i64 i = 0; i <= nx; ++i) {
      coords[2 * k] = (double)i / (double)nx;
      coords[2 * k + 1] = y;
      ++k;
    }
  }
  auto vid = [&](i64 i, i64 j) { return j * (nx + 1) + i; };
  i64 c = 0;
  for (i64 j = 0; j < ny; ++j)
    for (i64 i = 0; i < nx; ++i) {
      i64 v00 = vid(i, j), v10 = vid(i + 1, j), v01 = vid(i, j + 1), v11 = vid(i + 1, j + 1);
      i64* t = cells + 6 * c;
      t[0] = v00; t[1] = v10; t[2] = v11;
      t[3] = v00; t[4] = v11; t[5] = v01;
      ++c;
    }
}

void orc_box_beam(double L, double W, double H, i64 nx, i64 ny, i64 nz, double* coords, i64* cells) {
  i64 k = 0;
  for (i64 kk = 0; kk <= nz; ++kk) {
    double z = ((double)kk / (double)nz) * H;
    for (i64 j = 0; j <= ny; ++j) {
      double y = ((double)j / (double)ny) * W;
      for (i64 i = 0; i <= nx; ++i) {
        coords[3 * k] = ((double)i / (double)nx) * L;
        coords[3 * k + 1] = y;
        coords[3 * k + 2] = z;
        ++k;
      }
    }
  }
  auto vid = [&](i64 i, i64 j, i64 kk) { return kk * (nx + 1) * (ny + 1) + j * (nx + 1) + i; };
  i64 c = 0;
  for (i64 kk = 0; kk < nz; ++kk)
    for (i64 j = 0; j < ny; ++j)
      for (i64 i = 0; i < nx; ++i) {
        i64 p0 = vid(i, j, kk), p1 = vid(i + 1, j, kk), p2 = vid(i, j + 1, kk), p3 = vid(i + 1, j + 1, kk);
        i64 p4 = vid(i, j, kk + 1), p5 = vid(i + 1, j, kk + 1), p6 = vid(i, j + 1, kk + 1), p7 = vid(i + 1, j + 1, kk + 1);
        const i64 T[6][4] = {{p0, p1, p3, p7}, {p0, p3, p2, p7}, {p0, p2, p6, p7},
                             {p0, p6, p4, p7}, {p0, p4, p5, p7}, {p0, p5, p1, p7}};
        std::memcpy(cells + 24 * c, T, sizeof(T));
        ++c;
      }
}

// ---------------------------------------------------------------------------
// Boundary facets and dofs (mesh.rs:79-113, 145-210; poisson.rs:266-287).
// The reference iterates a HashMap, so its facet order is unspecified; the
// oracle returns facets sorted by their sorted vertex key.
// ---------------------------------------------------------------------------

i64 orc_boundary_facets_2d(i64 nc, const i64* cells, i64* out_verts, i64* out_cell, i64* out_local) {
  struct E { i64 a, b, cell, local; };
  std::vector<E> es;
  es.reserve(3 * nc);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 3 * c;
    i64 ed[3][2] = {{t[1], t[2]}, {t[2], t[0]}, {t[0], t[1]}};
    for (int l = 0; l < 3; ++l) {
      i64 a = std::min(ed[l][0], ed[l][1]), b = std::max(ed[l][0], ed[l][1]);
      es.push_back({a, b, c, l});
    }
  }
  std::stable_sort(es.begin(), es.end(), [](const E& x, const E& y) {
    return x.a != y.a ? x.a < y.a : x.b < y.b;
  });
  i64 nf = 0;
  for (size_t s = 0; s < es.size();) {
    size_t e = s;
    while (e < es.size() && es[e].a == es[s].a && es[e].b == es[s].b) ++e;
    if (e - s == 1) {
      if (out_verts) { out_verts[2 * nf] = es[s].a; out_verts[2 * nf + 1] = es[s].b; }
      if (out_cell) out_cell[nf] = es[s].cell;  // first inserter keeps (cell, local)
      if (out_local) out_local[nf] = es[s].local;
      ++nf;
    }
    s = e;
  }
  return nf;
}

i64 orc_boundary_facets_3d(const double* coords, i64 nc, const i64* cells, i64* out_verts, i64* out_cell,
                           i64* out_local) {
  struct F { i64 k[3]; i64 cell, local; i64 face[3]; i64 opp; };
  std::vector<F> fs;
  fs.reserve(4 * nc);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    const i64 faces[4][4] = {{t[1], t[2], t[3], t[0]}, {t[0], t[2], t[3], t[1]},
                             {t[0], t[1], t[3], t[2]}, {t[0], t[1], t[2], t[3]}};
    for (int l = 0; l < 4; ++l) {
      F f;
      f.face[0] = faces[l][0]; f.face[1] = faces[l][1]; f.face[2] = faces[l][2];
      f.opp = faces[l][3];
      f.k[0] = f.face[0]; f.k[1] = f.face[1]; f.k[2] = f.face[2];
      std::sort(f.k, f.k + 3);
      f.cell = c;
      f.local = l;
      fs.push_back(f);
    }
  }
  std::stable_sort(fs.begin(), fs.end(), [](const F& x, const F& y) {
    if (x.k[0] != y.k[0]) return x.k[0] < y.k[0];
    if (x.k[1] != y.k[1]) return x.k[1] < y.k[1];
    return x.k[2] < y.k[2];
  });
  i64 nf = 0;
  for (size_t s = 0; s < fs.size();) {
    size_t e = s;
    while (e < fs.size() && fs[e].k[0] == fs[s].k[0] && fs[e].k[1] == fs[s].k[1] && fs[e].k[2] == fs[s].k[2]) ++e;
    if (e - s == 1) {
      const F& f = fs[s];
      // Orientation: normal (b-a)x(c-a) must point away from the opposite
      // vertex (mesh.rs:166-192).
      const double* va = coords + 3 * f.face[0];
      const double* vb = coords + 3 * f.face[1];
      const double* vc = coords + 3 * f.face[2];
      const double* vo = coords + 3 * f.opp;
      double ab[3] = {vb[0] - va[0], vb[1] - va[1], vb[2] - va[2]};
      double ac[3] = {vc[0] - va[0], vc[1] - va[1], vc[2] - va[2]};
      double nrm[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
      double tf[3] = {va[0] - vo[0], va[1] - vo[1], va[2] - vo[2]};
      double dot = nrm[0] * tf[0] + nrm[1] * tf[1] + nrm[2] * tf[2];
      if (out_verts) {
        out_verts[3 * nf] = f.face[0];
        if (dot >= 0.0) { out_verts[3 * nf + 1] = f.face[1]; out_verts[3 * nf + 2] = f.face[2]; }
        else { out_verts[3 * nf + 1] = f.face[2]; out_verts[3 * nf + 2] = f.face[1]; }
      }
      if (out_cell) out_cell[nf] = f.cell;
      if (out_local) out_local[nf] = f.local;
      ++nf;
    }
    s = e;
  }
  return nf;
}

static i64 sorted_unique(std::vector<i64>& v, i64* out) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  if (out) std::copy(v.begin(), v.end(), out);
  return (i64)v.size();
}

// boundary_dofs_2d (poisson.rs:266-275)
i64 orc_boundary_dofs_2d(i64 nc, const i64* cells, i64* out) {
  i64 nf = orc_boundary_facets_2d(nc, cells, nullptr, nullptr, nullptr);
  std::vector<i64> fv(2 * nf);
  orc_boundary_facets_2d(nc, cells, fv.data(), nullptr, nullptr);
  return sorted_unique(fv, out);
}

// boundary_dofs_3d (poisson.rs:278-287)
i64 orc_boundary_dofs_3d(const double* coords, i64 nc, const i64* cells, i64* out) {
  i64 nf = orc_boundary_facets_3d(coords, nc, cells, nullptr, nullptr, nullptr);
  std::vector<i64> fv(3 * nf);
  orc_boundary_facets_3d(coords, nc, cells, fv.data(), nullptr, nullptr);
  return sorted_unique(fv, out);
}

// ---------------------------------------------------------------------------
// Scalar P1 stiffness (poisson.rs:23-69, 124-165). `kappa` (nullable) is the
// per-cell coefficient extension: entry = ((g_i . g_j) * measure) * kappa_e.
// ---------------------------------------------------------------------------

void* orc_assemble_stiffness_2d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* kappa,
                                int threads) {
  std::vector<i64> R(9 * nc), C(9 * nc);
  std::vector<double> V(9 * nc);
  std::vector<char> ok(nc, 0);
#pragma omp parallel for schedule(static) num_threads(nthreads_or_default(threads))
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 3 * c;
    Map2 m;
    if (!map_triangle(coords + 2 * t[0], coords + 2 * t[1], coords + 2 * t[2], m)) continue;
    ok[c] = 1;
    double area = 0.5 * std::fabs(m.det);
    double g[3][2];
    for (int i = 0; i < 3; ++i) tgrad2(m, P1TRI_G[i], g[i]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double v = (g[i][0] * g[j][0] + g[i][1] * g[j][1]) * area;
        if (kappa) v = v * kappa[c];
        R[9 * c + 3 * i + j] = t[i];
        C[9 * c + 3 * i + j] = t[j];
        V[9 * c + 3 * i + j] = v;
      }
  }
  // Compact away skipped (degenerate) cells, keeping cell order.
  i64 w = 0;
  for (i64 c = 0; c < nc; ++c)
    if (ok[c]) {
      for (int s = 0; s < 9; ++s) { R[w] = R[9 * c + s]; C[w] = C[9 * c + s]; V[w] = V[9 * c + s]; ++w; }
    }
  return build_csc(nv, w, R.data(), C.data(), V.data());
}

void* orc_assemble_stiffness_3d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* kappa,
                                int threads) {
  std::vector<i64> R(16 * nc), C(16 * nc);
  std::vector<double> V(16 * nc);
  std::vector<char> ok(nc, 0);
#pragma omp parallel for schedule(static) num_threads(nthreads_or_default(threads))
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) continue;
    ok[c] = 1;
    double vol = (1.0 / 6.0) * std::fabs(m.det);
    double g[4][3];
    for (int i = 0; i < 4; ++i) tgrad3(m, P1TET_G[i], g[i]);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        double v = (g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2]) * vol;
        if (kappa) v = v * kappa[c];
        R[16 * c + 4 * i + j] = t[i];
        C[16 * c + 4 * i + j] = t[j];
        V[16 * c + 4 * i + j] = v;
      }
  }
  i64 w = 0;
  for (i64 c = 0; c < nc; ++c)
    if (ok[c]) {
      for (int s = 0; s < 16; ++s) { R[w] = R[16 * c + s]; C[w] = C[16 * c + s]; V[w] = V[16 * c + s]; ++w; }
    }
  return build_csc(nv, w, R.data(), C.data(), V.data());
}

// ---------------------------------------------------------------------------
// Vector-P1 elasticity (elasticity.rs:33-47, 73-149). `cell_E` (nullable) is
// the per-cell Young's modulus extension: lambda_e, mu_e use E = cell_E[c]
// in the lame_lambda / lame_mu formulas.
// ---------------------------------------------------------------------------

static inline double lame_lambda(double e, double nu) { return (e * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu)); }
static inline double lame_mu(double e, double nu) { return e / (2.0 * (1.0 + nu)); }

void* orc_assemble_elasticity_3d(i64 nv, const double* coords, i64 nc, const i64* cells, double E, double nu,
                                 const double* cell_E, int threads) {
  const i64 K = 144;
  std::vector<i64> R(K * nc), C(K * nc);
  std::vector<double> V(K * nc);
  std::vector<char> ok(nc, 0);
  const double lam0 = lame_lambda(E, nu), mu0 = lame_mu(E, nu);
#pragma omp parallel for schedule(static) num_threads(nthreads_or_default(threads))
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) continue;
    ok[c] = 1;
    double lambda = lam0, mu = mu0;
    if (cell_E) { lambda = lame_lambda(cell_E[c], nu); mu = lame_mu(cell_E[c], nu); }
    double vol = (1.0 / 6.0) * std::fabs(m.det);
    double g[4][3];
    for (int i = 0; i < 4; ++i) tgrad3(m, P1TET_G[i], g[i]);
    i64 s = K * c;
    for (int i = 0; i < 4; ++i) {
      for (int j = 0; j < 4; ++j) {
        double gij = g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            double dab = (a == b) ? 1.0 : 0.0;
            double kv = vol * (lambda * g[j][b] * g[i][a] + mu * gij * dab + mu * g[j][a] * g[i][b]);
            R[s] = 3 * t[i] + a;
            C[s] = 3 * t[j] + b;
            V[s] = kv;
            ++s;
          }
      }
    }
  }
  i64 w = 0;
  for (i64 c = 0; c < nc; ++c)
    if (ok[c]) {
      for (i64 s = 0; s < K; ++s) { R[w] = R[K * c + s]; C[w] = C[K * c + s]; V[w] = V[K * c + s]; ++w; }
    }
  return build_csc(3 * nv, w, R.data(), C.data(), V.data());
}

// Unit-modulus element matrix K_e^1 (E = 1) of one cell, 12x12 row-major in
// interleaved local dofs (3*i + alpha); used by the adjoint gradient. Returns
// 0 for a degenerate cell.
int orc_elasticity_element_unit(const double* coords, const i64* cell, double nu, double* Ke) {
  Map3 m;
  if (!map_tet(coords + 3 * cell[0], coords + 3 * cell[1], coords + 3 * cell[2], coords + 3 * cell[3], m)) {
    std::fill(Ke, Ke + 144, 0.0);
    return 0;
  }
  double lambda = lame_lambda(1.0, nu), mu = lame_mu(1.0, nu);
  double vol = (1.0 / 6.0) * std::fabs(m.det);
  double g[4][3];
  for (int i = 0; i < 4; ++i) tgrad3(m, P1TET_G[i], g[i]);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double gij = g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double dab = (a == b) ? 1.0 : 0.0;
          Ke[(3 * i + a) * 12 + 3 * j + b] =
              vol * (lambda * g[j][b] * g[i][a] + mu * gij * dab + mu * g[j][a] * g[i][b]);
        }
    }
  return 1;
}

// ---------------------------------------------------------------------------
// Right-hand sides
// ---------------------------------------------------------------------------

// Physical quadrature points of assemble_rhs_2d's rule (poisson.rs:77, 98-100):
// out[(3c+q)*2 + d]. Degenerate cells get NaN points (their values are unused).
void orc_quadrature_points_2d(const double* coords, i64 nc, const i64* cells, double* out) {
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 3 * c;
    Map2 m;
    bool ok = map_triangle(coords + 2 * t[0], coords + 2 * t[1], coords + 2 * t[2], m);
    for (int q = 0; q < 3; ++q) {
      if (ok) phys2(m, coords + 2 * t[0], TRI_Q2[q], out + (3 * c + q) * 2);
      else out[(3 * c + q) * 2] = out[(3 * c + q) * 2 + 1] = NAN;
    }
  }
}

// assemble_rhs_2d (poisson.rs:72-121) with f given at the quadrature points:
// fq[3c+q] = f(x_q). Cell order serial scatter as in poisson.rs:116-120.
void orc_assemble_rhs_2d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* fq, double* b) {
  std::fill(b, b + nv, 0.0);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 3 * c;
    Map2 m;
    if (!map_triangle(coords + 2 * t[0], coords + 2 * t[1], coords + 2 * t[2], m)) continue;
    double detj = std::fabs(m.det);
    double lb[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 3; ++q) {
      const double* xi = TRI_Q2[q];
      double phi[3] = {1.0 - xi[0] - xi[1], xi[0], xi[1]};
      double f = fq[3 * c + q];
      for (int i = 0; i < 3; ++i) lb[i] += TRI_Q2_W * detj * f * phi[i];
    }
    for (int i = 0; i < 3; ++i) b[t[i]] += lb[i];
  }
}

void orc_quadrature_points_3d(const double* coords, i64 nc, const i64* cells, double* out) {
  double P[4][3], w;
  tet_q2(P, &w);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    bool ok = map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m);
    for (int q = 0; q < 4; ++q) {
      double* o = out + (4 * c + q) * 3;
      if (ok) phys3(m, coords + 3 * t[0], P[q], o);
      else o[0] = o[1] = o[2] = NAN;
    }
  }
}

// assemble_rhs_3d (poisson.rs:168-218)
void orc_assemble_rhs_3d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* fq, double* b) {
  double P[4][3], w;
  tet_q2(P, &w);
  std::fill(b, b + nv, 0.0);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) continue;
    double detj = std::fabs(m.det);
    double lb[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; ++q) {
      const double* xi = P[q];
      double phi[4] = {1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]};
      double f = fq[4 * c + q];
      for (int i = 0; i < 4; ++i) lb[i] += w * detj * f * phi[i];
    }
    for (int i = 0; i < 4; ++i) b[t[i]] += lb[i];
  }
}

// assemble_elasticity_body_force_3d (elasticity.rs:153-185): serial, lumped.
void orc_body_force_3d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* f, double* b) {
  std::fill(b, b + 3 * nv, 0.0);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) continue;
    double vol = (1.0 / 6.0) * std::fabs(m.det);
    double nl[3] = {f[0] * (vol * 0.25), f[1] * (vol * 0.25), f[2] * (vol * 0.25)};
    for (int i = 0; i < 4; ++i)
      for (int a = 0; a < 3; ++a) b[3 * t[i] + a] += nl[a];
  }
}

// Edge midpoints of each facet, the traction rule's evaluation points
// (boundary.rs:71-88): out[(3f+q)*3 + d].
void orc_traction_points_3d(const double* coords, i64 nf, const i64* facets, double* out) {
  for (i64 f = 0; f < nf; ++f) {
    const double* v0 = coords + 3 * facets[3 * f];
    const double* v1 = coords + 3 * facets[3 * f + 1];
    const double* v2 = coords + 3 * facets[3 * f + 2];
    for (int d = 0; d < 3; ++d) {
      out[(3 * f + 0) * 3 + d] = 0.5 * (v0[d] + v1[d]);
      out[(3 * f + 1) * 3 + d] = 0.5 * (v1[d] + v2[d]);
      out[(3 * f + 2) * 3 + d] = 0.5 * (v2[d] + v0[d]);
    }
  }
}

// assemble_surface_traction_3d (boundary.rs:48-108) with the traction given at
// the three edge midpoints of each facet: tq[(3f+q)*3 + d]. Adds into b.
void orc_surface_traction_3d(i64 nv, const double* coords, i64 nf, const i64* facets, const double* tq, double* b) {
  (void)nv;
  for (i64 f = 0; f < nf; ++f) {
    const i64* fv = facets + 3 * f;
    const double* v0 = coords + 3 * fv[0];
    const double* v1 = coords + 3 * fv[1];
    const double* v2 = coords + 3 * fv[2];
    double e1[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
    double e2[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
    double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double area = 0.5 * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    double w = area / 3.0;
    for (int q = 0; q < 3; ++q) {
      const double* t = tq + (3 * f + q) * 3;
      for (int k = 0; k < 3; ++k) {
        i64 node = fv[k];
        b[3 * node] += (w / 3.0) * t[0];
        b[3 * node + 1] += (w / 3.0) * t[1];
        b[3 * node + 2] += (w / 3.0) * t[2];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// P2 extension: numbering, stiffness, load, boundary dofs.
// Global numbering: vertices keep their ids; edge e (sorted by (min, max)
// vertex pair, ascending) gets dof nv + e. Cell-local order follows
// P2Tetrahedron: 4 corners, then edges 01, 12, 02, 03, 13, 23.
// ---------------------------------------------------------------------------

static void p2_edges(i64 nc, const i64* cells, std::vector<std::pair<i64, i64>>& edges) {
  edges.clear();
  edges.reserve(6 * nc);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    for (int e = 0; e < 6; ++e) {
      i64 a = t[P2_EDGE[e][0]], b = t[P2_EDGE[e][1]];
      edges.push_back({std::min(a, b), std::max(a, b)});
    }
  }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
}

i64 orc_p2_num_edges(i64 nc, const i64* cells) {
  std::vector<std::pair<i64, i64>> edges;
  p2_edges(nc, cells, edges);
  return (i64)edges.size();
}

void orc_p2_dofmap(i64 nv, i64 nc, const i64* cells, i64* cell_dofs, i64* edge_verts) {
  std::vector<std::pair<i64, i64>> edges;
  p2_edges(nc, cells, edges);
  if (edge_verts)
    for (size_t e = 0; e < edges.size(); ++e) { edge_verts[2 * e] = edges[e].first; edge_verts[2 * e + 1] = edges[e].second; }
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    i64* d = cell_dofs + 10 * c;
    for (int i = 0; i < 4; ++i) d[i] = t[i];
    for (int e = 0; e < 6; ++e) {
      i64 a = t[P2_EDGE[e][0]], b = t[P2_EDGE[e][1]];
      std::pair<i64, i64> key = {std::min(a, b), std::max(a, b)};
      i64 r = std::lower_bound(edges.begin(), edges.end(), key) - edges.begin();
      d[4 + e] = nv + r;
    }
  }
}

// K_e[a][b] = kappa_e * sum_q (w_q |det J|) (J^{-T} grad phi_a(xi_q)) . (J^{-T} grad phi_b(xi_q))
// with the degree-2 Keast rule (exact for piecewise-constant kappa).
void* orc_assemble_p2_stiffness_3d(i64 ndofs, const double* coords, i64 nc, const i64* cells, const i64* cell_dofs,
                                   const double* kappa, int threads) {
  const i64 K = 100;
  std::vector<i64> R(K * nc), C(K * nc);
  std::vector<double> V(K * nc);
  std::vector<char> ok(nc, 0);
  double P[4][3], wq;
  tet_q2(P, &wq);
#pragma omp parallel for schedule(static) num_threads(nthreads_or_default(threads))
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) continue;
    ok[c] = 1;
    double detj = std::fabs(m.det);
    double acc[10][10] = {{0}};
    for (int q = 0; q < 4; ++q) {
      double gr[10][3], g[10][3];
      p2_grads(P[q], gr);
      for (int a = 0; a < 10; ++a) tgrad3(m, gr[a], g[a]);
      double wd = wq * detj;
      for (int a = 0; a < 10; ++a)
        for (int b = 0; b < 10; ++b) acc[a][b] += wd * (g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2]);
    }
    double kap = kappa ? kappa[c] : 1.0;
    const i64* d = cell_dofs + 10 * c;
    for (int a = 0; a < 10; ++a)
      for (int b = 0; b < 10; ++b) {
        R[K * c + 10 * a + b] = d[a];
        C[K * c + 10 * a + b] = d[b];
        V[K * c + 10 * a + b] = acc[a][b] * kap;
      }
  }
  i64 w = 0;
  for (i64 c = 0; c < nc; ++c)
    if (ok[c]) {
      for (i64 s = 0; s < K; ++s) { R[w] = R[K * c + s]; C[w] = C[K * c + s]; V[w] = V[K * c + s]; ++w; }
    }
  return build_csc(ndofs, w, R.data(), C.data(), V.data());
}

// ---------------------------------------------------------------------------
// Mass matrices (mass.rs:10-250). Entry (i, j) of a cell is measure * factor
// (assemble_mass_2d: area * {1/6, 1/12}; assemble_mass_3d: vol * {1/10, 1/20};
// assemble_elasticity_mass_3d: density * vol * factor on each of the three
// components). Scalar P2 (this build's P2 numbering): density * |det J| *
// product, the products of build_reference_mass_products_p2. `coef`
// (nullable) is the per-cell extension: measure * coef_e before the factor.
// ---------------------------------------------------------------------------

// Barycentric moments over the reference tetrahedron (mass.rs:195-250):
// corner i is 2 l_i^2 - l_i, edge (i, j) is 4 l_i l_j; the products are
// summed term by term in that order.
void orc_p2_mass_products(double* out) {
  static const double F[12] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0, 362880.0, 3628800.0,
                               39916800.0};
  int mono[10][2][4] = {};
  double cf[10][2] = {};
  int nterm[10];
  for (int i = 0; i < 4; ++i) {
    mono[i][0][i] = 2;
    cf[i][0] = 2.0;
    mono[i][1][i] = 1;
    cf[i][1] = -1.0;
    nterm[i] = 2;
  }
  for (int e = 0; e < 6; ++e) {
    mono[4 + e][0][P2_EDGE[e][0]] = 1;
    mono[4 + e][0][P2_EDGE[e][1]] = 1;
    cf[4 + e][0] = 4.0;
    nterm[4 + e] = 1;
  }
  for (int a = 0; a < 10; ++a)
    for (int b = 0; b < 10; ++b) {
      double acc = 0.0;
      for (int ta = 0; ta < nterm[a]; ++ta)
        for (int tb = 0; tb < nterm[b]; ++tb) {
          int m[4], deg = 0;
          for (int q = 0; q < 4; ++q) {
            m[q] = mono[a][ta][q] + mono[b][tb][q];
            deg += m[q];
          }
          acc += cf[a][ta] * cf[b][tb] * F[m[0]] * F[m[1]] * F[m[2]] * F[m[3]] / F[deg + 3];
        }
      out[10 * a + b] = acc;
    }
}

// kind: 0 = P1 triangles, 1 = P1 tetrahedra, 2 = vector P1 tetrahedra,
// 3 = scalar P2 tetrahedra (cell_dofs gives the ten dofs of each cell),
// 4 = vector P2 (assemble_elasticity_mass_p2_3d, mass.rs:137-180: dof
// 3 node + component, cell_dofs the ten nodes of each cell).
void* orc_assemble_mass(i64 ndofs, const double* coords, i64 nc, const i64* cells, const i64* cell_dofs, int kind,
                        double density, const double* coef) {
  const int k = kind == 0 ? 3 : (kind >= 3 ? 10 : 4);
  const int bs = (kind == 2 || kind == 4) ? 3 : 1;
  const i64 per = (i64)k * k * bs;
  std::vector<i64> R(per * nc), C(per * nc);
  std::vector<double> V(per * nc);
  std::vector<char> ok(nc, 0);
  double prod[100];
  orc_p2_mass_products(prod);
  for (i64 c = 0; c < nc; ++c) {
    double meas;
    if (kind == 0) {
      const i64* t = cells + 3 * c;
      Map2 m;
      if (!map_triangle(coords + 2 * t[0], coords + 2 * t[1], coords + 2 * t[2], m)) continue;
      meas = 0.5 * std::fabs(m.det);
    } else {
      const i64* t = cells + 4 * c;
      Map3 m;
      if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) continue;
      meas = kind >= 3 ? std::fabs(m.det) : (1.0 / 6.0) * std::fabs(m.det);
    }
    ok[c] = 1;
    double s = density * meas;
    if (coef) s = s * coef[c];
    const i64* d = kind >= 3 ? cell_dofs + 10 * c : cells + (i64)k * c;
    i64 o = per * c;
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) {
        double f = kind >= 3 ? prod[10 * i + j] : (i == j ? (k == 3 ? 1.0 / 6.0 : 1.0 / 10.0)
                                                          : (k == 3 ? 1.0 / 12.0 : 1.0 / 20.0));
        double v = s * f;
        for (int a = 0; a < bs; ++a) {
          R[o] = bs * d[i] + a;
          C[o] = bs * d[j] + a;
          V[o] = v;
          ++o;
        }
      }
  }
  i64 w = 0;
  for (i64 c = 0; c < nc; ++c)
    if (ok[c])
      for (i64 q = 0; q < per; ++q) {
        R[w] = R[per * c + q];
        C[w] = C[per * c + q];
        V[w] = V[per * c + q];
        ++w;
      }
  return build_csc(ndofs, w, R.data(), C.data(), V.data());
}

// P2 load b_a = sum_q w_q |det J| f(x_q) phi_a(xi_q) with f given at the
// Keast points (fq[4c+q]); serial cell-order scatter.
void orc_assemble_p2_rhs_3d(i64 ndofs, const double* coords, i64 nc, const i64* cells, const i64* cell_dofs,
                            const double* fq, double* b) {
  double P[4][3], wq;
  tet_q2(P, &wq);
  std::fill(b, b + ndofs, 0.0);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) continue;
    double detj = std::fabs(m.det);
    double lb[10] = {0};
    for (int q = 0; q < 4; ++q) {
      double phi[10];
      p2_basis(P[q], phi);
      double f = fq[4 * c + q];
      for (int a = 0; a < 10; ++a) lb[a] += wq * detj * f * phi[a];
    }
    for (int a = 0; a < 10; ++a) b[cell_dofs[10 * c + a]] += lb[a];
  }
}

// Boundary dofs of the P2 space: vertices of boundary facets, plus the edges
// of boundary facets; sorted ascending (vertex dofs precede edge dofs).
i64 orc_p2_boundary_dofs(i64 nv, const double* coords, i64 nc, const i64* cells, i64* out) {
  i64 nf = orc_boundary_facets_3d(coords, nc, cells, nullptr, nullptr, nullptr);
  std::vector<i64> fv(3 * nf);
  orc_boundary_facets_3d(coords, nc, cells, fv.data(), nullptr, nullptr);
  std::vector<std::pair<i64, i64>> edges;
  p2_edges(nc, cells, edges);
  std::vector<i64> d(fv.begin(), fv.end());
  for (i64 f = 0; f < nf; ++f) {
    const i64 pr[3][2] = {{fv[3 * f], fv[3 * f + 1]}, {fv[3 * f + 1], fv[3 * f + 2]}, {fv[3 * f], fv[3 * f + 2]}};
    for (int e = 0; e < 3; ++e) {
      std::pair<i64, i64> key = {std::min(pr[e][0], pr[e][1]), std::max(pr[e][0], pr[e][1])};
      d.push_back(nv + (std::lower_bound(edges.begin(), edges.end(), key) - edges.begin()));
    }
  }
  return sorted_unique(d, out);
}

// ---------------------------------------------------------------------------
// Dirichlet elimination (poisson.rs:222-263; elasticity.rs:188-227).
// ---------------------------------------------------------------------------

void* orc_apply_dirichlet(void* h, const double* rhs, i64 nbc, const i64* dofs, const double* vals, double* new_b) {
  orc_csc* A = (orc_csc*)h;
  i64 n = A->n;
  std::vector<char> isd(n, 0);
  std::vector<double> g(n, 0.0);
  for (i64 k = 0; k < nbc; ++k) { isd[dofs[k]] = 1; g[dofs[k]] = vals[k]; }
  std::copy(rhs, rhs + n, new_b);
  std::vector<i64> R, C;
  std::vector<double> V;
  for (i64 col = 0; col < n; ++col) {
    for (i64 p = A->colptr[col]; p < A->colptr[col + 1]; ++p) {
      i64 row = A->rowidx[p];
      double v = A->vals[p];
      if (isd[col] && !isd[row]) new_b[row] -= v * g[col];
      else if (!isd[col] && !isd[row]) { R.push_back(row); C.push_back(col); V.push_back(v); }
    }
  }
  for (i64 k = 0; k < nbc; ++k) {
    R.push_back(dofs[k]); C.push_back(dofs[k]); V.push_back(1.0);
    new_b[dofs[k]] = vals[k];
  }
  return build_csc(n, (i64)R.size(), R.data(), C.data(), V.data());
}

// ---------------------------------------------------------------------------
// Jacobi-PCG (cg.rs:7-149). Returns 0 = Ok, 1 = breakdown, 2 = not converged.
// ---------------------------------------------------------------------------

static void spmv_csc(const orc_csc* A, const double* x, double* y) {
  std::fill(y, y + A->n, 0.0);
  for (i64 col = 0; col < A->n; ++col) {
    double xv = x[col];
    if (xv != 0.0)
      for (i64 p = A->colptr[col]; p < A->colptr[col + 1]; ++p) y[A->rowidx[p]] += A->vals[p] * xv;
  }
}
static double dotv(const double* a, const double* b, i64 n) {
  double s = 0.0;
  for (i64 i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

void orc_spmv(void* h, const double* x, double* y) { spmv_csc((orc_csc*)h, x, y); }

int orc_solve_cg(void* h, const double* b, const double* x0, double tol, i64 max_iter, double* x, i64* iters,
                 double* res) {
  const orc_csc* A = (const orc_csc*)h;
  i64 n = A->n;
  std::vector<double> inv(n, 1.0);
  for (i64 col = 0; col < n; ++col)
    for (i64 p = A->colptr[col]; p < A->colptr[col + 1]; ++p)
      if (A->rowidx[p] == col) {
        if (std::fabs(A->vals[p]) > 1e-15) inv[col] = 1.0 / A->vals[p];
        break;
      }
  if (x0) std::copy(x0, x0 + n, x);
  else std::fill(x, x + n, 0.0);
  std::vector<double> ax(n), r(n), z(n), p(n), ap(n);
  spmv_csc(A, x, ax.data());
  for (i64 i = 0; i < n; ++i) r[i] = b[i] - ax[i];
  double bn = std::sqrt(dotv(b, b, n));
  double r0 = std::sqrt(dotv(r.data(), r.data(), n));
  if (r0 < tol || (bn > 0.0 && r0 / bn < tol)) { *iters = 0; *res = r0; return 0; }
  for (i64 i = 0; i < n; ++i) z[i] = r[i] * inv[i];
  p = z;
  double rz = dotv(r.data(), z.data(), n);
  for (i64 it = 1; it <= max_iter; ++it) {
    spmv_csc(A, p.data(), ap.data());
    double pap = dotv(p.data(), ap.data(), n);
    if (std::fabs(pap) < 1e-30) { *iters = it; *res = std::sqrt(dotv(r.data(), r.data(), n)); return 1; }
    double alpha = rz / pap;
    for (i64 i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
    double rn = std::sqrt(dotv(r.data(), r.data(), n));
    double rel = bn > 0.0 ? rn / bn : rn;
    if (rel < tol) { *iters = it; *res = rn; return 0; }
    for (i64 i = 0; i < n; ++i) z[i] = r[i] * inv[i];
    double rzn = dotv(r.data(), z.data(), n);
    double beta = rzn / rz;
    rz = rzn;
    for (i64 i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  *iters = max_iter;
  *res = std::sqrt(dotv(r.data(), r.data(), n));
  return 2;
}

// Multi-threaded Jacobi-PCG (labelled as such wherever it is used; the
// reference's cg.rs is sequential): the recurrence and stopping rules of
// cg.rs:40-149 (x0 = 0 or given, the test ||r||/||b|| < tol after the x/r
// update, breakdown when |p.Ap| < 1e-30), with a row-gather SpMV (the CSC of
// a symmetric matrix read as its CSR) and the vector loops and dot products
// split over `threads` OpenMP threads, so sums are ordered per thread block.
// tol < 0 runs exactly max_iter iterations with no test (the timed-sample
// form). Returns 0 converged, 1 breakdown, 2 iteration limit.
static int cg_mt(const orc_csc* A, const double* b, const double* x0, double tol, i64 max_iter, int threads,
                 double* x, i64* iters, double* res) {
  const i64 n = A->n;
  const int nt = nthreads_or_default(threads);
  std::vector<double> inv(n, 1.0), r(n), z(n), p(n), ap(n);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (i64 col = 0; col < n; ++col)
    for (i64 q = A->colptr[col]; q < A->colptr[col + 1]; ++q)
      if (A->rowidx[q] == col) {
        if (std::fabs(A->vals[q]) > 1e-15) inv[col] = 1.0 / A->vals[q];
        break;
      }
  auto dot = [&](const double* u, const double* v) {
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s) num_threads(nt)
    for (i64 i = 0; i < n; ++i) s += u[i] * v[i];
    return s;
  };
  auto matvec = [&](const double* in, double* out) {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (i64 row = 0; row < n; ++row) {
      double s = 0.0;
      for (i64 q = A->colptr[row]; q < A->colptr[row + 1]; ++q) s += A->vals[q] * in[A->rowidx[q]];
      out[row] = s;
    }
  };
#pragma omp parallel for schedule(static) num_threads(nt)
  for (i64 i = 0; i < n; ++i) x[i] = x0 ? x0[i] : 0.0;
  if (x0) {
    matvec(x, ap.data());
#pragma omp parallel for schedule(static) num_threads(nt)
    for (i64 i = 0; i < n; ++i) r[i] = b[i] - ap[i];
  } else {
    std::copy(b, b + n, r.begin());
  }
  const double bn = std::sqrt(dot(b, b));
  double rn = std::sqrt(dot(r.data(), r.data()));
  *iters = 0;
  *res = rn;
  if (tol >= 0.0 && (rn < tol || (bn > 0.0 && rn / bn < tol))) return 0;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (i64 i = 0; i < n; ++i) {
    z[i] = r[i] * inv[i];
    p[i] = z[i];
  }
  double rz = dot(r.data(), z.data());
  for (i64 it = 1; it <= max_iter; ++it) {
    matvec(p.data(), ap.data());
    const double pap = dot(p.data(), ap.data());
    if (tol >= 0.0 && std::fabs(pap) < 1e-30) {
      *iters = it;
      *res = rn;
      return 1;
    }
    const double alpha = rz / pap;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (i64 i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * ap[i];
      z[i] = r[i] * inv[i];
    }
    rn = std::sqrt(dot(r.data(), r.data()));
    *iters = it;
    *res = rn;
    if (tol >= 0.0 && (bn > 0.0 ? rn / bn : rn) < tol) return 0;
    const double rzn = dot(r.data(), z.data());
    const double beta = rzn / rz;
    rz = rzn;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (i64 i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  return 2;
}

// Timed-sample form: exactly `iters` iterations, final relative residual.
double orc_cg_fixed_iters_mt(void* h, const double* b, i64 iters, double* x, int threads) {
  const orc_csc* A = (const orc_csc*)h;
  i64 it = 0;
  double rn = 0.0;
  cg_mt(A, b, nullptr, -1.0, iters, threads, x, &it, &rn);
  const double bn = std::sqrt(dotv(b, b, A->n));
  return bn > 0.0 ? rn / bn : rn;
}

// To tolerance (cg.rs stopping rules), multi-threaded.
int orc_solve_cg_mt(void* h, const double* b, const double* x0, double tol, i64 max_iter, int threads, double* x,
                    i64* iters, double* res) {
  return cg_mt((const orc_csc*)h, b, x0, tol, max_iter, threads, x, iters, res);
}

double orc_cg_fixed_iters(void* h, const double* b, i64 iters, double* x) {
  const orc_csc* A = (const orc_csc*)h;
  i64 n = A->n;
  std::vector<double> inv(n, 1.0);
  for (i64 col = 0; col < n; ++col)
    for (i64 p = A->colptr[col]; p < A->colptr[col + 1]; ++p)
      if (A->rowidx[p] == col) {
        if (std::fabs(A->vals[p]) > 1e-15) inv[col] = 1.0 / A->vals[p];
        break;
      }
  std::fill(x, x + n, 0.0);
  std::vector<double> r(b, b + n), z(n), p(n), ap(n);
  double bn = std::sqrt(dotv(b, b, n));
  for (i64 i = 0; i < n; ++i) z[i] = r[i] * inv[i];
  p = z;
  double rz = dotv(r.data(), z.data(), n), rn = bn;
  for (i64 it = 1; it <= iters; ++it) {
    spmv_csc(A, p.data(), ap.data());
    double alpha = rz / dotv(p.data(), ap.data(), n);
    for (i64 i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
    rn = std::sqrt(dotv(r.data(), r.data(), n));
    for (i64 i = 0; i < n; ++i) z[i] = r[i] * inv[i];
    double rzn = dotv(r.data(), z.data(), n);
    double beta = rzn / rz;
    rz = rzn;
    for (i64 i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  return bn > 0.0 ? rn / bn : rn;
}

// ---------------------------------------------------------------------------
// Error norms (poisson_solver.rs:62-96, 135-172) with u_exact given at the
// degree-3 quadrature points (ue[4c+q] in 2D, ue[5c+q] in 3D).
// ---------------------------------------------------------------------------

void orc_l2_points_2d(const double* coords, i64 nc, const i64* cells, double* out) {
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 3 * c;
    Map2 m;
    map_triangle(coords + 2 * t[0], coords + 2 * t[1], coords + 2 * t[2], m);
    for (int q = 0; q < 4; ++q) phys2(m, coords + 2 * t[0], TRI_Q3[q], out + (4 * c + q) * 2);
  }
}
double orc_l2_error_2d(const double* coords, i64 nc, const i64* cells, const double* uh, const double* ue) {
  double tot = 0.0;
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 3 * c;
    Map2 m;
    map_triangle(coords + 2 * t[0], coords + 2 * t[1], coords + 2 * t[2], m);
    double detj = std::fabs(m.det);
    for (int q = 0; q < 4; ++q) {
      const double* xi = TRI_Q3[q];
      double phi[3] = {1.0 - xi[0] - xi[1], xi[0], xi[1]};
      double ap = uh[t[0]] * phi[0] + uh[t[1]] * phi[1] + uh[t[2]] * phi[2];
      double err = ap - ue[4 * c + q];
      tot += TRI_Q3_W[q] * detj * err * err;
    }
  }
  return std::sqrt(tot);
}
void orc_l2_points_3d(const double* coords, i64 nc, const i64* cells, double* out) {
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m);
    for (int q = 0; q < 5; ++q) phys3(m, coords + 3 * t[0], TET_Q3[q], out + (5 * c + q) * 3);
  }
}
double orc_l2_error_3d(const double* coords, i64 nc, const i64* cells, const double* uh, const double* ue) {
  double tot = 0.0;
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m);
    double detj = std::fabs(m.det);
    for (int q = 0; q < 5; ++q) {
      const double* xi = TET_Q3[q];
      double phi[4] = {1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]};
      double ap = uh[t[0]] * phi[0] + uh[t[1]] * phi[1] + uh[t[2]] * phi[2] + uh[t[3]] * phi[3];
      double err = ap - ue[5 * c + q];
      tot += TET_Q3_W[q] * detj * err * err;
    }
  }
  return std::sqrt(tot);
}

// ---------------------------------------------------------------------------
// Stress recovery (elasticity.rs:230-320, 323-360): per-cell von Mises and
// the volume-weighted vertex average.
// ---------------------------------------------------------------------------

void orc_von_mises(i64 nv, const double* coords, i64 nc, const i64* cells, const double* u, double E, double nu,
                   double* cell_vm, double* vertex_vm) {
  double lambda = lame_lambda(E, nu), mu = lame_mu(E, nu);
  std::vector<double> vs(nv, 0.0), vw(nv, 0.0);
  for (i64 c = 0; c < nc; ++c) {
    const i64* t = cells + 4 * c;
    Map3 m;
    if (!map_tet(coords + 3 * t[0], coords + 3 * t[1], coords + 3 * t[2], coords + 3 * t[3], m)) {
      cell_vm[c] = 0.0;
      continue;
    }
    double g[4][3];
    for (int i = 0; i < 4; ++i) tgrad3(m, P1TET_G[i], g[i]);
    double gu[3][3] = {{0}};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int nd = 0; nd < 4; ++nd) gu[i][j] += u[3 * t[nd] + i] * g[nd][j];
    double eps[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) eps[i][j] = 0.5 * (gu[i][j] + gu[j][i]);
    double tr = eps[0][0] + eps[1][1] + eps[2][2];
    double s[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) s[i][j] = lambda * tr * (i == j ? 1.0 : 0.0) + 2.0 * mu * eps[i][j];
    double vm2 = 0.5 * ((s[0][0] - s[1][1]) * (s[0][0] - s[1][1]) + (s[1][1] - s[2][2]) * (s[1][1] - s[2][2]) +
                        (s[2][2] - s[0][0]) * (s[2][2] - s[0][0]) +
                        6.0 * (s[0][1] * s[0][1] + s[1][2] * s[1][2] + s[2][0] * s[2][0]));
    cell_vm[c] = std::sqrt(std::max(vm2, 0.0));
    double vol = (1.0 / 6.0) * std::fabs(m.det);
    for (int i = 0; i < 4; ++i) { vs[t[i]] += cell_vm[c] * vol; vw[t[i]] += vol; }
  }
  for (i64 i = 0; i < nv; ++i) vertex_vm[i] = vw[i] > 1e-15 ? vs[i] / vw[i] : vs[i];
}

// ---------------------------------------------------------------------------
// Adjoint extension: dJ/dtheta_e = -lambda_e^T (3 theta_e^2 E0 K_e^1) u_e for
// E_e = E0 theta_e^3. Dirichlet dofs carry zero in u and lambda.
// ---------------------------------------------------------------------------

void orc_adjoint_grad(const double* coords, i64 nc, const i64* cells, double nu, double E0, const double* theta,
                      const double* u, const double* lam, double* grad, int threads) {
#pragma omp parallel for schedule(static) num_threads(nthreads_or_default(threads))
  for (i64 c = 0; c < nc; ++c) {
    double Ke[144];
    const i64* t = cells + 4 * c;
    if (!orc_elasticity_element_unit(coords, t, nu, Ke)) { grad[c] = 0.0; continue; }
    double ue[12], le[12];
    for (int i = 0; i < 4; ++i)
      for (int a = 0; a < 3; ++a) { ue[3 * i + a] = u[3 * t[i] + a]; le[3 * i + a] = lam[3 * t[i] + a]; }
    double s = 0.0;
    for (int r = 0; r < 12; ++r) {
      double kr = 0.0;
      for (int q = 0; q < 12; ++q) kr += Ke[r * 12 + q] * ue[q];
      s += le[r] * kr;
    }
    grad[c] = -(3.0 * theta[c] * theta[c] * E0) * s;
  }
}

// ---------------------------------------------------------------------------
// Element-level probes for known-answer tests (jacobian.rs:107-147,
// lagrange.rs:480-559).
// ---------------------------------------------------------------------------

// verts: 3x2 (2D) row-major; out det, invT (row-major), ok flag as return.
int orc_affine_map_2d(const double* verts, double* det, double* invT) {
  Map2 m;
  bool ok = map_triangle(verts, verts + 2, verts + 4, m);
  *det = m.det;
  if (ok) for (int r = 0; r < 2; ++r) for (int c = 0; c < 2; ++c) invT[2 * r + c] = m.invT[r][c];
  return ok ? 1 : 0;
}
int orc_affine_map_3d(const double* verts, double* det, double* invT) {
  Map3 m;
  bool ok = map_tet(verts, verts + 3, verts + 6, verts + 9, m);
  *det = m.det;
  if (ok) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) invT[3 * r + c] = m.invT[r][c];
  return ok ? 1 : 0;
}
void orc_p2_basis(const double* xi, double* phi) { p2_basis(xi, phi); }
void orc_p2_grads(const double* xi, double* g) {
  double G[10][3];
  p2_grads(xi, G);
  std::memcpy(g, G, sizeof(G));
}

}  // extern "C"
