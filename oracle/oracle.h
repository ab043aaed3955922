// ORACLE — test infrastructure only (see oracle.cpp). C declarations of the
// CPU restatement of the fenics-rs assembly + Jacobi-PCG path.
#pragma once
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int64_t i64;
void* orc_csc_from_triplets(i64 n, i64 nt, const i64* rows, const i64* cols, const double* vals);
void* orc_csc_from_arrays(i64 n, const i64* colptr, const i64* rowidx, const double* vals);
i64 orc_csc_n(void* h);
i64 orc_csc_nnz(void* h);
void orc_csc_export(void* h, i64* colptr, i64* rowidx, double* vals);
void orc_csc_free(void* h);
void orc_unit_square(i64 nx, i64 ny, double* coords, i64* cells);
void orc_box_beam(double L, double W, double H, i64 nx, i64 ny, i64 nz, double* coords, i64* cells);
i64 orc_boundary_facets_2d(i64 nc, const i64* cells, i64* out_verts, i64* out_cell, i64* out_local);
i64 orc_boundary_facets_3d(const double* coords, i64 nc, const i64* cells, i64* out_verts, i64* out_cell, i64* out_local);
i64 orc_boundary_dofs_2d(i64 nc, const i64* cells, i64* out);
i64 orc_boundary_dofs_3d(const double* coords, i64 nc, const i64* cells, i64* out);
void* orc_assemble_stiffness_2d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* kappa, int threads);
void* orc_assemble_stiffness_3d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* kappa, int threads);
void* orc_assemble_elasticity_3d(i64 nv, const double* coords, i64 nc, const i64* cells, double E, double nu, const double* cell_E, int threads);
int orc_elasticity_element_unit(const double* coords, const i64* cell, double nu, double* Ke);
void orc_quadrature_points_2d(const double* coords, i64 nc, const i64* cells, double* out);
void orc_assemble_rhs_2d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* fq, double* b);
void orc_quadrature_points_3d(const double* coords, i64 nc, const i64* cells, double* out);
void orc_assemble_rhs_3d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* fq, double* b);
void orc_body_force_3d(i64 nv, const double* coords, i64 nc, const i64* cells, const double* f, double* b);
void orc_traction_points_3d(const double* coords, i64 nf, const i64* facets, double* out);
void orc_surface_traction_3d(i64 nv, const double* coords, i64 nf, const i64* facets, const double* tq, double* b);
i64 orc_p2_num_edges(i64 nc, const i64* cells);
void orc_p2_dofmap(i64 nv, i64 nc, const i64* cells, i64* cell_dofs, i64* edge_verts);
void* orc_assemble_p2_stiffness_3d(i64 ndofs, const double* coords, i64 nc, const i64* cells, const i64* cell_dofs, const double* kappa, int threads);
void orc_assemble_p2_rhs_3d(i64 ndofs, const double* coords, i64 nc, const i64* cells, const i64* cell_dofs, const double* fq, double* b);
i64 orc_p2_boundary_dofs(i64 nv, const double* coords, i64 nc, const i64* cells, i64* out);
void* orc_apply_dirichlet(void* h, const double* rhs, i64 nbc, const i64* dofs, const double* vals, double* new_b);
void orc_spmv(void* h, const double* x, double* y);
int orc_solve_cg(void* h, const double* b, const double* x0, double tol, i64 max_iter, double* x, i64* iters, double* res);
double orc_cg_fixed_iters(void* h, const double* b, i64 iters, double* x);
void orc_l2_points_2d(const double* coords, i64 nc, const i64* cells, double* out);
double orc_l2_error_2d(const double* coords, i64 nc, const i64* cells, const double* uh, const double* ue);
void orc_l2_points_3d(const double* coords, i64 nc, const i64* cells, double* out);
double orc_l2_error_3d(const double* coords, i64 nc, const i64* cells, const double* uh, const double* ue);
void orc_von_mises(i64 nv, const double* coords, i64 nc, const i64* cells, const double* u, double E, double nu, double* cell_vm, double* vertex_vm);
void orc_adjoint_grad(const double* coords, i64 nc, const i64* cells, double nu, double E0, const double* theta, const double* u, const double* lam, double* grad, int threads);
int orc_affine_map_2d(const double* verts, double* det, double* invT);
int orc_affine_map_3d(const double* verts, double* det, double* invT);
void orc_p2_basis(const double* xi, double* phi);
void orc_p2_grads(const double* xi, double* g);
void orc_p2_mass_products(double* out);
double orc_cg_fixed_iters_mt(void* h, const double* b, i64 iters, double* x, int threads);
int orc_solve_cg_mt(void* h, const double* b, const double* x0, double tol, i64 max_iter, int threads, double* x,
                    i64* iters, double* res);
void* orc_assemble_mass(i64 ndofs, const double* coords, i64 nc, const i64* cells, const i64* cell_dofs, int kind,
                        double density, const double* coef);
#ifdef __cplusplus
}
#endif
