/*
 * CPU restatement of the Hermes3D reference's hexahedral H1 assembly.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY: called by tests/, smoke() and the
 * CPU-baseline leg of bench.py as the checker; never by the product.
 *
 * Parity pin: checked against the reference itself (built from its sources
 * by oracle/Makefile) on the golden fixtures under tests/golden/.
 */
#ifndef H3D_PORT_H
#define H3D_PORT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CSC pattern from assembly lists (Discretization::create,
 * src/discretization.cc:164-230; SparseMatrix::sort_and_store_indices,
 * src/matrix.cc:169-189).  Pass Ai == NULL to get nnz in *nnz first. */
int h3d_port_pattern(int64_t ne, const int64_t *al_ptr, const int32_t *al_dof, int64_t ndof, int64_t *Ap,
                     int32_t *Ai, int64_t *nnz);

/* Numeric assembly (Discretization::assemble, src/discretization.cc:232-422)
 * with the explicit-order forms grad.grad (times gradcoef[e]) [+ mass] and
 * int F v, each pair integrated by its own point loop as in
 * src/integrals/h1.h:31-177.  nq is ne x 3 Gauss points per direction.
 * hex: ne x 8 zero-based vertex indices.  lf: 0 none, 1 constant lf_value,
 * 2 sin(pi x) sin(pi y) sin(pi z). */
int h3d_port_assemble(int64_t nv, const double *xyz, int64_t ne, const int64_t *hex, const int32_t *nq,
                      const int64_t *al_ptr, const int64_t *al_idx, const int32_t *al_dof, const double *al_coef,
                      int mass, const double *gradcoef, int lf, double lf_value, int64_t ndof, const int64_t *Ap,
                      const int32_t *Ai, double *Ax, double *rhs);

/* The same with the reference's stock quadrature: each pair (u, v) of
 * grad.grad / mass integrated with order(u) + order(v) + 1 per direction,
 * int F v with the maximal order 24 (src/integrals/h1.h:115-177). */
int h3d_port_assemble_stock(int64_t nv, const double *xyz, int64_t ne, const int64_t *hex, const int64_t *al_ptr,
                            const int64_t *al_idx, const int32_t *al_dof, const double *al_coef, int mass,
                            const double *gradcoef, int lf, double lf_value, int64_t ndof, const int64_t *Ap,
                            const int32_t *Ai, double *Ax, double *rhs);

/* Element matrix of one element in the assembly-list basis (cnt x cnt,
 * row = test, no coefficients applied): for element-level parity. */
int h3d_port_element_matrix(const double *X /* 8 x 3 */, int nqx, int nqy, int nqz, int cnt, const int64_t *idx,
                            int mass, double gradcoef, double *K);

/* Selected rows of the element matrix: K[r][j] for r in rows (test indices
 * into idx), all j; out is nrows x cnt. */
int h3d_port_element_rows(const double *X, int nqx, int nqy, int nqz, int cnt, const int64_t *idx, int nrows,
                          const int32_t *rows, int mass, double gradcoef, double *out);

#ifdef __cplusplus
}
#endif

#endif
