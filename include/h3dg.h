/*
 * h3dg.h -- C ABI of the B200 hp-FEM hexahedral assembly path.
 *
 * Plain C, extern "C", plain pointers and sizes; no torch or C++ types.
 * Every call returns an h3dg_status and never aborts; h3dg_last_error()
 * returns a message for the last failing call on the calling thread.
 *
 * Each entry point replaces one piece of the Hermes3D reference's call
 * surface for assembling a linear system (cited as file:line within the
 * reference project).  The reference's own C++ objects are
 *   Mesh          src/mesh.h:522-698      (+ Mesh3DReader, src/loader/mesh3d.cc)
 *   H1Space       src/space.h:76-458, src/space/h1.h
 *   Discretization src/discretization.h:39-101
 *   UMFPackMatrix / UMFPackVector  src/linsolver/umfpack.h:26-64 (CSC Ap/Ai/Ax, v)
 * and weak forms are C function pointers (src/integrals/h1.h).  A GPU
 * cannot run opaque CPU form callbacks, so the stock forms are selected
 * by descriptor (H3DG_BF_*, H3DG_LF_*); anything else is rejected with
 * H3DG_ERR_UNSUPPORTED_FORM.  There is no CPU fallback: assembly calls
 * fail with H3DG_ERR_CUDA when no device is usable.
 */
#ifndef H3DG_H
#define H3DG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int h3dg_status;
#define H3DG_OK                   0
#define H3DG_ERR_INVALID_ARG      1
#define H3DG_ERR_CUDA             2
#define H3DG_ERR_OUT_OF_MEMORY    3
#define H3DG_ERR_UNSUPPORTED_FORM 4
#define H3DG_ERR_MESH             5
#define H3DG_ERR_STATE            6
#define H3DG_ERR_TIMEOUT          7
#define H3DG_ERR_TOO_LARGE        8

/* boundary-condition types, as EBCType (src/space.h:44-48) */
#define H3DG_BC_ESSENTIAL 0
#define H3DG_BC_NATURAL   1
#define H3DG_BC_NONE      2

/* bilinear forms (src/integrals/h1.h:115-177) */
#define H3DG_BF_GRAD_GRAD       1   /* int_grad_u_grad_v, optionally times a per-element coefficient */
#define H3DG_BF_GRAD_GRAD_MASS  2   /* int_grad_u_grad_v + int_u_v */

/* exact solutions for h3dg_disc_norms */
#define H3DG_EXACT_ZERO      0   /* u = 0: the errors are the norms */
#define H3DG_EXACT_QUADRATIC 1   /* u = x^2 + y^2 + z^2 */
#define H3DG_EXACT_SIN       2   /* u = sin(pi x) sin(pi y) sin(pi z) */

/* surface forms (src/integrals/h1.h:184-242) */
#define H3DG_SBF_NONE 0
#define H3DG_SBF_U_V  1   /* surf_int_u_v */
#define H3DG_SLF_NONE 0
#define H3DG_SLF_G_V  1   /* surf_int_G_v, g constant per boundary marker */

/* linear forms (int_F_v, src/integrals/h1.h:136-152) */
#define H3DG_LF_NONE   0
#define H3DG_LF_CONST  1   /* F(x,y,z) = c */
#define H3DG_LF_SIN    2   /* F(x,y,z) = sin(pi x) sin(pi y) sin(pi z) */

/* volume quadrature: n Gauss points per direction, or p_d + n per direction */
#define H3DG_QUAD_FIXED   0
#define H3DG_QUAD_P_PLUS  1
#define H3DG_QUAD_STOCK   2   /* the reference's stock rule: per pair order(u) + order(v) + 1, int_F_v order 24 */

/* arithmetic of the element-matrix contraction */
#define H3DG_PREC_FP64    0
/* Split precision: geometry, load vector, lifting and coefficient products
 * in FP64; the z / y sum-factorisation stages in FP32; the x stage on the
 * tensor cores as three TF32 products (hi*hi + hi*lo + lo*hi) with FP32
 * accumulation.  Normwise relative error of the matrix below 1e-6.  Used by
 * the high-order path; where the FP64 kernels are the faster choice (low
 * orders) the matrix is assembled in FP64. */
#define H3DG_PREC_TF32X3  1
/* FP64-accurate split (no reference counterpart): geometry, load vector,
 * lifting and the z / y stages in FP64; the x stage on the tensor cores with
 * each FP64 operand cut into 7 int8 slices (Ozaki-style), exact int32
 * accumulation per slice level, recombined in FP64.  Relative error of the
 * matrix below 1e-12.  High-order path; low orders assemble in FP64. */
#define H3DG_PREC_OZAKI   2

typedef struct h3dg_mesh h3dg_mesh;
typedef struct h3dg_space h3dg_space;
typedef struct h3dg_disc h3dg_disc;

typedef int (*h3dg_bc_type_fn)(int marker, void *ctx);
typedef double (*h3dg_bc_value_fn)(int marker, double x, double y, double z, void *ctx);

int h3dg_version(void);
const char *h3dg_status_string(h3dg_status s);
const char *h3dg_last_error(void);

/* ---------------------------------------------------------------- mesh */
/* new Mesh (src/mesh.h:522) */
h3dg_status h3dg_mesh_create(h3dg_mesh **mesh);
h3dg_status h3dg_mesh_destroy(h3dg_mesh *mesh);
/* Mesh::add_vertex (src/mesh.cc:915-920), n vertices, ids 1..n in order */
h3dg_status h3dg_mesh_add_vertices(h3dg_mesh *mesh, const double *xyz, int64_t n);
/* Mesh::add_hex (src/mesh.cc:975-1000); vtx is n x 8, 1-based, RefHex order */
h3dg_status h3dg_mesh_add_hexes(h3dg_mesh *mesh, const int64_t *vtx, int64_t n);
/* Mesh::add_quad_boundary (src/mesh.cc:1061-1078); vtx is n x 4, 1-based */
h3dg_status h3dg_mesh_add_quad_boundaries(h3dg_mesh *mesh, const int64_t *vtx, const int32_t *marker, int64_t n);
/* Mesh::ugh (src/mesh.cc:1080-1102) + Mesh3DReader's outer-face check (src/loader/mesh3d.cc:272-282) */
h3dg_status h3dg_mesh_finalize(h3dg_mesh *mesh);
/* sizes: vertices, elements, facets, edges */
h3dg_status h3dg_mesh_counts(const h3dg_mesh *mesh, int64_t *nv, int64_t *ne, int64_t *nfacets, int64_t *nedges);
/* Mesh::refine_element (src/mesh.cc:1262-1279) with refinement REFT_HEX_XYZ (7,
 * src/mesh.h:97) of an active base element (one refinement level): the 8 children
 * get the next element ids, the new vertices the next vertex ids (refine_hex_8,
 * src/mesh.cc:1555-1633).  Other refinement types return H3DG_ERR_MESH. */
h3dg_status h3dg_mesh_refine_element(h3dg_mesh *mesh, int64_t elem_id, int reft);
/* The same for n elements (1-based ids, in order), rebuilding the topology once */
h3dg_status h3dg_mesh_refine_elements(h3dg_mesh *mesh, const int64_t *elem_ids, int64_t n, int reft);
/* Current arrays (sizes from h3dg_mesh_counts): xyz nv x 3, hex ne x 8 (1-based
 * vertex ids), parent ne (1-based parent id, 0 for base elements); any may be NULL */
h3dg_status h3dg_mesh_get_arrays(const h3dg_mesh *mesh, double *xyz, int64_t *hex, int64_t *parent);

/* ---------------------------------------------------------------- space */
/* H1Space(mesh, H1ShapesetLobattoHex) (src/space/h1.cc:33-37) */
h3dg_status h3dg_space_create(h3dg_mesh *mesh, h3dg_space **space);
h3dg_status h3dg_space_destroy(h3dg_space *space);
/* Space::set_bc_types / set_bc_values (src/space.cc:2087-2098); NULL = reference defaults
 * (every marker essential, value 0) */
h3dg_status h3dg_space_set_bc_types(h3dg_space *space, h3dg_bc_type_fn fn, void *ctx);
h3dg_status h3dg_space_set_bc_values(h3dg_space *space, h3dg_bc_value_fn fn, void *ctx);
/* Space::set_uniform_order / set_element_order (src/space.cc:108-150); orders is ne x 3 */
h3dg_status h3dg_space_set_uniform_order(h3dg_space *space, int px, int py, int pz);
h3dg_status h3dg_space_set_element_orders(h3dg_space *space, const int32_t *orders, int64_t ne);
/* Space::assign_dofs (src/space.cc:1991-2028), returns get_dof_count() */
h3dg_status h3dg_space_assign_dofs(h3dg_space *space, int first_dof, int stride, int64_t *ndof);
/* H1Space::get_element_assembly_list (src/space/h1.cc:130-137); elem_id is 1-based.
 * Writes min(cap, cnt) entries; *cnt receives the full length. */
h3dg_status h3dg_space_get_element_assembly_list(const h3dg_space *space, int64_t elem_id,
	int64_t *idx, int32_t *dof, double *coef, int32_t cap, int32_t *cnt);

/* ---------------------------------------------------------------- discretization */
/* Discretization() + set_num_equations(1) (src/discretization.cc:36-88); device = CUDA ordinal */
h3dg_status h3dg_disc_create(h3dg_disc **disc, int device);
h3dg_status h3dg_disc_destroy(h3dg_disc *disc);
/* set_spaces(1, &space) + set_pss (src/discretization.cc:102-134) */
h3dg_status h3dg_disc_set_space(h3dg_disc *disc, h3dg_space *space);
/* Block (m, n) of a multi-equation system whose test space (equation m)
 * differs from the trial space (equation n) (Discretization::set_spaces with
 * neq > 1, src/discretization.cc:290-325): the next create_pattern plans the
 * block with rows from the test space and columns from the trial space, each
 * counted from its own first DOF; the trial space's Dirichlet lifting goes to
 * the test rows.  nullptr (or the trial space): one space.  FP64, one mesh,
 * uniform orders per space, no refinement, partition, surface forms or stock
 * rule (H3DG_ERR_INVALID_ARG at create_pattern). */
h3dg_status h3dg_disc_set_test_space(h3dg_disc *disc, h3dg_space *test);
/* set_bilinear_form(0, 0, form) (src/discretization.cc:136-148); elem_coef: one value per
 * element id (ne values, multiplies the grad-grad term), or NULL for 1 */
h3dg_status h3dg_disc_set_bilinear_form(h3dg_disc *disc, int form, const double *elem_coef, int64_t ne);
/* set_linear_form(0, lf) (src/discretization.cc:151-161); value is the constant for H3DG_LF_CONST */
h3dg_status h3dg_disc_set_linear_form(h3dg_disc *disc, int form, double value);
/* No reference counterpart (the reference solves with UMFPACK,
 * src/linsolver/umfpack.cc:280-330): Jacobi-preconditioned conjugate gradients on the
 * assembled matrix (d_Ax in the plan's CSC pattern; the forms are symmetric) for the
 * RHS d_rhs, starting from d_x and overwriting it, until ||r|| <= rtol ||b|| or maxit
 * iterations; bitwise reproducible.  Synchronises `stream` every iteration. */
h3dg_status h3dg_disc_solve_cg(h3dg_disc *disc, const double *d_Ax, const double *d_rhs, double *d_x, double rtol,
                               int maxit, int *iters, double *relres, void *stream);
/* Norms of the finite-element function with coefficient vector d_sol (device,
 * ndof doubles; Dirichlet parts from the space's lifting), as calc_error /
 * calc_norm with the H1 and L2 functions (src/norm.cc:33-180): out[0] = L2 error,
 * out[1] = H1 error against the exact solution `exact` (H3DG_EXACT_*), out[2] = L2
 * norm, out[3] = H1 norm of the function itself; each integral with the rule of
 * the assembly (set_quadrature), the square root taken above 1e-14 as in the
 * reference.  Synchronises `stream`. */
h3dg_status h3dg_disc_norms(h3dg_disc *disc, const double *d_sol, int exact, double *out, void *stream);
/* surface forms on the outer faces whose marker is natural (set_bilinear_form's
 * and set_linear_form's surf arguments, src/discretization.cc:136-161, assembled as
 * src/discretization.cc:345-412): bilinear H3DG_SBF_U_V = surf_int_u_v, linear
 * H3DG_SLF_G_V = surf_int_G_v with g constant per boundary marker (g[marker], ng values,
 * markers 0..15; src/integrals/h1.h:200-242), each integrated with the element's rule on
 * the face's two directions.  As in the reference, the surface pass runs only when the
 * matrix is assembled, and its Dirichlet lifting reaches the RHS only with a surface
 * linear form.  Set before create_pattern; not supported on refined meshes. */
h3dg_status h3dg_disc_set_surface_forms(h3dg_disc *disc, int bilinear, int linear, const double *g, int ng);
/* quadrature of the forms: mode H3DG_QUAD_FIXED (n points per direction) or
 * H3DG_QUAD_P_PLUS (p_d + n points per direction), as the explicit-order forms
 * of tests/integrals/hex-h1-real/h1-hex-real.cc:55-103 fix it; or
 * H3DG_QUAD_STOCK (n ignored), the rule of the stock int_grad_u_grad_v /
 * int_u_v / int_F_v (src/integrals/h1.h:115-177): each pair integrated with
 * order(u) + order(v) + 1 per direction, the load vector with order 24.
 * STOCK: uniform orders 1..3, FP64, no refinement or surface forms
 * (H3DG_ERR_INVALID_ARG at create_pattern otherwise). */
h3dg_status h3dg_disc_set_quadrature(h3dg_disc *disc, int mode, int n);
/* Discretization::create (src/discretization.cc:164-230) + UMFPackMatrix::alloc
 * (src/linsolver/umfpack.cc:46-71): builds the CSC pattern and the device plan */
h3dg_status h3dg_disc_create_pattern(h3dg_disc *disc, int64_t *ndof, int64_t *nnz);
/* No reference counterpart: the precision the next create_pattern plans for.
 * With H3DG_PREC_TF32X3 the plan takes the high-order (tensor-core capable)
 * form from order 4 up instead of 5, where the 3xTF32 kernel is already the
 * faster one; assemble's precision argument still selects the arithmetic. */
h3dg_status h3dg_disc_set_precision(h3dg_disc *disc, int precision);
/* No reference counterpart (multi-GPU sharding, one process per GPU): build
 * the next plan for part `part` of `nparts` z-slabs of the mesh.  The part
 * assembles its slab of elements plus the one-element halo that touches its
 * DOFs and produces the full CSC columns (and rhs entries) of the DOFs it
 * owns -- equal to those of the whole-mesh assembly -- with empty columns
 * elsewhere; no data moves between parts.  A DOF belongs to the part whose
 * slab holds the lowest-numbered element listing it.  rhs entries of DOFs
 * not owned hold partial sums: read the owned ones.  nparts = 1 (default):
 * the whole mesh. */
h3dg_status h3dg_disc_set_partition(h3dg_disc *disc, int nparts, int part);
/* owned-DOF mask (ndof bytes, 1 = owned) and element counts of the current
 * plan's part; any pointer may be NULL */
h3dg_status h3dg_disc_get_partition(const h3dg_disc *disc, uint8_t *owned, int64_t *nslab, int64_t *nhalo, int64_t *nowned);
/* elements the current plan's part assembles (slab + halo): ne bytes, 1 = in the part */
h3dg_status h3dg_disc_get_partition_elements(const h3dg_disc *disc, uint8_t *in_part, int64_t ne);
/* UMFPackMatrix Ap (ndof+1, widened to int64: nnz can exceed INT_MAX) and Ai (nnz) */
h3dg_status h3dg_disc_get_pattern(const h3dg_disc *disc, int64_t *Ap, int32_t *Ai);
/* Discretization::assemble (src/discretization.cc:232-422) into device arrays
 * d_Ax (nnz, CSC order of the pattern) and d_rhs (ndof); either may be NULL.
 * stream: a cudaStream_t, or NULL for the default stream. */
h3dg_status h3dg_disc_assemble(h3dg_disc *disc, int precision, double *d_Ax, double *d_rhs, void *stream);
/* the same into host arrays (UMFPackMatrix::Ax / UMFPackVector::v); copies inside */
h3dg_status h3dg_disc_assemble_host(h3dg_disc *disc, int precision, double *Ax, double *rhs);
/* No reference counterpart.  h3dg_disc_assemble_host without any device
 * allocation, for callers that must not allocate: an application whose
 * device memory is fully reserved by its own pool (cudaMalloc would fail),
 * or one that cannot afford the implicit device-wide synchronisation of
 * cudaFree while other streams run.  Ax and rhs are staged in a fixed
 * 16 MiB device array of the library (H3DG_NOALLOC_SCRATCH_DOUBLES doubles,
 * shared by Ax and rhs, the rhs part starting on a 256-byte boundary);
 * larger problems are rejected with H3DG_ERR_TOO_LARGE.  Preconditions
 * (H3DG_ERR_STATE otherwise): one allocating device call on this disc with
 * the same precision came first on the current plan (h3dg_disc_assemble or
 * h3dg_disc_assemble_host), so the device plan, the autotuned variant and
 * the split-precision scatter stream and work area exist.  Every call looks
 * up the array's address (cudaGetSymbolAddress, which allocates nothing once
 * the library's module is loaded) with the disc's device current, so a
 * cudaDeviceReset between calls leaves no stale address; make the first call
 * outside any stream capture, since it may load the module.  The array is
 * zeroed by the assembly itself.  Calls that overlap in time on one device
 * share the array and race: serialise them. */
#define H3DG_NOALLOC_SCRATCH_DOUBLES (2u << 20)
h3dg_status h3dg_disc_assemble_host_noalloc(h3dg_disc *disc, int precision, double *Ax, double *rhs);
/* replace the vertex coordinates (same topology) from host memory, nv x 3 */
h3dg_status h3dg_disc_update_vertices(h3dg_disc *disc, const double *xyz, int64_t nv);
/* replace the per-element coefficient (ne values, element-id order) from host memory */
h3dg_status h3dg_disc_update_coefficients(h3dg_disc *disc, const double *elem_coef, int64_t ne);
/* the same from device memory, ordered on `stream` (no host copy, no
 * synchronisation; the host-side copy of the coefficients is not updated) */
h3dg_status h3dg_disc_update_coefficients_device(h3dg_disc *disc, const double *d_elem_coef, int64_t ne, void *stream);
/* number of kernels launched by the last assemble call */
h3dg_status h3dg_disc_last_launch_count(const h3dg_disc *disc, int32_t *count);
/* the element-matrix kernel family of the last volume assembly (no reference
 * counterpart; for tests and measurement): */
#define H3DG_KERNEL_OTHER 0          /* low orders, mixed orders, stock rule */
#define H3DG_KERNEL_HO_FP64_FMA 1    /* high order, FP64 on the FMA pipe */
#define H3DG_KERNEL_HO_FP64_DMMA 2   /* high order, FP64 on the FP64 tensor cores (p >= 4, one space) */
#define H3DG_KERNEL_HO_TF32X3 3      /* high order, 3xTF32 on tcgen05 */
#define H3DG_KERNEL_HO_OZAKI 4       /* high order, int8 slices on tcgen05 */
h3dg_status h3dg_disc_last_kernel(const h3dg_disc *disc, int32_t *kind);

/* the kernel variant the autotuner picked on the first assembly of the
 * current plan: threads per CTA, elements per CTA pass, and the time of one
 * assembly with it in milliseconds (all -1 / 0 before the first assembly).
 * No reference counterpart. */
h3dg_status h3dg_disc_get_tuning(const h3dg_disc *disc, int32_t *threads, int32_t *elems_per_cta, float *ms);
/* which scatter the picked low-order variant uses: 1 segmented (element
 * matrices into an L2-resident ring, every CSC column summed in assembly
 * order and written once), 0 colour sweeps, -1 not tuned.  Both give the
 * same bits.  No reference counterpart. */
h3dg_status h3dg_disc_tuned_scatter(const h3dg_disc *disc, int32_t *segmented);
/* statistics of the last segmented assembly (a measurement hook, no
 * reference counterpart): out[0..3] element items that waited and their
 * polls, column items that waited and their polls; out[4..7] items, ring
 * windows, CTAs, column span in windows. */
h3dg_status h3dg_disc_seg_stats(const h3dg_disc *disc, int64_t *out);

/* Kernel-only timing (no reference counterpart; a measurement hook): when
 * enabled with capacity n, each assemble call records a CUDA event pair on its
 * launch stream around its kernel launches (after the output zeroing), up to
 * n calls.  h3dg_disc_kernel_times synchronises those events and returns the
 * elapsed milliseconds of each recorded call, then clears the records. */
h3dg_status h3dg_disc_enable_kernel_timing(h3dg_disc *disc, int32_t n);
h3dg_status h3dg_disc_kernel_times(h3dg_disc *disc, float *ms, int32_t cap, int32_t *n);

/* Adjoint of the coefficient-weighted assembly (no reference counterpart: the
 * reference has no adjoint).  For nfields fields k with per-element
 * log-coefficients g_k (a = exp(g) multiplies the grad-grad term, as the
 * coefficient of h3dg_disc_set_bilinear_form does) and vectors u_k, lambda_k:
 *   L_k = lambda_k^T K(a_k) u_k - lambda_k^T f(a_k),
 *   d_S[k][e]    = lambda_e^T K_e^(1) (u_e + d_e)   (unit coefficient; d_e Dirichlet lifting
 *                  when a linear form is set)
 *   d_grad[k][e] = dL_k / dg_{k,e} = exp(g_{k,e}) d_S[k][e].
 * Device arrays: d_logcoef nfields x ne (element-id order, or NULL for a = 1),
 * d_u and d_lambda nfields x ndof, d_S and d_grad nfields x ne (either may be NULL).
 * Uniform and mixed-order plans, hanging nodes included (orders up to 8, rules up to
 * 10 points per direction on the mixed path); ne counts every element id, and ids
 * of refined (inactive) elements get zero. */
h3dg_status h3dg_disc_adjoint(h3dg_disc *disc, int nfields, const double *d_logcoef, const double *d_u,
	const double *d_lambda, double *d_S, double *d_grad, void *stream);

/* Diagnostic (no reference counterpart): one 128 x 128 tcgen05 MMA tile,
 * C = A B^T, A and B 128 x K row-major floats (K = 32 for kind 2 = tf32,
 * K = 64 for kind 1 = bf16 and kind 8 = int8, integer values in -128..127;
 * the int32 result is returned as floats), C 128 x 128; device pointers.
 * Checks the tensor-core layer the split-precision kernels use. */
h3dg_status h3dg_tc_selftest(int kind, const float *d_A, const float *d_B, float *d_C, int device);

/* Test hooks (no reference counterpart): drive the failure paths of an
 * assembly without any device fault.
 *   H3DG_DEBUG_WAIT_GIVES_UP: the next FP64 low-order assembly gives its
 *     bounded table-staging wait no polls at all, so every CTA records a
 *     timeout, drains its copy and leaves; h3dg_disc_assemble_host then
 *     returns H3DG_ERR_TIMEOUT and the following assembly runs normally.
 *   H3DG_DEBUG_CORRUPT_POSITION: one entry of the device position map of a
 *     low-order plan is set past the end of its CSC column; the bounds check
 *     skips that store and assemblies report H3DG_ERR_STATE until
 *     h3dg_disc_create_pattern builds the plan again. */
#define H3DG_DEBUG_WAIT_GIVES_UP    1
#define H3DG_DEBUG_CORRUPT_POSITION 2
h3dg_status h3dg_disc_debug_inject(h3dg_disc *disc, int what);

/* RefMap (src/refmap.cc:177-231, 265-316): per element (id order) and per point of the
 * disc's volume rule, the signed Jacobian determinant (get_jacobian without the
 * weight), the transposed inverse Jacobian irm[r][c] = (J^-1)[c][r] (get_inv_ref_map)
 * and the physical coordinates (get_phys_x/y/z).  Device arrays: d_jac ne*nq,
 * d_irm ne*nq*9, d_xyz ne*nq*3 (any may be NULL). */
h3dg_status h3dg_disc_geometry(h3dg_disc *disc, double *d_jac, double *d_irm, double *d_xyz, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* H3DG_H */
