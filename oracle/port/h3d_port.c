/*
 * CPU restatement of the Hermes3D reference's hexahedral H1 assembly.
 * ORACLE / TEST INFRASTRUCTURE ONLY (see h3d_port.h).
 *
 * Follows, in plain C:
 *   shape index decoding     src/shapeset/h1lobattohex.cc:36-130 (h1_hex_index_t, decompose)
 *   shape values/gradients   src/shapeset/h1lobattohex.cc:134-213 (calc_fn/dx/dy/dz_value)
 *   1D Lobatto functions     src/shapeset/lobatto.h:80-109
 *   reference map            src/refmap.cc:177-231 (calc_inv_ref_map), 265-316 (calc_phys_*)
 *   integrands               src/integrals/h1.h:31-177 (T_DUDX.., H1_INTEGRATE_*)
 *   element loop / lifting   src/discretization.cc:232-338
 *   CSC insert               src/linsolver/umfpack.cc:80-152 (update, insert_value)
 *   pattern                  src/discretization.cc:164-230, src/matrix.cc:156-189
 */
#include "h3d_port.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- 1D Lobatto functions: l0, l1 linear; l_k = (P_k - P_{k-2}) / sqrt(2(2k-1)),
 *      l_k' = sqrt((2k-1)/2) P_{k-1}  (the reference writes the same polynomials
 *      as (1-x^2)/4 * phi_{k-2}(x)) */
static void legendre(int n, double x, double *P) {
	P[0] = 1.0;
	if (n >= 1) P[1] = x;
	for (int k = 1; k < n; k++) P[k + 1] = ((2 * k + 1) * x * P[k] - k * P[k - 1]) / (k + 1);
}

static double lob(int k, double x) {
	double P[16];
	if (k == 0) return (1.0 - x) * 0.5;
	if (k == 1) return (1.0 + x) * 0.5;
	legendre(k, x, P);
	return (P[k] - P[k - 2]) / sqrt(2.0 * (2 * k - 1));
}

static double dlob(int k, double x) {
	double P[16];
	if (k == 0) return -0.5;
	if (k == 1) return 0.5;
	legendre(k - 1, x, P);
	return sqrt((2.0 * k - 1) / 2.0) * P[k - 1];
}

/* ---- decompose(): directional indices and argument flips of a shape index */
static void decompose(int64_t index, int ind[3], int ori[3]) {
	int o = (int) ((index >> 12) & 7);
	int permut[3] = { 0, 1, 2 }, n01 = 0, t;
	ind[0] = (int) ((index >> 8) & 15);
	ind[1] = (int) ((index >> 4) & 15);
	ind[2] = (int) (index & 15);
	/* find_permutation */
	if (ind[0] < 2) n01++;
	if (ind[1] < 2) {
		n01++;
		if (n01 == 1) { t = permut[0]; permut[0] = permut[1]; permut[1] = t; }
	}
	if (ind[2] < 2) {
		n01++;
		if (n01 == 1) {
			t = permut[1]; permut[1] = permut[2]; permut[2] = t;
			t = permut[0]; permut[0] = permut[1]; permut[1] = t;
		}
		if (n01 == 2) { t = permut[1]; permut[1] = permut[2]; permut[2] = t; }
	}
	ori[0] = ori[1] = ori[2] = 0;
	if (n01 == 2) ori[permut[2]] = o;
	else if (n01 == 1) {
		if (o % 2 == 1) ori[permut[1]] = 1;
		if (o % 4 >= 2) ori[permut[2]] = 1;
		if (o >= 4) {
			t = ind[permut[1]]; ind[permut[1]] = ind[permut[2]]; ind[permut[2]] = t;
			t = ori[permut[1]]; ori[permut[1]] = ori[permut[2]]; ori[permut[2]] = t;
		}
	}
}

/* value, d/dxi, d/deta, d/dzeta of shape `index` at a reference point */
static void shape_eval(int64_t index, double x, double y, double z, double out[4]) {
	int ind[3], ori[3];
	decompose(index, ind, ori);
	if (ori[0]) x = -x;
	if (ori[1]) y = -y;
	if (ori[2]) z = -z;
	double lx = lob(ind[0], x), ly = lob(ind[1], y), lz = lob(ind[2], z);
	out[0] = lx * ly * lz;
	out[1] = dlob(ind[0], x) * ly * lz;
	out[2] = lx * dlob(ind[1], y) * lz;
	out[3] = lx * ly * dlob(ind[2], z);
	if (ori[0]) out[1] = -out[1];
	if (ori[1]) out[2] = -out[2];
	if (ori[2]) out[3] = -out[3];
}

/* ---- Gauss-Legendre rule (ascending, symmetric) */
static void gauss(int n, double *pts, double *wts) {
	for (int i = 0; i < (n + 1) / 2; i++) {
		long double x = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L)), dp = 0;
		for (int it = 0; it < 100; it++) {
			long double p0 = 1, p1 = x;
			for (int k = 1; k < n; k++) {
				long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
				p0 = p1;
				p1 = p2;
			}
			if (n == 1) { p1 = x; p0 = 1; }
			dp = n * (x * p1 - p0) / (x * x - 1);
			long double dx = p1 / dp;
			x -= dx;
			if (fabsl(dx) < 1e-19L) {
				p0 = 1; p1 = x;
				for (int k = 1; k < n; k++) {
					long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
					p0 = p1;
					p1 = p2;
				}
				if (n == 1) { p1 = x; p0 = 1; }
				dp = n * (x * p1 - p0) / (x * x - 1);
				break;
			}
		}
		long double w = 2.0L / ((1 - x * x) * dp * dp);
		pts[n - 1 - i] = (double) x;
		pts[i] = -(double) x;
		wts[n - 1 - i] = wts[i] = (double) w;
	}
	if (n % 2) pts[n / 2] = 0.0;
}

static const int kVtxXYZ[8][3] = { { 0, 0, 0 }, { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 },
                                   { 0, 0, 1 }, { 1, 0, 1 }, { 1, 1, 1 }, { 0, 1, 1 } };

/* RefMap at one point: jac = signed det, irm = transposed inverse, phys point */
static void refmap(const double *X, double x, double y, double z, double *jac, double irm[3][3], double xp[3]) {
	double m[3][3] = { { 0 } };
	xp[0] = xp[1] = xp[2] = 0.0;
	for (int v = 0; v < 8; v++) {
		double lx = lob(kVtxXYZ[v][0], x), ly = lob(kVtxXYZ[v][1], y), lz = lob(kVtxXYZ[v][2], z);
		double dx = dlob(kVtxXYZ[v][0], x) * ly * lz, dy = lx * dlob(kVtxXYZ[v][1], y) * lz, dz = lx * ly * dlob(kVtxXYZ[v][2], z);
		for (int r = 0; r < 3; r++) {
			m[r][0] += X[3 * v + r] * dx;
			m[r][1] += X[3 * v + r] * dy;
			m[r][2] += X[3 * v + r] * dz;
			xp[r] += X[3 * v + r] * (lx * ly * lz);
		}
	}
	double d = m[0][0] * m[1][1] * m[2][2] + m[0][1] * m[1][2] * m[2][0] + m[0][2] * m[1][0] * m[2][1] -
	           m[2][0] * m[1][1] * m[0][2] - m[2][1] * m[1][2] * m[0][0] - m[2][2] * m[1][0] * m[0][1];
	double ij = 1.0 / d;
	irm[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * ij;
	irm[1][0] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * ij;
	irm[2][0] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * ij;
	irm[0][1] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * ij;
	irm[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * ij;
	irm[2][1] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * ij;
	irm[0][2] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * ij;
	irm[1][2] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * ij;
	irm[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * ij;
	*jac = d;
}

static double source(int lf, double val, const double xp[3]) {
	if (lf == 1) return val;
	if (lf == 2) {
		const double pi = 3.141592653589793238462643383279502884;
		return sin(pi * xp[0]) * sin(pi * xp[1]) * sin(pi * xp[2]);
	}
	return 0.0;
}

typedef struct {
	int np;
	double *w, *jac, *irm, *xp;   /* per point */
	double *sv;                   /* per (entry, point): value, dx, dy, dz */
} ElemCache;

static int elem_cache(const double *X, int nqx, int nqy, int nqz, int cnt, const int64_t *idx, ElemCache *c) {
	double qx[16], wx[16], qy[16], wy[16], qz[16], wz[16];
	gauss(nqx, qx, wx);
	gauss(nqy, qy, wy);
	gauss(nqz, qz, wz);
	int np = nqx * nqy * nqz;
	c->np = np;
	c->w = malloc(sizeof(double) * np);
	c->jac = malloc(sizeof(double) * np);
	c->irm = malloc(sizeof(double) * 9 * np);
	c->xp = malloc(sizeof(double) * 3 * np);
	c->sv = malloc(sizeof(double) * 4 * (size_t) np * (cnt > 0 ? cnt : 1));
	if (!c->w || !c->jac || !c->irm || !c->xp || !c->sv) return -1;
	/* tensor points, x outermost, z innermost (src/quadstd.cc:4367-4388) */
	for (int k = 0, n = 0; k < nqx; k++)
		for (int l = 0; l < nqy; l++)
			for (int p = 0; p < nqz; p++, n++) {
				c->w[n] = wx[k] * wy[l] * wz[p];
				refmap(X, qx[k], qy[l], qz[p], &c->jac[n], (double(*)[3]) & c->irm[9 * n], &c->xp[3 * n]);
				for (int i = 0; i < cnt; i++) shape_eval(idx[i], qx[k], qy[l], qz[p], &c->sv[4 * ((size_t) i * np + n)]);
			}
	return 0;
}

static void elem_free(ElemCache *c) {
	free(c->w); free(c->jac); free(c->irm); free(c->xp); free(c->sv);
}

/* int_grad_u_grad_v (+ int_u_v) between entries j (u) and i (v) */
static double biform(const ElemCache *c, int j, int i, int mass, double gcoef) {
	double result = 0.0;
	for (int q = 0; q < c->np; q++) {
		const double *mu = &c->irm[9 * q];
		const double *u = &c->sv[4 * ((size_t) j * c->np + q)], *v = &c->sv[4 * ((size_t) i * c->np + q)];
		double ux = u[1] * mu[0] + u[2] * mu[1] + u[3] * mu[2];
		double uy = u[1] * mu[3] + u[2] * mu[4] + u[3] * mu[5];
		double uz = u[1] * mu[6] + u[2] * mu[7] + u[3] * mu[8];
		double vx = v[1] * mu[0] + v[2] * mu[1] + v[3] * mu[2];
		double vy = v[1] * mu[3] + v[2] * mu[4] + v[3] * mu[5];
		double vz = v[1] * mu[6] + v[2] * mu[7] + v[3] * mu[8];
		result += c->w[q] * c->jac[q] * (ux * vx + uy * vy + uz * vz);
	}
	result *= gcoef;
	if (mass) {
		double m = 0.0;
		for (int q = 0; q < c->np; q++)
			m += c->w[q] * c->jac[q] * (c->sv[4 * ((size_t) j * c->np + q)] * c->sv[4 * ((size_t) i * c->np + q)]);
		result += m;
	}
	return result;
}

static double liform(const ElemCache *c, int i, int lf, double val) {
	double result = 0.0;
	for (int q = 0; q < c->np; q++)
		result += c->w[q] * c->jac[q] * (c->sv[4 * ((size_t) i * c->np + q)] * source(lf, val, &c->xp[3 * q]));
	return result;
}

static int cmp_i32(const void *a, const void *b) {
	int32_t x = *(const int32_t *) a, y = *(const int32_t *) b;
	return (x > y) - (x < y);
}

int h3d_port_pattern(int64_t ne, const int64_t *al_ptr, const int32_t *al_dof, int64_t ndof, int64_t *Ap,
                     int32_t *Ai, int64_t *nnz) {
	/* per column: rows of every element holding the column DOF */
	int64_t *cnt = calloc(ndof + 1, sizeof(int64_t));
	if (!cnt) return -1;
	for (int64_t e = 0; e < ne; e++) {
		int64_t m = 0;
		for (int64_t k = al_ptr[e]; k < al_ptr[e + 1]; k++) m += al_dof[k] >= 0;
		for (int64_t k = al_ptr[e]; k < al_ptr[e + 1]; k++)
			if (al_dof[k] >= 0) cnt[al_dof[k] + 1] += m;
	}
	for (int64_t d = 0; d < ndof; d++) cnt[d + 1] += cnt[d];
	int32_t *rows = malloc(sizeof(int32_t) * (cnt[ndof] > 0 ? cnt[ndof] : 1));
	int64_t *fill = malloc(sizeof(int64_t) * (ndof + 1));
	if (!rows || !fill) { free(cnt); free(rows); free(fill); return -1; }
	memcpy(fill, cnt, sizeof(int64_t) * (ndof + 1));
	for (int64_t e = 0; e < ne; e++)
		for (int64_t k = al_ptr[e]; k < al_ptr[e + 1]; k++) {
			if (al_dof[k] < 0) continue;
			for (int64_t r = al_ptr[e]; r < al_ptr[e + 1]; r++)
				if (al_dof[r] >= 0) rows[fill[al_dof[k]]++] = al_dof[r];
		}
	int64_t pos = 0;
	for (int64_t d = 0; d < ndof; d++) {
		int32_t *b = rows + cnt[d];
		int64_t n = cnt[d + 1] - cnt[d];
		qsort(b, (size_t) n, sizeof(int32_t), cmp_i32);
		if (Ap) Ap[d] = pos;
		int32_t last = -1;
		for (int64_t i = 0; i < n; i++)
			if (b[i] != last) {
				if (Ai) Ai[pos] = b[i];
				pos++;
				last = b[i];
			}
	}
	if (Ap) Ap[ndof] = pos;
	*nnz = pos;
	free(cnt); free(rows); free(fill);
	return 0;
}

static int insert_value(const int32_t *ai, double *ax, int64_t len, int32_t row, double v) {
	int64_t lo = 0, hi = len - 1;
	while (lo <= hi) {
		int64_t mid = (lo + hi) >> 1;
		if (row < ai[mid]) hi = mid - 1;
		else if (row > ai[mid]) lo = mid + 1;
		else { ax[mid] += v; return 0; }
	}
	return -1;   /* "Sparse matrix entry not found." */
}

int h3d_port_assemble(int64_t nv, const double *xyz, int64_t ne, const int64_t *hex, const int32_t *nq,
                      const int64_t *al_ptr, const int64_t *al_idx, const int32_t *al_dof, const double *al_coef,
                      int mass, const double *gradcoef, int lf, double lf_value, int64_t ndof, const int64_t *Ap,
                      const int32_t *Ai, double *Ax, double *rhs) {
	(void) nv;
	if (Ax) memset(Ax, 0, sizeof(double) * Ap[ndof]);
	if (rhs) memset(rhs, 0, sizeof(double) * ndof);
	for (int64_t e = 0; e < ne; e++) {
		double X[24];
		for (int v = 0; v < 8; v++)
			for (int r = 0; r < 3; r++) X[3 * v + r] = xyz[3 * hex[8 * e + v] + r];
		int cnt = (int) (al_ptr[e + 1] - al_ptr[e]);
		const int64_t *idx = al_idx + al_ptr[e];
		const int32_t *dof = al_dof + al_ptr[e];
		const double *coef = al_coef + al_ptr[e];
		ElemCache c;
		if (elem_cache(X, nq[3 * e], nq[3 * e + 1], nq[3 * e + 2], cnt, idx, &c) != 0) return -1;
		double gc = gradcoef ? gradcoef[e] : 1.0;
		double *lsm = calloc((size_t) cnt * cnt + 1, sizeof(double));
		double *lrhs = calloc((size_t) cnt + 1, sizeof(double));
		for (int j = 0; j < cnt; j++)
			for (int i = 0; i < cnt; i++) {
				if (dof[i] < 0) continue;
				double bi = biform(&c, j, i, mass, gc) * coef[j] * coef[i];
				if (dof[j] >= 0) lsm[(size_t) i * cnt + j] += bi;
				else lrhs[i] -= bi;
			}
		if (Ax)
			for (int i = 0; i < cnt; i++)
				for (int j = 0; j < cnt; j++) {
					double v = lsm[(size_t) i * cnt + j];
					if (v != 0.0 && dof[i] >= 0 && dof[j] >= 0)
						if (insert_value(Ai + Ap[dof[j]], Ax + Ap[dof[j]], Ap[dof[j] + 1] - Ap[dof[j]], dof[i], v) != 0) {
							free(lsm); free(lrhs); elem_free(&c);
							return -2;
						}
				}
		if (rhs && lf) {
			for (int i = 0; i < cnt; i++)
				if (dof[i] >= 0) lrhs[i] += liform(&c, i, lf, lf_value) * coef[i];
			for (int i = 0; i < cnt; i++)
				if (dof[i] >= 0) rhs[dof[i]] += lrhs[i];
		}
		free(lsm);
		free(lrhs);
		elem_free(&c);
	}
	return 0;
}

int h3d_port_element_matrix(const double *X, int nqx, int nqy, int nqz, int cnt, const int64_t *idx, int mass,
                            double gradcoef, double *K) {
	ElemCache c;
	if (elem_cache(X, nqx, nqy, nqz, cnt, idx, &c) != 0) return -1;
	for (int i = 0; i < cnt; i++)
		for (int j = 0; j < cnt; j++) K[(size_t) i * cnt + j] = biform(&c, j, i, mass, gradcoef);
	elem_free(&c);
	return 0;
}

int h3d_port_element_rows(const double *X, int nqx, int nqy, int nqz, int cnt, const int64_t *idx, int nrows,
                          const int32_t *rows, int mass, double gradcoef, double *out) {
	ElemCache c;
	if (elem_cache(X, nqx, nqy, nqz, cnt, idx, &c) != 0) return -1;
	for (int r = 0; r < nrows; r++)
		for (int j = 0; j < cnt; j++) out[(size_t) r * cnt + j] = biform(&c, j, rows[r], mass, gradcoef);
	elem_free(&c);
	return 0;
}

/* ---- the reference's stock quadrature (src/integrals/h1.h:115-177):
 * int_grad_u_grad_v and int_u_v integrate each pair with the order
 * order(u) + order(v) + (1,1,1) per direction (the inverse map's order of a
 * hexahedron, src/refmap.cc:140-142), capped at 24 (order.h limit()); the 1D
 * order of Lobatto function k is max(k, 1) (src/shapeset/lobatto.cc:23); a
 * rule of order o has o / 2 + 1 Gauss points (src/quadstd.cc:179-205).
 * int_F_v uses the maximal order 24 (13 points) in every direction. */
static int stock_ord1d(int k) { return k < 2 ? 1 : k; }
static int stock_npts(int o) { return (o > 24 ? 24 : o) / 2 + 1; }

int h3d_port_assemble_stock(int64_t nv, const double *xyz, int64_t ne, const int64_t *hex, const int64_t *al_ptr,
                            const int64_t *al_idx, const int32_t *al_dof, const double *al_coef, int mass,
                            const double *gradcoef, int lf, double lf_value, int64_t ndof, const int64_t *Ap,
                            const int32_t *Ai, double *Ax, double *rhs) {
	(void) nv;
	if (Ax) memset(Ax, 0, sizeof(double) * Ap[ndof]);
	if (rhs) memset(rhs, 0, sizeof(double) * ndof);
	for (int64_t e = 0; e < ne; e++) {
		double X[24];
		for (int v = 0; v < 8; v++)
			for (int r = 0; r < 3; r++) X[3 * v + r] = xyz[3 * hex[8 * e + v] + r];
		int cnt = (int) (al_ptr[e + 1] - al_ptr[e]);
		const int64_t *idx = al_idx + al_ptr[e];
		const int32_t *dof = al_dof + al_ptr[e];
		const double *coef = al_coef + al_ptr[e];
		int (*ord)[3] = malloc(sizeof(int[3]) * (cnt > 0 ? cnt : 1));
		for (int i = 0; i < cnt; i++) {
			int ind[3], ori[3];
			decompose(idx[i], ind, ori);
			for (int d = 0; d < 3; d++) ord[i][d] = stock_ord1d(ind[d]);
		}
		/* one cache per rule triple met (2..13 points per direction) */
		ElemCache *cache[14 * 14 * 14];
		memset(cache, 0, sizeof(cache));
		double gc = gradcoef ? gradcoef[e] : 1.0;
		double *lsm = calloc((size_t) cnt * cnt + 1, sizeof(double));
		double *lrhs = calloc((size_t) cnt + 1, sizeof(double));
		int rc = 0;
		for (int j = 0; j < cnt && !rc; j++)
			for (int i = 0; i < cnt && !rc; i++) {
				if (dof[i] < 0) continue;
				int n[3];
				for (int d = 0; d < 3; d++) n[d] = stock_npts(ord[j][d] + ord[i][d] + 1);
				ElemCache **cp = &cache[(n[0] * 14 + n[1]) * 14 + n[2]];
				if (!*cp) {
					*cp = malloc(sizeof(ElemCache));
					if (!*cp || elem_cache(X, n[0], n[1], n[2], cnt, idx, *cp) != 0) { rc = -1; break; }
				}
				double bi = biform(*cp, j, i, mass, gc) * coef[j] * coef[i];
				if (dof[j] >= 0) lsm[(size_t) i * cnt + j] += bi;
				else lrhs[i] -= bi;
			}
		if (!rc && Ax)
			for (int i = 0; i < cnt && !rc; i++)
				for (int j = 0; j < cnt; j++) {
					double v = lsm[(size_t) i * cnt + j];
					if (v != 0.0 && dof[i] >= 0 && dof[j] >= 0)
						if (insert_value(Ai + Ap[dof[j]], Ax + Ap[dof[j]], Ap[dof[j] + 1] - Ap[dof[j]], dof[i], v) != 0) {
							rc = -2;
							break;
						}
				}
		if (!rc && rhs && lf) {
			ElemCache c13;
			if (elem_cache(X, 13, 13, 13, cnt, idx, &c13) != 0) rc = -1;
			else {
				for (int i = 0; i < cnt; i++)
					if (dof[i] >= 0) lrhs[i] += liform(&c13, i, lf, lf_value) * coef[i];
				for (int i = 0; i < cnt; i++)
					if (dof[i] >= 0) rhs[dof[i]] += lrhs[i];
				elem_free(&c13);
			}
		}
		for (int k = 0; k < 14 * 14 * 14; k++)
			if (cache[k]) {
				elem_free(cache[k]);
				free(cache[k]);
			}
		free(lsm);
		free(lrhs);
		free(ord);
		if (rc) return rc;
	}
	return 0;
}

