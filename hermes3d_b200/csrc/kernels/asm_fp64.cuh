// FP64 element-matrix + deterministic scatter, EB elements per CTA pass.
//
// Replaces the per-pair form calls of Discretization::assemble
// (src/discretization.cc:290-325) with int_grad_u_grad_v / int_u_v / int_F_v
// (src/integrals/h1.h:115-177), and the binary-search insert of
// UMFPackMatrix::update (src/linsolver/umfpack.cc:80-152).
//
// Element matrix.  With G_q = w_q det J_q J_q^-1 J_q^-T (times the element
// coefficient) the grad-grad matrix in the canonical tensor basis
// phi_abc = L_a(xi) L_b(eta) L_c(zeta) is
//     K_ij = sum_q sum_rs G_q[r][s] d_r phi_i(q) d_s phi_j(q).
// It is formed as K = A + A^T with
//     A = sum_r (G_rr/2) B_r^T B_r + sum_{r<s} G_rs B_r^T B_s  (+ (M/2) V^T V)
// and every one of the 7 terms is contracted by sum factorisation over the
// three quadrature directions, because each factor d_r phi_i(q) is a
// product of 1D table entries:
//   stage 1  T1_t[q1][q2][c][c'] = sum_q3 G_t[q1][q2][q3] Wz_t[c][c'][q3]
//   stage 2  T2_t[q1][b][b'][cc'] = sum_q2 Wy_t[b][b'][q2] T1_t[q1][q2][cc']
//   stage 3  A[(a,b,c)][(a',b',c')] = sum_t sum_q1 Wx_t[a][a'][q1] T2_t[q1][bb'cc']
// Work per element is O(nq p^6) instead of the O(nq^3 p^6) of the dense
// per-pair loops.  The 7 terms use only 3 distinct x tables (value/value,
// derivative/value, derivative/derivative) and share y and z tables, so the
// contraction is evaluated as a tree: stage 1 forms 6 products T1_k (zz and
// mass share one), stage 2 accumulates them into 3 x-classes, stage 3
// applies the 3 x tables.  Stage 1 runs into shared memory; in stages 2+3
// each thread owns one (b,b',c,c') column, keeps its stage-2 values and the
// (a,a') rows of A in registers, and reads the x tables as broadcasts.
//
// Scatter.  Entry (a, b) of the element's assembly list goes to
// Ax[Ap[dof_b] + off[b][a]] (CSC: column = trial DOF).  Elements of one
// colour share no DOF, so the read-modify-write needs no atomics and the
// summation order of every entry (colour order) is fixed: bitwise
// reproducible.  The add is a posted reduction (red.global.add.f64): no
// two elements of a launch target the same entry, so it changes nothing in
// the arithmetic and lets the thread move on without waiting for the line.  Dirichlet lifting follows src/discretization.cc:316-317, the
// RHS :329-338 (lifting only enters the RHS when a linear form is set, as
// in the reference).
#pragma once

#include "common.cuh"

namespace h3dg {

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int EB>
struct SfShape {
	static constexpr int NX = PX + 1, NY = PY + 1, NZ = PZ + 1;
	static constexpr int NL = NX * NY * NZ;
	static constexpr int NQ = NQX * NQY * NQZ;
	static constexpr int NQ1X = NQX, NQ1Y = NQY, NQ1Z = NQZ;
	static constexpr int NT_TERMS = 6;   // stage-1 products (zz and mass share one)
	// 1D tables blob: Vx Dx Vy Dy Vz Dz (k-major, q fastest) then q/w per direction
	static constexpr int OVX = 0, ODX = OVX + NX * NQX, OVY = ODX + NX * NQX, ODY = OVY + NY * NQY;
	static constexpr int OVZ = ODY + NY * NQY, ODZ = OVZ + NZ * NQZ;
	static constexpr int OQX = ODZ + NZ * NQZ, OWX = OQX + NQX, OQY = OWX + NQX, OWY = OQY + NQY;
	static constexpr int OQZ = OWY + NQY, OWZ = OQZ + NQZ;
	static constexpr int TAB = OWZ + NQZ;
	static constexpr int TABP = (TAB + 1) & ~1;
	// products W^f[k][k'][q] = E^(f>>1)[k][q] E^(f&1)[k'][q], E^0 = V, E^1 = D
	static constexpr int WX = 4 * NX * NX * NQX, WY = 4 * NY * NY * NQY, WZ = 4 * NZ * NZ * NQZ;
	static constexpr int T1N = NQX * NQY * NZ * NZ;           // per term
	static constexpr int T2N = NQX * NY * NY * NZ * NZ;       // per term
	static constexpr int COLS = NY * NY * NZ * NZ;            // stage-3 columns (b,b',c,c')
	// per-element area: [G (8 NQ) | T1 (7 terms)]; A (NL^2) overwrites it once
	// every thread has finished reading T1 (block barrier in between).
	static constexpr int E_G = 0;
	static constexpr int E_T1 = 8 * NQ;
	static constexpr int E_A = 0;
	static constexpr int T1_END = E_T1 + NT_TERMS * T1N;
	static constexpr int E_F = T1_END > NL * NL ? T1_END : NL * NL;   // NL
	static constexpr int E_X = E_F + NL;        // 24
	static constexpr int E_M = E_X + 24;        // 24 trilinear monomial coefficients
	static constexpr int E_C = E_M + 24;        // NL coefficients
	static constexpr int E_CS = E_C + NL;       // NL column starts (int64)
	static constexpr int E_CE = E_CS + NL;      // NL column ends (int64)
	static constexpr int E_I = E_CE + NL;       // ints: dof NL, s NL (NL doubles)
	static constexpr int E_SIZE = (E_I + NL + 1) & ~1;
	static constexpr int S_TAB = 0;
	static constexpr int S_W = S_TAB + TABP;
	static constexpr int S_E = S_W + WX + WY + WZ;
	static constexpr int SMEM_DOUBLES = S_E + EB * E_SIZE;
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

// flags of the 7 terms: per direction, f = 2*alpha + beta (alpha: test side
// differentiated, beta: trial side differentiated)
static __device__ __constant__ int kTermFlags[7][3] = {
	{ 3, 0, 0 }, { 0, 3, 0 }, { 0, 0, 3 },   // xx yy zz
	{ 2, 1, 0 }, { 2, 0, 1 }, { 0, 2, 1 },   // xy xz yz
	{ 0, 0, 0 }                               // mass
};

// stage-1 products k = xx, yy, zz(+mass), xy, xz, yz: (x, y, z) table flags
// and the x-class each feeds (0: Wx^0, 1: Wx^2, 2: Wx^3)
static __device__ __constant__ int kT1Flags[6][3] = {
	{ 3, 0, 0 }, { 0, 3, 0 }, { 0, 0, 3 }, { 2, 1, 0 }, { 2, 0, 1 }, { 0, 2, 1 }
};

// ---- phases of the element computation, shared by the colour-sweep kernel
// below and the segmented-scatter kernel (asm_fp64_seg.cuh).  Each works on
// the EB element areas of a batch (layout of SfShape) with NT threads; the
// caller puts a block barrier between consecutive phases.

// 1D product tables W^f[k][k'][q], once per CTA
template <class S, int NT>
__device__ __forceinline__ void sf_product_tables(const double *tab, double *Wx, double *Wy, double *Wz) {
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ;
	constexpr int NQX = S::NQ1X, NQY = S::NQ1Y, NQZ = S::NQ1Z;
	const int tid = threadIdx.x;
	for (int i = tid; i < S::WX; i += NT) {
		int q = i % NQX, kk = (i / NQX) % NX, k = (i / (NQX * NX)) % NX, f = i / (NQX * NX * NX);
		double e0 = (f >> 1) ? tab[S::ODX + k * NQX + q] : tab[S::OVX + k * NQX + q];
		double e1 = (f & 1) ? tab[S::ODX + kk * NQX + q] : tab[S::OVX + kk * NQX + q];
		Wx[i] = e0 * e1;
	}
	for (int i = tid; i < S::WY; i += NT) {
		int q = i % NQY, kk = (i / NQY) % NY, k = (i / (NQY * NY)) % NY, f = i / (NQY * NY * NY);
		double e0 = (f >> 1) ? tab[S::ODY + k * NQY + q] : tab[S::OVY + k * NQY + q];
		double e1 = (f & 1) ? tab[S::ODY + kk * NQY + q] : tab[S::OVY + kk * NQY + q];
		Wy[i] = e0 * e1;
	}
	for (int i = tid; i < S::WZ; i += NT) {
		int q = i % NQZ, kk = (i / NQZ) % NZ, k = (i / (NQZ * NZ)) % NZ, f = i / (NQZ * NZ * NZ);
		double e0 = (f >> 1) ? tab[S::ODZ + k * NQZ + q] : tab[S::OVZ + k * NQZ + q];
		double e1 = (f & 1) ? tab[S::ODZ + kk * NQZ + q] : tab[S::OVZ + kk * NQZ + q];
		Wz[i] = e0 * e1;
	}
}

// trilinear map as monomials: x_r = sum_m c_m[r] mono_m(xi, eta, zeta),
// mono = 1, xi, eta, zeta, xi eta, xi zeta, eta zeta, xi eta zeta;
// c_m = (1/8) sum_v X_v prod_{d in m} s_d(v), s_d(v) = +-1 the vertex's
// reference coordinate (src/refdomain.cc:96-105)
template <class S, int NT, int EB>
__device__ __forceinline__ void sf_monomials(double *E0) {
	for (int i = threadIdx.x; i < EB * 24; i += NT) {
		const int e = i / 24, mr = i % 24, mo = mr / 3, r = mr % 3;
		double *Eb = E0 + e * S::E_SIZE;
		const int usex = mo == 1 || mo == 4 || mo == 5 || mo == 7;
		const int usey = mo == 2 || mo == 4 || mo == 6 || mo == 7;
		const int usez = mo == 3 || mo == 5 || mo == 6 || mo == 7;
		double c = 0.0;
#pragma unroll
		for (int v = 0; v < 8; v++) {
			const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
			const int neg = (usex && !bx) ^ (usey && !by) ^ (usez && !bz);
			const double xv = Eb[S::E_X + 3 * v + r];
			c += neg ? -xv : xv;
		}
		Eb[S::E_M + mr] = 0.125 * c;
	}
}

// geometry at one quadrature point -> the 8 term weights (xx yy zz xy xz yz
// mass source).  Jacobian, signed determinant and inverse as in
// RefMap::calc_inv_ref_map (src/refmap.cc:177-231);
// G = w det J^-1 J^-T = (w / det) adj(J) adj(J)^T.  cm: the 24 monomial
// coefficients of the element's map, (x, y, z) the point, w its weight.
__device__ __forceinline__ void sf_point_terms(const double *cm, double x, double y, double z, double w, double cg, int lf,
                                               double lf_value, double t[8]) {
	const double xy = x * y, xz = x * z, yz = y * z, xyz = xy * z;
	double m[3][3], xp[3];
#pragma unroll
	for (int r = 0; r < 3; r++) {
		const double c0 = cm[r], c1 = cm[3 + r], c2 = cm[6 + r], c3 = cm[9 + r];
		const double c4 = cm[12 + r], c5 = cm[15 + r], c6 = cm[18 + r], c7 = cm[21 + r];
		m[r][0] = c1 + c4 * y + c5 * z + c7 * yz;
		m[r][1] = c2 + c4 * x + c6 * z + c7 * xz;
		m[r][2] = c3 + c5 * x + c6 * y + c7 * xy;
		xp[r] = c0 + c1 * x + c2 * y + c3 * z + c4 * xy + c5 * xz + c6 * yz + c7 * xyz;
	}
	// cofactors: adj(J)[c][k] = C[k][c]; J^-1 = adj(J) / det
	const double C00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
	const double C01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
	const double C02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
	const double C10 = m[0][2] * m[2][1] - m[0][1] * m[2][2];
	const double C11 = m[0][0] * m[2][2] - m[0][2] * m[2][0];
	const double C12 = m[0][1] * m[2][0] - m[0][0] * m[2][1];
	const double C20 = m[0][1] * m[1][2] - m[0][2] * m[1][1];
	const double C21 = m[0][2] * m[1][0] - m[0][0] * m[1][2];
	const double C22 = m[0][0] * m[1][1] - m[0][1] * m[1][0];
	const double det = m[0][0] * C00 + m[0][1] * C01 + m[0][2] * C02;
	const double wd = w * det;
	const double s = w * cg / det;
	// (J^-1)[c][k] = C[k][c] / det  =>  G[c][d] = sum_k C[k][c] C[k][d] / det^2
	t[0] = 0.5 * s * (C00 * C00 + C10 * C10 + C20 * C20);
	t[1] = 0.5 * s * (C01 * C01 + C11 * C11 + C21 * C21);
	t[2] = 0.5 * s * (C02 * C02 + C12 * C12 + C22 * C22);
	t[3] = s * (C00 * C01 + C10 * C11 + C20 * C21);
	t[4] = s * (C00 * C02 + C10 * C12 + C20 * C22);
	t[5] = s * (C01 * C02 + C11 * C12 + C21 * C22);
	t[6] = 0.5 * wd;
	t[7] = wd * source_value(lf, lf_value, xp);
}

// geometry at the quadrature points of the batch -> term weights G
template <class S, int NT, int EB>
__device__ __forceinline__ void sf_geometry(const double *tab, double *E0, const double *s_cg, int lf, double lf_value) {
	constexpr int NQY = S::NQ1Y, NQZ = S::NQ1Z, NQ = S::NQ;
	for (int i = threadIdx.x; i < EB * NQ; i += NT) {
		const int e = i / NQ, q = i % NQ;
		double *Eb = E0 + e * S::E_SIZE;
		const int q1 = q / (NQY * NQZ), q2 = (q / NQZ) % NQY, q3 = q % NQZ;
		const double w = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3];
		double t[8];
		sf_point_terms(Eb + S::E_M, tab[S::OQX + q1], tab[S::OQY + q2], tab[S::OQZ + q3], w, s_cg[e], lf, lf_value, t);
#pragma unroll
		for (int r = 0; r < 8; r++) Eb[S::E_G + r * NQ + q] = t[r];
	}
}

// element load vector F_i = sum_q (w det f)(q) phi_i(q) of one (a, b) line,
// by sum factorisation: contracts q3, then q2, then q1 for all c.  src: the
// source weights at the NQ points, out: F[(a, b, *)] (NZ values).
template <class S>
__device__ __forceinline__ void sf_load_line(const double *tab, const double *src, int a, int b, double *out) {
	constexpr int NZ = S::NZ;
	constexpr int NQX = S::NQ1X, NQY = S::NQ1Y, NQZ = S::NQ1Z;
	double fc[NZ];
#pragma unroll
	for (int c = 0; c < NZ; c++) fc[c] = 0.0;
	for (int q1 = 0; q1 < NQX; q1++) {
		double s1[NZ];
#pragma unroll
		for (int c = 0; c < NZ; c++) s1[c] = 0.0;
		for (int q2 = 0; q2 < NQY; q2++) {
			const double vy = tab[S::OVY + b * NQY + q2];
#pragma unroll
			for (int q3 = 0; q3 < NQZ; q3++) {
				const double w = src[(q1 * NQY + q2) * NQZ + q3] * vy;
#pragma unroll
				for (int c = 0; c < NZ; c++) s1[c] += w * tab[S::OVZ + c * NQZ + q3];
			}
		}
		const double vx = tab[S::OVX + a * NQX + q1];
#pragma unroll
		for (int c = 0; c < NZ; c++) fc[c] += vx * s1[c];
	}
#pragma unroll
	for (int c = 0; c < NZ; c++) out[c] = fc[c];
}

// element load vectors of the batch: thread (e, a, b)
template <class S, int NT, int EB>
__device__ __forceinline__ void sf_load_vector(const double *tab, double *E0) {
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NQ = S::NQ;
	for (int i = threadIdx.x; i < EB * NX * NY; i += NT) {
		const int e = i / (NX * NY), ab = i % (NX * NY);
		double *Eb = E0 + e * S::E_SIZE;
		sf_load_line<S>(tab, Eb + S::E_G + 7 * NQ, ab / NY, ab % NY, Eb + S::E_F + ab * NZ);
	}
}

// stage 1: item (e, k, q1, q2) produces T1_k[q1][q2][*][*]
//   k: 0 xx, 1 yy, 2 zz (+ mass), 3 xy, 4 xz, 5 yz
template <class S, int NT, int EB>
__device__ __forceinline__ void sf_stage1(double *E0, const double *Wz, int mass) {
	constexpr int NZ = S::NZ;
	constexpr int NQX = S::NQ1X, NQY = S::NQ1Y, NQZ = S::NQ1Z, NQ = S::NQ;
	for (int i = threadIdx.x; i < EB * 6 * NQX * NQY; i += NT) {
		const int e = i / (6 * NQX * NQY), r = i % (6 * NQX * NQY);
		const int kk = r / (NQX * NQY), q12 = r % (NQX * NQY);
		double *Eb = E0 + e * S::E_SIZE;
		const double *gp = Eb + S::E_G + kk * NQ + q12 * NQZ;
		const double *wz = Wz + kT1Flags[kk][2] * NZ * NZ * NQZ;
		double g[NQZ];
#pragma unroll
		for (int q3 = 0; q3 < NQZ; q3++) g[q3] = gp[q3];
		double *out = Eb + S::E_T1 + kk * S::T1N + q12 * NZ * NZ;
		if (kk == 2 && mass) {
			const double *gm = Eb + S::E_G + 6 * NQ + q12 * NQZ;
			const double *wz0 = Wz;
			double h[NQZ];
#pragma unroll
			for (int q3 = 0; q3 < NQZ; q3++) h[q3] = gm[q3];
#pragma unroll
			for (int cc = 0; cc < NZ * NZ; cc++) {
				double s = 0.0;
#pragma unroll
				for (int q3 = 0; q3 < NQZ; q3++) s += g[q3] * wz[cc * NQZ + q3] + h[q3] * wz0[cc * NQZ + q3];
				out[cc] = s;
			}
		}
		else {
#pragma unroll
			for (int cc = 0; cc < NZ * NZ; cc++) {
				double s = 0.0;
#pragma unroll
				for (int q3 = 0; q3 < NQZ; q3++) s += g[q3] * wz[cc * NQZ + q3];
				out[cc] = s;
			}
		}
	}
}

// stages 2+3: thread owns column (e, b, b', c, c'); it accumulates the
// stage-2 values of the 3 x-classes in registers,
//   V_f[q1] = sum_k(class f) sum_q2 Wy_k[b][b'][q2] T1_k[q1][q2][c][c'],
// then A[(a,b,c)][(a',b',c')] = sum_f sum_q1 Wx_f[a][a'][q1] V_f[q1], which
// overwrites the element's G / T1 area (block barrier in between).
template <class S, int NT, int EB>
__device__ __forceinline__ void sf_stage23(double *E0, const double *Wx, const double *Wy) {
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL;
	constexpr int NQX = S::NQ1X, NQY = S::NQ1Y;
	constexpr int COLS = S::COLS;
	static_assert(EB * COLS <= NT, "one stage-3 column per thread");
	const int tid = threadIdx.x;
	const int e = tid / COLS, col = tid % COLS;
	const bool active = tid < EB * COLS;
	double acc[NX * NX];
	const int bb = col / (NZ * NZ), cc = col % (NZ * NZ);
	if (active) {
		const double *Eb = E0 + e * S::E_SIZE;
		double V[3][NQX];
#pragma unroll
		for (int f = 0; f < 3; f++)
#pragma unroll
			for (int q1 = 0; q1 < NQX; q1++) V[f][q1] = 0.0;
#pragma unroll
		for (int kk = 0; kk < 6; kk++) {
			// compile-time after unrolling, so V stays in registers
			constexpr int kFy[6] = { 0, 3, 0, 1, 0, 2 };
			constexpr int kCls[6] = { 2, 0, 0, 1, 1, 0 };
			const double *wy = Wy + kFy[kk] * NY * NY * NQY + bb * NQY;
			const double *t1 = Eb + S::E_T1 + kk * S::T1N + cc;
			const int f = kCls[kk];
			double wyr[NQY];
#pragma unroll
			for (int q2 = 0; q2 < NQY; q2++) wyr[q2] = wy[q2];
#pragma unroll
			for (int q1 = 0; q1 < NQX; q1++) {
				double s2 = V[f][q1];
#pragma unroll
				for (int q2 = 0; q2 < NQY; q2++) s2 += wyr[q2] * t1[(q1 * NQY + q2) * NZ * NZ];
				V[f][q1] = s2;
			}
		}
		const double *wx0 = Wx, *wx2 = Wx + 2 * NX * NX * NQX, *wx3 = Wx + 3 * NX * NX * NQX;
#pragma unroll
		for (int r = 0; r < NX * NX; r++) {
			double s3 = 0.0;
#pragma unroll
			for (int q1 = 0; q1 < NQX; q1++)
				s3 += wx0[r * NQX + q1] * V[0][q1] + wx2[r * NQX + q1] * V[1][q1] + wx3[r * NQX + q1] * V[2][q1];
			acc[r] = s3;
		}
	}
	__syncthreads();   // T1 fully consumed: A may overwrite it
	if (active) {
		const int b = bb / NY, b2 = bb % NY, c = cc / NZ, c2 = cc % NZ;
		double *A = E0 + e * S::E_SIZE + S::E_A;
#pragma unroll
		for (int a = 0; a < NX; a++)
#pragma unroll
			for (int a2 = 0; a2 < NX; a2++)
				A[((a * NY + b) * NZ + c) * NL + (a2 * NY + b2) * NZ + c2] = acc[a * NX + a2];
	}
}

// PF: software prefetch.  The plan data of the CTA's next batch (position
// map, DOFs, coefficients, shape indices, column bounds, vertex coordinates)
// are loaded into registers while the current batch is being computed, so
// their global-memory latency overlaps the arithmetic; the arithmetic itself
// is unchanged (bitwise identical results).
template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int NT, int EB, int MINB, bool PF = false>
__global__ void __launch_bounds__(NT, MINB) k_assemble_fp64(KArgs args, int64_t kbeg, int64_t kend) {
	using S = SfShape<PX, PY, PZ, NQX, NQY, NQZ, EB>;
	constexpr int NL = S::NL;
	constexpr int NL2 = NL * NL;
	constexpr int CH = 4;   // scatter chunk per thread
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int s_m[EB], s_l[EB];
	__shared__ double s_cg[EB];
	double *tab = sm + S::S_TAB;
	double *Wx = sm + S::S_W, *Wy = Wx + S::WX, *Wz = Wy + S::WY;
	double *E0 = sm + S::S_E;
	const int tid = threadIdx.x;

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar, args.status, args.wait_limit)) return;

	sf_product_tables<S, NT>(tab, Wx, Wy, Wz);
	__syncthreads();

	const bool do_rhs = args.rhs && args.lf;
	const int64_t nbatch = (kend - kbeg + EB - 1) / EB;

	// prefetch registers (PF): per thread its share of the batch's items
	constexpr int UOFF = PF ? (EB * NL2 + NT - 1) / NT : 1;   // position-map entries
	constexpr int VEL = PF ? (EB * NL + NT - 1) / NT : 1;     // functions
	constexpr int VX = PF ? (EB * 24 + NT - 1) / NT : 1;      // vertex coordinates
	uint16_t off_n[UOFF], off_c[UOFF];
	int dof_n[VEL], vtx_n[VX], m_n = 0, l_n = 0, id_n = 0;
	double coef_n[VEL], x_n[VX], cg_n = 1.0;
	uint16_t s_n[VEL];
	int64_t cs_n[VEL], ce_n[VEL];
	// first-level loads of batch bt (no dependent addresses)
	auto prefetch1 = [&](int64_t bt) {
		const int64_t k0 = kbeg + bt * EB;
		const int ne = (int) (kend - k0 < EB ? kend - k0 : EB);
#pragma unroll
		for (int u = 0; u < UOFF; u++) {
			const int p = tid + u * NT;
			off_n[u] = p < ne * NL2 ? args.el_off[k0 * NL2 + p] : (uint16_t) 0;
		}
#pragma unroll
		for (int v = 0; v < VEL; v++) {
			const int i = tid + v * NT, e = i / NL, j = i % NL;
			const bool live = i < EB * NL && e < ne;
			const int64_t g = (k0 + e) * NL + j;
			dof_n[v] = live ? args.el_dof[g] : -1;
			coef_n[v] = live ? args.el_coef[g] : 0.0;
			s_n[v] = live ? args.el_s[g] : (uint16_t) 0;
		}
#pragma unroll
		for (int v = 0; v < VX; v++) {
			const int i = tid + v * NT, e = i / 24, r = i % 24;
			vtx_n[v] = i < EB * 24 && e < ne ? args.el_vtx[8 * (k0 + e) + r / 3] : -1;
		}
		if (tid < EB) {
			const bool live = tid < ne;
			m_n = live ? args.el_cnt[2 * (k0 + tid)] : 0;
			l_n = live ? args.el_cnt[2 * (k0 + tid) + 1] : 0;
			id_n = live ? args.el_id[k0 + tid] : -1;
		}
	};
	// second-level loads (addresses from the first level)
	auto prefetch2 = [&]() {
#pragma unroll
		for (int v = 0; v < VEL; v++) {
			cs_n[v] = dof_n[v] >= 0 ? args.Ap[dof_n[v]] : 0;
			ce_n[v] = dof_n[v] >= 0 ? args.Ap[dof_n[v] + 1] : 0;
		}
#pragma unroll
		for (int v = 0; v < VX; v++) {
			const int r = (tid + v * NT) % 24;
			x_n[v] = vtx_n[v] >= 0 ? args.xyz[3 * (int64_t) vtx_n[v] + r % 3] : 0.0;
		}
		if (tid < EB) cg_n = id_n >= 0 && args.ecoef ? args.ecoef[id_n] : 1.0;
	};
	if (PF && (int64_t) blockIdx.x < nbatch) {
		prefetch1(blockIdx.x);
		prefetch2();
	}

	for (int64_t bt = blockIdx.x; bt < nbatch; bt += gridDim.x) {
		const int64_t k0 = kbeg + bt * EB;
		const int ne = (int) (kend - k0 < EB ? kend - k0 : EB);

		// ---- element data
		if (PF) {
			// this batch's data are in the prefetch registers; start the next batch's loads
			if (tid < EB) {
				s_m[tid] = m_n;
				s_l[tid] = l_n;
				s_cg[tid] = cg_n;
			}
#pragma unroll
			for (int v = 0; v < VX; v++) {
				const int i = tid + v * NT;
				if (i < EB * 24) E0[(i / 24) * S::E_SIZE + S::E_X + i % 24] = x_n[v];
			}
#pragma unroll
			for (int v = 0; v < VEL; v++) {
				const int i = tid + v * NT;
				if (i < EB * NL) {
					const int e = i / NL, j = i % NL;
					double *Eb = E0 + e * S::E_SIZE;
					int *ei = reinterpret_cast<int *>(Eb + S::E_I);
					int64_t *cs = reinterpret_cast<int64_t *>(Eb + S::E_CS);
					Eb[S::E_C + j] = coef_n[v];
					ei[j] = dof_n[v];
					ei[NL + j] = s_n[v];
					cs[j] = cs_n[v];
					cs[NL + j] = ce_n[v];
				}
			}
#pragma unroll
			for (int u = 0; u < UOFF; u++) off_c[u] = off_n[u];
			if (bt + gridDim.x < nbatch) prefetch1(bt + gridDim.x);
		}
		else {
			if (tid < EB) {
				const bool live = tid < ne;
				s_m[tid] = live ? args.el_cnt[2 * (k0 + tid)] : 0;
				s_l[tid] = live ? args.el_cnt[2 * (k0 + tid) + 1] : 0;
				s_cg[tid] = live && args.ecoef ? args.ecoef[args.el_id[k0 + tid]] : 1.0;
			}
			for (int i = tid; i < EB * 24; i += NT) {
				const int e = i / 24, r = i % 24;
				E0[e * S::E_SIZE + S::E_X + r] = e < ne ? args.xyz[3 * (int64_t) args.el_vtx[8 * (k0 + e) + r / 3] + r % 3] : 0.0;
			}
			for (int i = tid; i < EB * NL; i += NT) {
				const int e = i / NL, j = i % NL;
				double *Eb = E0 + e * S::E_SIZE;
				int *ei = reinterpret_cast<int *>(Eb + S::E_I);
				const int64_t g = (k0 + e) * NL + j;
				const int dof = e < ne ? args.el_dof[g] : -1;
				Eb[S::E_C + j] = e < ne ? args.el_coef[g] : 0.0;
				ei[j] = dof;
				ei[NL + j] = e < ne ? args.el_s[g] : 0;
				int64_t *cs = reinterpret_cast<int64_t *>(Eb + S::E_CS);
				cs[j] = dof >= 0 ? args.Ap[dof] : 0;
				cs[NL + j] = dof >= 0 ? args.Ap[dof + 1] : 0;
			}
		}
		__syncthreads();

		sf_monomials<S, NT, EB>(E0);
		__syncthreads();
		sf_geometry<S, NT, EB>(tab, E0, s_cg, args.lf, args.lf_value);
		__syncthreads();
		if (do_rhs) sf_load_vector<S, NT, EB>(tab, E0);
		sf_stage1<S, NT, EB>(E0, Wz, args.mass);
		__syncthreads();
		if (PF && bt + gridDim.x < nbatch) prefetch2();   // the first-level loads have had stage 1 to land
		sf_stage23<S, NT, EB>(E0, Wx, Wy);
		__syncthreads();

		// ---- scatter into the CSC matrix (exclusive within a colour)
		if (args.Ax) {
			double *__restrict__ Ax = args.Ax;
#pragma unroll
			for (int base = 0; base < EB * NL2; base += NT * CH) {
				int64_t pos[CH];
				double val[CH];
#pragma unroll
				for (int r = 0; r < CH; r++) {
					const int p = base + tid + r * NT;
					pos[r] = -1;
					val[r] = 0.0;
					if (p < EB * NL2) {
						const int e = p / NL2, pp = p % NL2;
						const int m = s_m[e];
						const int b = pp / NL, a = pp % NL;
						if (a < m && b < m) {
							const double *Eb = E0 + e * S::E_SIZE;
							const int *ei = reinterpret_cast<const int *>(Eb + S::E_I);
							const int64_t *cs = reinterpret_cast<const int64_t *>(Eb + S::E_CS);
							const int sa = ei[NL + a], sb = ei[NL + b];
							const double *A = Eb + S::E_A;
							val[r] = Eb[S::E_C + a] * Eb[S::E_C + b] * (A[sa * NL + sb] + A[sb * NL + sa]);
							const int uu = (base / (NT * CH)) * CH + r;     // = (p - tid) / NT, compile-time when unrolled
							const int64_t t = cs[b] + (PF ? (int64_t) off_c[uu < UOFF ? uu : UOFF - 1]
							                              : (int64_t) args.el_off[(k0 + e) * NL2 + b * NL + a]);
							if (t < cs[NL + b]) pos[r] = t;
							else if (cs[NL + b] > cs[b]) atomicOr(args.status, kErrBounds);   // empty: column not owned
						}
					}
				}
#pragma unroll
				for (int r = 0; r < CH; r++)
					if (pos[r] >= 0) posted_add(Ax + pos[r], val[r]);
			}
		}
		if (do_rhs) {
			for (int i = tid; i < EB * NL; i += NT) {
				const int e = i / NL, a = i % NL;
				if (a >= s_m[e]) continue;
				const double *Eb = E0 + e * S::E_SIZE;
				const int *ei = reinterpret_cast<const int *>(Eb + S::E_I);
				const double *A = Eb + S::E_A;
				const int sa = ei[NL + a];
				const double ca = Eb[S::E_C + a];
				double lr = 0.0;
				for (int j = s_m[e]; j < s_m[e] + (args.Ax ? s_l[e] : 0); j++) {      // lifting only with the matrix (src/discretization.cc:296-317)
					const int sj = ei[NL + j];
					lr -= ca * Eb[S::E_C + j] * (A[sa * NL + sj] + A[sj * NL + sa]);
				}
				lr += Eb[S::E_F + sa] * ca;
				posted_add(args.rhs + ei[a], lr);
			}
		}
		__syncthreads();
	}
}

} // namespace h3dg
