// FP64 assembly for high orders (the element matrix does not fit in shared
// memory): per element, never materialised.
//
// Same mathematics as k_assemble_fp64 (src/integrals/h1.h:115-177 per pair,
// restated as sum factorisation), organised for (p+1)^3 up to ~1000:
//   * the gradient part uses all 9 (r,s) terms with the full G (no A + A^T
//     split), so every entry K_ij is produced whole by one thread;
//   * the test-side z index c is processed in chunks: stage 1 forms the 9
//     products T1_k[q1][q2][c'] = sum_q3 G_g(k)(q) E_z[c][q3] E_z[c'][q3] for
//     the chunk's c into shared memory;
//   * stages 2+3: a thread owns a column (b, b', c'), accumulates
//     V_f[q1] = sum_{k in class f} sum_q2 E_y[b][q2] E_y[b'][q2] T1_k[q1][q2][c']
//     for the 4 x-classes in registers and then produces
//     K[(a,b,c)][(a',b',c')] = sum_q1 E0_a (E0_a' V_0 + E1_a' V_1) + E1_a (E0_a' V_2 + E1_a' V_3)
//     for all (a, a'), each added straight into the CSC matrix.  The row
//     position map is indexed canonically ([i][j], i test, j trial), so a
//     warp reads it contiguously.
//   * Dirichlet lifting and the load vector use the matrix-free element
//     operator y = K g (interpolate g to the points, apply G, integrate
//     back), so no K row is ever needed: lrhs_i = c_i (F_i - (K g)_i)
//     (src/discretization.cc:316-338).
// Determinism: within one launch (one colour) each Ax entry receives exactly
// one posted add, each rhs entry exactly one; launches are stream-ordered.
#pragma once

#include "common.cuh"

namespace h3dg {

struct KArgsHO {
	const double *xyz;
	const int32_t *el_vtx;     // assembly order, ne x 8
	const int32_t *el_id;
	const double *ecoef;       // per element id, or nullptr
	const int32_t *cdof;       // ne x nl: DOF of canonical function i, -1 if not a matrix entry
	const double *ccoef;       // ne x nl: sign x AsmList coefficient (lifting value when cdof = -1), 0 if absent
	const uint16_t *offc;      // ne x nl x nl: [i][j] row position of cdof_i in column cdof_j
	const uint16_t *offt;      // tensor-core scatter stream (k_build_offt), or nullptr
	const int64_t *Ap;
	const double *tables;
	int table_bytes;
	int mass, lf;
	double lf_value;
	double *Ax, *rhs;
	int *status;
	double *gscratch;          // per-CTA global work area (kernels that keep G out of shared memory), or nullptr
	const int32_t *tcdof;      // test side of a two-space block (ne x nl), or nullptr: the trial tables
	const double *tccoef;
	const uint16_t *offd;      // FP64 tensor-core scatter stream (k_build_offd), or nullptr
	int64_t split_from;        // FP64 tensor-core kernel: elements from here on are done in two halves
};

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ>
struct HoShape {
	static constexpr int NX = PX + 1, NY = PY + 1, NZ = PZ + 1;
	static constexpr int NL = NX * NY * NZ;
	static constexpr int NQ = NQX * NQY * NQZ;
	static constexpr int QX = NQX, QY = NQY, QZ = NQZ;
	static constexpr int OVX = 0, ODX = OVX + NX * NQX, OVY = ODX + NX * NQX, ODY = OVY + NY * NQY;
	static constexpr int OVZ = ODY + NY * NQY, ODZ = OVZ + NZ * NQZ;
	static constexpr int OQX = ODZ + NZ * NQZ, OWX = OQX + NQX, OQY = OWX + NQX, OWY = OQY + NQY;
	static constexpr int OQZ = OWY + NQY, OWZ = OQZ + NQZ;
	static constexpr int TAB = OWZ + NQZ;
	static constexpr int TABP = (TAB + 1) & ~1;
	static constexpr int NPROD = 9;
	static constexpr int T1C = NPROD * NQX * NQY * NZ;                 // one c chunk
	// matrix-free work area: U (4 NQ), P (3 NX NQY NQZ), Q (2 NX NY NQZ)
	static constexpr int MF = 4 * NQ + 3 * NX * NQY * NQZ + 2 * NX * NY * NQZ;
	static constexpr int UNION = T1C > MF ? T1C : MF;
	static constexpr int S_TAB = 0;
	static constexpr int S_G = S_TAB + TABP;                            // 8 NQ: xx yy zz xy xz yz mass src
	static constexpr int S_U = S_G + 8 * NQ;                            // UNION
	static constexpr int S_X = S_U + UNION;                             // 24
	static constexpr int S_M = S_X + 24;                                // 24 monomials
	static constexpr int S_C = S_M + 24;                                // NL ccoef
	static constexpr int S_Y = S_C + NL;                                // NL (K g, then F)
	static constexpr int S_CS = S_Y + NL;                               // NL int64 column start
	static constexpr int S_CE = S_CS + NL;                              // NL int64 column end
	static constexpr int S_D = S_CE + NL;                               // NL int dof (NL/2 doubles)
	static constexpr int S_TD = S_D + (NL + 1) / 2;                     // test side of a two-space block: NL int dof
	static constexpr int S_TC = S_TD + (NL + 1) / 2;                    //   and NL coefficients
	static constexpr int SMEM_DOUBLES = S_TC + NL + 2;
	static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

// ---- pieces shared by the high-order kernels (FP64 and tensor-core)

// Element set-up: vertex coordinates, per-function DOF / coefficient and
// column bounds, the count of lifting functions, trilinear monomial
// coefficients of the map.  Returns the grad-grad coefficient.
template <class S, int NT>
__device__ __forceinline__ double ho_element_setup(const KArgsHO &args, int64_t k, double *X, double *Mo, double *cc, int *cd,
                                                   int64_t *cs, int64_t *ce, int *s_nlift) {
	constexpr int NL = S::NL;
	const int tid = threadIdx.x;
	if (tid == 0) *s_nlift = 0;
	if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.el_vtx[8 * k + tid / 3] + tid % 3];
	__syncthreads();
	int nl_local = 0;
	for (int i = tid; i < NL; i += NT) {
		const int d = args.cdof[k * NL + i];
		const double c = args.ccoef[k * NL + i];
		cd[i] = d;
		cc[i] = c;
		cs[i] = d >= 0 ? args.Ap[d] : 0;
		ce[i] = d >= 0 ? args.Ap[d + 1] : 0;
		if (d < 0 && c != 0.0) nl_local++;
	}
	if (nl_local) atomicAdd(s_nlift, nl_local);
	for (int i = tid; i < 24; i += NT) {
		const int mo = i / 3, r = i % 3;
		const int usex = mo == 1 || mo == 4 || mo == 5 || mo == 7;
		const int usey = mo == 2 || mo == 4 || mo == 6 || mo == 7;
		const int usez = mo == 3 || mo == 5 || mo == 6 || mo == 7;
		double c = 0.0;
#pragma unroll
		for (int v = 0; v < 8; v++) {
			const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
			const int neg = (usex && !bx) ^ (usey && !by) ^ (usez && !bz);
			c += neg ? -X[3 * v + r] : X[3 * v + r];
		}
		Mo[i] = 0.125 * c;
	}
	const double cgrad = args.ecoef ? args.ecoef[args.el_id[k]] : 1.0;
	__syncthreads();
	return cgrad;
}

// Geometric factors at every quadrature point (FP64): the 6 entries of
// w J^-1 J^-T |J| (times the grad-grad coefficient), the mass weight w |J|
// and the source weight w |J| f(x).  G is [8][NQ].
template <class S, int NT>
__device__ __forceinline__ void ho_geometry(const KArgsHO &args, const double *tab, const double *Mo, double cgrad, double *G) {
	constexpr int NQ = S::NQ, NQY = S::QY, NQZ = S::QZ;
	const int tid = threadIdx.x;
	// ---- geometry: full G (no halving), mass weight, source weight
	for (int q = tid; q < NQ; q += NT) {
		const int q1 = q / (NQY * NQZ), q2 = (q / NQZ) % NQY, q3 = q % NQZ;
		const double x = tab[S::OQX + q1], y = tab[S::OQY + q2], z = tab[S::OQZ + q3];
		const double xy = x * y, xz = x * z, yz = y * z, xyz = xy * z;
		double m[3][3], xp[3];
#pragma unroll
		for (int r = 0; r < 3; r++) {
			const double c0 = Mo[r], c1 = Mo[3 + r], c2 = Mo[6 + r], c3 = Mo[9 + r];
			const double c4 = Mo[12 + r], c5 = Mo[15 + r], c6 = Mo[18 + r], c7 = Mo[21 + r];
			m[r][0] = c1 + c4 * y + c5 * z + c7 * yz;
			m[r][1] = c2 + c4 * x + c6 * z + c7 * xz;
			m[r][2] = c3 + c5 * x + c6 * y + c7 * xy;
			xp[r] = c0 + c1 * x + c2 * y + c3 * z + c4 * xy + c5 * xz + c6 * yz + c7 * xyz;
		}
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
		const double w = tab[S::OWX + q1] * tab[S::OWY + q2] * tab[S::OWZ + q3];
		const double wd = w * det, s = w * cgrad / det;
		G[0 * NQ + q] = s * (C00 * C00 + C10 * C10 + C20 * C20);
		G[1 * NQ + q] = s * (C01 * C01 + C11 * C11 + C21 * C21);
		G[2 * NQ + q] = s * (C02 * C02 + C12 * C12 + C22 * C22);
		G[3 * NQ + q] = s * (C00 * C01 + C10 * C11 + C20 * C21);
		G[4 * NQ + q] = s * (C00 * C02 + C10 * C12 + C20 * C22);
		G[5 * NQ + q] = s * (C01 * C02 + C11 * C12 + C21 * C22);
		G[6 * NQ + q] = args.mass ? wd : 0.0;
		G[7 * NQ + q] = wd * source_value(args.lf, args.lf_value, xp);
	}
	__syncthreads();
}

// Load vector with Dirichlet lifting, matrix-free (FP64):
// lrhs_i = c_i (F_i - (K g)_i), posted into rhs.  U is a work area of
// HoShape::MF doubles.  g: the trial side's lifting (cd < 0, value cc);
// rows i: the test side (td, tc; the same tables unless the block has two
// spaces).
template <class S, int NT>
__device__ __forceinline__ void ho_rhs(const KArgsHO &args, const double *tab, const double *G, double *U, const int *cd,
                                       const double *cc, const int *td, const double *tc, bool lift) {
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL, NQ = S::NQ;
	constexpr int NQX = S::QX, NQY = S::QY, NQZ = S::QZ;
	const int tid = threadIdx.x;
	const double *Vx = tab + S::OVX, *Dx = tab + S::ODX, *Vy = tab + S::OVY, *Dy = tab + S::ODY;
	const double *Vz = tab + S::OVZ, *Dz = tab + S::ODZ;
	double *Pw = U + 4 * NQ;                       // P: [3][NX][NQY][NQZ]
	double *Qw = Pw + 3 * NX * NQY * NQZ;          // Q: [2][NX][NY][NQZ]
	if (lift) {
		// interpolate g (value, d/dxi, d/deta, d/dzeta) to the points
		for (int i = tid; i < NX * NY * NQZ; i += NT) {   // Q0 = sum_c g V_z, Q1 = sum_c g D_z
			const int ab = i / NQZ, q3 = i % NQZ;
			double s0 = 0.0, s1 = 0.0;
			for (int c = 0; c < NZ; c++) {
				const int j = ab * NZ + c;
				const double g = cd[j] < 0 ? cc[j] : 0.0;
				s0 += g * Vz[c * NQZ + q3];
				s1 += g * Dz[c * NQZ + q3];
			}
			Qw[i] = s0;
			Qw[NX * NY * NQZ + i] = s1;
		}
		__syncthreads();
		for (int i = tid; i < NX * NQY * NQZ; i += NT) {   // P00, P10 (d/deta), P01 (d/dzeta)
			const int a = i / (NQY * NQZ), q2 = (i / NQZ) % NQY, q3 = i % NQZ;
			double s00 = 0.0, s10 = 0.0, s01 = 0.0;
			for (int b = 0; b < NY; b++) {
				const double q0v = Qw[(a * NY + b) * NQZ + q3], q1v = Qw[NX * NY * NQZ + (a * NY + b) * NQZ + q3];
				s00 += q0v * Vy[b * NQY + q2];
				s10 += q0v * Dy[b * NQY + q2];
				s01 += q1v * Vy[b * NQY + q2];
			}
			Pw[i] = s00;
			Pw[NX * NQY * NQZ + i] = s10;
			Pw[2 * NX * NQY * NQZ + i] = s01;
		}
		__syncthreads();
		for (int q = tid; q < NQ; q += NT) {
			const int q1 = q / (NQY * NQZ), q23 = q % (NQY * NQZ);
			double u0 = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
			for (int a = 0; a < NX; a++) {
				const double p00 = Pw[a * NQY * NQZ + q23], p10 = Pw[NX * NQY * NQZ + a * NQY * NQZ + q23];
				const double p01 = Pw[2 * NX * NQY * NQZ + a * NQY * NQZ + q23];
				u0 += p00 * Vx[a * NQX + q1];
				ux += p00 * Dx[a * NQX + q1];
				uy += p10 * Vx[a * NQX + q1];
				uz += p01 * Vx[a * NQX + q1];
			}
			// W = G grad g (+ mass g), minus the source weight (integrated with V)
			const double gxx = G[q], gyy = G[NQ + q], gzz = G[2 * NQ + q];
			const double gxy = G[3 * NQ + q], gxz = G[4 * NQ + q], gyz = G[5 * NQ + q];
			U[q] = G[6 * NQ + q] * u0 - G[7 * NQ + q];
			U[NQ + q] = gxx * ux + gxy * uy + gxz * uz;
			U[2 * NQ + q] = gxy * ux + gyy * uy + gyz * uz;
			U[3 * NQ + q] = gxz * ux + gyz * uy + gzz * uz;
		}
	}
	else {
		for (int q = tid; q < NQ; q += NT) {
			U[q] = -G[7 * NQ + q];
			U[NQ + q] = U[2 * NQ + q] = U[3 * NQ + q] = 0.0;
		}
	}
	__syncthreads();
	// integrate back: Y_i = sum_q W_0 phi_i + sum_r W_r d_r phi_i  (= (K g)_i - F_i)
	for (int i = tid; i < NX * NQY * NQZ; i += NT) {
		const int a = i / (NQY * NQZ), q23 = i % (NQY * NQZ);
		double s00 = 0.0, s10 = 0.0, s01 = 0.0;
		for (int q1 = 0; q1 < NQX; q1++) {
			const int q = q1 * NQY * NQZ + q23;
			s00 += U[q] * Vx[a * NQX + q1] + U[NQ + q] * Dx[a * NQX + q1];
			s10 += U[2 * NQ + q] * Vx[a * NQX + q1];
			s01 += U[3 * NQ + q] * Vx[a * NQX + q1];
		}
		Pw[i] = s00;
		Pw[NX * NQY * NQZ + i] = s10;
		Pw[2 * NX * NQY * NQZ + i] = s01;
	}
	__syncthreads();
	for (int i = tid; i < NX * NY * NQZ; i += NT) {
		const int a = i / (NY * NQZ), b = (i / NQZ) % NY, q3 = i % NQZ;
		double s0 = 0.0, s1 = 0.0;
		for (int q2 = 0; q2 < NQY; q2++) {
			const int o = (a * NQY + q2) * NQZ + q3;
			s0 += Pw[o] * Vy[b * NQY + q2] + Pw[NX * NQY * NQZ + o] * Dy[b * NQY + q2];
			s1 += Pw[2 * NX * NQY * NQZ + o] * Vy[b * NQY + q2];
		}
		Qw[i] = s0;
		Qw[NX * NY * NQZ + i] = s1;
	}
	__syncthreads();
	for (int i = tid; i < NL; i += NT) {
		if (td[i] < 0) continue;                      // rows: the test functions
		const int ab = i / NZ, c = i % NZ;
		double s = 0.0;
		for (int q3 = 0; q3 < NQZ; q3++)
			s += Qw[ab * NQZ + q3] * Vz[c * NQZ + q3] + Qw[NX * NY * NQZ + ab * NQZ + q3] * Dz[c * NQZ + q3];
		posted_add(args.rhs + td[i], -tc[i] * s);
	}
	__syncthreads();

}

// stage-1 products: G index, z flag, y flag, x class (f = 2 alpha + beta)
//   xx, yy, zz(+mass), xy, yx, xz, zx, yz, zy
static __device__ __constant__ int kHoG[9] = { 0, 1, 2, 3, 3, 4, 4, 5, 5 };
static __device__ __constant__ int kHoFz[9] = { 0, 0, 3, 0, 0, 1, 2, 1, 2 };

template <int PX, int PY, int PZ, int NQX, int NQY, int NQZ, int NT>
__global__ void __launch_bounds__(NT, 1) k_assemble_fp64_ho(KArgsHO args, int64_t kbeg, int64_t kend) {
	using S = HoShape<PX, PY, PZ, NQX, NQY, NQZ>;
	constexpr int NX = S::NX, NY = S::NY, NZ = S::NZ, NL = S::NL, NQ = S::NQ;
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int s_nlift;
	const double *tab = sm + S::S_TAB;
	double *G = sm + S::S_G, *U = sm + S::S_U, *T1 = sm + S::S_U;
	double *X = sm + S::S_X, *Mo = sm + S::S_M, *cc = sm + S::S_C, *Y = sm + S::S_Y;
	int64_t *cs = reinterpret_cast<int64_t *>(sm + S::S_CS), *ce = reinterpret_cast<int64_t *>(sm + S::S_CE);
	int *cd = reinterpret_cast<int *>(sm + S::S_D);
	// test side: its own tables in a two-space block, else the trial tables
	int *td = args.tcdof ? reinterpret_cast<int *>(sm + S::S_TD) : cd;
	double *tc = args.tcdof ? sm + S::S_TC : cc;
	const int tid = threadIdx.x;
	if (!stage_tables(sm + S::S_TAB, args.tables, args.table_bytes, &bar, args.status)) return;
	const double *Vx = tab + S::OVX, *Dx = tab + S::ODX, *Vy = tab + S::OVY, *Dy = tab + S::ODY;
	const double *Vz = tab + S::OVZ, *Dz = tab + S::ODZ;
	const bool do_rhs = args.rhs && args.lf;

	for (int64_t k = kbeg + blockIdx.x; k < kend; k += gridDim.x) {
		if (args.tcdof)
			for (int i = tid; i < NL; i += NT) {
				td[i] = args.tcdof[k * NL + i];
				tc[i] = args.tccoef[k * NL + i];
			}
		const double cgrad = ho_element_setup<S, NT>(args, k, X, Mo, cc, cd, cs, ce, &s_nlift);
		ho_geometry<S, NT>(args, tab, Mo, cgrad, G);
		if (do_rhs) ho_rhs<S, NT>(args, tab, G, U, cd, cc, td, tc, s_nlift > 0 && args.Ax);

		// ---- matrix: chunks of the test z index c
		if (args.Ax) {
			for (int c = 0; c < NZ; c++) {
				// stage 1: T1_k[q1][q2][c'] = sum_q3 G_g(k) E_z^alpha[c][q3] E_z^beta[c'][q3] (+ mass into k = 2)
				for (int i = tid; i < S::NPROD * NQX * NQY; i += NT) {
					const int kk = i / (NQX * NQY), q12 = i % (NQX * NQY);
					const int fz = kHoFz[kk];
					const double *ea = (fz >> 1) ? Dz + c * NQZ : Vz + c * NQZ;
					const double *gp = G + kHoG[kk] * NQ + q12 * NQZ;
					const double *gm = G + 6 * NQ + q12 * NQZ;
					double h[NQZ];
#pragma unroll
					for (int q3 = 0; q3 < NQZ; q3++) h[q3] = gp[q3] * ea[q3];
					double hm[NQZ];
					const bool addm = kk == 2 && args.mass;
#pragma unroll
					for (int q3 = 0; q3 < NQZ; q3++) hm[q3] = addm ? gm[q3] * Vz[c * NQZ + q3] : 0.0;
					double *out = T1 + (kk * NQX * NQY + q12) * NZ;
					for (int c2 = 0; c2 < NZ; c2++) {
						const double *eb = (fz & 1) ? Dz + c2 * NQZ : Vz + c2 * NQZ;
						double s = 0.0;
#pragma unroll
						for (int q3 = 0; q3 < NQZ; q3++) s += h[q3] * eb[q3];
						if (addm) {
#pragma unroll
							for (int q3 = 0; q3 < NQZ; q3++) s += hm[q3] * Vz[c2 * NQZ + q3];
						}
						out[c2] = s;
					}
				}
				__syncthreads();
				// stages 2 + 3 per column (b, b', c'), b slowest
				for (int col = tid; col < NY * NY * NZ; col += NT) {
					const int b = col / (NY * NZ), b2 = (col / NZ) % NY, c2 = col % NZ;
					double V[4][NQX];
#pragma unroll
					for (int f = 0; f < 4; f++)
#pragma unroll
						for (int q1 = 0; q1 < NQX; q1++) V[f][q1] = 0.0;
#pragma unroll
					for (int kk = 0; kk < 9; kk++) {
						// y flag and x class of product kk (compile-time after unrolling)
						constexpr int kFy[9] = { 0, 3, 0, 1, 2, 0, 0, 2, 1 };
						constexpr int kCls[9] = { 3, 0, 0, 2, 1, 2, 1, 0, 0 };
						const int fy = kFy[kk], f = kCls[kk];
						const double *ea = (fy >> 1) ? Dy + b * NQY : Vy + b * NQY;
						const double *eb = (fy & 1) ? Dy + b2 * NQY : Vy + b2 * NQY;
						double wy[NQY];
#pragma unroll
						for (int q2 = 0; q2 < NQY; q2++) wy[q2] = ea[q2] * eb[q2];
						const double *t1 = T1 + kk * NQX * NQY * NZ + c2;
#pragma unroll
						for (int q1 = 0; q1 < NQX; q1++) {
							double s = V[f][q1];
#pragma unroll
							for (int q2 = 0; q2 < NQY; q2++) s += wy[q2] * t1[(q1 * NQY + q2) * NZ];
							V[f][q1] = s;
						}
					}
					const int jbase = b2 * NZ + c2;               // j = (a2*NY + b2)*NZ + c2
					const int ibase = b * NZ + c;                 // i = (a*NY + b)*NZ + c
					for (int a2 = 0; a2 < NX; a2++) {
						const int j = a2 * NY * NZ + jbase;
						const int dj = cd[j];
						if (dj < 0) continue;
						double Z0[NQX], Z1[NQX];
#pragma unroll
						for (int q1 = 0; q1 < NQX; q1++) {
							const double e0 = Vx[a2 * NQX + q1], e1 = Dx[a2 * NQX + q1];
							Z0[q1] = e0 * V[0][q1] + e1 * V[1][q1];
							Z1[q1] = e0 * V[2][q1] + e1 * V[3][q1];
						}
						const double cj = cc[j];
						const int64_t c0 = cs[j], c1 = ce[j];
						const uint16_t *offrow = args.offc + (k * NL) * NL + j;
						for (int a = 0; a < NX; a++) {
							const int i = a * NY * NZ + ibase;
							if (td[i] < 0) continue;
							double s = 0.0;
#pragma unroll
							for (int q1 = 0; q1 < NQX; q1++) s += Vx[a * NQX + q1] * Z0[q1] + Dx[a * NQX + q1] * Z1[q1];
							const int64_t pos = c0 + offrow[(int64_t) i * NL];
							if (pos < c1) posted_add(args.Ax + pos, tc[i] * cj * s);
							else if (c1 > c0) atomicOr(args.status, kErrBounds);   // empty: column not owned
						}
					}
				}
				__syncthreads();
			}
		}
	}
}

} // namespace h3dg
