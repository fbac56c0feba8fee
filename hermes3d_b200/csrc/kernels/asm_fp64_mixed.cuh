// FP64 assembly for meshes with mixed (anisotropic, per-element) orders.
//
// Same element matrix as the uniform kernels (src/integrals/h1.h:115-177 per
// pair, restated as sum factorisation; Dirichlet lifting and load vector as
// src/discretization.cc:316-338), with the order triple (px, py, pz) and the
// rule (nqx, nqy, nqz) read per element from its descriptor.  One kernel
// instance serves a class of elements (orders <= PM, points <= QM per
// direction): loop bounds are the element's own, block-uniform, and the
// register arrays are sized by the class maxima.  The host groups the
// elements of each colour by class and orders them by decreasing work; the
// CTAs of a launch are persistent and fetch elements through an atomic
// counter, so the expensive elements start first and the tail is short.
//
// The matrix is produced per TRIAL z index c' (stage 1 over zeta, stage 2
// over eta, stage 3 over xi).  A thread owns one row set (b', b, c) (trial
// y, test y, test z; c fastest) and, for each trial x index a', posts the
// entries of CSC column j = (a', b', c') for all test x indices a: the lanes
// of a warp share b' and so post into the same column at nearby rows, and
// read the column-major position map (rows of one column contiguous)
// contiguously.  Determinism: within one launch each Ax / rhs entry receives
// at most one posted add (elements of a colour share no DOF); launches of
// different classes of one colour touch disjoint entries, and colours are
// ordered.
#pragma once

#include "common.cuh"

namespace h3dg {

struct KArgsMixed {
	const double *xyz;
	const int32_t *el_vtx;     // assembly order, ne x 8
	const int32_t *el_id;
	const double *ecoef;       // per element id, or nullptr
	const int32_t *el_desc;    // ne x 12: px py pz nqx nqy nqz ox oy oz nl class -
	const int64_t *el_base;    // ne + 1: start of the element's canonical entries
	const int64_t *el_obase;   // ne + 1: start of the element's position map
	const int32_t *cdof;       // DOF of canonical function i, -1 if not a matrix entry
	const double *ccoef;       // sign x AsmList coefficient (lifting value when cdof = -1), 0 if absent
	const uint16_t *offm;      // [j][i]: row position of cdof_i in column cdof_j
	const int64_t *Ap;
	const double *tables;      // table sets: V[(p+1) nq], D[(p+1) nq], q[nq], w[nq]
	int table_bytes;
	int mass, lf;
	double lf_value;
	double *Ax, *rhs;
	int *status;
	unsigned int *counters;    // one work counter per launch, zero at the start
};

template <int PM, int QM>
struct MixShape {
	static constexpr int NM = PM + 1;
	static constexpr int NLM = NM * NM * NM;
	static constexpr int Q3 = QM * QM * QM;
	static constexpr int T1 = 9 * QM * QM * NM;
	static constexpr int MF = 4 * Q3 + 3 * NM * QM * QM + 2 * NM * NM * QM;
	static constexpr int UNION = T1 > MF ? T1 : MF;
	// doubles after the staged tables
	static constexpr int R_G = 0;                  // 8 x nq: xx yy zz xy xz yz mass src
	static constexpr int R_U = R_G + 8 * Q3;
	static constexpr int R_X = R_U + UNION;
	static constexpr int R_M = R_X + 24;
	static constexpr int R_C = R_M + 24;
	static constexpr int R_CS = R_C + NLM;
	static constexpr int R_CE = R_CS + NLM;
	static constexpr int R_D = R_CE + NLM;
	static constexpr int END = R_D + (NLM + 1) / 2 + 2;
	static size_t smem_bytes(int table_bytes) { return (size_t) ((table_bytes + 15) / 16) * 16 + sizeof(double) * END; }
};

// stage-1 products: G index and z flags, in the order xx, yy, zz(+mass), xy, yx, xz, zx, yz, zy
static __device__ __constant__ int kMxG[9] = { 0, 1, 2, 3, 3, 4, 4, 5, 5 };
static __device__ __constant__ int kMxFz[9] = { 0, 0, 3, 0, 0, 1, 2, 1, 2 };

template <int PM, int QM, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_assemble_fp64_mixed(KArgsMixed args, int64_t kbeg, int64_t kend, int launch) {
	using S = MixShape<PM, QM>;
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int s_nlift;
	__shared__ int64_t s_k;
	const int tid = threadIdx.x;
	if (!stage_tables(sm, args.tables, args.table_bytes, &bar, args.status)) return;
	const double *tab = sm;
	double *R = sm + ((args.table_bytes + 15) / 16) * 2;
	double *G = R + S::R_G, *U = R + S::R_U, *T1 = R + S::R_U;
	double *X = R + S::R_X, *Mo = R + S::R_M, *cc = R + S::R_C;
	int64_t *cs = reinterpret_cast<int64_t *>(R + S::R_CS), *ce = reinterpret_cast<int64_t *>(R + S::R_CE);
	int *cd = reinterpret_cast<int *>(R + S::R_D);
	const bool do_rhs = args.rhs && args.lf;

	for (;;) {
		if (tid == 0) s_k = kbeg + (int64_t) atomicAdd(&args.counters[launch], 1u);
		__syncthreads();
		const int64_t k = s_k;
		if (k >= kend) break;                                   // block-uniform
		const int32_t *dsc = args.el_desc + k * 12;
		const int px = dsc[0], py = dsc[1], pz = dsc[2];
		const int nqx = dsc[3], nqy = dsc[4], nqz = dsc[5];
		const int NX = px + 1, NY = py + 1, NZ = pz + 1, NL = NX * NY * NZ;
		const int NQ = nqx * nqy * nqz;
		const double *Vx = tab + dsc[6], *Dx = Vx + NX * nqx, *Qx = Dx + NX * nqx, *Wx = Qx + nqx;
		const double *Vy = tab + dsc[7], *Dy = Vy + NY * nqy, *Qy = Dy + NY * nqy, *Wy = Qy + nqy;
		const double *Vz = tab + dsc[8], *Dz = Vz + NZ * nqz, *Qz = Dz + NZ * nqz, *Wz = Qz + nqz;
		const int64_t base = args.el_base[k];

		// ---- set-up: vertices, per-function DOF / coefficient / column bounds, monomials
		if (tid == 0) s_nlift = 0;
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.el_vtx[8 * k + tid / 3] + tid % 3];
		__syncthreads();
		int nl_local = 0;
		for (int i = tid; i < NL; i += NT) {
			const int d = args.cdof[base + i];
			const double c = args.ccoef[base + i];
			cd[i] = d;
			cc[i] = c;
			cs[i] = d >= 0 ? args.Ap[d] : 0;
			ce[i] = d >= 0 ? args.Ap[d + 1] : 0;
			if (d < 0 && c != 0.0) nl_local++;
		}
		if (nl_local) atomicAdd(&s_nlift, nl_local);
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

		// ---- geometry (FP64): w J^-1 J^-T |J| (x coefficient), mass and source weights
		for (int q = tid; q < NQ; q += NT) {
			const int q1 = q / (nqy * nqz), q2 = (q / nqz) % nqy, q3 = q % nqz;
			const double x = Qx[q1], y = Qy[q2], z = Qz[q3];
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
			const double w = Wx[q1] * Wy[q2] * Wz[q3];
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

		// ---- load vector with lifting, matrix-free: lrhs_i = c_i (F_i - (K g)_i)
		if (do_rhs) {
			double *Pw = U + 4 * NQ;                       // P: [3][NX][nqy][nqz]
			double *Qw = Pw + 3 * NX * nqy * nqz;          // Q: [2][NX][NY][nqz]
			const int PS = NX * nqy * nqz, QS = NX * NY * nqz;
			if (s_nlift > 0 && args.Ax) {          // lifting only with the matrix (src/discretization.cc:296-317)
				for (int i = tid; i < QS; i += NT) {
					const int ab = i / nqz, q3 = i % nqz;
					double s0 = 0.0, s1 = 0.0;
					for (int c = 0; c < NZ; c++) {
						const int j = ab * NZ + c;
						const double g = cd[j] < 0 ? cc[j] : 0.0;
						s0 += g * Vz[c * nqz + q3];
						s1 += g * Dz[c * nqz + q3];
					}
					Qw[i] = s0;
					Qw[QS + i] = s1;
				}
				__syncthreads();
				for (int i = tid; i < PS; i += NT) {
					const int a = i / (nqy * nqz), q2 = (i / nqz) % nqy, q3 = i % nqz;
					double s00 = 0.0, s10 = 0.0, s01 = 0.0;
					for (int b = 0; b < NY; b++) {
						const double q0v = Qw[(a * NY + b) * nqz + q3], q1v = Qw[QS + (a * NY + b) * nqz + q3];
						s00 += q0v * Vy[b * nqy + q2];
						s10 += q0v * Dy[b * nqy + q2];
						s01 += q1v * Vy[b * nqy + q2];
					}
					Pw[i] = s00;
					Pw[PS + i] = s10;
					Pw[2 * PS + i] = s01;
				}
				__syncthreads();
				for (int q = tid; q < NQ; q += NT) {
					const int q1 = q / (nqy * nqz), q23 = q % (nqy * nqz);
					double u0 = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
					for (int a = 0; a < NX; a++) {
						const double p00 = Pw[a * nqy * nqz + q23], p10 = Pw[PS + a * nqy * nqz + q23];
						const double p01 = Pw[2 * PS + a * nqy * nqz + q23];
						u0 += p00 * Vx[a * nqx + q1];
						ux += p00 * Dx[a * nqx + q1];
						uy += p10 * Vx[a * nqx + q1];
						uz += p01 * Vx[a * nqx + q1];
					}
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
			for (int i = tid; i < PS; i += NT) {
				const int a = i / (nqy * nqz), q23 = i % (nqy * nqz);
				double s00 = 0.0, s10 = 0.0, s01 = 0.0;
				for (int q1 = 0; q1 < nqx; q1++) {
					const int q = q1 * nqy * nqz + q23;
					s00 += U[q] * Vx[a * nqx + q1] + U[NQ + q] * Dx[a * nqx + q1];
					s10 += U[2 * NQ + q] * Vx[a * nqx + q1];
					s01 += U[3 * NQ + q] * Vx[a * nqx + q1];
				}
				Pw[i] = s00;
				Pw[PS + i] = s10;
				Pw[2 * PS + i] = s01;
			}
			__syncthreads();
			for (int i = tid; i < QS; i += NT) {
				const int a = i / (NY * nqz), b = (i / nqz) % NY, q3 = i % nqz;
				double s0 = 0.0, s1 = 0.0;
				for (int q2 = 0; q2 < nqy; q2++) {
					const int o = (a * nqy + q2) * nqz + q3;
					s0 += Pw[o] * Vy[b * nqy + q2] + Pw[PS + o] * Dy[b * nqy + q2];
					s1 += Pw[2 * PS + o] * Vy[b * nqy + q2];
				}
				Qw[i] = s0;
				Qw[QS + i] = s1;
			}
			__syncthreads();
			for (int i = tid; i < NL; i += NT) {
				if (cd[i] < 0) continue;
				const int ab = i / NZ, c = i % NZ;
				double s = 0.0;
				for (int q3 = 0; q3 < nqz; q3++)
					s += Qw[ab * nqz + q3] * Vz[c * nqz + q3] + Qw[QS + ab * nqz + q3] * Dz[c * nqz + q3];
				posted_add(args.rhs + cd[i], -cc[i] * s);
			}
			__syncthreads();
		}

		// ---- matrix, per trial z index c'
		if (args.Ax) {
			const uint16_t *offe = args.offm + args.el_obase[k];
			for (int c2 = 0; c2 < NZ; c2++) {
				// stage 1: T1_kk[q1][q2][c] = sum_q3 G_g(kk) E_z^alpha[c][q3] E_z^beta[c'][q3] (+ mass into kk = 2)
				for (int i = tid; i < 9 * nqx * nqy; i += NT) {
					const int kk = i / (nqx * nqy), q12 = i % (nqx * nqy);
					const int fz = kMxFz[kk];
					const double *eb = (fz & 1) ? Dz + c2 * nqz : Vz + c2 * nqz;
					const double *gp = G + kMxG[kk] * NQ + q12 * nqz;
					const double *gm = G + 6 * NQ + q12 * nqz;
					const bool addm = kk == 2 && args.mass;
					double h[QM], hm[QM];
#pragma unroll
					for (int q3 = 0; q3 < QM; q3++) {
						h[q3] = q3 < nqz ? gp[q3] * eb[q3] : 0.0;
						hm[q3] = (addm && q3 < nqz) ? gm[q3] * Vz[c2 * nqz + q3] : 0.0;
					}
					double *out = T1 + (kk * nqx * nqy + q12) * NZ;
					for (int c = 0; c < NZ; c++) {
						const double *ea = (fz >> 1) ? Dz + c * nqz : Vz + c * nqz;
						double s = 0.0;
#pragma unroll
						for (int q3 = 0; q3 < QM; q3++)
							if (q3 < nqz) s += h[q3] * ea[q3];
						if (addm) {
#pragma unroll
							for (int q3 = 0; q3 < QM; q3++)
								if (q3 < nqz) s += hm[q3] * Vz[c * nqz + q3];
						}
						out[c] = s;
					}
				}
				__syncthreads();
				// stages 2 + 3 per row set (b', b, c)
				for (int r = tid; r < NY * NY * NZ; r += NT) {
					const int b2 = r / (NY * NZ), b = (r / NZ) % NY, c = r % NZ;
					double V[4][QM];
#pragma unroll
					for (int f = 0; f < 4; f++)
#pragma unroll
						for (int q1 = 0; q1 < QM; q1++) V[f][q1] = 0.0;
#pragma unroll
					for (int kk = 0; kk < 9; kk++) {
						// y flag and x class of product kk (compile-time after unrolling)
						constexpr int kFy[9] = { 0, 3, 0, 1, 2, 0, 0, 2, 1 };
						constexpr int kCls[9] = { 3, 0, 0, 2, 1, 2, 1, 0, 0 };
						const int fy = kFy[kk], f = kCls[kk];
						const double *ea = (fy >> 1) ? Dy + b * nqy : Vy + b * nqy;
						const double *eb = (fy & 1) ? Dy + b2 * nqy : Vy + b2 * nqy;
						double wy[QM];
#pragma unroll
						for (int q2 = 0; q2 < QM; q2++) wy[q2] = q2 < nqy ? ea[q2] * eb[q2] : 0.0;
						const double *t1 = T1 + kk * nqx * nqy * NZ + c;
#pragma unroll
						for (int q1 = 0; q1 < QM; q1++) {
							if (q1 < nqx) {
								double s = V[f][q1];
#pragma unroll
								for (int q2 = 0; q2 < QM; q2++)
									if (q2 < nqy) s += wy[q2] * t1[(q1 * nqy + q2) * NZ];
								V[f][q1] = s;
							}
						}
					}
					const int ibase = b * NZ + c;                  // i = a NY NZ + ibase
					for (int a2 = 0; a2 < NX; a2++) {
						const int j = (a2 * NY + b2) * NZ + c2;
						if (cd[j] < 0) continue;
						double Z0[QM], Z1[QM];
#pragma unroll
						for (int q1 = 0; q1 < QM; q1++) {
							const double e0 = q1 < nqx ? Vx[a2 * nqx + q1] : 0.0, e1 = q1 < nqx ? Dx[a2 * nqx + q1] : 0.0;
							Z0[q1] = e0 * V[0][q1] + e1 * V[1][q1];
							Z1[q1] = e0 * V[2][q1] + e1 * V[3][q1];
						}
						const double cj = cc[j];
						const int64_t c0 = cs[j], c1 = ce[j];
						const uint16_t *offcol = offe + (int64_t) j * NL;
						for (int a = 0; a < NX; a++) {
							const int i = a * NY * NZ + ibase;
							if (cd[i] < 0) continue;
							double s = 0.0;
#pragma unroll
							for (int q1 = 0; q1 < QM; q1++)
								if (q1 < nqx) s += Vx[a * nqx + q1] * Z0[q1] + Dx[a * nqx + q1] * Z1[q1];
							const int64_t pos = c0 + offcol[i];
							if (pos < c1) posted_add(args.Ax + pos, cc[i] * cj * s);
							else if (c1 > c0) atomicOr(args.status, kErrBounds);   // empty: column not owned
						}
					}
				}
				__syncthreads();
			}
		}
		__syncthreads();
	}
}

} // namespace h3dg
