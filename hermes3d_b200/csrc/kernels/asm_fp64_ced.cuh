// FP64 assembly of elements with constrained (hanging) nodes.
//
// Such an element's assembly list maps its functions onto global functions
// through weights (the restrictions of the constraining functions,
// src/space.cc:296-450 with the CED combinations of
// src/shapeset/h1lobattohex.cc:428-719): column u of the element's W lists
// (canonical function s, weight w) pairs for one global DOF, and one extra
// column holds the Dirichlet lifting.
//
// Two kernels.  k_assemble_fp64_ced computes, for every constrained element
// in one persistent launch (no colouring: it writes only its own output),
// the element matrix K and load vector F in the element's canonical basis
// (orders raised to those of the constraining functions, rule of the
// element's own orders; the sum-factorised stages of the mixed-order kernel)
// into a per-CTA scratch block, then the element's entries in the global
// functions
//   E[v][u] = sum_{a in u} w_a sum_{b in v} w_b K[s_b][s_a]
//   r[u]    = sum_{a in u} w_a (F[s_a] - sum_{b in lift} w_b K[s_b][s_a])
// into its slice of an output buffer: the reference posts every pair of its
// assembly list (src/discretization.cc:293-342), whose sums these are.
// k_scatter_ced then posts E and r for the elements of one colour; elements
// of a colour share no DOF, so each entry receives at most one add per
// launch and the result is bitwise reproducible.
#pragma once

#include "common.cuh"

namespace h3dg {

struct KArgsCed {
	const double *xyz;
	const int32_t *el_vtx;     // nce x 8
	const int32_t *el_id;
	const double *ecoef;       // per element id, or nullptr
	const int32_t *el_desc;    // nce x 12: px py pz nqx nqy nqz ox oy oz nl class -
	const int64_t *ubase;      // nce + 1: the element's columns
	const int32_t *udof;       // per column: DOF, -1 = lifting (last)
	const int64_t *wptr;       // columns + 1
	const uint16_t *ws;        // canonical function of each weight
	const double *ww;          // weights
	const int64_t *obase;      // nce + 1
	const uint16_t *off;       // [v][u]: row position of DOF u in column DOF v
	const int64_t *Ap;
	const double *tables;
	int table_bytes;
	int mass, lf;
	double lf_value;
	double *Ax, *rhs;
	int *status;
	unsigned int *counters;
	double *scratch;           // per CTA: K (nl x nl, [j][i]), F (nl), Y (columns x nl)
	int64_t scratch_stride;    // doubles per CTA
	const int32_t *order;      // compute order (class, decreasing work) -> element
	const int64_t *ebase;      // nce + 1: the element's slice of out: E (nu x nu, [v][u]) then r (nu)
	double *out;
};

template <int PM, int QM>
struct CedShape {
	static constexpr int NM = PM + 1;
	static constexpr int Q3 = QM * QM * QM;
	static constexpr int T1 = 9 * QM * QM * NM;
	static constexpr int MF = 4 * Q3 + 3 * NM * QM * QM + 2 * NM * NM * QM;
	static constexpr int UNION = T1 > MF ? T1 : MF;
	static constexpr int R_G = 0;                  // 8 x nq: xx yy zz xy xz yz mass src
	static constexpr int R_U = R_G + 8 * Q3;
	static constexpr int R_X = R_U + UNION;
	static constexpr int R_M = R_X + 24;
	static constexpr int END = R_M + 24;
	static size_t smem_bytes(int table_bytes) { return (size_t) ((table_bytes + 15) / 16) * 16 + sizeof(double) * END; }
};

static __device__ __constant__ int kCeG[9] = { 0, 1, 2, 3, 3, 4, 4, 5, 5 };
static __device__ __constant__ int kCeFz[9] = { 0, 0, 3, 0, 0, 1, 2, 1, 2 };

template <int PM, int QM, int NT>
__global__ void __launch_bounds__(NT, 1) k_assemble_fp64_ced(KArgsCed args, int64_t kbeg, int64_t kend, int launch) {
	using S = CedShape<PM, QM>;
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar;
	__shared__ int64_t s_k;
	const int tid = threadIdx.x;
	if (!stage_tables(sm, args.tables, args.table_bytes, &bar, args.status)) return;
	const double *tab = sm;
	double *R = sm + ((args.table_bytes + 15) / 16) * 2;
	double *G = R + S::R_G, *U = R + S::R_U, *T1 = R + S::R_U;
	double *X = R + S::R_X, *Mo = R + S::R_M;
	double *Ks = args.scratch + (int64_t) blockIdx.x * args.scratch_stride;

	for (;;) {
		if (tid == 0) s_k = kbeg + (int64_t) atomicAdd(&args.counters[launch], 1u);
		__syncthreads();
		const int64_t k = s_k;
		if (k >= kend) break;                                   // block-uniform
		const int64_t el = args.order[k];
		const int32_t *dsc = args.el_desc + el * 12;
		const int px = dsc[0], py = dsc[1], pz = dsc[2];
		const int nqx = dsc[3], nqy = dsc[4], nqz = dsc[5];
		const int NX = px + 1, NY = py + 1, NZ = pz + 1, NL = NX * NY * NZ;
		const int NQ = nqx * nqy * nqz;
		const double *Vx = tab + dsc[6], *Dx = Vx + NX * nqx, *Qx = Dx + NX * nqx, *Wx = Qx + nqx;
		const double *Vy = tab + dsc[7], *Dy = Vy + NY * nqy, *Qy = Dy + NY * nqy, *Wy = Qy + nqy;
		const double *Vz = tab + dsc[8], *Dz = Vz + NZ * nqz, *Qz = Dz + NZ * nqz, *Wz = Qz + nqz;
		double *Fs = Ks + (int64_t) NL * NL;
		const int64_t u0 = args.ubase[el], u1 = args.ubase[el + 1];
		const bool has_lift = u1 > u0 && args.udof[u1 - 1] < 0;
		const int nu = (int) (u1 - u0) - (has_lift ? 1 : 0);
		const bool do_rhs = args.rhs && args.lf;      // no linear form: no rhs update at all (src/discretization.cc:328-338)
		const bool need_k = args.Ax != nullptr;          // the lifting enters only with the matrix (src/discretization.cc:296-317)

		// ---- set-up: vertices, monomial coefficients of the trilinear map
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.el_vtx[8 * el + tid / 3] + tid % 3];
		__syncthreads();
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
		const double cgrad = args.ecoef ? args.ecoef[args.el_id[el]] : 1.0;
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

		// ---- load vector in the canonical basis: F_i = sum_q w |J| f phi_i
		if (do_rhs) {
			double *Pw = U + NQ;                           // P: [NX][nqy][nqz]
			double *Qw = Pw + NX * nqy * nqz;              // Q: [NX][NY][nqz]
			const int PS = NX * nqy * nqz, QS = NX * NY * nqz;
			for (int i = tid; i < PS; i += NT) {
				const int a = i / (nqy * nqz), q23 = i % (nqy * nqz);
				double s = 0.0;
				for (int q1 = 0; q1 < nqx; q1++) s += G[7 * NQ + q1 * nqy * nqz + q23] * Vx[a * nqx + q1];
				Pw[i] = s;
			}
			__syncthreads();
			for (int i = tid; i < QS; i += NT) {
				const int a = i / (NY * nqz), b = (i / nqz) % NY, q3 = i % nqz;
				double s = 0.0;
				for (int q2 = 0; q2 < nqy; q2++) s += Pw[(a * nqy + q2) * nqz + q3] * Vy[b * nqy + q2];
				Qw[i] = s;
			}
			__syncthreads();
			for (int i = tid; i < NL; i += NT) {
				const int ab = i / NZ, c = i % NZ;
				double s = 0.0;
				for (int q3 = 0; q3 < nqz; q3++) s += Qw[ab * nqz + q3] * Vz[c * nqz + q3];
				Fs[i] = s;
			}
			__syncthreads();
		}

		// ---- element matrix in the canonical basis, per trial z index c'
		if (need_k) {
			for (int c2 = 0; c2 < NZ; c2++) {
				// stage 1: T1_kk[q1][q2][c] = sum_q3 G_g(kk) E_z^alpha[c][q3] E_z^beta[c'][q3] (+ mass into kk = 2)
				for (int i = tid; i < 9 * nqx * nqy; i += NT) {
					const int kk = i / (nqx * nqy), q12 = i % (nqx * nqy);
					const int fz = kCeFz[kk];
					const double *eb = (fz & 1) ? Dz + c2 * nqz : Vz + c2 * nqz;
					const double *gp = G + kCeG[kk] * NQ + q12 * nqz;
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
						double Z0[QM], Z1[QM];
#pragma unroll
						for (int q1 = 0; q1 < QM; q1++) {
							const double e0 = q1 < nqx ? Vx[a2 * nqx + q1] : 0.0, e1 = q1 < nqx ? Dx[a2 * nqx + q1] : 0.0;
							Z0[q1] = e0 * V[0][q1] + e1 * V[1][q1];
							Z1[q1] = e0 * V[2][q1] + e1 * V[3][q1];
						}
						double *kcol = Ks + (int64_t) j * NL;
						for (int a = 0; a < NX; a++) {
							double s = 0.0;
#pragma unroll
							for (int q1 = 0; q1 < QM; q1++)
								if (q1 < nqx) s += Vx[a * nqx + q1] * Z0[q1] + Dx[a * nqx + q1] * Z1[q1];
							kcol[a * NY * NZ + ibase] = s;
						}
					}
				}
				__syncthreads();
			}
		}

		// ---- entries in the global functions, into the element's output slice:
		// Y[v][i] = sum_{b in v} w_b K[s_b][i] (coalesced over the rows i), then
		// E[v][u] = sum_{a in u} w_a Y[v][s_a]; the lifting column last
		double *E = args.out + args.ebase[el];
		double *Y = Fs + NL;
		const int nv = (int) (u1 - u0);
		if (need_k) {
			const int vb = args.Ax ? 0 : nu;                 // without Ax only the lifting column
			for (int p = tid; p < (nv - vb) * NL; p += NT) {
				const int v = vb + p / NL, i = p % NL;
				const int64_t b0 = args.wptr[u0 + v], b1 = args.wptr[u0 + v + 1];
				double s = 0.0;
				for (int64_t bi = b0; bi < b1; bi++) s += args.ww[bi] * Ks[(int64_t) args.ws[bi] * NL + i];
				Y[(int64_t) v * NL + i] = s;
			}
			__syncthreads();
		}
		if (args.Ax) {
			for (int p = tid; p < nu * nu; p += NT) {
				const int v = p / nu, u = p % nu;
				const int64_t a0 = args.wptr[u0 + u], a1 = args.wptr[u0 + u + 1];
				const double *yv = Y + (int64_t) v * NL;
				double s = 0.0;
				for (int64_t ai = a0; ai < a1; ai++) s += args.ww[ai] * yv[args.ws[ai]];
				E[p] = s;
			}
		}
		if (do_rhs) {
			const double *yl = Y + (int64_t) nu * NL;
			for (int u = tid; u < nu; u += NT) {
				const int64_t a0 = args.wptr[u0 + u], a1 = args.wptr[u0 + u + 1];
				double s = 0.0;
				if (args.lf)
					for (int64_t ai = a0; ai < a1; ai++) s += args.ww[ai] * Fs[args.ws[ai]];
				if (has_lift && args.Ax)
					for (int64_t ai = a0; ai < a1; ai++) s -= args.ww[ai] * yl[args.ws[ai]];
				E[(int64_t) nu * nu + u] = s;
			}
		}
		__syncthreads();
	}
}

// posts the entries of the constrained elements kbeg..kend-1 (one colour):
// one CTA per element at a time
template <int NT>
__global__ void __launch_bounds__(NT) k_scatter_ced(KArgsCed args, int64_t kbeg, int64_t kend) {
	for (int64_t k = kbeg + blockIdx.x; k < kend; k += gridDim.x) {
		const int64_t u0 = args.ubase[k], u1 = args.ubase[k + 1];
		const bool has_lift = u1 > u0 && args.udof[u1 - 1] < 0;
		const int nu = (int) (u1 - u0) - (has_lift ? 1 : 0);
		const double *E = args.out + args.ebase[k];
		if (args.Ax) {
			const uint16_t *offe = args.off + args.obase[k];
			for (int p = threadIdx.x; p < nu * nu; p += NT) {
				const int v = p / nu, u = p % nu;
				const int dv = args.udof[u0 + v];
				const int64_t c0 = args.Ap[dv], c1 = args.Ap[dv + 1];
				const int64_t pos = c0 + offe[p];
				if (pos < c1) posted_add(args.Ax + pos, E[p]);
				else if (c1 > c0) atomicOr(args.status, kErrBounds);
				(void) u;
			}
		}
		if (args.rhs && args.lf)
			for (int u = threadIdx.x; u < nu; u += NT) posted_add(args.rhs + args.udof[u0 + u], E[(int64_t) nu * nu + u]);
	}
}

} // namespace h3dg
