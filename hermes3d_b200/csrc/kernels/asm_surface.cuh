// Surface forms on natural boundary faces (FP64): Discretization::assemble's
// surface loop (src/discretization.cc:345-412) with surf_int_u_v and
// surf_int_G_v (src/integrals/h1.h:200-242), the integrals taken with the
// element's rule on the face's two directions.  Per face: the surface
// Jacobian |dx/dxi_1 x dx/dxi_2| of the trilinear map at the face points
// (RefMap::calc_face_jacobian, src/refmap.cc:416-475), the trace functions
// l_a(xi_1) l_b(xi_2) of the boundary assembly list, and
//   Ax[slot(i, j)] += c_i c_j int u_j v_i            (DOF_j >= 0)
//   lrhs_i          -= c_i c_j int u_j v_i            (DOF_j Dirichlet)
//   rhs[DOF_i]      += lrhs_i + c_i int g v_i         (only with a surface linear form)
// The whole surface pass runs only with a matrix, as in the reference.  Faces
// of one launch (one colour) share no DOF: one posted add per entry.
#pragma once

#include "common.cuh"

namespace h3dg {

constexpr int kSurfMarkers = 16;

struct KArgsSurf {
	const double *xyz;
	const int32_t *desc;       // nsf x 8: element, face, marker, n, nq1, nq2, t1, t2
	const int32_t *vtx;        // nsf x 8
	const int64_t *base, *obase;
	const int32_t *dof;
	const double *coef;
	const int16_t *ab;         // 2 per trace function
	const uint16_t *off;       // [j][i]
	const int64_t *Ap;
	const double *tables;      // per (order, points) set: q[nq], w[nq], V[(p+1) nq]
	int bf, lf;
	double g[kSurfMarkers];    // g by boundary marker
	double *Ax, *rhs;
	int *status;
};

// dynamic shared memory: wJ[nq], then Phi[n][nq] (sized by the host from the largest face)
template <int NT>
__global__ void __launch_bounds__(NT) k_assemble_surface(KArgsSurf args, int64_t kbeg, int64_t kend) {
	extern __shared__ __align__(16) double sd[];
	__shared__ double X[24];
	__shared__ double Fg[1];
	const int tid = threadIdx.x;
	for (int64_t k = kbeg + blockIdx.x; k < kend; k += gridDim.x) {
		const int32_t *d = args.desc + 8 * k;
		const int f = d[1], marker = d[2], n = d[3], nq1 = d[4], nq2 = d[5];
		const double *Q1 = args.tables + d[6], *W1 = Q1 + nq1, *V1 = W1 + nq1;
		const double *Q2 = args.tables + d[7], *W2 = Q2 + nq2, *V2 = W2 + nq2;
		const int NQ = nq1 * nq2;
		double *wJ = sd, *Phi = sd + NQ;
		const int64_t b = args.base[k];
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.vtx[8 * k + tid / 3] + tid % 3];
		if (tid == 0) Fg[0] = (marker >= 0 && marker < kSurfMarkers) ? args.g[marker] : 0.0;
		__syncthreads();
		// RefHex faces: x = -1, x = 1, y = -1, y = 1, z = -1, z = 1; face directions ascending
		const int dn = f >> 1, d1 = dn == 0 ? 1 : 0, d2 = dn == 2 ? 1 : 2;
		const double xn = (f & 1) ? 1.0 : -1.0;
		for (int q = tid; q < NQ; q += NT) {
			const int i1 = q / nq2, i2 = q % nq2;
			double xi[3];
			xi[dn] = xn;
			xi[d1] = Q1[i1];
			xi[d2] = Q2[i2];
			// tangents dx/dxi_d1, dx/dxi_d2 of the trilinear map (vertex v: corner (bx, by, bz))
			double t1[3] = { 0.0, 0.0, 0.0 }, t2[3] = { 0.0, 0.0, 0.0 };
#pragma unroll
			for (int v = 0; v < 8; v++) {
				const int bc[3] = { ((v + 1) >> 1) & 1, (v >> 1) & 1, v >> 2 };
				double l[3], dl[3];
#pragma unroll
				for (int r = 0; r < 3; r++) {
					l[r] = bc[r] ? 0.5 * (1.0 + xi[r]) : 0.5 * (1.0 - xi[r]);
					dl[r] = bc[r] ? 0.5 : -0.5;
				}
				double g1 = dl[d1], g2 = dl[d2];
#pragma unroll
				for (int r = 0; r < 3; r++) {
					if (r != d1) g1 *= l[r];
					if (r != d2) g2 *= l[r];
				}
#pragma unroll
				for (int r = 0; r < 3; r++) {
					t1[r] += X[3 * v + r] * g1;
					t2[r] += X[3 * v + r] * g2;
				}
			}
			const double cx = t1[1] * t2[2] - t1[2] * t2[1], cy = t1[2] * t2[0] - t1[0] * t2[2], cz = t1[0] * t2[1] - t1[1] * t2[0];
			wJ[q] = W1[i1] * W2[i2] * sqrt(cx * cx + cy * cy + cz * cz);
		}
		for (int p = tid; p < n * NQ; p += NT) {
			const int i = p / NQ, q = p % NQ;
			const int a = args.ab[2 * (b + i)], c = args.ab[2 * (b + i) + 1];
			Phi[p] = V1[a * nq1 + q / nq2] * V2[c * nq2 + q % nq2];
		}
		__syncthreads();
		if (args.bf) {
			const uint16_t *offe = args.off + args.obase[k];
			for (int p = tid; p < n * n; p += NT) {
				const int j = p / n, i = p % n;
				const int di = args.dof[b + i], dj = args.dof[b + j];
				if (di < 0 || dj < 0) continue;
				const double *pi = Phi + i * NQ, *pj = Phi + j * NQ;
				double s = 0.0;
				for (int q = 0; q < NQ; q++) s += wJ[q] * pi[q] * pj[q];
				const int64_t c0 = args.Ap[dj], c1 = args.Ap[dj + 1], pos = c0 + offe[p];
				if (pos < c1) posted_add(args.Ax + pos, args.coef[b + i] * args.coef[b + j] * s);
				else atomicOr(args.status, kErrBounds);
			}
		}
		if (args.lf && args.rhs) {
			const double gm = Fg[0];
			for (int i = tid; i < n; i += NT) {
				const int di = args.dof[b + i];
				if (di < 0) continue;
				const double *pi = Phi + i * NQ;
				double r = 0.0;
				if (args.bf)
					for (int j = 0; j < n; j++) {
						if (args.dof[b + j] >= 0) continue;
						const double *pj = Phi + j * NQ;
						double s = 0.0;
						for (int q = 0; q < NQ; q++) s += wJ[q] * pi[q] * pj[q];
						r -= args.coef[b + i] * args.coef[b + j] * s;
					}
				double s = 0.0;
				for (int q = 0; q < NQ; q++) s += wJ[q] * pi[q];
				posted_add(args.rhs + di, r + args.coef[b + i] * (gm * s));
			}
		}
		__syncthreads();
	}
}

} // namespace h3dg
