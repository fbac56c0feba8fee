// Error and solution norms of a finite-element function (FP64), as the
// reference's calc_error / calc_norm with error_fn_h1 / norm_fn_h1 and the
// L2 variants (src/norm.cc:33-180): per active element, the coefficient
// tensor of u_h from the assembly list (sum of coef x solution[DOF], the
// Dirichlet lifting value for DOF -1), values and reference gradients at the
// element's rule by sum factorisation, physical gradients J^-T grad_xi, and
//   e_L2 = sum w |J| (u_h - u)^2,  e_H1 = e_L2 + sum w |J| |grad u_h - grad u|^2,
//   n_L2 = sum w |J| u_h^2,        n_H1 = n_L2 + sum w |J| |grad u_h|^2
// for an exact solution u of a built-in kind.  Per-element partial sums are
// reduced in a fixed order (bitwise reproducible).
#pragma once

#include "common.cuh"

namespace h3dg {

constexpr int kExactZero = 0, kExactQuadratic = 1, kExactSin = 2;

struct KArgsNorm {
	const double *xyz;
	const int32_t *el_vtx;     // ne x 8
	const int32_t *el_desc;    // ne x 12: px py pz nqx nqy nqz ox oy oz nl - -
	const int64_t *gptr;       // ne + 1: groups (one per canonical function present, ascending)
	const int64_t *eptr;       // groups + 1: entries of each group
	const uint16_t *gs;        // canonical function of each group
	const int32_t *edof;       // entry DOF (-1: lifting)
	const double *ecoef;       // entry coefficient (sign included)
	const double *tables;      // per set: V[(p+1) nq], D[(p+1) nq], q[nq], w[nq]
	const double *sol;         // ndof
	int exact;
	double *partial;           // ne x 4
};

__device__ __forceinline__ void exact_value(int kind, const double x[3], double &u, double g[3]) {
	if (kind == kExactQuadratic) {
		u = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
		g[0] = 2.0 * x[0]; g[1] = 2.0 * x[1]; g[2] = 2.0 * x[2];
	}
	else if (kind == kExactSin) {
		const double sx = sinpi(x[0]), sy = sinpi(x[1]), sz = sinpi(x[2]);
		const double pi = 3.141592653589793;
		u = sx * sy * sz;
		g[0] = pi * cospi(x[0]) * sy * sz;
		g[1] = pi * sx * cospi(x[1]) * sz;
		g[2] = pi * sx * sy * cospi(x[2]);
	}
	else { u = 0.0; g[0] = g[1] = g[2] = 0.0; }
}

// dynamic shared memory: C[nl], A[2][nx][ny][nqz], B[3][nx][nqy][nqz], red[4][NT]
template <int NT>
__global__ void __launch_bounds__(NT) k_norms(KArgsNorm args, int64_t ne, int nlmax, int amax, int bmax) {
	extern __shared__ __align__(16) double sd[];
	__shared__ double X[24], Mo[24];
	double *Cf = sd, *A = Cf + nlmax, *B = A + amax, *red = B + bmax;
	const int tid = threadIdx.x;
	for (int64_t k = blockIdx.x; k < ne; k += gridDim.x) {
		const int32_t *dsc = args.el_desc + k * 12;
		const int px = dsc[0], py = dsc[1], pz = dsc[2], nqx = dsc[3], nqy = dsc[4], nqz = dsc[5];
		const int NX = px + 1, NY = py + 1, NZ = pz + 1, NL = NX * NY * NZ;
		const double *Vx = args.tables + dsc[6], *Dx = Vx + NX * nqx, *Qx = Dx + NX * nqx, *Wx = Qx + nqx;
		const double *Vy = args.tables + dsc[7], *Dy = Vy + NY * nqy, *Qy = Dy + NY * nqy, *Wy = Qy + nqy;
		const double *Vz = args.tables + dsc[8], *Dz = Vz + NZ * nqz, *Qz = Dz + NZ * nqz, *Wz = Qz + nqz;
		if (tid < 24) X[tid] = args.xyz[3 * (int64_t) args.el_vtx[8 * k + tid / 3] + tid % 3];
		for (int i = tid; i < NL; i += NT) Cf[i] = 0.0;
		__syncthreads();
		// coefficient tensor, one thread per canonical function, entries in order
		for (int64_t g = args.gptr[k] + tid; g < args.gptr[k + 1]; g += NT) {
			double s = 0.0;
			for (int64_t e = args.eptr[g]; e < args.eptr[g + 1]; e++) {
				const int d = args.edof[e];
				s += args.ecoef[e] * (d >= 0 ? args.sol[d] : 1.0);
			}
			Cf[args.gs[g]] = s;
		}
		for (int i = tid; i < 24; i += NT) {
			const int mo = i / 3, r = i % 3;
			const int usex = mo == 1 || mo == 4 || mo == 5 || mo == 7;
			const int usey = mo == 2 || mo == 4 || mo == 6 || mo == 7;
			const int usez = mo == 3 || mo == 5 || mo == 6 || mo == 7;
			double c = 0.0;
			for (int v = 0; v < 8; v++) {
				const int bx = ((v + 1) >> 1) & 1, by = (v >> 1) & 1, bz = v >> 2;
				const int neg = (usex && !bx) ^ (usey && !by) ^ (usez && !bz);
				c += neg ? -X[3 * v + r] : X[3 * v + r];
			}
			Mo[i] = 0.125 * c;
		}
		__syncthreads();
		// z, then y: A0/A1 = C x (V_z | D_z); B00/B10/B01
		const int AS = NX * NY * nqz, BS = NX * nqy * nqz;
		for (int i = tid; i < AS; i += NT) {
			const int ab = i / nqz, q3 = i % nqz;
			double s0 = 0.0, s1 = 0.0;
			for (int c = 0; c < NZ; c++) {
				const double cf = Cf[ab * NZ + c];
				s0 += cf * Vz[c * nqz + q3];
				s1 += cf * Dz[c * nqz + q3];
			}
			A[i] = s0;
			A[AS + i] = s1;
		}
		__syncthreads();
		for (int i = tid; i < BS; i += NT) {
			const int a = i / (nqy * nqz), q2 = (i / nqz) % nqy, q3 = i % nqz;
			double s00 = 0.0, s10 = 0.0, s01 = 0.0;
			for (int b = 0; b < NY; b++) {
				const double a0 = A[(a * NY + b) * nqz + q3], a1 = A[AS + (a * NY + b) * nqz + q3];
				s00 += a0 * Vy[b * nqy + q2];
				s10 += a0 * Dy[b * nqy + q2];
				s01 += a1 * Vy[b * nqy + q2];
			}
			B[i] = s00;
			B[BS + i] = s10;
			B[2 * BS + i] = s01;
		}
		__syncthreads();
		// x, geometry and the integrands per point
		double acc[4] = { 0.0, 0.0, 0.0, 0.0 };
		const int NQ = nqx * nqy * nqz;
		for (int q = tid; q < NQ; q += NT) {
			const int q1 = q / (nqy * nqz), q23 = q % (nqy * nqz), q2 = q23 / nqz, q3 = q23 % nqz;
			double u = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
			for (int a = 0; a < NX; a++) {
				const double b00 = B[a * nqy * nqz + q23], b10 = B[BS + a * nqy * nqz + q23], b01 = B[2 * BS + a * nqy * nqz + q23];
				u += b00 * Vx[a * nqx + q1];
				ux += b00 * Dx[a * nqx + q1];
				uy += b10 * Vx[a * nqx + q1];
				uz += b01 * Vx[a * nqx + q1];
			}
			const double x = Qx[q1], y = Qy[q2], z = Qz[q3];
			const double xy = x * y, xz = x * z, yz = y * z, xyz = xy * z;
			double m[3][3], xp[3];
			for (int r = 0; r < 3; r++) {
				const double c0 = Mo[r], c1 = Mo[3 + r], c2 = Mo[6 + r], c3 = Mo[9 + r];
				const double c4 = Mo[12 + r], c5 = Mo[15 + r], c6 = Mo[18 + r], c7 = Mo[21 + r];
				m[r][0] = c1 + c4 * y + c5 * z + c7 * yz;
				m[r][1] = c2 + c4 * x + c6 * z + c7 * xz;
				m[r][2] = c3 + c5 * x + c6 * y + c7 * xy;
				xp[r] = c0 + c1 * x + c2 * y + c3 * z + c4 * xy + c5 * xz + c6 * yz + c7 * xyz;
			}
			// cofactors C_rk: grad_x u = (1/det) sum_k C_rk du/dxi_k
			double C[3][3];
			C[0][0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
			C[0][1] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
			C[0][2] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
			C[1][0] = m[0][2] * m[2][1] - m[0][1] * m[2][2];
			C[1][1] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
			C[1][2] = m[0][1] * m[2][0] - m[0][0] * m[2][1];
			C[2][0] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
			C[2][1] = m[0][2] * m[1][0] - m[0][0] * m[1][2];
			C[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
			const double det = m[0][0] * C[0][0] + m[0][1] * C[0][1] + m[0][2] * C[0][2];
			const double wd = Wx[q1] * Wy[q2] * Wz[q3] * det;          // signed, as the assembly
			double gh[3];
			for (int r = 0; r < 3; r++) gh[r] = (C[r][0] * ux + C[r][1] * uy + C[r][2] * uz) / det;
			double ue, ge[3];
			exact_value(args.exact, xp, ue, ge);
			const double du = u - ue;
			const double dg = (gh[0] - ge[0]) * (gh[0] - ge[0]) + (gh[1] - ge[1]) * (gh[1] - ge[1]) + (gh[2] - ge[2]) * (gh[2] - ge[2]);
			acc[0] += wd * du * du;
			acc[1] += wd * (du * du + dg);
			acc[2] += wd * u * u;
			acc[3] += wd * (u * u + gh[0] * gh[0] + gh[1] * gh[1] + gh[2] * gh[2]);
		}
		// fixed-order block reduction
		for (int j = 0; j < 4; j++) red[j * NT + tid] = acc[j];
		__syncthreads();
		for (int s = NT / 2; s > 0; s >>= 1) {
			if (tid < s)
				for (int j = 0; j < 4; j++) red[j * NT + tid] += red[j * NT + tid + s];
			__syncthreads();
		}
		if (tid < 4) args.partial[4 * k + tid] = red[tid * NT];
		__syncthreads();
	}
}

// sum of the per-element partials, one CTA, fixed order
template <int NT>
__global__ void __launch_bounds__(NT) k_norms_reduce(const double *partial, int64_t ne, double *out) {
	__shared__ double red[4][NT];
	double acc[4] = { 0.0, 0.0, 0.0, 0.0 };
	for (int64_t e = threadIdx.x; e < ne; e += NT)
		for (int j = 0; j < 4; j++) acc[j] += partial[4 * e + j];
	for (int j = 0; j < 4; j++) red[j][threadIdx.x] = acc[j];
	__syncthreads();
	for (int s = NT / 2; s > 0; s >>= 1) {
		if ((int) threadIdx.x < s)
			for (int j = 0; j < 4; j++) red[j][threadIdx.x] += red[j][threadIdx.x + s];
		__syncthreads();
	}
	if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

} // namespace h3dg
