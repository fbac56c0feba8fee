// Jacobi-preconditioned conjugate gradients on the assembled matrix (FP64),
// the on-device consumer of the assembly (the reference hands its
// UMFPackMatrix to UMFPACK, src/linsolver/umfpack.cc:280-330).  The matrix
// is the plan's CSC (Ap, Ai, Ax); the forms are symmetric, so column i is
// also row i and y = A x is a gather per column (one warp per column, fixed
// shuffle order).  Dot products reduce per-block partial sums in a fixed
// order: the iteration is bitwise reproducible.
#pragma once

#include "common.cuh"

namespace h3dg {

constexpr int kCgThreads = 256;
constexpr int kCgBlocks = 296;   // partial sums of the dot products

// y = A x (column i read as row i)
__global__ void __launch_bounds__(kCgThreads) k_cg_spmv(const int64_t *Ap, const int32_t *Ai, const double *Ax,
                                                        const double *x, double *y, int64_t n) {
	const int lane = threadIdx.x & 31;
	for (int64_t i = (blockIdx.x * (int64_t) blockDim.x + threadIdx.x) >> 5; i < n; i += ((int64_t) gridDim.x * blockDim.x) >> 5) {
		double s = 0.0;
		for (int64_t k = Ap[i] + lane; k < Ap[i + 1]; k += 32) s += Ax[k] * x[Ai[k]];
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) y[i] = s;
	}
}

// inverse diagonal (1 where the diagonal entry is missing or zero)
__global__ void k_cg_invdiag(const int64_t *Ap, const int32_t *Ai, const double *Ax, double *dinv, int64_t n) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		int64_t lo = Ap[i], hi = Ap[i + 1];
		while (lo < hi) {
			const int64_t mid = (lo + hi) / 2;
			if (Ai[mid] < i) lo = mid + 1;
			else hi = mid;
		}
		const double d = (lo < Ap[i + 1] && Ai[lo] == i) ? Ax[lo] : 0.0;
		dinv[i] = d != 0.0 ? 1.0 / d : 1.0;
	}
}

// partial[b] = sum over the block's fixed slice of a . b
__global__ void __launch_bounds__(kCgThreads) k_cg_dot_partial(const double *a, const double *b, int64_t n, double *partial) {
	__shared__ double red[kCgThreads];
	double s = 0.0;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) s += a[i] * b[i];
	red[threadIdx.x] = s;
	__syncthreads();
	for (int o = kCgThreads / 2; o > 0; o >>= 1) {
		if ((int) threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
		__syncthreads();
	}
	if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(kCgThreads) k_cg_dot_final(const double *partial, int nb, double *out) {
	__shared__ double red[kCgThreads];
	double s = 0.0;
	for (int i = threadIdx.x; i < nb; i += kCgThreads) s += partial[i];
	red[threadIdx.x] = s;
	__syncthreads();
	for (int o = kCgThreads / 2; o > 0; o >>= 1) {
		if ((int) threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
		__syncthreads();
	}
	if (threadIdx.x == 0) *out = red[0];
}

// x += alpha p, r -= alpha q, z = dinv r
__global__ void k_cg_update_xr(double *x, double *r, double *z, const double *p, const double *q, const double *dinv,
                               double alpha, int64_t n) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		x[i] += alpha * p[i];
		r[i] -= alpha * q[i];
		z[i] = dinv[i] * r[i];
	}
}

// p = z + beta p
__global__ void k_cg_update_p(double *p, const double *z, double beta, int64_t n) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
		p[i] = z[i] + beta * p[i];
}

// r = b - A x (from q = A x), z = dinv r, p = z
__global__ void k_cg_init(const double *b, const double *q, const double *dinv, double *r, double *z, double *p, int64_t n) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		r[i] = b[i] - q[i];
		z[i] = dinv[i] * r[i];
		p[i] = z[i];
	}
}

} // namespace h3dg
