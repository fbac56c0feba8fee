// Kernel variant table (see kernel_tables.h): FP64 tensor-core high-order kernels.
#include "kernel_tables.h"
#include "kernels/asm_fp64_dm.cuh"

namespace h3dg_tables {

template <int P, int NQ, int PHV = 0>
static DmSpec dm_spec() {
	using S = h3dg::DmShape<P, NQ, PHV>;
	return DmSpec { P, NQ, &h3dg::k_assemble_fp64_dm<P, NQ, PHV>, S::NT, S::SMEM_BYTES, false, (size_t) S::EPE,
	                &h3dg::k_build_offd<P, NQ> };
}

// Per (order, rule), the variants in order of preference; the first is used
// unless H3DG_DM_VARIANT=i picks the i-th (measurement).  Variants of one
// (order, rule) give the same bits.  The smaller CTAs (fewer pairs per
// iteration) let two CTAs share an SM: faster at p = 4 (32^3, 5.27 against
// 5.99 ms), slower at p = 5 (2.19 / 2.11) and p = 6 (5.64 / 4.95).
std::vector<DmSpec> &dm_table() {
	static std::vector<DmSpec> t = {
		dm_spec<4, 6, 3>(), dm_spec<4, 6>(), dm_spec<5, 6>(), dm_spec<5, 6, 2>(), dm_spec<5, 7>(), dm_spec<5, 7, 2>(),
		dm_spec<6, 7>(), dm_spec<6, 7, 1>(), dm_spec<6, 8>(), dm_spec<6, 8, 1>(),
		dm_spec<7, 8>(), dm_spec<7, 9>(), dm_spec<8, 9>(), dm_spec<8, 10>(),
	};
	return t;
}

cudaError_t build_offd(const DmSpec &k, const uint16_t *offc, const int32_t *cdof, const int64_t *Ap, int64_t ne,
                       const int64_t *color_ptr, int ncolors, int64_t nnz, uint16_t **offd, size_t *count,
                       unsigned long long *stores, int *status, cudaStream_t st) {
	const size_t n = (size_t) ne * k.epe;
	cudaError_t e = cudaMalloc((void **) offd, sizeof(uint16_t) * n);
	if (e != cudaSuccess) return e;
	*count = n;
	// first-touch flags: colour by colour over a byte per Ax slot (temporary)
	uint8_t *touched = nullptr;
	unsigned long long *d_st = nullptr;
	if (nnz > 0) {
		if (cudaMalloc((void **) &touched, (size_t) nnz) != cudaSuccess || cudaMalloc((void **) &d_st, sizeof(unsigned long long)) != cudaSuccess) {
			cudaGetLastError();
			if (touched) cudaFree(touched);
			touched = nullptr;
		}
	}
	*stores = 0;
	if (touched) {
		cudaMemsetAsync(touched, 0, (size_t) nnz, st);
		cudaMemsetAsync(d_st, 0, sizeof(unsigned long long), st);
		for (int c = 0; c < ncolors; c++)
			if (color_ptr[c + 1] > color_ptr[c])
				k.build<<<148 * 8, 256, 0, st>>>(offc, cdof, Ap, color_ptr[c], color_ptr[c + 1], *offd, status, touched, d_st);
		e = cudaMemcpyAsync(stores, d_st, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
		if (e == cudaSuccess) e = cudaStreamSynchronize(st);
		cudaFree(touched);
		cudaFree(d_st);
		if (e != cudaSuccess) return e;
	}
	else
		k.build<<<148 * 8, 256, 0, st>>>(offc, cdof, Ap, 0, ne, *offd, status, nullptr, nullptr);
	return cudaGetLastError();
}

} // namespace h3dg_tables
