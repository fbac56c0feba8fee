// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"
#include "kernels/asm_ho_tc.cuh"

namespace h3dg_tables {

template <int P, int NQ, int MINB = 1>
static HoSpec ho_tc_spec() {
	return HoSpec { P, NQ, &h3dg::k_assemble_ho_tc<P, P, P, NQ, NQ, NQ, MINB>, 256,
	                h3dg::HoTcShape<P, P, P, NQ, NQ, NQ>::SMEM_BYTES, false };
}

std::vector<HoSpec> &ho_tc_table() {
	static std::vector<HoSpec> t = {
		ho_tc_spec<1, 3, 2>(), ho_tc_spec<2, 4, 2>(), ho_tc_spec<3, 5, 2>(), ho_tc_spec<4, 6, 2>(), ho_tc_spec<5, 6>(), ho_tc_spec<5, 7>(), ho_tc_spec<6, 7>(),
		ho_tc_spec<6, 8>(), ho_tc_spec<7, 8>(), ho_tc_spec<7, 9>(), ho_tc_spec<8, 9>(), ho_tc_spec<8, 10>(),
	};
	return t;
}

cudaError_t build_offt(const uint16_t *offc, const int32_t *cdof, const int64_t *Ap, int64_t ne, int px, int nq,
                       const int64_t *color_ptr, int ncolors, int64_t nnz, uint16_t **offt, size_t *count,
                       unsigned long long *stores, int *status, cudaStream_t st) {
	(void) nq;
	const int nx = px + 1, nb = (nx * nx + 15) / 16 * 16;
	const size_t n = (size_t) ne * nx * (size_t) (nx * nx * nx) * nb;
	cudaError_t e = cudaMalloc((void **) offt, sizeof(uint16_t) * n);
	if (e != cudaSuccess) return e;
	*count = n;
	// first-touch flags: colour by colour over a byte per Ax slot (temporary)
	uint8_t *touched = nullptr;
	unsigned long long *d_st = nullptr;
	if (color_ptr && nnz > 0) {
		if (cudaMalloc((void **) &touched, (size_t) nnz) != cudaSuccess || cudaMalloc((void **) &d_st, sizeof(unsigned long long)) != cudaSuccess) {
			cudaGetLastError();
			if (touched) cudaFree(touched);
			touched = nullptr;
		}
	}
	if (touched) {
		cudaMemsetAsync(touched, 0, (size_t) nnz, st);
		cudaMemsetAsync(d_st, 0, sizeof(unsigned long long), st);
		for (int c = 0; c < ncolors; c++)
			if (color_ptr[c + 1] > color_ptr[c])
				h3dg::k_build_offt<<<148 * 8, 256, 0, st>>>(offc, cdof, Ap, color_ptr[c], color_ptr[c + 1], nx, nx, nx, nb, *offt,
				                                             status, touched, d_st);
		e = cudaMemcpyAsync(stores, d_st, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
		if (e == cudaSuccess) e = cudaStreamSynchronize(st);
		cudaFree(touched);
		cudaFree(d_st);
		if (e != cudaSuccess) return e;
	}
	else {
		*stores = 0;
		h3dg::k_build_offt<<<148 * 8, 256, 0, st>>>(offc, cdof, Ap, 0, ne, nx, nx, nx, nb, *offt, status, nullptr, nullptr);
	}
	return cudaGetLastError();
}

} // namespace h3dg_tables
