// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"
#include "kernels/asm_fp64.cuh"
#include "kernels/asm_fp64_seq.cuh"
#include "kernels/asm_fp64_warp.cuh"

namespace h3dg_tables {

template <int P, int NQ, int NT, int EB, int MINB = 1, bool PF = false>
static KernelSpec spec() {
	return KernelSpec { P, NQ, &h3dg::k_assemble_fp64<P, P, P, NQ, NQ, NQ, NT, EB, MINB, PF>, NT, EB,
	                    h3dg::SfShape<P, P, P, NQ, NQ, NQ, EB>::SMEM_BYTES, false };
}

// one element per warp, W warps per CTA
template <int P, int NQ, int W, int MINB>
static KernelSpec spec_warp() {
	return KernelSpec { P, NQ, &h3dg::k_assemble_fp64_warp<P, P, P, NQ, NQ, NQ, W, MINB>, 32 * W, W,
	                    h3dg::WarpShape<P, P, P, NQ, NQ, NQ, W>::SMEM_BYTES, false };
}

template <int P, int NQ, int NT, int EB>
static KernelSpec spec_seq() {
	return KernelSpec { P, NQ, &h3dg::k_assemble_fp64_seq<P, P, P, NQ, NQ, NQ, NT, EB>, NT, EB,
	                    h3dg::SfShapeSeq<P, P, P, NQ, NQ, NQ, EB>::SMEM_BYTES, false };
}

std::vector<KernelSpec> &kernel_table() {
	static std::vector<KernelSpec> t = {
		spec<1, 2, 64, 4, 8>(), spec<1, 3, 64, 4, 8>(), spec<1, 2, 128, 8, 4>(), spec<1, 3, 128, 8, 4>(),
		spec<2, 3, 96, 1, 8>(), spec<2, 3, 192, 2, 4>(),
		spec<2, 4, 96, 1>(), spec<2, 4, 96, 1, 8>(), spec<2, 4, 96, 1, 10>(), spec<2, 4, 128, 1, 8>(),
		spec<2, 4, 192, 2, 4>(), spec<2, 4, 192, 2, 5>(), spec<2, 4, 256, 3, 3>(),
		spec_warp<2, 4, 4, 4>(), spec_warp<2, 4, 4, 3>(), spec_warp<2, 4, 8, 2>(), spec_warp<2, 4, 2, 8>(),
		spec<2, 4, 96, 1, 4, true>(), spec<2, 4, 96, 1, 6, true>(), spec<2, 4, 128, 1, 4, true>(),
		spec<2, 4, 192, 2, 2, true>(), spec<2, 4, 192, 2, 3, true>(),
		spec<2, 5, 96, 1, 8>(), spec<2, 5, 192, 2, 4>(), spec<2, 6, 96, 1, 4>(),
		spec<3, 4, 256, 1, 3>(), spec<3, 5, 256, 1>(), spec<3, 5, 256, 1, 3>(), spec<3, 5, 512, 2>(),
		spec<3, 5, 256, 1, 1, true>(), spec<3, 5, 256, 1, 2, true>(),
		spec<3, 6, 256, 1, 2>(),
		spec<4, 5, 640, 1>(), spec<4, 6, 640, 1>(), spec_seq<4, 6, 512, 1>(),
	};
	return t;
}

} // namespace h3dg_tables
