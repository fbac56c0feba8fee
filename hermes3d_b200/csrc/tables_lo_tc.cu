// Batched split-precision low-order kernels (see kernel_tables.h).
#include "kernel_tables.h"
#include "kernels/asm_lo_tc.cuh"

namespace h3dg_tables {

template <int P, int NQ>
static KernelSpec spec() {
	return KernelSpec { P, NQ, &h3dg::k_assemble_lo_tc<P, NQ, 256>, 256, h3dg::LoTcShape<P, NQ>::EBT,
	                    h3dg::LoTcShape<P, NQ>::SMEM_BYTES, false };
}

std::vector<KernelSpec> &lo_tc_table() {
	static std::vector<KernelSpec> t = { spec<1, 2>(), spec<1, 3>(), spec<2, 3>(), spec<2, 4>() };
	return t;
}

} // namespace h3dg_tables
