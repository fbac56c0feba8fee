// Stock-quadrature kernels (see kernel_tables.h).
#include "kernel_tables.h"
#include "kernels/asm_stock.cuh"

namespace h3dg_tables {

template <int P>
static KernelSpec spec() {
	return KernelSpec { P, 0, &h3dg::k_assemble_stock<P, 256>, 256, 1, h3dg::StockShape<P>::SMEM_BYTES, false };
}

std::vector<KernelSpec> &stock_table() {
	static std::vector<KernelSpec> t = { spec<1>(), spec<2>(), spec<3>() };
	return t;
}

} // namespace h3dg_tables
