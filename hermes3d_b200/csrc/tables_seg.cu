// Segmented-scatter kernel variants (see kernel_tables.h).
#include "kernel_tables.h"

namespace h3dg_tables {

template <int P, int NQ, int NT, int EB, int MINB, int PER_ITEM>
static SegSpec spec() {
	struct Sz {
		static size_t smem(int colcap) {
			using S = h3dg::SfShape<P, P, P, NQ, NQ, NQ, EB>;
			using G = h3dg::SegStage<S::NL>;
			const size_t el = (size_t) EB * S::E_SIZE, stage = G::doubles(NT / 32, colcap);
			return sizeof(double) * ((size_t) S::S_E + (el > stage ? el : stage));
		}
	};
	return SegSpec { P, NQ, &h3dg::k_assemble_seg<P, NQ, NT, EB, MINB>, NT, EB, PER_ITEM, &Sz::smem, false, 0 };
}

std::vector<SegSpec> &seg_table() {
	static std::vector<SegSpec> t = {
		spec<1, 2, 64, 4, 8, 16>(), spec<1, 3, 64, 4, 8, 16>(),
		spec<2, 3, 96, 1, 8, 4>(),
		spec<2, 4, 96, 1, 4, 2>(), spec<2, 4, 96, 1, 4, 4>(), spec<2, 4, 96, 1, 4, 8>(),
		spec<2, 5, 96, 1, 8, 4>(),
		spec<3, 4, 256, 1, 3, 1>(), spec<3, 5, 256, 1, 2, 1>(), spec<3, 5, 256, 1, 3, 1>(),
		spec<3, 6, 256, 1, 2, 1>(),
	};
	return t;
}

} // namespace h3dg_tables
