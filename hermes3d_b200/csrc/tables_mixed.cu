// Kernel variant table (see kernel_tables.h).
#include "kernel_tables.h"

namespace h3dg_tables {

template <int CLS, int PM, int QM, int NT, int MINB>
static MixSpec mix_spec() {
	return MixSpec { CLS, &h3dg::k_assemble_fp64_mixed<PM, QM, NT, MINB>, NT, &h3dg::MixShape<PM, QM>::smem_bytes, false, 0 };
}

// classes: (orders <= 2, <= 4 points), (<= 4, <= 6), (<= 6, <= 8)
std::vector<MixSpec> &mix_table() {
	static std::vector<MixSpec> t = {
		mix_spec<0, 2, 4, 64, 8>(), mix_spec<0, 2, 4, 128, 4>(),
		mix_spec<1, 4, 6, 128, 3>(), mix_spec<1, 4, 6, 256, 1>(),
		mix_spec<2, 6, 8, 128, 2>(), mix_spec<2, 6, 8, 256, 1>(),
	};
	return t;
}

template <int CLS, int PM, int QM, int NT>
static CedSpec ced_spec() {
	return CedSpec { CLS, (PM + 1) * (PM + 1) * (PM + 1), &h3dg::k_assemble_fp64_ced<PM, QM, NT>, NT,
	                 &h3dg::CedShape<PM, QM>::smem_bytes, false, 0 };
}

// classes: (orders <= 4, <= 6 points), (<= 6, <= 8), (<= 8, <= 10)
std::vector<CedSpec> &ced_table() {
	static std::vector<CedSpec> t = { ced_spec<0, 4, 6, 256>(), ced_spec<1, 6, 8, 128>(), ced_spec<2, 8, 10, 256>() };
	return t;
}

CedScatterFn ced_scatter_fn() { return &h3dg::k_scatter_ced<kCedScatterThreads>; }

SurfFn surf_fn() { return &h3dg::k_assemble_surface<kSurfThreads>; }

NormFn norm_fn() { return &h3dg::k_norms<kNormThreads>; }
NormReduceFn norm_reduce_fn() { return &h3dg::k_norms_reduce<kNormThreads>; }

} // namespace h3dg_tables
