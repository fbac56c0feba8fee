// Kernel variant tables.  Each table lives in its own translation unit so
// the template instantiations compile in parallel; the dispatcher in
// h3dg_capi.cu only sees function pointers, launch shapes and shared-memory
// sizes.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "kernels/common.cuh"
#include "kernels/asm_fp64_ho.cuh"
#include "kernels/adjoint.cuh"
#include "kernels/asm_fp64_mixed.cuh"
#include "kernels/asm_fp64_ced.cuh"
#include "kernels/asm_surface.cuh"
#include "kernels/norms.cuh"
#include "kernels/asm_fp64_seg.cuh"

namespace h3dg_tables {

using KernelFn = void (*)(h3dg::KArgs, int64_t, int64_t);

struct KernelSpec {
	int p, nq;
	KernelFn fn;
	int threads, eb;
	size_t smem;
	bool configured;
};

using HoFn = void (*)(h3dg::KArgsHO, int64_t, int64_t);

struct HoSpec {
	int p, nq;
	HoFn fn;
	int threads;
	size_t smem;
	bool configured;
};

// FP64 tensor-core (DMMA) high-order kernels and the builders of their scatter streams
using OffdFn = void (*)(const uint16_t *, const int32_t *, const int64_t *, int64_t, int64_t, uint16_t *, int *, uint8_t *,
                        unsigned long long *);

struct DmSpec {
	int p, nq;
	HoFn fn;
	int threads;
	size_t smem;
	bool configured;
	size_t epe;                   // scatter-stream entries per element
	OffdFn build;
};

using AdjFn = void (*)(h3dg::AdjArgs);

struct AdjSpec {
	int p, nq;
	AdjFn fn;
	size_t smem;
	bool configured;
};

using MixFn = void (*)(h3dg::KArgsMixed, int64_t, int64_t, int);

struct MixSpec {
	int cls;                      // kernel class (Plan::kClassP / kClassQ)
	MixFn fn;
	int threads;
	size_t (*smem)(int table_bytes);
	bool configured;
	size_t configured_smem;
};

// FP64 low-order kernels (register / shared-memory element matrix); the
// autotuner times each candidate for an (order, points) pair on the actual
// plan at the first assembly and keeps the fastest.
std::vector<KernelSpec> &kernel_table();
// FP64 high-order kernels (element matrix never materialised)
std::vector<HoSpec> &ho_table();
// FP64 high-order kernels with stages 2 and 3 on the FP64 tensor cores
std::vector<DmSpec> &dm_table();
// their scatter stream, colour by colour with first-touch store flags (async on st)
cudaError_t build_offd(const DmSpec &k, const uint16_t *offc, const int32_t *cdof, const int64_t *Ap, int64_t ne,
                       const int64_t *color_ptr, int ncolors, int64_t nnz, uint16_t **offd, size_t *count,
                       unsigned long long *stores, int *status, cudaStream_t st);
// split-precision high-order kernels (tcgen05 3xTF32 stage 3)
std::vector<HoSpec> &ho_tc_table();
// FP64-accurate high-order kernels (int8-sliced tcgen05 stage 3)
std::vector<HoSpec> &ho_oz_table();
// tensor-core scatter stream from the canonical position map (async on st)
// (colour by colour, with first-touch store flags; *stores = the number of flagged entries)
cudaError_t build_offt(const uint16_t *offc, const int32_t *cdof, const int64_t *Ap, int64_t ne, int px, int nq,
                       const int64_t *color_ptr, int ncolors, int64_t nnz, uint16_t **offt, size_t *count,
                       unsigned long long *stores, int *status, cudaStream_t st);
// mixed-order kernels, several variants per class (timed once per plan)
std::vector<MixSpec> &mix_table();
// adjoint (element sensitivity) kernels
std::vector<AdjSpec> &adj_table();

using CedFn = void (*)(h3dg::KArgsCed, int64_t, int64_t, int);

struct CedSpec {
	int cls;                      // Plan::kCedClassP / kCedClassQ
	int nlm;                      // largest canonical basis of the class
	CedFn fn;
	int threads;
	size_t (*smem)(int table_bytes);
	bool configured;
	size_t configured_smem;
};

// elements with constrained (hanging) nodes, one kernel per class, and the
// scatter of their entries
std::vector<CedSpec> &ced_table();
using CedScatterFn = void (*)(h3dg::KArgsCed, int64_t, int64_t);
CedScatterFn ced_scatter_fn();
constexpr int kCedScatterThreads = 256;

// surface forms on natural boundary faces
using SurfFn = void (*)(h3dg::KArgsSurf, int64_t, int64_t);
SurfFn surf_fn();
constexpr int kSurfThreads = 128;

// norms of a finite-element function (per element, then a fixed-order reduction)
using NormFn = void (*)(h3dg::KArgsNorm, int64_t, int, int, int);
using NormReduceFn = void (*)(const double *, int64_t, double *);
NormFn norm_fn();
NormReduceFn norm_reduce_fn();
constexpr int kNormThreads = 128;



// segmented-scatter FP64 kernels (uniform orders p <= 3): one persistent
// launch per assembly
using SegFn = void (*)(h3dg::KArgs, h3dg::SegArgs);

struct SegSpec {
	int p, nq;
	SegFn fn;
	int threads, eb;
	int per_item;                 // elements per element item
	size_t (*smem)(int colcap);
	bool configured;
	size_t configured_smem;
};
std::vector<SegSpec> &seg_table();

// split-precision (3xTF32) low-order kernels, elements batched on the tensor
// cores (one launch per colour, one CTA per SM; KernelSpec::eb = elements per batch)
std::vector<KernelSpec> &lo_tc_table();

// FP64 kernels with the reference's stock per-pair quadrature (uniform p <= 3;
// KernelSpec::nq unused)
std::vector<KernelSpec> &stock_table();

} // namespace h3dg_tables
