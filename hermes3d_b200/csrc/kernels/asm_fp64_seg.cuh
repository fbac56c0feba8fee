// FP64 assembly with a segmented scatter (uniform orders p <= 3).
//
// Replaces the element loop of Discretization::assemble
// (src/discretization.cc:290-342) and the insert of UMFPackMatrix::update /
// insert_value and UMFPackVector::update (src/linsolver/umfpack.cc:80-152,
// 183-192) without colour sweeps or float atomics:
//
//  * element items compute the element matrices (the phases of
//    asm_fp64.cuh, same arithmetic) in element order and write them, with
//    the AsmList coefficients applied, into a ring of slots in global memory
//    that stays resident in L2: slot column b holds K[b][a] for the
//    element's rows a, then the element's load-vector entry of b;
//  * column items take a batch of CSC columns whose elements are all done,
//    bring the columns' element-matrix slices and row positions into shared
//    memory with bulk copies (cp.async.bulk, mbarrier completion), sum every
//    slot in assembly order (colour, then element: the order in which the
//    colour sweeps add, so the result is bitwise that of k_assemble_fp64) and
//    write each column of Ax, and each RHS entry, exactly once.
//
// One persistent launch; CTAs take items from a ticket counter.  An item
// waits only on items with smaller tickets (elements of the windows a column
// batch reads; column batches that still read a ring window an element item
// overwrites), which were taken by CTAs that are running, so the waits end.
// Every wait is bounded: on timeout the kernel records kErrTimeout, raises
// the abort flag that stops every CTA, and leaves.
#pragma once

#include "asm_fp64.cuh"

namespace h3dg {

struct SegArgs {
	const int32_t *kof;       // plan element -> assembly index k
	const int32_t *items;     // nitems x 4: element item (window, -1, first, end element);
	                          //             column item (ready window, first window, first, end column)
	int nitems;
	const int32_t *col;       // columns in processing order: DOF
	const int64_t *cptr;      // pair ranges of the columns
	const int32_t *pe;        // per pair: plan element
	const uint16_t *plm;      // per pair: element-local index of the column's DOF | matrix entries << 8
	const uint16_t *off;      // per pair x nl: row position of the element's row a inside the column
	const int32_t *p1n;       // per window: element items
	const int32_t *p2n;       // per ready window: column items
	unsigned *ctr;            // [0] ticket, [1] abort, [2, 2 + nwin) element items done, then column items done,
	                          // then 4 wait statistics
	int nwin;
	int ring_win;             // windows the ring holds (>= nwin: no slot is reused)
	int span;                 // max ready window - first window over the columns
	int ring_slots;           // ring_win x window elements
	double *ring;             // ring_slots x nl x CW doubles
	int colcap;               // rows of a per-warp column buffer in shared memory (longer columns: in Ax)
};

// Poll until *p >= target (relaxed loads, then one acquire fence), at most
// `limit` polls; on timeout record kErrTimeout and raise the abort flag.
// Gives up at once when another CTA has aborted.  Returns the polls that
// found the count short (0: no wait), or -1 on timeout / abort.
__device__ __forceinline__ int seg_wait(const unsigned *p, unsigned target, unsigned *abort, int *status, unsigned limit) {
	for (unsigned it = 0; it < limit; it++) {
		if (*(const volatile unsigned *) p >= target) {
			__threadfence();
			return (int) it;
		}
		if ((it & 63) == 63 && *(volatile unsigned *) abort) return -1;
		__nanosleep(64);
	}
	atomicOr(status, kErrTimeout);
	atomicExch(abort, 1u);
	return -1;
}

// Staging layout of a column batch in shared memory (host and device)
template <int NL>
struct SegStage {
	static constexpr int CW = (NL + 1 + 1) & ~1;                   // ring column: NL rows + load-vector entry, 16-byte multiple
	static constexpr int PB = NL <= 27 ? 128 : 64;                 // pairs per batch (seg_batch_pairs)
	static constexpr int CB = 32;                                  // columns per batch (kSegBatchCols)
	static constexpr int OFFD = (2 * PB * NL + 32 + 15) / 16 * 2;  // row positions (u16), 16-byte-rounded copy
	static constexpr int VALS = OFFD;                              // PB x CW ring columns
	static constexpr int BUFS = VALS + PB * CW;                    // per-warp column buffers
	static size_t doubles(int nwarps, int colcap) { return (size_t) BUFS + (size_t) nwarps * colcap; }
};

template <int P, int NQ, int NT, int EB, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_assemble_seg(KArgs args, SegArgs sg) {
	using S = SfShape<P, P, P, NQ, NQ, NQ, EB>;
	using G = SegStage<S::NL>;
	constexpr int NL = S::NL, NL2 = NL * NL, CW = G::CW;
	constexpr int NW = NT / 32;
	static_assert(NT % 32 == 0, "whole warps");
	extern __shared__ __align__(128) double sm[];
	__shared__ uint64_t bar, bar2;
	__shared__ int s_m[EB], s_l[EB];
	__shared__ int64_t s_slot[EB];                // ring offset (doubles) of the batch's elements
	__shared__ double s_cg[EB];
	__shared__ int s_item[4];
	__shared__ int64_t s_pb[G::PB];               // ring offset (doubles) of each pair's column
	__shared__ uint16_t s_plm[G::PB];
	__shared__ int s_cd[G::CB], s_clen[G::CB], s_cp[G::CB + 1];
	__shared__ int64_t s_c0[G::CB];
	double *tab = sm + S::S_TAB;
	double *Wx = sm + S::S_W, *Wy = Wx + S::WX, *Wz = Wy + S::WY;
	double *E0 = sm + S::S_E;                     // element areas, or the staging of a column batch
	uint16_t *offs = reinterpret_cast<uint16_t *>(E0);
	double *vals = E0 + G::VALS;
	const int tid = threadIdx.x, lane = tid & 31, wi = tid >> 5;
	unsigned *ticket = sg.ctr, *abort = sg.ctr + 1, *p1done = sg.ctr + 2, *p2done = sg.ctr + 2 + sg.nwin;
	unsigned *waits = sg.ctr + 2 + 2 * sg.nwin;   // element items waited / their polls, column items waited / polls
	const unsigned limit = args.wait_limit ? (args.wait_limit >> 4) + 1 : 0;   // polls of a counter wait

	if (!stage_tables(tab, args.tables, args.table_bytes, &bar, args.status, args.wait_limit)) {
		atomicExch(abort, 1u);
		return;
	}
	if (tid == 0) {
		mbar_init(&bar2, 1);
		fence_mbar_init();
	}
	sf_product_tables<S, NT>(tab, Wx, Wy, Wz);
	__syncthreads();

	const bool do_mat = args.Ax != nullptr;
	const bool do_rhs = args.rhs && args.lf;
	uint32_t ph2 = 0;
	double *colbuf = E0 + G::BUFS + (size_t) wi * sg.colcap;

	// element data of a batch, loaded ahead into registers in three levels
	// (the assembly index, then the tables it addresses, then coordinates and
	// coefficient) while the previous batch computes
	constexpr int VEL = (EB * NL + NT - 1) / NT, VX = (EB * 24 + NT - 1) / NT;
	int kc[VEL], kx[VX], vtx_n[VX], kk = 0, m_n = 0, l_n = 0, id_n = -1;
	double coef_n[VEL], x_n[VX], cg_n = 1.0;
	uint16_t s_n[VEL];
	auto pre_a = [&](int i0, int ne) {
#pragma unroll
		for (int v = 0; v < VEL; v++) {
			const int j = tid + v * NT, e = j / NL;
			kc[v] = j < EB * NL && e < ne ? sg.kof[i0 + e] : -1;
		}
#pragma unroll
		for (int v = 0; v < VX; v++) {
			const int j = tid + v * NT, e = j / 24;
			kx[v] = j < EB * 24 && e < ne ? sg.kof[i0 + e] : -1;
		}
		if (tid < EB) kk = tid < ne ? sg.kof[i0 + tid] : -1;
	};
	auto pre_b = [&]() {
#pragma unroll
		for (int v = 0; v < VEL; v++) {
			const int j = (tid + v * NT) % NL;
			coef_n[v] = kc[v] >= 0 ? args.el_coef[(int64_t) kc[v] * NL + j] : 0.0;
			s_n[v] = kc[v] >= 0 ? args.el_s[(int64_t) kc[v] * NL + j] : (uint16_t) 0;
		}
#pragma unroll
		for (int v = 0; v < VX; v++) vtx_n[v] = kx[v] >= 0 ? args.el_vtx[8 * (int64_t) kx[v] + ((tid + v * NT) % 24) / 3] : -1;
		if (tid < EB) {
			m_n = kk >= 0 ? args.el_cnt[2 * (int64_t) kk] : 0;
			l_n = kk >= 0 ? args.el_cnt[2 * (int64_t) kk + 1] : 0;
			id_n = kk >= 0 ? args.el_id[kk] : -1;
		}
	};
	auto pre_c = [&]() {
#pragma unroll
		for (int v = 0; v < VX; v++) x_n[v] = vtx_n[v] >= 0 ? args.xyz[3 * (int64_t) vtx_n[v] + ((tid + v * NT) % 24) % 3] : 0.0;
		if (tid < EB) cg_n = id_n >= 0 && args.ecoef ? args.ecoef[id_n] : 1.0;
	};

	// warp 0 schedules: lane 0 holds the next ticket, taken while the current
	// item is processed (an item never waits on a later ticket, so holding one
	// cannot block); the windows an item waits on are polled one per lane
	int next = 0;
	if (tid == 0) next = (int) atomicAdd(ticket, 1u);
	for (;;) {
		if (wi == 0) {
			int it = __shfl_sync(0xffffffffu, next, 0);
			if (*(volatile unsigned *) abort) it = sg.nitems;
			bool live = it < sg.nitems;
			int4 d = make_int4(-2, 0, 0, 0);
			if (live) {
				if (lane == 0) next = (int) atomicAdd(ticket, 1u);
				d = reinterpret_cast<const int4 *>(sg.items)[it];
				int polls = 0;
				bool ok = true;
				if (d.y < 0) {
					// element item: the column items still reading the ring window it overwrites
					if (sg.ring_win < sg.nwin && d.x >= sg.ring_win) {
						const int v1 = min(d.x - sg.ring_win + sg.span, sg.nwin - 1);
						for (int v = d.x - sg.ring_win + lane; v <= v1 && ok; v += 32) {
							const int r = seg_wait(p2done + v, (unsigned) sg.p2n[v], abort, args.status, limit);
							ok = r >= 0;
							polls += r > 0 ? r : 0;
						}
					}
				}
				else {
					// column item: every element of its windows is in the ring
					for (int w = d.y + lane; w <= d.x && ok; w += 32) {
						const int r = seg_wait(p1done + w, (unsigned) sg.p1n[w], abort, args.status, limit);
						ok = r >= 0;
						polls += r > 0 ? r : 0;
					}
				}
				live = __all_sync(0xffffffffu, ok);
				// statistics: items that had to wait, and their polls
				const int wp = __reduce_add_sync(0xffffffffu, (unsigned) polls);
				if (lane == 0 && wp > 0) {
					atomicAdd(waits + (d.y < 0 ? 0 : 2), 1u);
					atomicAdd(waits + (d.y < 0 ? 1 : 3), (unsigned) wp);
				}
			}
			if (lane == 0) {
				s_item[0] = live ? d.x : -2;
				s_item[1] = d.y;
				s_item[2] = d.z;
				s_item[3] = d.w;
			}
		}
		__syncthreads();
		if (s_item[0] == -2) break;
		const int iw = s_item[0], iu = s_item[1], ib = s_item[2], ie = s_item[3];

		if (iu < 0) {
			// ---------------------------------------------- element item
			{
				const int ne = ie - ib < EB ? ie - ib : EB;
				pre_a(ib, ne);
				pre_b();
				pre_c();
			}
			for (int i0 = ib; i0 < ie; i0 += EB) {
				const int ne = ie - i0 < EB ? ie - i0 : EB;
				const int nn = ie - i0 - EB < EB ? ie - i0 - EB : EB;     // elements of the next batch (<= 0: none)
				if (tid < EB) {
					s_m[tid] = m_n;
					s_l[tid] = l_n;
					s_cg[tid] = cg_n;
					s_slot[tid] = (int64_t) ((unsigned) (i0 + tid) % (unsigned) sg.ring_slots) * (NL * CW);
				}
#pragma unroll
				for (int v = 0; v < VX; v++) {
					const int j = tid + v * NT;
					if (j < EB * 24) E0[(j / 24) * S::E_SIZE + S::E_X + j % 24] = x_n[v];
				}
#pragma unroll
				for (int v = 0; v < VEL; v++) {
					const int j = tid + v * NT;
					if (j < EB * NL) {
						double *Eb = E0 + (j / NL) * S::E_SIZE;
						Eb[S::E_C + j % NL] = coef_n[v];
						reinterpret_cast<int *>(Eb + S::E_I)[NL + j % NL] = s_n[v];
					}
				}
				if (nn > 0) pre_a(i0 + EB, nn);
				__syncthreads();
				sf_monomials<S, NT, EB>(E0);
				__syncthreads();
				if (nn > 0) pre_b();
				sf_geometry<S, NT, EB>(tab, E0, s_cg, args.lf, args.lf_value);
				__syncthreads();
				if (do_rhs) sf_load_vector<S, NT, EB>(tab, E0);
				sf_stage1<S, NT, EB>(E0, Wz, args.mass);
				__syncthreads();
				if (nn > 0) pre_c();
				sf_stage23<S, NT, EB>(E0, Wx, Wy);
				__syncthreads();
				// element matrix (AsmList order, coefficients applied) and load vector into the ring
				if (do_mat) {
					for (int p = tid; p < EB * NL2; p += NT) {
						const int e = p / NL2, pp = p % NL2, b = pp / NL, a = pp % NL;
						const int m = s_m[e];
						if (e < ne && a < m && b < m) {
							const double *Eb = E0 + e * S::E_SIZE;
							const int *ei = reinterpret_cast<const int *>(Eb + S::E_I);
							const int sa = ei[NL + a], sb = ei[NL + b];
							const double *A = Eb + S::E_A;
							const double val = Eb[S::E_C + a] * Eb[S::E_C + b] * (A[sa * NL + sb] + A[sb * NL + sa]);
							sg.ring[s_slot[e] + b * CW + a] = val;
						}
					}
				}
				if (do_rhs) {
					for (int i = tid; i < EB * NL; i += NT) {
						const int e = i / NL, a = i % NL;
						if (e >= ne || a >= s_m[e]) continue;
						const double *Eb = E0 + e * S::E_SIZE;
						const int *ei = reinterpret_cast<const int *>(Eb + S::E_I);
						const double *A = Eb + S::E_A;
						const int sa = ei[NL + a];
						const double ca = Eb[S::E_C + a];
						double lr = 0.0;
						for (int j = s_m[e]; j < s_m[e] + (do_mat ? s_l[e] : 0); j++) {      // lifting only with the matrix (src/discretization.cc:296-317)
							const int sj = ei[NL + j];
							lr -= ca * Eb[S::E_C + j] * (A[sa * NL + sj] + A[sj * NL + sa]);
						}
						lr += Eb[S::E_F + sa] * ca;
						sg.ring[s_slot[e] + a * CW + NL] = lr;
					}
				}
				__syncthreads();
			}
			// publish: the ring writes of every thread, then the count (release)
			__threadfence();
			__syncthreads();
			if (tid == 0) atomicAdd(p1done + iw, 1u);
		}
		else {
			// ---------------------------------------------- column item
			const int nc = ie - ib;
			const int64_t pb = sg.cptr[ib];
			const int np = (int) (sg.cptr[ie] - pb);
			for (int t = tid; t < np; t += NT) {
				const int e = sg.pe[pb + t];
				const uint16_t lm = sg.plm[pb + t];
				s_plm[t] = lm;
				s_pb[t] = (int64_t) ((unsigned) e % (unsigned) sg.ring_slots) * (NL * CW) + (lm & 0xff) * CW;
			}
			if (tid < nc) {
				const int d = sg.col[ib + tid];
				const int64_t c0 = args.Ap[d];
				s_cd[tid] = d;
				s_c0[tid] = c0;
				s_clen[tid] = (int) (args.Ap[d + 1] - c0);
				s_cp[tid] = (int) (sg.cptr[ib + tid] - pb);
			}
			if (tid == 0) s_cp[nc] = np;
			__syncthreads();
			// bulk copies: the batch's row positions (one range, widened to 16-byte
			// boundaries) and the ring column of every pair; many small copies stay
			// in flight at once, which loads from a few warps would not
			const uintptr_t oa = reinterpret_cast<uintptr_t>(sg.off + pb * NL);
			const uintptr_t o0 = oa & ~(uintptr_t) 15, o1 = (oa + 2 * (uintptr_t) np * NL + 15) & ~(uintptr_t) 15;
			const int odelta = (int) (oa - o0) / 2;
			if (wi == 0) {
				// the ring was written through the generic proxy and is read by bulk
				// copies (async proxy) after the acquire of its counters
				asm volatile("fence.proxy.async.global;" ::: "memory");
				if (lane == 0) mbar_arrive_expect_tx(&bar2, (uint32_t) ((do_mat ? o1 - o0 : 0) + (size_t) np * CW * 8));
				__syncwarp();
				if (lane == 0 && do_mat) bulk_g2s(offs, reinterpret_cast<const void *>(o0), (uint32_t) (o1 - o0), &bar2);
				for (int t = lane; t < np; t += 32) bulk_g2s(vals + t * CW, sg.ring + s_pb[t], CW * 8, &bar2);
			}
			bool ok = mbar_wait_bounded(&bar2, ph2, args.status, args.wait_limit);
			if (!ok) mbar_wait_bounded(&bar2, ph2, nullptr, 1u << 26);   // no copy left in flight
			ph2 ^= 1;
			if (__syncthreads_or(ok ? 0 : 1)) {
				if (tid == 0) atomicExch(abort, 1u);
				break;
			}
			// every column: its slots summed in pair order, the pairs' loads hoisted
			// into registers in groups of PG (the adds of a group stay ordered)
			constexpr int PG = 8, RA = (NL + 31) / 32;
			for (int jc = wi; jc < nc; jc += NW) {
				const int t0 = s_cp[jc], t1 = s_cp[jc + 1];
				const int len = s_clen[jc];
				if (do_mat && len > 0) {
					double *buf = len <= sg.colcap ? colbuf : args.Ax + s_c0[jc];
					for (int r = lane; r < len; r += 32) buf[r] = 0.0;
					__syncwarp();
					for (int tg = t0; tg < t1; tg += PG) {
						int o[PG][RA];
						double v[PG][RA];
#pragma unroll
						for (int g = 0; g < PG; g++) {
							const int m = tg + g < t1 ? s_plm[tg + g] >> 8 : 0;
#pragma unroll
							for (int r = 0; r < RA; r++) {
								const int a = lane + 32 * r;
								o[g][r] = a < m ? offs[odelta + (tg + g) * NL + a] : -1;
								v[g][r] = a < m ? vals[(tg + g) * CW + a] : 0.0;
							}
						}
#pragma unroll
						for (int g = 0; g < PG; g++) {
							if (tg + g >= t1) break;
#pragma unroll
							for (int r = 0; r < RA; r++)
								if (o[g][r] >= 0) {
									if (o[g][r] < len) buf[o[g][r]] += v[g][r];
									else atomicOr(args.status, kErrBounds);
								}
							__syncwarp();
						}
					}
					if (len <= sg.colcap) {
						double *dst = args.Ax + s_c0[jc];
						for (int r = lane; r < len; r += 32) __stcs(dst + r, buf[r]);
					}
					__syncwarp();
				}
				if (do_rhs) {
					// load-vector entries of the pairs, summed in pair order by every lane
					double racc = 0.0;
					for (int tg = t0; tg < t1; tg += 32) {
						const double mine = tg + lane < t1 ? vals[(tg + lane) * CW + NL] : 0.0;
						const int ng = t1 - tg < 32 ? t1 - tg : 32;
						for (int g = 0; g < ng; g++) racc += __shfl_sync(0xffffffffu, mine, g);
					}
					if (lane == 0) args.rhs[s_cd[jc]] = racc;
				}
			}
			__syncthreads();
			if (tid == 0) atomicAdd(p2done + iw, 1u);   // the ring reads ended with the bulk copies
		}
	}
}

} // namespace h3dg
