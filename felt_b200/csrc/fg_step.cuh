// The whole global update of every surface of a pool as ONE persistent launch.
//
// Surface::update(fn) (include/Felt/Surface.hpp:254-296, update_end_global 739-762) is a chain
// of dependent global phases: the resets of update_start, the delta track_children copy, the
// speed functor over the zero layer, update_zero_layer, 2L distance passes of two sub-passes
// each, the status-change flush, the band expansion and the brick retirement, then the same
// passes again over the changed nodes until no layer changes. Launched one kernel per phase a
// step is ~100 dependent launches. Here the kernel bodies of fg_kernels.cuh run as the phases of
// one cooperative launch whose blocks are all resident: a grid-wide barrier separates phases
// that depend on each other, single-block steps (entry-offset scans) run on block 0 while the
// rest wait at the next barrier, and the convergence loop runs on the device. The phases, their
// order and what each does are exactly those of the multi-launch path, so every list, order and
// value is the same.
//
// Every wait is bounded: a barrier that has not completed after `wait_ns` records EB_TIMEOUT
// (FG_ERR_TIMEOUT on the host) and the kernel returns; the entry barrier comes before any work,
// so a launch that cannot gather its blocks changes nothing.
#pragma once

#include "fg_kernels.cuh"

namespace fg {

struct StepArgs {
	const Speed* speeds;       // [S] builtin speeds (device)
	unsigned* bar;             // [2] grid barrier: arrivals, generation (zero before the launch)
	int* out;                  // [4] iterations run, final buffer, surfaces stopped, 0
	int* newfrozen;            // [S] set for a surface stopped by this launch
	unsigned long long* acc;   // node-update accumulator
	unsigned long long wait_ns;  // bound of every barrier wait
	int stall;                 // check of the bounded wait: the entry barrier expects one block
	                           // more than the launch has, so it can never complete
	int do_begin, do_delta, do_finish;  // parts of the update to run (see k_update_step)
	int clear_status, clear_buf0, clear_buf1;  // resets of update_start that are due
	int delta_smem;            // speed functor over a staged brick + halo (curvature speeds)
	int block_passes;          // a block (else a warp) per partition entry in record passes
	int flush_smem;            // flush with staged removal windows (else one thread per brick)
	int split;                 // warps per partition entry in the first distance pass
	int max_iters;             // convergence iterations after which changing surfaces stop
};

static __device__ __forceinline__ unsigned long long globaltimer_ns()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

static __device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
	unsigned v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

/// Grid-wide barrier of the resident blocks of a cooperative launch (arrival counter and
/// generation in bar[0..1]; the last block to arrive resets the counter and bumps the
/// generation). Writes before it are visible to every block after it. Returns false when the
/// wait gave up after wait_ns (EB_TIMEOUT set) or another block gave up before.
static __device__ __noinline__ bool grid_sync(unsigned* bar, unsigned expected, unsigned& gen,
                                              int* err, unsigned long long wait_ns)
{
	__shared__ int ok_s;
	__syncthreads();
	if (threadIdx.x == 0) {
		int ok = 1;
		__threadfence();
		const unsigned g = gen;
		const unsigned arrived = atomicAdd(&bar[0], 1u) + 1u;
		if (arrived == expected) {
			atomicExch(&bar[0], 0u);
			__threadfence();
			atomicExch(&bar[1], g + 1u);
		} else {
			const unsigned long long t0 = globaltimer_ns();
			while (ld_acquire(&bar[1]) == g) {
				if (globaltimer_ns() - t0 > wait_ns) {
					atomicOr(err, EB_TIMEOUT);
					ok = 0;
					break;
				}
				__nanosleep(100);
			}
		}
		gen = g + 1u;
		__threadfence();
		if (ok && (*(volatile int*)err & EB_TIMEOUT)) ok = 0;
		ok_s = ok;
	}
	__syncthreads();
	return ok_s != 0;
}

/// Zeroes n ints with every thread of the launch.
static __device__ __forceinline__ void grid_zero(int* p, int n, GridPos G)
{
	for (int i = G.bid * blockDim.x + threadIdx.x; i < n; i += G.nb * blockDim.x) p[i] = 0;
}

#define FG_SYNC()                                                                  \
	do {                                                                           \
		if (!grid_sync(A.bar, expect, gen, P.err, A.wait_ns)) return;              \
	} while (0)

/// The 2L layer passes of update_distance (Surface.hpp:989-1125) over the lists of lv,
/// recording status changes into buffer b; `ca` is a compaction still due from the pass before
/// (it rides on the first pass, as in the multi-launch path). Returns false if a barrier gave
/// up.
template <int D, int L>
__device__ bool step_distance(const Dev& P, const StepArgs& A, ListView lv, int b, CompactArgs ca,
                              GridPos G, unsigned expect, unsigned& gen)
{
	constexpr int NL = 2 * L + 1;
	if (G.bid == 0) d_scan_layers(lv.pcnt, NL, P.S, P.woffl, P.sfrozen);
	if (!grid_sync(A.bar, expect, gen, P.err, A.wait_ns)) return false;
	for (int i = 0; i < 2 * L; i++) {
		const int k = i < L ? -(i + 1) : i - L + 1;
		const float side = k < 0 ? -1.0f : 1.0f;
		const int* woff = P.woffl + (size_t)(k + L) * (P.S + 1);
		d_dist1<D, L>(P, woff, lv, k, side, A.split, ca, G);
		if (!grid_sync(A.bar, expect, gen, P.err, A.wait_ns)) return false;
		if (A.block_passes)
			d_dist2<D, L>(P, woff, lv, k, b, G);
		else
			d_dist2_warp<D, L>(P, woff, lv, k, b, G);
		if (!grid_sync(A.bar, expect, gen, P.err, A.wait_ns)) return false;
		ca = CompactArgs{P.S, woff, lv.plist, k + L, b};
	}
	for (int s = G.bid; s < ca.nblocks; s += G.nb) {
		compact_surface<L>(P, ca, s);
		__syncthreads();
	}
	return grid_sync(A.bar, expect, gen, P.err, A.wait_ns);
}

/// flush_status_change, expand_narrow_band and the retirement of bricks whose partitions left
/// the band (Surface.hpp:1183-1355).
template <int D, int L>
__device__ bool step_flush_expand(const Dev& P, const StepArgs& A, unsigned char* dsm, GridPos G,
                                  unsigned expect, unsigned& gen)
{
	constexpr int NL = 2 * L + 1;
	auto sync = [&] { return grid_sync(A.bar, expect, gen, P.err, A.wait_ns); };
	if (A.flush_smem)
		d_flush_smem<D, L>(P, G, dsm);
	else
		d_flush_leaf<D, L>(P, G);
	if (!sync()) return false;
	d_flush_plist<L>(P, G);
	if (!sync()) return false;
	if (G.bid == 0) {
		d_scan_counts(P.spcnt, NL, 0, 1, P.S, P.woff, P.sfrozen);
		if (threadIdx.x == 0) {
			P.counters[CNT_ACT] = 0;
			P.counters[CNT_TOUCH] = 0;
			P.counters[CNT_CAND] = 0;
		}
	}
	if (!sync()) return false;
	d_expand_gen<D, L>(P, 0, G);
	if (!sync()) return false;
	d_activate<L>(P, G);
	if (!sync()) return false;
	d_expand_gen<D, L>(P, 1, G);
	if (!sync()) return false;
	d_expand_gen<D, L>(P, 2, G);
	if (!sync()) return false;
	d_expand_append<L>(P, G, reinterpret_cast<unsigned long long*>(dsm));
	if (!sync()) return false;
	d_expand_plist<L>(P, G);
	if (!sync()) return false;
	d_retire(P, G);
	if (!sync()) return false;
	if (G.bid == 0 && threadIdx.x == 0) P.counters[CNT_RETIRE] = 0;
	return true;
}

/// The global update as one launch. do_begin: update_start's due resets, the delta
/// track_children copy, the band count and the zero layer's entry offsets
/// (Surface.hpp:257-263, 393-399). do_delta: the builtin speed functor over the zero layer
/// (Surface.hpp:263-294). do_finish: update_end_global (Surface.hpp:739-762): the zero-layer
/// update, the distance passes, flush, expansion and retirement, then the convergence loop,
/// stopping the surfaces still changing after every max_iters iterations.
template <int D, int L>
__global__ void __launch_bounds__(256) k_update_step(Dev P, StepArgs A)
{
	constexpr int NL = 2 * L + 1;
	constexpr int B = 1, Abuf = 0;  // affected buffers: B = the buffer the first passes record
	extern __shared__ __align__(16) unsigned char dsm[];
	const GridPos G = hw_grid();
	const bool lead = G.bid == 0;
	unsigned gen = 0;
	const unsigned expect = gridDim.x + (A.stall ? 1u : 0u);
	FG_SYNC();  // every block resident before any work
	if (A.do_begin) {
		if (A.clear_status) {
			d_clear_status<L>(P, G);
			FG_SYNC();
			grid_zero(P.spcnt, P.S * NL, G);
			if (lead && threadIdx.x == 0) P.counters[CNT_SUNION] = 0;
			FG_SYNC();
		}
		for (int b = 0; b < 2; b++) {
			if (!(b ? A.clear_buf1 : A.clear_buf0)) continue;
			if (lead) d_scan_counts(P.apcnt[b], NL, 0, 2, P.S, P.woff, P.sfrozen);
			FG_SYNC();
			d_clear_buffer<L>(P, b, G);
			FG_SYNC();
			grid_zero(P.apcnt[b], P.S * NL, G);
			FG_SYNC();
		}
		d_copy_plists(P, NL, G);
		if (lead) d_scan_counts(P.pcnt, NL, 0, 2, P.S, P.woff, P.sfrozen);
		FG_SYNC();
		d_band_size<L>(P, A.acc, G);
		FG_SYNC();
		if (lead) d_scan_counts(P.pcnt, NL, L, 0, P.S, P.woff, P.sfrozen);
		FG_SYNC();
	}
	if (A.do_delta) {
		if (A.delta_smem)
			d_delta_smem<D, L>(P, A.speeds, G, reinterpret_cast<float*>(dsm));
		else
			d_delta_builtin<D, L>(P, A.speeds, G);
		FG_SYNC();
	}
	if (!A.do_finish) return;
	if (lead) {
		d_scan_counts(P.pcnt, NL, L, 0, P.S, P.woff, P.sfrozen);
		if (threadIdx.x == 0) *P.changed = 0;
	}
	FG_SYNC();
	const ListView iso{P.plist, P.pcnt, P.lst, P.lcnt};
	if (A.block_passes)
		d_zero_apply<D, L>(P, iso, nullptr, B, G);
	else
		d_zero_apply_warp<D, L>(P, iso, nullptr, B, G);
	FG_SYNC();
	if (!step_distance<D, L>(P, A, iso, B, CompactArgs{P.S, P.woff, P.plist, L, B}, G, expect, gen))
		return;
	if (!step_flush_expand<D, L>(P, A, dsm, G, expect, gen)) return;
	int cur = B, oth = Abuf, iters = 1, stopped = 0;
	FG_SYNC();
	int changed = *(volatile int*)P.changed;
	while (changed) {
		// one iteration after the first: the passes over the nodes that changed (buffer cur),
		// recording into buffer oth, then flush, expansion, and the reset of buffer cur
		d_clear_status<L>(P, G);
		FG_SYNC();
		grid_zero(P.spcnt, P.S * NL, G);
		if (lead && threadIdx.x == 0) {
			P.counters[CNT_SUNION] = 0;
			*P.changed = 0;
		}
		FG_SYNC();
		const ListView bv{P.aplist[cur], P.apcnt[cur], P.alst[cur], P.acnt[cur]};
		if (!step_distance<D, L>(P, A, bv, oth, CompactArgs{0, nullptr, nullptr, 0, 0}, G, expect,
		                         gen))
			return;
		if (!step_flush_expand<D, L>(P, A, dsm, G, expect, gen)) return;
		if (lead) d_scan_counts(P.apcnt[cur], NL, 0, 2, P.S, P.woff, P.sfrozen);
		FG_SYNC();
		d_clear_buffer<L>(P, cur, G);
		FG_SYNC();
		grid_zero(P.apcnt[cur], P.S * NL, G);
		const int t = cur;
		cur = oth;
		oth = t;
		iters++;
		FG_SYNC();
		changed = *(volatile int*)P.changed;
		if (changed && iters % A.max_iters == 0) {
			// the surfaces still changing stop here (their buffer cur is not empty): the
			// reference's loop has no bound and would cycle for ever on them
			for (int s = G.bid * blockDim.x + threadIdx.x; s < P.S; s += G.nb * blockDim.x) {
				if (P.sfrozen[s]) continue;
				int tot = 0;
				for (int l = 0; l < NL; l++) tot += P.apcnt[cur][s * NL + l];
				if (tot) {
					P.sfrozen[s] = 1;
					A.newfrozen[s] = 1;
				}
			}
			stopped = 1;
			FG_SYNC();
		}
	}
	if (lead && threadIdx.x == 0) {
		A.out[0] = iters;
		A.out[1] = cur;
		A.out[2] = stopped;
	}
}

#undef FG_SYNC

}  // namespace fg
