// Kernels of one global update step, templated on dimension D and narrow-band half-width L.
//
// Work is spread as one warp per (surface, partition) list entry; every per-partition list
// operation is done by the warp that owns the partition, in lane order, so the ordered leaf
// lists come out exactly as the reference's sequential traversal builds them. Orderings across
// partitions (children lists) are rebuilt by per-surface compaction kernels in the reference's
// iteration order.
#pragma once

#include "fg_dev.cuh"

namespace fg {

constexpr unsigned FULL = 0xffffffffu;

/// A partition-list + leaf-list pair: the isogrid's own lists, or one affected buffer's.
struct ListView {
	const int* plist;
	const int* pcnt;
	const uint16_t* lst;
	const int* lcnt;
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

/// Exclusive block scan of one int per thread; returns the prefix, total in *total.
__device__ __forceinline__ int block_excl_scan(int v, int* total)
{
	__shared__ int ws[32];
	const int lane = lane_id(), w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	int x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int y = __shfl_up_sync(FULL, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) ws[w] = x;
	__syncthreads();
	if (w == 0) {
		int t = lane < nw ? ws[lane] : 0;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(FULL, t, o);
			if (lane >= o) t += y;
		}
		if (lane < nw) ws[lane] = t;
	}
	__syncthreads();
	const int before = (w > 0 ? ws[w - 1] : 0) + x - v;
	*total = ws[nw - 1];
	__syncthreads();
	return before;
}

// ---------------------------------------------------------------------------------------------
// Entry offsets: woff[s] = sum of per-surface counts before s.
// mode 0: cnt[s*NL + l]; mode 1: cnt[s*NL] + cnt[s*NL + NL-1]; mode 2: sum over layers.
// ---------------------------------------------------------------------------------------------
static __global__ void k_scan_counts(const int* cnt, int NL, int l, int mode, int S, int* woff)
{
	__shared__ int carry;
	if (threadIdx.x == 0) {
		carry = 0;
		woff[0] = 0;
	}
	__syncthreads();
	for (int base = 0; base < S; base += blockDim.x) {
		const int s = base + threadIdx.x;
		int v = 0;
		if (s < S) {
			if (mode == 0)
				v = cnt[s * NL + l];
			else if (mode == 1)
				v = cnt[s * NL] + cnt[s * NL + NL - 1];
			else
				for (int t = 0; t < NL; t++) v += cnt[s * NL + t];
		}
		int tot;
		const int ex = block_excl_scan(v, &tot);
		if (s < S) woff[s + 1] = carry + ex + v;
		__syncthreads();
		if (threadIdx.x == 0) carry += tot;
		__syncthreads();
	}
}

#define FG_WARP_LOOP(woff_)                                                         \
	const int lane = lane_id();                                                     \
	const int nwarps = (gridDim.x * blockDim.x) >> 5;                              \
	const int total = (woff_)[P.S];                                                 \
	for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < total; e += nwarps)

// ---------------------------------------------------------------------------------------------
// status_change (Surface.hpp:1138-1178) for one 32-leaf chunk of partition gp processed by a
// warp in pass `from`: records the status grid entry (list per from-layer, value = to) and
// tracks the leaf into affected buffer b under its new layer. Per-entry flags: bit 31 = the
// partition must join the status partition list of `from`; bit t = it must join the buffer's
// partition list t.
// ---------------------------------------------------------------------------------------------
template <int L>
__device__ __forceinline__ void status_chunk(const Dev& P, int gp, int sl, int from, bool valid,
                                             int leaf, int to, int b, unsigned& flags,
                                             bool& any_change)
{
	constexpr int NL = 2 * L + 1;
	const int lane = lane_id();
	const unsigned lt = (1u << lane) - 1u;
	const bool chgd = valid && to != from;
	if (__ballot_sync(FULL, chgd) == 0) return;
	any_change = true;
	const size_t bv = (size_t)P.BV;
	bool app = false;
	if (chgd) {
		const int cur = P.sto[sl * bv + leaf];
		app = cur == L + 1;
		P.sto[sl * bv + leaf] = (int8_t)to;
	}
	const unsigned ma = __ballot_sync(FULL, app);
	if (ma) {
		const int fi = from + L;
		const int base = P.ccnt[sl * NL + fi];
		if (app) P.chg[((size_t)sl * NL + fi) * bv + base + __popc(ma & lt)] = (uint16_t)leaf;
		__syncwarp();
		if (lane == 0) P.ccnt[sl * NL + fi] = base + __popc(ma);
		flags |= 0x80000000u;
	}
	const bool inb = chgd && inside_band(to, L);
	if (__ballot_sync(FULL, inb)) {
		const int t = inb ? to + L : -1;
		const unsigned grp = __match_any_sync(FULL, t);
		const bool isnew = inb && P.alkp[b][sl * bv + leaf] == NUL16;
		const unsigned mn = __ballot_sync(FULL, isnew) & grp;
		int base = 0;
		if (inb) base = P.acnt[b][sl * NL + t];
		__syncwarp();
		if (isnew) {
			const int pos = base + __popc(mn & lt);
			P.alst[b][((size_t)sl * NL + t) * bv + pos] = (uint16_t)leaf;
			P.alkp[b][sl * bv + leaf] = (uint16_t)pos;
		}
		const bool leader = inb && (__ffs(grp) - 1) == lane;
		if (leader) {
			P.acnt[b][sl * NL + t] = base + __popc(mn);
			if (P.appos[b][gp * NL + t] < 0) flags |= 1u << t;
		}
		__syncwarp();
	}
}

__device__ __forceinline__ unsigned warp_or(unsigned v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(FULL, v, o);
	return v;
}

// ---------------------------------------------------------------------------------------------
// update(fn) functor loop (Surface.hpp:263-294) with a builtin speed: delta of every zero-layer
// leaf, written to the brick's delta array.
// ---------------------------------------------------------------------------------------------
template <int D, int L>
__global__ void __launch_bounds__(256) k_delta_builtin(Dev P, const Speed* speeds)
{
	constexpr int NL = 2 * L + 1;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const Speed sp = speeds[s];
		const int gp = g.pbase + P.plist[(size_t)L * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		const int n = P.lcnt[sl * NL + L];
		const uint16_t* lst = P.lst + ((size_t)sl * NL + L) * P.BV;
		for (int j = lane; j < n; j += 32) {
			const int leaf = lst[j];
			P.dlt[(size_t)sl * P.BV + leaf] = speed_eval<D, L>(P, g, sp, leaf_pos<D>(P, gp, leaf));
		}
		if (lane == 0) atomicAdd(&P.kstat[KS_ZERO], (unsigned long long)n);
	}
}

/// update_zero_layer (Surface.hpp:920-979) over the isogrid's zero-layer lists, which the delta
/// grid mirrors in the global update.
template <int D, int L>
__global__ void __launch_bounds__(256) k_zero_apply(Dev P, int b)
{
	constexpr int NL = 2 * L + 1;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const int gp = g.pbase + P.plist[(size_t)L * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		const int n = P.lcnt[sl * NL + L];
		const uint16_t* lst = P.lst + ((size_t)sl * NL + L) * P.BV;
		unsigned flags = 0;
		bool any = false;
		for (int base = 0; base < n; base += 32) {
			const int j = base + lane;
			const bool valid = j < n;
			int leaf = 0, to = 0;
			if (valid) {
				leaf = lst[j];
				const size_t k = (size_t)sl * P.BV + leaf;
				const float nw = __fadd_rn(P.phi[k], P.dlt[k]);
				to = layer_id(nw, P.err);
				P.phi[k] = nw;
			}
			status_chunk<L>(P, gp, sl, 0, valid, leaf, to, b, flags, any);
		}
		flags = warp_or(flags);
		if (lane == 0) P.eflag[e] = flags;
	}
}

/// update_distance first pass (Surface.hpp:1028-1073): distance of every leaf of layer k to
/// the zero curve, into the delta array.
template <int D, int L>
__global__ void __launch_bounds__(256) k_dist1(Dev P, ListView lv, int k, float side)
{
	constexpr int NL = 2 * L + 1;
	const int li = k + L;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const int gp = g.pbase + lv.plist[(size_t)li * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		const int n = lv.lcnt[sl * NL + li];
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
		for (int j = lane; j < n; j += 32) {
			const int leaf = lst[j];
			const size_t kk = (size_t)sl * P.BV + leaf;
			P.dlt[kk] = distance<D, L>(P, g, leaf_pos<D>(P, gp, leaf), P.phi[kk], side);
		}
		if (lane == 0) atomicAdd(&P.kstat[KS_DIST], (unsigned long long)n);
	}
}

/// update_distance second pass (Surface.hpp:1075-1121): apply and record status changes.
template <int D, int L>
__global__ void __launch_bounds__(256) k_dist2(Dev P, ListView lv, int k, int b)
{
	constexpr int NL = 2 * L + 1;
	const int li = k + L;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const int gp = g.pbase + lv.plist[(size_t)li * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		const int n = lv.lcnt[sl * NL + li];
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
		unsigned flags = 0;
		bool any = false;
		for (int base = 0; base < n; base += 32) {
			const int j = base + lane;
			const bool valid = j < n;
			int leaf = 0, to = 0;
			if (valid) {
				leaf = lst[j];
				const size_t kk = (size_t)sl * P.BV + leaf;
				const float d = P.dlt[kk];
				to = layer_id(d, P.err);
				P.phi[kk] = d;
			}
			status_chunk<L>(P, gp, sl, k, valid, leaf, to, b, flags, any);
		}
		flags = warp_or(flags);
		if (lane == 0) {
			P.eflag[e] = flags;
			if (any) atomicOr(P.changed, 1);
		}
	}
}

/// Appends, in the pass's partition order, the partitions that gained status changes to the
/// status partition list of layer index `li`, and those newly tracked in buffer b's partition
/// lists (the children-level track_child calls of status_change, PartitionedMixin.hpp:201-213).
/// One block per surface.
template <int L>
__global__ void k_compact(Dev P, const int* plist, int li, int b)
{
	constexpr int NL = 2 * L + 1;
	const int s = blockIdx.x;
	const SurfGeom& g = P.geom[s];
	const int e0 = P.woff[s], e1 = P.woff[s + 1];
	__shared__ int cnt_s, cnt_a[NL];
	if (threadIdx.x == 0) cnt_s = P.spcnt[s * NL + li];
	if (threadIdx.x < NL) cnt_a[threadIdx.x] = P.apcnt[b][s * NL + threadIdx.x];
	__syncthreads();
	for (int base = e0; base < e1; base += blockDim.x) {
		const int e = base + threadIdx.x;
		unsigned f = 0;
		int lp = 0;
		if (e < e1) {
			f = P.eflag[e];
			lp = plist[(size_t)li * P.NP + g.pbase + (e - e0)];
		}
		const int gp = g.pbase + lp;
		int tot;
		const bool fs = (f & 0x80000000u) != 0;
		const int ps = block_excl_scan(fs ? 1 : 0, &tot);
		if (fs) {
			const int pos = cnt_s + ps;
			P.splist[(size_t)li * P.NP + g.pbase + pos] = lp;
			P.sppos[gp * NL + li] = pos;
			if (atomicExch(&P.sflag[gp], 1) == 0)
				P.q_sunion[atomicAdd(&P.counters[CNT_SUNION], 1)] = gp;
		}
		__syncthreads();
		if (threadIdx.x == 0) cnt_s += tot;
		for (int t = 0; t < NL; t++) {
			const bool ft = (f >> t) & 1u;
			int tt;
			const int pt = block_excl_scan(ft ? 1 : 0, &tt);
			if (ft) {
				const int pos = cnt_a[t] + pt;
				P.aplist[b][(size_t)t * P.NP + g.pbase + pos] = lp;
				P.appos[b][gp * NL + t] = pos;
			}
			__syncthreads();
			if (threadIdx.x == 0) cnt_a[t] += tt;
		}
		__syncthreads();
	}
	__syncthreads();
	if (threadIdx.x == 0) P.spcnt[s * NL + li] = cnt_s;
	if (threadIdx.x < NL) P.apcnt[b][s * NL + threadIdx.x] = cnt_a[threadIdx.x];
}

// ---------------------------------------------------------------------------------------------
// flush_status_change (Surface.hpp:1183-1244) with Untrack::retrack / untrack
// (PartitionedMixin.hpp:489-558), leaf level: each partition with status changes replays its
// own edits in the reference's order (from-layer ascending, status list order), one thread per
// partition, and records the children-level events for k_flush_plist.
// ---------------------------------------------------------------------------------------------
template <int D, int L>
__global__ void k_flush_leaf(Dev P)
{
	constexpr int NL = 2 * L + 1;
	const int n = P.counters[CNT_SUNION];
	for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
		const int gp = P.q_sunion[e];
		const int sl = P.slot[gp];
		const size_t bv = (size_t)P.BV;
		int cnt[NL];
		int live = 0;
		for (int l = 0; l < NL; l++) {
			cnt[l] = P.lcnt[sl * NL + l];
			live += cnt[l];
		}
		unsigned remb = 0;
		bool dead = false;
		for (int fi = 0; fi < NL; fi++) {
			unsigned appf = 0;
			const int nc = P.ccnt[sl * NL + fi];
			const uint16_t* ch = P.chg + ((size_t)sl * NL + fi) * bv;
			uint16_t* lf = P.lst + ((size_t)sl * NL + fi) * bv;
			for (int c = 0; c < nc; c++) {
				const int leaf = ch[c];
				const int to = P.sto[sl * bv + leaf];
				// LookupMixin.hpp:339-371: swap-with-last removal from list fi.
				const int pos = P.lkp[sl * bv + leaf];
				const int last = cnt[fi] - 1;
				if (pos < last) {
					const int moved = lf[last];
					lf[pos] = (uint16_t)moved;
					P.lkp[sl * bv + moved] = (uint16_t)pos;
				}
				P.lkp[sl * bv + leaf] = NUL16;
				cnt[fi] = last;
				if (inside_band(to, L)) {
					const int ti = to + L;
					uint16_t* lt = P.lst + ((size_t)sl * NL + ti) * bv;
					lt[cnt[ti]] = (uint16_t)leaf;
					P.lkp[sl * bv + leaf] = (uint16_t)cnt[ti];
					if (cnt[ti] == 0) appf |= 1u << ti;
					cnt[ti]++;
					if (last == 0) remb |= 1u << fi;
				} else {
					P.phi[sl * bv + leaf] = (float)to;
					live--;
					if (last == 0) {
						remb |= 1u << fi;
						if (live == 0) {
							P.bg[gp] = (float)to;
							dead = true;
						}
					}
				}
			}
			P.app[gp * NL + fi] = appf;
		}
		for (int l = 0; l < NL; l++) P.lcnt[sl * NL + l] = cnt[l];
		P.rem[gp] = remb;
		{
			int edits = 0;
			for (int fi = 0; fi < NL; fi++) edits += P.ccnt[sl * NL + fi];
			atomicAdd(&P.kstat[KS_FLUSH], (unsigned long long)edits);
		}
		if (dead) {
			P.oslot[gp] = sl;
			P.slot[gp] = -1;
			P.q_retire[atomicAdd(&P.counters[CNT_RETIRE], 1)] = sl;
		}
	}
}

/// Children-level half of the flush: one warp per (surface, list k) replays, in the reference's
/// order (from-layer ascending, then status partition list order), the appends to list k and
/// the swap-with-last removals from it (LookupMixin.hpp:483-556).
template <int L>
__global__ void k_flush_plist(Dev P)
{
	constexpr int NL = 2 * L + 1;
	const int lane = lane_id();
	const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (w >= P.S * NL) return;
	const int s = w / NL, k = w % NL;
	const SurfGeom& g = P.geom[s];
	int* pl = P.plist + (size_t)k * P.NP + g.pbase;
	int cnt = P.pcnt[s * NL + k];
	for (int fi = 0; fi < NL; fi++) {
		const int ns = P.spcnt[s * NL + fi];
		const int* sp = P.splist + (size_t)fi * P.NP + g.pbase;
		for (int base = 0; base < ns; base += 32) {
			const int i = base + lane;
			int lp = 0, ev = 0;
			if (i < ns) {
				lp = sp[i];
				const int gp = g.pbase + lp;
				if (fi == k)
					ev = ((P.rem[gp] >> k) & 1u) ? 2 : 0;
				else
					ev = ((P.app[gp * NL + fi] >> k) & 1u) ? 1 : 0;
			}
			unsigned m = __ballot_sync(FULL, ev != 0);
			while (m) {
				const int src = __ffs(m) - 1;
				m &= m - 1;
				const int lps = __shfl_sync(FULL, lp, src);
				const int evs = __shfl_sync(FULL, ev, src);
				if (lane == 0) {
					const int gp = g.pbase + lps;
					int* at = &P.ppos[gp * NL + k];
					if (evs == 1) {
						if (*at < 0) {
							pl[cnt] = lps;
							*at = cnt;
							cnt++;
						}
					} else if (*at >= 0) {
						const int last = cnt - 1;
						if (*at < last) {
							const int mv = pl[last];
							pl[*at] = mv;
							P.ppos[(g.pbase + mv) * NL + k] = *at;
						}
						*at = -1;
						cnt = last;
					}
				}
				__syncwarp();
			}
		}
	}
	if (lane == 0) P.pcnt[s * NL + k] = cnt;
}

// ---------------------------------------------------------------------------------------------
// expand_narrow_band (Surface.hpp:1249-1355). The sequential reference walks the status lists
// of layers -L then +L (partition list order, leaf list order, neighbour order) and tracks each
// out-of-band in-grid neighbour into the outermost layer on first encounter. Here every
// (source, neighbour) candidate gets a key in that order; the smallest key claims the node.
// A claimed node's distance only depends on neighbours already in the band (the band is
// consistent, so a newly added node never undercuts the source that adds it), so all values
// are computed from the post-flush state. Modes: 0 mark partitions to activate, 1 claim,
// 2 compute the winners' distances into the delta array.
// ---------------------------------------------------------------------------------------------
template <int D, int L>
__global__ void __launch_bounds__(256) k_expand_gen(Dev P, int mode)
{
	constexpr int NL = 2 * L + 1;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const int i = e - P.woff[s];
		const int n0 = P.spcnt[s * NL];
		const int phase = i < n0 ? 0 : 1;
		const int rank = phase ? i - n0 : i;
		const int fi = phase ? NL - 1 : 0;
		const int gp = g.pbase + P.splist[(size_t)fi * P.NP + g.pbase + rank];
		const int sl = P.slot[gp] >= 0 ? P.slot[gp] : P.oslot[gp];
		const int side = phase ? 1 : -1;
		const int want = L * side - side;
		const int nc = P.ccnt[sl * NL + fi];
		const uint16_t* ch = P.chg + ((size_t)sl * NL + fi) * P.BV;
		for (int c = lane; c < nc; c += 32) {
			const int leaf = ch[c];
			if (P.sto[(size_t)sl * P.BV + leaf] != want) continue;
			const Vec<D> pos = leaf_pos<D>(P, gp, leaf);
#pragma unroll
			for (int nb = 0; nb < 2 * D; nb++) {
				Vec<D> q = pos;
				q[nb >> 1] += (nb & 1) ? 1 : -1;
				if (!in_grid<D>(g, q)) continue;
				const float v = get_phi<D, L>(P, g, q);
				if (inside_band(layer_id(v, P.err), L)) continue;
				int gpn, leafn;
				locate<D>(P, g, q, gpn, leafn);
				// key: phase (1 bit) | rank (24) | position in status list (16) | neighbour (3)
				const unsigned long long key = ((unsigned long long)phase << 43) |
				                               ((unsigned long long)rank << 19) |
				                               ((unsigned long long)c << 3) | (unsigned long long)nb;
				if (mode == 0) {
					if (P.slot[gpn] < 0 && atomicExch(&P.actflag[gpn], 1) == 0)
						P.q_act[atomicAdd(&P.counters[CNT_ACT], 1)] = gpn;
				} else {
					const int sn = P.slot[gpn];
					if (sn < 0) {
						atomicOr(P.err, EB_POOL);
						continue;
					}
					unsigned long long* cl = &P.claim[(size_t)sn * P.BV + leafn];
					if (mode == 1) {
						atomicMin(cl, key);
						if (atomicExch(&P.touched[sn], 1) == 0)
							P.q_touch[atomicAdd(&P.counters[CNT_TOUCH], 1)] = sn;
					} else if (*cl == key) {
						P.dlt[(size_t)sn * P.BV + leafn] = distance<D, L>(P, g, q, v, (float)side);
					}
				}
			}
		}
	}
}

/// Reset a brick to an activated, empty partition: values = background, no lists.
template <int L>
__device__ void brick_init(const Dev& P, int sl, float bgv, int tid, int nth)
{
	constexpr int NL = 2 * L + 1;
	const size_t base = (size_t)sl * P.BV;
	for (int i = tid; i < P.BV; i += nth) {
		P.phi[base + i] = bgv;
		P.lkp[base + i] = NUL16;
		P.sto[base + i] = (int8_t)(L + 1);
		P.alkp[0][base + i] = NUL16;
		P.alkp[1][base + i] = NUL16;
		P.claim[base + i] = NOCLAIM;
	}
	for (int i = tid; i < NL; i += nth) {
		P.lcnt[sl * NL + i] = 0;
		P.ccnt[sl * NL + i] = 0;
		P.acnt[0][sl * NL + i] = 0;
		P.acnt[1][sl * NL + i] = 0;
	}
}

/// Child activation (TrackedMixin.hpp:37-41) of queued partitions: one block per partition.
template <int L>
__global__ void k_activate(Dev P)
{
	__shared__ int sl;
	const int n = P.counters[CNT_ACT];
	for (int q = blockIdx.x; q < n; q += gridDim.x) {
		const int gp = P.q_act[q];
		if (threadIdx.x == 0) {
			const int t = atomicSub(&P.counters[CNT_FREE_TOP], 1) - 1;
			if (t < 0) {
				atomicAdd(&P.counters[CNT_FREE_TOP], 1);
				atomicOr(P.err, EB_POOL);
				sl = -1;
			} else {
				sl = P.free_stack[t];
			}
		}
		__syncthreads();
		const int my = sl;
		if (my >= 0) {
			brick_init<L>(P, my, P.bg[gp], threadIdx.x, blockDim.x);
			if (threadIdx.x == 0) {
				P.slot_gp[my] = gp;
				P.touched[my] = 0;
			}
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			if (my >= 0) P.slot[gp] = my;
			P.actflag[gp] = 0;
		}
		__syncthreads();
	}
}

/// Appends each touched brick's claimed nodes to its outermost lists in claim-key order (the
/// reference's sequential track order) and records the partition's first key per side for the
/// children-level append. One block per touched brick; keys sorted in shared memory.
template <int L>
__global__ void k_expand_append(Dev P)
{
	constexpr int NL = 2 * L + 1;
	extern __shared__ unsigned long long sk[];
	__shared__ int ns, n0, base0, base1;
	const int n = P.counters[CNT_TOUCH];
	const size_t bv = (size_t)P.BV;
	for (int q = blockIdx.x; q < n; q += gridDim.x) {
		const int sl = P.q_touch[q];
		const int gp = P.slot_gp[sl];
		if (threadIdx.x == 0) ns = 0;
		__syncthreads();
		for (int leaf = threadIdx.x; leaf < P.BV; leaf += blockDim.x) {
			const unsigned long long k = P.claim[sl * bv + leaf];
			if (k != NOCLAIM) {
				// keys use 44 bits; the leaf is packed below them.
				sk[atomicAdd(&ns, 1)] = (k << 16) | (unsigned long long)leaf;
				P.claim[sl * bv + leaf] = NOCLAIM;
			}
		}
		__syncthreads();
		const int m = ns;
		int p2 = 1;
		while (p2 < m) p2 <<= 1;
		for (int i = m + threadIdx.x; i < p2; i += blockDim.x) sk[i] = ~0ull;
		__syncthreads();
		// bitonic sort, ascending
		for (int kk = 2; kk <= p2; kk <<= 1)
			for (int j = kk >> 1; j > 0; j >>= 1) {
				for (int i = threadIdx.x; i < p2; i += blockDim.x) {
					const int ixj = i ^ j;
					if (ixj > i) {
						const unsigned long long a = sk[i], c = sk[ixj];
						const bool up = (i & kk) == 0;
						if ((a > c) == up) {
							sk[i] = c;
							sk[ixj] = a;
						}
					}
				}
				__syncthreads();
			}
		if (threadIdx.x == 0) {
			int c0 = 0;
			while (c0 < m && ((sk[c0] >> 16) >> 43) == 0) c0++;
			n0 = c0;
			base0 = P.lcnt[sl * NL + 0];
			base1 = P.lcnt[sl * NL + NL - 1];
		}
		__syncthreads();
		for (int i = threadIdx.x; i < m; i += blockDim.x) {
			const int leaf = (int)(sk[i] & 0xFFFFu);
			const int ph = i < n0 ? 0 : 1;
			const int li = ph ? NL - 1 : 0;
			const int pos = ph ? base1 + (i - n0) : base0 + i;
			P.phi[sl * bv + leaf] = P.dlt[sl * bv + leaf];
			P.lst[((size_t)sl * NL + li) * bv + pos] = (uint16_t)leaf;
			P.lkp[sl * bv + leaf] = (uint16_t)pos;
		}
		if (threadIdx.x == 0) {
			P.lcnt[sl * NL + 0] = base0 + n0;
			P.lcnt[sl * NL + NL - 1] = base1 + (m - n0);
			const int s = P.surf_of[gp];
			const int pb = P.geom[s].pbase;
			if (n0 > 0 && P.ppos[gp * NL + 0] < 0) {
				const int at = atomicAdd(&P.papn[s], 1);
				P.pap[2 * (size_t)pb + at] = sk[0] >> 16;
				P.papg[2 * (size_t)pb + at] = gp - pb;
			}
			if (m - n0 > 0 && P.ppos[gp * NL + NL - 1] < 0) {
				const int at = atomicAdd(&P.papn[s], 1);
				P.pap[2 * (size_t)pb + at] = sk[n0] >> 16;
				P.papg[2 * (size_t)pb + at] = gp - pb;
			}
			P.touched[sl] = 0;
		}
		__syncthreads();
	}
}

/// Children-level appends of the expansion (track_child of PartitionedMixin.hpp:201-213, in
/// first-claim order). One block per surface; entries ranked by key.
template <int L>
__global__ void k_expand_plist(Dev P)
{
	constexpr int NL = 2 * L + 1;
	const int s = blockIdx.x;
	if (s >= P.S) return;
	const int m = P.papn[s];
	if (m == 0) return;
	const SurfGeom& g = P.geom[s];
	const unsigned long long* ent = P.pap + 2 * (size_t)g.pbase;
	const int* entg = P.papg + 2 * (size_t)g.pbase;
	__shared__ int c0, c1;
	if (threadIdx.x == 0) {
		c0 = P.pcnt[s * NL + 0];
		c1 = P.pcnt[s * NL + NL - 1];
	}
	__syncthreads();
	for (int i = threadIdx.x; i < m; i += blockDim.x) {
		const unsigned long long ki = ent[i];
		const int ph = (int)(ki >> 43);
		int rank = 0;
		for (int j = 0; j < m; j++) {
			const unsigned long long kj = ent[j];
			if ((int)(kj >> 43) == ph && kj < ki) rank++;
		}
		const int lp = entg[i];
		const int li = ph ? NL - 1 : 0;
		const int pos = (ph ? c1 : c0) + rank;
		P.plist[(size_t)li * P.NP + g.pbase + pos] = lp;
		P.ppos[(g.pbase + lp) * NL + li] = pos;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		int a0 = 0, a1 = 0;
		for (int j = 0; j < m; j++) {
			if ((int)(ent[j] >> 43) == 0)
				a0++;
			else
				a1++;
		}
		P.pcnt[s * NL + 0] = c0 + a0;
		P.pcnt[s * NL + NL - 1] = c1 + a1;
		P.papn[s] = 0;
	}
}

// ---------------------------------------------------------------------------------------------
// Resets between iterations
// ---------------------------------------------------------------------------------------------

/// status_change grid reset (Reset::MultiList::reset, PartitionedMixin.hpp:336-360).
template <int L>
__global__ void k_clear_status(Dev P)
{
	constexpr int NL = 2 * L + 1;
	const int n = P.counters[CNT_SUNION];
	const int lane = lane_id();
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < n; e += nwarps) {
		const int gp = P.q_sunion[e];
		const int sl = P.slot[gp];
		if (sl >= 0) {
			for (int fi = 0; fi < NL; fi++) {
				const int nc = P.ccnt[sl * NL + fi];
				const uint16_t* ch = P.chg + ((size_t)sl * NL + fi) * P.BV;
				for (int c = lane; c < nc; c += 32) P.sto[(size_t)sl * P.BV + ch[c]] = (int8_t)(L + 1);
			}
			__syncwarp();
			if (lane < NL) P.ccnt[sl * NL + lane] = 0;
		}
		if (lane < NL) P.sppos[gp * NL + lane] = -1;
		if (lane == 0) P.sflag[gp] = 0;
	}
}

/// Affected buffer reset: clears the leaf lookups and lists of buffer b.
template <int L>
__global__ void k_clear_buffer(Dev P, int b)
{
	constexpr int NL = 2 * L + 1;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		int i = e - P.woff[s];
		int t = 0;
		while (i >= P.apcnt[b][s * NL + t]) {
			i -= P.apcnt[b][s * NL + t];
			t++;
		}
		const int gp = g.pbase + P.aplist[b][(size_t)t * P.NP + g.pbase + i];
		const int sl = P.slot[gp];
		if (sl >= 0) {
			const int nc = P.acnt[b][sl * NL + t];
			const uint16_t* al = P.alst[b] + ((size_t)sl * NL + t) * P.BV;
			for (int c = lane; c < nc; c += 32) P.alkp[b][(size_t)sl * P.BV + al[c]] = NUL16;
			__syncwarp();
			if (lane == 0) P.acnt[b][sl * NL + t] = 0;
		}
		if (lane == 0) P.appos[b][gp * NL + t] = -1;
	}
}

/// Returns the bricks of partitions deactivated in this iteration to the free pool.
static __global__ void k_retire(Dev P)
{
	const int n = P.counters[CNT_RETIRE];
	for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
		const int sl = P.q_retire[e];
		const int gp = P.slot_gp[sl];
		if (P.oslot[gp] == sl) P.oslot[gp] = -1;
		P.slot_gp[sl] = -1;
		P.free_stack[atomicAdd(&P.counters[CNT_FREE_TOP], 1)] = sl;
	}
}

/// Copies the isogrid partition lists to the delta partition lists (track_children of the
/// delta grid at update start, Surface.hpp:261 / PartitionedMixin.hpp:319-334, which mirrors
/// the isogrid lists into the freshly reset delta lists). Grid y = s*NL + l.
static __global__ void k_copy_plists(Dev P, int NL)
{
	const int s = blockIdx.y / NL, l = blockIdx.y % NL;
	const SurfGeom& g = P.geom[s];
	const int n = P.pcnt[s * NL + l];
	const size_t o = (size_t)l * P.NP + g.pbase;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		P.dplist[o + i] = P.plist[o + i];
	if (blockIdx.x == 0 && threadIdx.x == 0) P.dpcnt[s * NL + l] = n;
}

/// Narrow-band size: sum over all isogrid lists of the leaf counts (64-bit accumulator).
template <int L>
__global__ void k_band_size(Dev P, unsigned long long* acc)
{
	constexpr int NL = 2 * L + 1;
	unsigned long long local = 0;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		int i = e - P.woff[s];
		int t = 0;
		while (i >= P.pcnt[s * NL + t]) {
			i -= P.pcnt[s * NL + t];
			t++;
		}
		const int gp = g.pbase + P.plist[(size_t)t * P.NP + g.pbase + i];
		if (lane == 0) local += (unsigned long long)P.lcnt[P.slot[gp] * NL + t];
	}
	if (lane_id() == 0 && local) atomicAdd(acc, local);
}

/// Dense snapshot (PartitionedMixin.hpp:642-660) of surface s.
template <int D, int L>
__global__ void k_snapshot(Dev P, int s, float* out, long long total)
{
	const SurfGeom& g = P.geom[s];
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
	     i += (long long)gridDim.x * blockDim.x) {
		Vec<D> p;
		long long r = i;
		for (int a = D - 1; a >= 0; a--) {
			p[a] = (int)(r % g.size[a]) + g.off[a];
			r /= g.size[a];
		}
		out[i] = get_phi<D, L>(P, g, p);
	}
}

/// seed (Surface.hpp:207-241) executed by one thread: the window walk and its track calls are
/// sequential in the reference and set the initial list orders.
template <int D, int L>
__global__ void k_seed(Dev P, int s, Vec<D> centre)
{
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	int win = 2 * L + 1;
	long long nmax = 1;
	for (int a = 0; a < D; a++) nmax *= win;
	for (long long i = 0; i <= nmax; i++) {
		Vec<D> p;
		long long r = i;
		for (int a = D - 1; a >= 1; a--) {
			p[a] = (int)(r % win);
			r /= win;
		}
		p[0] = (int)(r % win);
		int l1 = 0;
		for (int a = 0; a < D; a++) {
			p[a] += centre[a] - L;
			l1 += abs(p[a] - centre[a]);
		}
		const float dist = (float)l1;
		const int lid = layer_id(dist, P.err);
		if (!inside_band(lid, L)) continue;
		if (!in_grid<D>(g, p)) {
			atomicOr(P.err, EB_OUTSIDE);
			continue;
		}
		const int li = lid + L;
		int gp, leaf;
		locate<D>(P, g, p, gp, leaf);
		// track_child (PartitionedMixin.hpp:201-213)
		if (P.ppos[gp * NL + li] < 0) {
			if (P.slot[gp] < 0) {
				const int t = atomicSub(&P.counters[CNT_FREE_TOP], 1) - 1;
				if (t < 0) {
					atomicAdd(&P.counters[CNT_FREE_TOP], 1);
					atomicOr(P.err, EB_POOL);
					return;
				}
				const int sl = P.free_stack[t];
				brick_init<L>(P, sl, P.bg[gp], 0, 1);
				P.slot_gp[sl] = gp;
				P.touched[sl] = 0;
				P.slot[gp] = sl;
			}
			const int c = P.pcnt[s * NL + li];
			P.plist[(size_t)li * P.NP + g.pbase + c] = gp - g.pbase;
			P.ppos[gp * NL + li] = c;
			P.pcnt[s * NL + li] = c + 1;
		}
		const int sl = P.slot[gp];
		P.phi[(size_t)sl * P.BV + leaf] = dist;
		if (P.lkp[(size_t)sl * P.BV + leaf] == NUL16) {
			const int c = P.lcnt[sl * NL + li];
			P.lst[((size_t)sl * NL + li) * P.BV + c] = (uint16_t)leaf;
			P.lkp[(size_t)sl * P.BV + leaf] = (uint16_t)c;
			P.lcnt[sl * NL + li] = c + 1;
		}
	}
}

}  // namespace fg
