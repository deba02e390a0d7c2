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

/// A partition-list + leaf-list pair: the isogrid's own lists, or one affected buffer's, with
/// the leaf lookup (a leaf's position in its list) where a kernel needs it.
struct ListView {
	const int* plist;
	const int* pcnt;
	const uint16_t* lst;
	const int* lcnt;
	const uint16_t* lkp = nullptr;
	const int* ppos = nullptr;  // [NP*NL] position of a partition in plist's list, -1 = none
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

/// Adds every thread's count to a global work counter with one atomic per block instead of one
/// per partition entry on the same word. Every thread of the block calls it once, at the end
/// of the kernel's work.
__device__ __forceinline__ void block_add(unsigned long long* dst, unsigned long long v)
{
	__shared__ unsigned long long acc;
	if (threadIdx.x == 0) acc = 0;
	__syncthreads();
	if (v) atomicAdd(&acc, v);
	__syncthreads();
	if (threadIdx.x == 0 && acc) atomicAdd(dst, acc);
}

/// True in exactly one block of the launch, the last to arrive; every thread of every block
/// calls it once, after the block's work. The arrival counter is left at zero for the next
/// launch. Where it returns true, every other block's global reads and writes are complete, so
/// that block may reset what the launch read (the update's graph then needs no memset nodes,
/// which would break the chain of programmatic launches).
__device__ __forceinline__ bool last_block(int* counter)
{
	__shared__ int last;
	__syncthreads();
	if (threadIdx.x == 0) {
		__threadfence();
		last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
		if (last) *counter = 0;
	}
	__syncthreads();
	if (last) __threadfence();
	return last;
}

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
// Frozen surfaces (frozen[s] != 0) contribute no entries, so no kernel works on them.
// ---------------------------------------------------------------------------------------------
/// One surface count per lane of warp 0 (S <= 32): the scan in registers, no block barrier.
/// cg: the counts were written by other blocks of the same launch, read past L1.
static __device__ __forceinline__ int count_at(const int* cnt, int i, bool cg)
{
	return cg ? __ldcg(cnt + i) : cnt[i];
}
static __device__ __forceinline__ int surface_count(const int* cnt, int NL, int l, int mode, int s,
                                                    const int* frozen, bool cg = false)
{
	if (frozen && frozen[s]) return 0;
	if (mode == 0) return count_at(cnt, s * NL + l, cg);
	if (mode == 1) return count_at(cnt, s * NL, cg) + count_at(cnt, s * NL + NL - 1, cg);
	int v = 0;
	for (int t = 0; t < NL; t++) v += count_at(cnt, s * NL + t, cg);
	return v;
}
static __device__ __forceinline__ void warp_scan_counts(const int* cnt, int NL, int l, int mode,
                                                        int S, int* woff, const int* frozen,
                                                        bool cg = false)
{
	const int lane = lane_id();
	int v = lane < S ? surface_count(cnt, NL, l, mode, lane, frozen, cg) : 0;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int y = __shfl_up_sync(FULL, v, o);
		if (lane >= o) v += y;
	}
	if (lane == 0) woff[0] = 0;
	if (lane < S) woff[lane + 1] = v;
}

static __device__ __noinline__ void d_scan_counts(const int* cnt, int NL, int l, int mode, int S,
                                                  int* woff, const int* frozen, bool cg = false)
{
	if (S <= 32) {
		if (threadIdx.x < 32) warp_scan_counts(cnt, NL, l, mode, S, woff, frozen, cg);
		__syncthreads();
		return;
	}
	__shared__ int carry;
	if (threadIdx.x == 0) {
		carry = 0;
		woff[0] = 0;
	}
	__syncthreads();
	for (int base = 0; base < S; base += blockDim.x) {
		const int s = base + threadIdx.x;
		const int v = s < S ? surface_count(cnt, NL, l, mode, s, frozen, cg) : 0;
		int tot;
		const int ex = block_excl_scan(v, &tot);
		if (s < S) woff[s + 1] = carry + ex + v;
		__syncthreads();
		if (threadIdx.x == 0) carry += tot;
		__syncthreads();
	}
}
static __global__ void k_scan_counts(const int* cnt, int NL, int l, int mode, int S, int* woff,
                                     const int* frozen)
{
	pdl_enter();
	d_scan_counts(cnt, NL, l, mode, S, woff, frozen);
}

/// k_scan_counts mode 0 for every layer index at once: woffl[l*(S+1) + s].
static __device__ __noinline__ void d_scan_layers(const int* cnt, int NL, int S, int* woffl,
                                                  const int* frozen)
{
	if (S <= 32 && (int)(blockDim.x >> 5) >= NL) {
		// a warp per layer
		const int w = threadIdx.x >> 5;
		if (w < NL) warp_scan_counts(cnt, NL, w, 0, S, woffl + (size_t)w * (S + 1), frozen);
		__syncthreads();
		return;
	}
	__shared__ int carry;
	for (int l = 0; l < NL; l++) {
		int* woff = woffl + (size_t)l * (S + 1);
		if (threadIdx.x == 0) {
			carry = 0;
			woff[0] = 0;
		}
		__syncthreads();
		for (int base = 0; base < S; base += blockDim.x) {
			const int s = base + threadIdx.x;
			const int v = (s < S && !(frozen && frozen[s])) ? cnt[s * NL + l] : 0;
			int tot;
			const int ex = block_excl_scan(v, &tot);
			if (s < S) woff[s + 1] = carry + ex + v;
			__syncthreads();
			if (threadIdx.x == 0) carry += tot;
			__syncthreads();
		}
	}
}
static __global__ void k_scan_layers(const int* cnt, int NL, int S, int* woffl, const int* frozen)
{
	pdl_enter();
	d_scan_layers(cnt, NL, S, woffl, frozen);
}

/// Entry-offset scans run inside the kernel that needs them, every block for itself from
/// shared memory, for pools of at most this many surfaces; larger pools scan in a launch of
/// their own.
constexpr int kScanHereMax = 512;

/// The block index and block count a kernel body works with (the hardware grid's, or another
/// grid dimension's where the launch is two-dimensional).
struct GridPos {
	int bid, nb;
};
__device__ __forceinline__ GridPos hw_grid() { return GridPos{(int)blockIdx.x, (int)gridDim.x}; }

#define FG_WARP_LOOP_G(woff_, G_)                                                   \
	const int lane = lane_id();                                                     \
	const int nwarps = ((G_).nb * blockDim.x) >> 5;                                \
	const int total = (woff_)[P.S];                                                 \
	for (int e = ((G_).bid * blockDim.x + threadIdx.x) >> 5; e < total; e += nwarps)
#define FG_WARP_LOOP(woff_) FG_WARP_LOOP_G(woff_, G)

// ---------------------------------------------------------------------------------------------
// status_change (Surface.hpp:1138-1178) for one 32-leaf chunk of partition gp processed by a
// warp in pass `from`: records the status grid entry (list per from-layer, value = to) and
// tracks the leaf into affected buffer b under its new layer. Per-entry flags: bit 31 = the
// partition must join the status partition list of `from`; bit t = it must join the buffer's
// partition list t.
//
// While a warp records one partition entry nothing else writes that partition's list counts,
// so they stay in registers for the whole entry (StatusCache): every lane holds the status
// list count of `from`; lane t < NL holds buffer list t's leaf count and whether the partition
// is already in the buffer's partition list t (compaction, which changes that, runs after the
// pass). They are loaded at the entry's first change (most chunks have none). A chunk with
// changes then costs one round of loads (the leaves' status and buffer lookups).
// ---------------------------------------------------------------------------------------------
struct StatusCache {
	int ccnt = 0;         // leaves in the status list of `from`
	int acnt = 0;         // lane t < NL: leaves in buffer list t
	bool tracked = true;  // lane t < NL: the partition is in the buffer's partition list t
	bool loaded = false;
};

template <int L>
__device__ __forceinline__ StatusCache status_load(const Dev& P, int gp, int sl, int from, int b)
{
	constexpr int NL = 2 * L + 1;
	const int lane = lane_id();
	StatusCache c;
	c.ccnt = P.ccnt[sl * NL + from + L];
	c.acnt = lane < NL ? P.acnt[b][sl * NL + lane] : 0;
	c.tracked = lane < NL ? P.appos[b][gp * NL + lane] >= 0 : true;
	c.loaded = true;
	return c;
}

template <int L>
__device__ __forceinline__ void status_store(const Dev& P, int sl, int from, int b,
                                             const StatusCache& c)
{
	constexpr int NL = 2 * L + 1;
	const int lane = lane_id();
	if (!c.loaded) return;
	if (lane == 0) P.ccnt[sl * NL + from + L] = c.ccnt;
	if (lane < NL) P.acnt[b][sl * NL + lane] = c.acnt;
}

template <int L>
__device__ __forceinline__ void status_chunk(const Dev& P, int gp, int sl, int from, bool valid,
                                             int leaf, int to, int b, unsigned& flags,
                                             bool& any_change, StatusCache& sc)
{
	constexpr int NL = 2 * L + 1;
	const int lane = lane_id();
	const unsigned lt = (1u << lane) - 1u;
	const bool chgd = valid && to != from;
	if (__ballot_sync(FULL, chgd) == 0) return;
	any_change = true;
	if (!sc.loaded) sc = status_load<L>(P, gp, sl, from, b);
	const size_t bv = (size_t)P.BV;
	const bool inb = chgd && inside_band(to, L);
	const int t = inb ? to + L : -1;
	bool app = false, isnew = false;
	if (chgd) {
		const int cur = P.sto[sl * bv + leaf];
		if (inb) isnew = P.alkp[b][sl * bv + leaf] == NUL16;
		app = cur == L + 1;
		P.sto[sl * bv + leaf] = (int8_t)to;
	}
	const unsigned ma = __ballot_sync(FULL, app);
	if (ma) {
		const int fi = from + L;
		if (app) P.chg[((size_t)sl * NL + fi) * bv + sc.ccnt + __popc(ma & lt)] = (uint16_t)leaf;
		sc.ccnt += __popc(ma);
		flags |= 0x80000000u;
	}
	if (__ballot_sync(FULL, inb)) {
		const unsigned grp = __match_any_sync(FULL, t);
		const unsigned mn = __ballot_sync(FULL, isnew) & grp;
		const int base = __shfl_sync(FULL, sc.acnt, inb ? t : 0);
		const bool trk = __shfl_sync(FULL, sc.tracked, inb ? t : 0);
		if (isnew) {
			const int pos = base + __popc(mn & lt);
			P.alst[b][((size_t)sl * NL + t) * bv + pos] = (uint16_t)leaf;
			P.alkp[b][sl * bv + leaf] = (uint16_t)pos;
		}
		if (inb && !trk) flags |= 1u << t;
#pragma unroll
		for (int l = 0; l < NL; l++) {
			const int add = __popc(__ballot_sync(FULL, isnew && t == l));
			if (lane == l) sc.acnt += add;
		}
	}
}

__device__ __forceinline__ unsigned warp_or(unsigned v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(FULL, v, o);
	return v;
}

/// The status records of one block-wide round over a partition's list: the block's changed
/// leaves (ch: to != from) are compacted in list order into shared memory, and warp 0 records
/// them 32 at a time with status_chunk, which keeps the reference's order. Every thread of the
/// block calls it; flags and any_change accumulate in warp 0.
template <int L>
__device__ __forceinline__ void status_round(const Dev& P, int gp, int sl, int from, bool ch,
                                             int leaf, int to, int b, unsigned& flags,
                                             bool& any_change, uint16_t* cl, int* ct,
                                             StatusCache& sc)
{
	if (!__syncthreads_or(ch)) return;
	int tot;
	const int pos = block_excl_scan(ch ? 1 : 0, &tot);
	if (ch) {
		cl[pos] = (uint16_t)leaf;
		ct[pos] = to;
	}
	__syncthreads();
	if (threadIdx.x < 32) {
		for (int c0 = 0; c0 < tot; c0 += 32) {
			const int c = c0 + (int)threadIdx.x;
			const bool v = c < tot;
			status_chunk<L>(P, gp, sl, from, v, v ? cl[c] : 0, v ? ct[c] : from, b, flags,
			                any_change, sc);
		}
	}
	__syncthreads();
}

// ---------------------------------------------------------------------------------------------
// update(fn) functor loop (Surface.hpp:263-294) with a builtin speed: delta of every zero-layer
// leaf, written to the brick's delta array.
// ---------------------------------------------------------------------------------------------
/// `split` warps per partition entry take interleaved 32-leaf chunks of its zero layer; the
/// stencil reads inside the brick skip the partition lookup (BrickGet).
template <int D, int L>
__device__ void d_delta_builtin(const Dev& P, const Speed* speeds, int split, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	const int lane = lane_id();
	const int nwarps = (G.nb * blockDim.x) >> 5;
	const int total = P.woff[P.S] * split;
	unsigned long long done = 0;
	for (int v = (G.bid * blockDim.x + threadIdx.x) >> 5; v < total; v += nwarps) {
		const int e = v / split, part = v - e * split;
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const Speed sp = speeds[s];
		const int gp = g.pbase + P.plist[(size_t)L * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		const int n = P.lcnt[sl * NL + L];
		const uint16_t* lst = P.lst + ((size_t)sl * NL + L) * P.BV;
		BrickGet<D, L> get{P, g, P.phi + (size_t)sl * P.BV, Vec<D>()};
#pragma unroll
		for (int a = 0; a < D; a++) get.org[a] = P.porig[gp * 3 + a];
		for (int j = part * 32 + lane; j < n; j += 32 * split) {
			const int leaf = lst[j];
			P.dlt[(size_t)sl * P.BV + leaf] = speed_eval_g<D>(get, sp, leaf_pos<D>(P, gp, leaf));
		}
		if (lane == 0 && part == 0) done += n;
	}
	block_add(&P.kstat[KS_ZERO], done);
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_delta_builtin(Dev P, const Speed* speeds, int split)
{
	pdl_enter();
	d_delta_builtin<D, L>(P, speeds, split, hw_grid());
}

/// The staged box of k_delta_smem: the partition and a one-node halo, row-major with the last
/// axis fastest. Along the last axis a row holds 3 unused slots, the -1 halo node, the brick's
/// row and the +1 halo node, padded to a multiple of 4 floats, so that every brick row starts on
/// a 16-byte boundary and arrives by one bulk copy.
struct HaloBox {
	int ext[3];  // extents: csz + 2 on the leading axes, the padded row on the last
	int vol;
	__host__ __device__ HaloBox(int D, const int* csz)
	{
		vol = 1;
		for (int a = 0; a < D; a++) {
			ext[a] = a == D - 1 ? ((csz[a] + 5 + 3) & ~3) : csz[a] + 2;
			vol *= ext[a];
		}
	}
};

/// Fills the box of partition gp (brick slot sl). The slots (or backgrounds) of the 3^D
/// partitions around it are looked up once. Each row of the box along the last axis is one
/// thread's: a row inside the brick and the grid takes its brick row by one bulk copy
/// (cp.async.bulk completing on bar; rows = number issued, returned) and loads its two halo
/// nodes; every other node is one load from the neighbour partition's brick, its background
/// (inactive), or L+1 outside the grid: the values get_phi reads there. bulk = false: every
/// node by a load.
template <int D, int L>
__device__ int stage_halo(const Dev& P, const SurfGeom& g, int gp, float* box, const HaloBox& hb,
                          bool bulk, unsigned long long* bar)
{
	constexpr int ND = D == 3 ? 27 : 9;
	__shared__ int nsl[27];    // slot of the partition in each direction (-1 inactive)
	__shared__ float nbg[27];  // its background
	if (threadIdx.x < ND) {
		// a node of the neighbour partition: one outside the brick on the axes the direction
		// leaves it, the brick's first node elsewhere
		int r = threadIdx.x;
		Vec<D> p;
		for (int a = D - 1; a >= 0; a--) {
			const int d = r % 3 - 1;
			r /= 3;
			p[a] = P.porig[gp * 3 + a] + (d < 0 ? -1 : d > 0 ? P.csz[a] : 0);
		}
		int s2 = -1;
		float b2 = (float)(L + 1);
		if (in_grid<D>(g, p)) {
			int gp2, leaf2;
			locate<D>(P, g, p, gp2, leaf2);
			s2 = P.slot[gp2];
			b2 = P.bg[gp2];
		}
		nsl[threadIdx.x] = s2;
		nbg[threadIdx.x] = b2;
	}
	__syncthreads();
	constexpr int X = D - 1;
	const int cx = P.csz[X];
	const int ex = hb.ext[X];
	const int nrows = hb.vol / ex;
	const int ox = P.porig[gp * 3 + X];
	const bool rows_bulk = bulk && (cx * sizeof(float)) % 16 == 0;
	int issued = 0;
	for (int row = threadIdx.x; row < nrows; row += blockDim.x) {
		// the row's coordinates on the leading axes (-1..csz), its direction digits and leaf base
		int r = row, dir = 0, mul = 3, leaf0 = 0;
		bool ing = true, inner = true;
#pragma unroll
		for (int a = D - 2; a >= 0; a--) {
			const int c = r % hb.ext[a] - 1;
			r /= hb.ext[a];
			const int cs = P.csz[a];
			dir += (c < 0 ? 0 : c >= cs ? 2 : 1) * mul;
			mul *= 3;
			leaf0 += (c < 0 ? cs - 1 : c >= cs ? 0 : c) * P.lstr[a];
			const int pa = P.porig[gp * 3 + a] + c;
			ing = ing && pa >= g.off[a] && pa < g.hi[a];
			inner = inner && c >= 0 && c < cs;
		}
		float* out = box + (size_t)row * ex + 3;  // node x = -1 of the row
		// the brick's row in one bulk copy when it lies wholly inside the grid
		const bool copy = rows_bulk && inner && ing && ox + cx <= g.hi[X];
		if (copy) {
			bulk_g2s(out + 1, P.phi + (size_t)P.slot[gp] * P.BV + leaf0,
			         (unsigned)(cx * sizeof(float)), bar);
			issued++;
		}
		for (int x = -1; x <= cx; x++) {
			if (copy && x >= 0 && x < cx) continue;
			const int d = x < 0 ? 0 : x >= cx ? 2 : 1;
			const int leaf = leaf0 + (x < 0 ? cx - 1 : x >= cx ? 0 : x);
			const int px = ox + x;
			float v = (float)(L + 1);
			if (ing && px >= g.off[X] && px < g.hi[X]) {
				const int s2 = nsl[dir + d];
				v = s2 >= 0 ? P.phi[(size_t)s2 * P.BV + leaf] : nbg[dir + d];
			}
			out[x + 1] = v;
		}
	}
	return issued;
}

/// Reads a staged box (stage_halo) by world position.
template <int D>
struct BoxGet {
	const float* box;
	int org[D];  // world position of the box's first node on each axis (the -1 halo node)
	int ext[D];
	__device__ float operator()(const Vec<D>& p) const
	{
		int i = 0;
#pragma unroll
		for (int a = 0; a < D; a++) i = i * ext[a] + (p[a] - org[a]);
		return box[i + 3];  // the 3 unused slots at the start of each row
	}
};

/// Shared-memory bytes of k_delta_smem's box.
__host__ __device__ inline size_t halo_smem_bytes(int D, const int* csz)
{
	return (size_t)HaloBox(D, csz).vol * sizeof(float);
}

/// k_delta_builtin with the partition and its halo staged in shared memory, for speeds with a
/// curvature term: every stencil read of the zero-layer nodes hits shared memory. One block per
/// zero-layer partition. The brick's rows arrive by bulk copies (cp.async.bulk on an mbarrier,
/// one per row, issued by the threads that stage the halo around them); a brick whose rows are
/// not a multiple of 16 bytes is loaded by the threads.
template <int D, int L>
__device__ void d_delta_smem(const Dev& P, const Speed* speeds, GridPos G, float* hbox)
{
	constexpr int NL = 2 * L + 1;
	constexpr int WAIT_TRIES = 1 << 20;  // bound of the copies' wait (each poll may suspend)
	__shared__ __align__(8) unsigned long long bar;
	__shared__ int copy_ok, any_copy;
	const int total = P.woff[P.S];
	const HaloBox hb(D, P.csz);
	unsigned long long done = 0;
	if (threadIdx.x == 0) mbar_init(&bar);
	__syncthreads();
	unsigned parity = 0;
	for (int e = G.bid; e < total; e += G.nb) {
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const Speed sp = speeds[s];
		const int gp = g.pbase + P.plist[(size_t)L * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		if (threadIdx.x == 0) any_copy = 0;
		fence_proxy_async();  // the previous entry's reads of the box come before the copies
		const int issued = stage_halo<D, L>(P, g, gp, hbox, hb, true, &bar);
		if (issued) atomicOr(&any_copy, 1);
		__syncthreads();  // every copy of the phase issued
		if (any_copy) {
			if (threadIdx.x == 0) {
				mbar_arrive(&bar);
				copy_ok = mbar_wait(&bar, parity, WAIT_TRIES) ? 1 : 0;
			}
			__syncthreads();
			if (!copy_ok) {
				// the copies did not land: report it and leave; a last bounded wait lets late
				// copies finish before the block's shared memory goes
				if (threadIdx.x == 0) {
					atomicOr(P.err, EB_TIMEOUT);
					mbar_wait(&bar, parity, WAIT_TRIES);
				}
				return;
			}
			mbar_wait(&bar, parity, WAIT_TRIES);  // completed: every thread observes it
			parity ^= 1u;
		}
		__syncthreads();
		BoxGet<D> get;
		get.box = hbox;
#pragma unroll
		for (int a = 0; a < D; a++) {
			get.org[a] = P.porig[gp * 3 + a] - 1;
			get.ext[a] = hb.ext[a];
		}
		const int n = P.lcnt[sl * NL + L];
		const uint16_t* lst = P.lst + ((size_t)sl * NL + L) * P.BV;
		for (int j = threadIdx.x; j < n; j += blockDim.x) {
			const int leaf = lst[j];
			P.dlt[(size_t)sl * P.BV + leaf] = speed_eval_g<D>(get, sp, leaf_pos<D>(P, gp, leaf));
		}
		if (threadIdx.x == 0) done += n;
		__syncthreads();
	}
	block_add(&P.kstat[KS_ZERO], done);
}
template <int D, int L>
__global__ void __launch_bounds__(128) k_delta_smem(Dev P, const Speed* speeds)
{
	pdl_enter();
	extern __shared__ __align__(16) float hbox[];
	d_delta_smem<D, L>(P, speeds, hw_grid(), hbox);
}

/// update_zero_layer (Surface.hpp:920-979) over the isogrid's zero-layer lists, which the delta
/// grid mirrors in the global update. One block per partition entry (bricks of thousands of
/// leaves): every thread applies one leaf, and the rare layer changes are recorded in list order
/// (status_round).
template <int D, int L>
__device__ void d_zero_apply(const Dev& P, ListView lv, const int* ncount, int b, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	__shared__ uint16_t cl[256];
	__shared__ int ct[256];
	const int total = P.woff[P.S];
	for (int e = G.bid; e < total; e += G.nb) {
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const int gp = g.pbase + lv.plist[(size_t)L * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		// the delta grid's zero-layer leaves: the isogrid list in the global update, a prefix of
		// the affected list (the delta() calls' leaves) in the local update
		const int n = ncount ? ncount[sl] : lv.lcnt[sl * NL + L];
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + L) * P.BV;
		const size_t b0 = (size_t)sl * P.BV;
		unsigned flags = 0;
		bool any = false;
		StatusCache sc;
		for (int base = 0; base < n; base += blockDim.x) {
			const int j = base + threadIdx.x;
			int leaf = 0, to = 0;
			if (j < n) {
				leaf = lst[j];
				const float nw = __fadd_rn(P.phi[b0 + leaf], P.dlt[b0 + leaf]);
				to = layer_id(nw, P.err);
				P.phi[b0 + leaf] = nw;
			}
			status_round<L>(P, gp, sl, 0, j < n && to != 0, leaf, to, b, flags, any, cl, ct, sc);
		}
		if (threadIdx.x < 32) {
			status_store<L>(P, sl, 0, b, sc);
			flags = warp_or(flags);
			if (threadIdx.x == 0) P.eflag[e] = flags;
		}
	}
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_zero_apply(Dev P, ListView lv, const int* ncount, int b)
{
	pdl_enter();
	d_zero_apply<D, L>(P, lv, ncount, b, hw_grid());
}

/// update_zero_layer (Surface.hpp:920-979) over the isogrid's zero-layer lists, which the delta
/// grid mirrors in the global update. One warp per partition entry (bricks of few leaves).
template <int D, int L>
__device__ void d_zero_apply_warp(const Dev& P, ListView lv, const int* ncount, int b, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	FG_WARP_LOOP(P.woff)
	{
		const int s = entry_surface(P.woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const int gp = g.pbase + lv.plist[(size_t)L * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		// the delta grid's zero-layer leaves: the isogrid list in the global update, a prefix of
		// the affected list (the delta() calls' leaves) in the local update
		const int n = ncount ? ncount[sl] : lv.lcnt[sl * NL + L];
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + L) * P.BV;
		unsigned flags = 0;
		bool any = false;
		StatusCache sc;
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
			status_chunk<L>(P, gp, sl, 0, valid, leaf, to, b, flags, any, sc);
		}
		status_store<L>(P, sl, 0, b, sc);
		flags = warp_or(flags);
		if (lane == 0) P.eflag[e] = flags;
	}
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_zero_apply_warp(Dev P, ListView lv, const int* ncount, int b)
{
	pdl_enter();
	d_zero_apply_warp<D, L>(P, lv, ncount, b, hw_grid());
}

/// Appends, in the pass's partition order, the partitions that gained status changes to the
/// status partition list of layer index `li`, and those newly tracked in buffer b's partition
/// lists (the children-level track_child calls of status_change, PartitionedMixin.hpp:201-213),
/// for surface s, by one block. The block stages a tile of the entries' flags and partition
/// indices in shared memory; each warp owns whole lists (list t < NL: buffer list t, list NL:
/// the status list) and ranks the entries that join it with ballots (stores only, nothing
/// waited on); then the whole block adds the tile's partitions with status changes to the
/// flush's work queue (any order).
struct CompactArgs {
	int nblocks;        // blocks of the launch that compact (one per surface), 0 = none
	const int* woff;    // entry offsets of the pass being compacted
	const int* plist;   // its partition lists
	int li;             // its layer index
	int b;              // affected buffer its changes went to
	const unsigned* ef = nullptr;  // its entry flags (nullptr = Dev::eflag)
	int dedup = 0;      // 1: a partition already in a buffer list is not appended again (the
	                    // pass recorded before the compaction of the passes ahead of it)
};

template <int L>
__device__ void compact_surface(const Dev& P, const CompactArgs& a, int s)
{
	constexpr int NL = 2 * L + 1;
	constexpr int TILE = 1024;
	__shared__ unsigned sf[TILE];
	__shared__ int slp[TILE];
	__shared__ int scnt[NL + 1];
	const int li = a.li, b = a.b;
	const unsigned* ef = a.ef ? a.ef : P.eflag;
	const SurfGeom& g = P.geom[s];
	const int e0 = a.woff[s], e1 = a.woff[s + 1];
	if (e0 == e1) return;  // no entries in this pass: every count stays as it is
	const int lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	const unsigned lt = (1u << lane) - 1u;
	if (threadIdx.x <= NL)
		scnt[threadIdx.x] = threadIdx.x == NL ? P.spcnt[s * NL + li]
		                                      : P.apcnt[b][s * NL + threadIdx.x];
	for (int t0 = e0; t0 < e1; t0 += TILE) {
		const int nt = min(TILE, e1 - t0);
		__syncthreads();
		for (int i = threadIdx.x; i < nt; i += blockDim.x) {
			const unsigned f = ef[t0 + i];
			sf[i] = f;
			slp[i] = f ? a.plist[(size_t)li * P.NP + g.pbase + (t0 + i - e0)] : 0;
		}
		__syncthreads();
		for (int t = warp; t <= NL; t += nwarps) {
			const bool status = t == NL;
			const unsigned bit = status ? 0x80000000u : (1u << t);
			int* list = status ? P.splist + (size_t)li * P.NP + g.pbase
			                   : P.aplist[b] + (size_t)t * P.NP + g.pbase;
			int cnt = scnt[t];
			for (int base = 0; base < nt; base += 32) {
				const int i = base + lane;
				const bool hit = i < nt && (sf[i] & bit) &&
				                 (status || !a.dedup ||
				                  P.appos[b][(g.pbase + slp[i]) * NL + t] < 0);
				const unsigned m = __ballot_sync(FULL, hit);
				if (hit) {
					const int lp = slp[i];
					const int gp = g.pbase + lp;
					const int pos = cnt + __popc(m & lt);
					list[pos] = lp;
					if (status)
						P.sppos[gp * NL + li] = pos;
					else
						P.appos[b][gp * NL + t] = pos;
				}
				cnt += __popc(m);
			}
			if (lane == 0) scnt[t] = cnt;
		}
		for (int i = threadIdx.x; i < nt; i += blockDim.x) {
			if (!(sf[i] & 0x80000000u)) continue;
			const int gp = g.pbase + slp[i];
			if (*(volatile int*)&P.sflag[gp] == 0 && atomicExch(&P.sflag[gp], 1) == 0)
				P.q_sunion[atomicAdd(&P.counters[CNT_SUNION], 1)] = gp;
		}
	}
	__syncthreads();
	if (threadIdx.x <= NL) {
		if (threadIdx.x == NL)
			P.spcnt[s * NL + li] = scnt[NL];
		else
			P.apcnt[b][s * NL + threadIdx.x] = scnt[threadIdx.x];
	}
}

/// The compaction of one pass on its own launch, one block per surface.
template <int L>
__global__ void __launch_bounds__(256) k_compact(Dev P, CompactArgs a, int expand_prep)
{
	constexpr int NL = 2 * L + 1;
	pdl_enter();
	compact_surface<L>(P, a, blockIdx.x);
	if (!expand_prep) return;
	// The last pass's compaction completes the status partition lists; its last block to
	// finish prepares the expansion: the entry offsets of the outer status lists (the counts
	// the other blocks wrote, read past L1) and the expansion's counters reset.
	__shared__ int last;
	__syncthreads();
	if (threadIdx.x == 0) {
		__threadfence();
		last = atomicAdd(&P.counters[CNT_CDONE], 1) == (int)gridDim.x - 1;
	}
	__syncthreads();
	if (!last) return;
	__threadfence();
	d_scan_counts(P.spcnt, NL, 0, 1, P.S, P.woff, P.sfrozen, true);
	if (threadIdx.x == 0) {
		P.counters[CNT_ACT] = 0;
		P.counters[CNT_TOUCH] = 0;
		P.counters[CNT_CAND] = 0;
		P.counters[CNT_CDONE] = 0;
	}
}

/// update_distance first pass (Surface.hpp:1028-1073): distance of every leaf of layer k to
/// the zero curve, into the delta array. The pass is bound by load latency, so each partition
/// entry gets `split` warps that take interleaved 32-leaf chunks (large bricks: the fullest
/// partitions no longer set the pass's length alone), and each lane takes two leaves per round
/// so that their neighbour reads are in flight together. The order of the writes does not
/// matter (Jacobi). The launch's first ca.nblocks blocks compact the previous pass instead
/// (compact_surface): that work only touches the previous pass's records and the status and
/// buffer lists, none of which this pass reads, so it overlaps this pass instead of taking a
/// launch of its own.
template <int D, int L>
__device__ void d_dist1_work(const Dev& P, const int* woff, ListView lv, int k, float side,
                             int split, int first_warp, int nwarps)
{
	constexpr int NL = 2 * L + 1;
	const int li = k + L;
	const int lane = lane_id();
	const int total = woff[P.S] * split;
	unsigned long long done = 0;
	for (int v = first_warp; v < total; v += nwarps) {
		const int e = v / split, part = v - e * split;
		const int4 et = P.etab[(size_t)li * P.NP + e];  // entry_table
		const SurfGeom& g = P.geom[et.z];
		const int gp = et.x, sl = et.y, n = et.w;
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
		const size_t b0 = (size_t)sl * P.BV;
		const int STRIDE = 32 * split;
		for (int j = part * 32 + lane; j < n; j += 2 * STRIDE) {
			const bool two = j + STRIDE < n;
			const int l1 = lst[j];
			const int l2 = two ? lst[j + STRIDE] : l1;
			const float p1 = P.phi[b0 + l1], p2 = P.phi[b0 + l2];
			const float d1 = distance_leaf<D, L>(P, g, gp, sl, l1, p1, side);
			const float d2 = distance_leaf<D, L>(P, g, gp, sl, l2, p2, side);
			P.dlt[b0 + l1] = d1;
			if (two) P.dlt[b0 + l2] = d2;
		}
		if (lane == 0 && part == 0) done += n;
	}
	block_add(&P.kstat[KS_DIST], done);
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_dist1(Dev P, const int* woff, ListView lv, int k,
                                               float side, int split, CompactArgs ca)
{
	pdl_enter();
	if ((int)blockIdx.x < ca.nblocks) {
		compact_surface<L>(P, ca, blockIdx.x);
		return;
	}
	d_dist1_work<D, L>(P, woff, lv, k, side, split,
	                   ((blockIdx.x - ca.nblocks) * blockDim.x + threadIdx.x) >> 5,
	                   ((gridDim.x - ca.nblocks) * blockDim.x) >> 5);
}
/// update_distance second pass (Surface.hpp:1075-1121): apply and record status changes. One
/// block per partition entry (bricks of thousands of leaves): every thread commits one leaf,
/// and the rare layer changes are recorded in list order (status_round).
template <int D, int L>
__device__ void d_dist2(const Dev& P, const int* woff, ListView lv, int k, int b, GridPos G,
                        unsigned* eflag)
{
	constexpr int NL = 2 * L + 1;
	const int li = k + L;
	__shared__ uint16_t cl[256];
	__shared__ int ct[256];
	const int total = woff[P.S];
	for (int e = G.bid; e < total; e += G.nb) {
		const int4 et = P.etab[(size_t)li * P.NP + e];  // entry_table
		const int gp = et.x, sl = et.y, n = et.w;
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
		const size_t b0 = (size_t)sl * P.BV;
		unsigned flags = 0;
		bool any = false;
		StatusCache sc;
		for (int base = 0; base < n; base += blockDim.x) {
			const int j = base + threadIdx.x;
			int leaf = 0, to = k;
			if (j < n) {
				leaf = lst[j];
				const float d = P.dlt[b0 + leaf];
				to = layer_id(d, P.err);
				P.phi[b0 + leaf] = d;
			}
			status_round<L>(P, gp, sl, k, j < n && to != k, leaf, to, b, flags, any, cl, ct, sc);
		}
		if (threadIdx.x < 32) {
			status_store<L>(P, sl, k, b, sc);
			flags = warp_or(flags);
			if (threadIdx.x == 0) {
				eflag[e] = flags;
				if (any && !*(volatile int*)P.changed) atomicOr(P.changed, 1);
			}
		}
	}
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_dist2(Dev P, const int* woff, ListView lv, int k, int b)
{
	pdl_enter();
	d_dist2<D, L>(P, woff, lv, k, b, hw_grid(), P.eflag);
}

/// k_dist2 with one warp per partition entry (bricks of few leaves). The next chunk's list
/// entry and delta are loaded before the current chunk's status records (which must stay in
/// list order), so the two load latencies overlap the record work.
template <int D, int L>
__device__ void d_dist2_warp(const Dev& P, const int* woff, ListView lv, int k, int b, GridPos G,
                             unsigned* eflag)
{
	constexpr int NL = 2 * L + 1;
	const int li = k + L;
	FG_WARP_LOOP(woff)
	{
		const int4 et = P.etab[(size_t)li * P.NP + e];  // entry_table
		const int gp = et.x, sl = et.y, n = et.w;
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
		const size_t b0 = (size_t)sl * P.BV;
		unsigned flags = 0;
		bool any = false;
		StatusCache sc;
		bool vnext = lane < n;
		int lnext = vnext ? lst[lane] : 0;
		float dnext = vnext ? P.dlt[b0 + lnext] : 0.0f;
		for (int base = 0; base < n; base += 32) {
			const bool valid = vnext;
			const int leaf = lnext;
			const float d = dnext;
			const int jn = base + 32 + lane;
			vnext = jn < n;
			if (vnext) {
				lnext = lst[jn];
				dnext = P.dlt[b0 + lnext];
			}
			int to = 0;
			if (valid) {
				to = layer_id(d, P.err);
				P.phi[b0 + leaf] = d;
			}
			status_chunk<L>(P, gp, sl, k, valid, leaf, to, b, flags, any, sc);
		}
		status_store<L>(P, sl, k, b, sc);
		flags = warp_or(flags);
		if (lane == 0) {
			eflag[e] = flags;
			if (any && !*(volatile int*)P.changed) atomicOr(P.changed, 1);
		}
	}
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_dist2_warp(Dev P, const int* woff, ListView lv, int k, int b)
{
	pdl_enter();
	d_dist2_warp<D, L>(P, woff, lv, k, b, hw_grid(), P.eflag);
}

// ---------------------------------------------------------------------------------------------
// Fused distance passes. update_distance (Surface.hpp:989-1125) runs, per layer in the order
// -1..-L, +1..+L, a first pass (the distance of every leaf of the layer's list into the delta
// grid) and a second pass (the delta into the isogrid, status changes recorded). The first pass
// of layer j only depends on the second pass of layer j-1 through the values it commits, and
// those are the delta values the first pass of j-1 computed. So one launch runs the second pass
// of layer j-1 and the first pass of layer j together, the latter reading the delta value of
// every leaf the pass of j-1 processed (a leaf of that layer's list) and the isogrid elsewhere:
// the same values the reference reads, 2L+1 launches per iteration instead of 4L. The two
// passes touch different leaves (a leaf is in one list), and the compaction of the records of
// layer j-2 rides in the same launch on entry flags of the other parity.
// ---------------------------------------------------------------------------------------------

/// The value the first pass of a layer reads at leaf `leaf` of brick sl when the second pass of
/// the layer before (layer index lip, -1 = none) runs in the same launch: that pass's new value
/// for a leaf in its list (lv's list lip of the brick, found through the lookup), else the
/// isogrid value. The isogrid value is loaded alongside the lookup and discarded for a listed
/// leaf (its commit may be in flight).
template <int L>
__device__ __forceinline__ float fused_value(const Dev& P, const ListView& lv, int lip, int sl,
                                             int leaf)
{
	constexpr int NL = 2 * L + 1;
	const size_t i = (size_t)sl * P.BV + leaf;
	const float v = P.phi[i];
	if (lip < 0) return v;
	const int p = lv.lkp[i];
	if (p == NUL16 || p >= lv.lcnt[sl * NL + lip]) return v;
	if (lv.lst[((size_t)sl * NL + lip) * P.BV + p] != leaf) return v;
	return P.dlt[i];
}

/// distance_leaf with every neighbour read through fused_value (same result as distance() on
/// the values the reference's pass reads).
template <int D, int L>
__device__ __forceinline__ float distance_leaf_fused(const Dev& P, const SurfGeom& g,
                                                     const ListView& lv, int lip, int gp, int sl,
                                                     int leaf, float dist, float dir)
{
	dist = __fmul_rn(dist, dir);
	int q[D];
	Vec<D> pos;
	int rem = leaf;
#pragma unroll
	for (int a = 0; a < D; a++) {
		q[a] = rem / P.lstr[a];
		rem -= q[a] * P.lstr[a];
		pos[a] = P.porig[gp * 3 + a] + q[a];
	}
	Vec<D> n = pos;
#pragma unroll
	for (int a = 0; a < D; a++) {
#pragma unroll
		for (int s = -1; s <= 1; s += 2) {
			n[a] = pos[a] + s;
			if (in_grid<D>(g, n)) {
				const int qa = q[a] + s;
				float v;
				if (qa >= 0 && qa < P.csz[a]) {
					v = fused_value<L>(P, lv, lip, sl, leaf + s * P.lstr[a]);
				} else {
					int gp2, leaf2;
					next_partition<D>(P, g, gp, leaf, a, s, gp2, leaf2);
					const int sl2 = P.slot[gp2];
					v = sl2 < 0 ? P.bg[gp2] : fused_value<L>(P, lv, lip, sl2, leaf2);
				}
				const float dn = __fmul_rn(v, dir);
				if (dn < dist) dist = dn;
			}
		}
		n[a] = pos[a];
	}
	return __fadd_rn(__fmul_rn(dist, dir), dir);
}

/// One pass of the fused sequence: the layer, its entry offsets, nullptr = no such pass.
struct FusedPass {
	const int* woff;
	int k;
};

/// Second pass of layer p2 (records into buffer b, entry flags into ef2) and first pass of
/// layer p1 (side `side`, `split` warps per entry), after the compaction of the pass before p2
/// in the first ca.nblocks blocks. With both passes, the even blocks after those run the
/// second pass and the odd ones the first, so that their chains of dependent loads overlap
/// instead of following each other on the same warps.
template <int D, int L>
__global__ void __launch_bounds__(256) k_dist_fused(Dev P, ListView lv, FusedPass p2, FusedPass p1,
                                                    float side, int split, int b, unsigned* ef2,
                                                    CompactArgs ca, int block_passes)
{
	constexpr int NL = 2 * L + 1;
	pdl_enter();
	if ((int)blockIdx.x < ca.nblocks) {
		compact_surface<L>(P, ca, blockIdx.x);
		return;
	}
	GridPos G{(int)blockIdx.x - ca.nblocks, (int)gridDim.x - ca.nblocks};
	// the layer the first pass reads new values of: the second pass's, in this launch
	const int lip = p2.woff ? p2.k + L : -1;
	const bool both = p2.woff && p1.woff;
	if (both) {
		const bool second = (G.bid & 1) == 0;
		G = GridPos{G.bid >> 1, second ? (G.nb + 1) >> 1 : G.nb >> 1};
		if (!second) p2.woff = nullptr;
	}
	if (p2.woff) {
		if (block_passes)
			d_dist2<D, L>(P, p2.woff, lv, p2.k, b, G, ef2);
		else
			d_dist2_warp<D, L>(P, p2.woff, lv, p2.k, b, G, ef2);
		return;
	}
	if (!p1.woff) return;
	const int li = p1.k + L;
	const int lane = lane_id();
	const int nwarps = (G.nb * blockDim.x) >> 5;
	const int total = p1.woff[P.S] * split;
	unsigned long long done = 0;
	for (int v = (G.bid * blockDim.x + threadIdx.x) >> 5; v < total; v += nwarps) {
		const int e = v / split, part = v - e * split;
		const int4 et = P.etab[(size_t)li * P.NP + e];  // entry_table
		const SurfGeom& g = P.geom[et.z];
		const int gp = et.x, sl = et.y, n = et.w;
		const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
		const size_t b0 = (size_t)sl * P.BV;
		const int STRIDE = 32 * split;
		for (int j = part * 32 + lane; j < n; j += 2 * STRIDE) {
			const bool two = j + STRIDE < n;
			const int l1 = lst[j];
			const int l2 = two ? lst[j + STRIDE] : l1;
			const float q1 = P.phi[b0 + l1], q2 = P.phi[b0 + l2];
			const float d1 = distance_leaf_fused<D, L>(P, g, lv, lip, gp, sl, l1, q1, side);
			const float d2 = distance_leaf_fused<D, L>(P, g, lv, lip, gp, sl, l2, q2, side);
			P.dlt[b0 + l1] = d1;
			if (two) P.dlt[b0 + l2] = d2;
		}
		if (lane == 0 && part == 0) done += n;
	}
	block_add(&P.kstat[KS_DIST], done);
}

// ---------------------------------------------------------------------------------------------
// Tiled distance passes. The 2L passes of update_distance (Surface.hpp:989-1125; layers -1..-L,
// then +1..+L, each a first loop writing distance() of every leaf of the layer's list into the
// delta grid and a second loop committing it) run for one brick at a time in shared memory: the
// block stages the brick with a halo of H = 2L nodes on every side (isogrid values, the list
// each node belongs to), runs every pass over the whole tile, and keeps the brick's own results.
// A node's value after pass m depends on nodes at most m steps away, so after the 2L passes the
// brick's nodes hold exactly what the reference's passes give them; the halo's work is
// redundant (other blocks own those nodes). The status changes of each pass are recorded over
// the brick's own list in list order, as in the untiled second pass; the entry flags of every
// pass go to their own array (Dev::eflagl), and the next launch commits the values and compacts
// the passes' records in pass order. Nothing is written to the isogrid during the passes,
// because other blocks are still staging their halos from it: the results go to the delta grid
// (where the untiled first pass puts them too) and the next launch copies them over.
// ---------------------------------------------------------------------------------------------

/// The staged tile: the brick (partition shape) with a halo of H nodes on every side.
struct TileShape {
	int T[3];   // extent per axis
	int ts[3];  // strides, row-major, last axis fastest
	int NT;     // nodes
	int H;      // halo width
};

/// Dynamic shared memory of k_dist_tiled: values and new values (float), the status-round
/// scratch (int, uint16 per thread) and the list index of every node (byte).
__host__ __device__ inline size_t tiled_smem_bytes(int NT, int threads)
{
	return (size_t)NT * 9 + (size_t)threads * 6 + 16;
}

/// Layer index of the list that holds `leaf` of brick sl (lookup position lk, not NUL16), or
/// 0xFF: the list its value rounds to is tried first, then the others.
template <int L>
__device__ __forceinline__ int tiled_member(const ListView& lv, const int* cnt, int sl, int BV,
                                            int leaf, int lk, float v)
{
	constexpr int NL = 2 * L + 1;
	const float x = __fadd_rn(v, 1.1920928955078125e-07f);
	int h = 0;
	if (isfinite(x)) h = x >= (float)L ? L : x <= (float)-L ? -L : (int)roundf(x);
	const int h0 = h + L;
	if (lk < cnt[h0] && lv.lst[((size_t)sl * NL + h0) * BV + lk] == leaf) return h0;
	for (int l = 0; l < NL; l++)
		if (l != h0 && lk < cnt[l] && lv.lst[((size_t)sl * NL + l) * BV + lk] == leaf) return l;
	return 0xFF;
}

/// One block per queued partition (persistent grid): stage, 2L passes, records per pass.
template <int D, int L>
__global__ void __launch_bounds__(1024, 1) k_dist_tiled(Dev P, ListView lv, int b, TileShape ts)
{
	constexpr int NL = 2 * L + 1;
	constexpr int NN = D == 3 ? 27 : 9;  // the partition and its neighbours, offsets in {-1,0,1}^D
	constexpr int CTR = (NN - 1) / 2;     // the partition itself
	extern __shared__ __align__(16) unsigned char tsm[];
	float* ph = reinterpret_cast<float*>(tsm);
	float* nv = ph + ts.NT;
	int* ct = reinterpret_cast<int*>(nv + ts.NT);
	uint16_t* cl = reinterpret_cast<uint16_t*>(ct + blockDim.x);
	uint8_t* mb = reinterpret_cast<uint8_t*>(cl + blockDim.x);
	__shared__ int nsl[NN];
	__shared__ float nbg[NN];
	__shared__ int ncnt[NN * NL];
	pdl_enter();
	const int nq = P.counters[CNT_DQ];
	const int H = ts.H;
	const float qnan = __int_as_float(0x7fc00000);
	unsigned long long done = 0;
	for (int q = blockIdx.x; q < nq; q += gridDim.x) {
		const int gp = P.dq[q];
		const int sl = P.slot[gp];
		const int s = P.surf_of[gp];
		const SurfGeom& g = P.geom[s];
		__syncthreads();  // the previous partition's shared state is no longer read
		if (threadIdx.x < NN) {
			int lp = gp - g.pbase, r = threadIdx.x, gp2 = gp, cst = 1;
			bool ok = true;
#pragma unroll
			for (int a = D - 1; a >= 0; a--) {
				const int c = lp % g.ccount[a];
				lp /= g.ccount[a];
				const int o = r % 3 - 1;
				r /= 3;
				if (c + o < 0 || c + o >= g.ccount[a]) ok = false;
				gp2 += o * cst;
				cst *= g.ccount[a];
			}
			const int sl2 = ok ? P.slot[gp2] : -2;
			nsl[threadIdx.x] = sl2;
			nbg[threadIdx.x] = (ok && sl2 < 0) ? P.bg[gp2] : 0.0f;
			for (int l = 0; l < NL; l++)
				ncnt[threadIdx.x * NL + l] = sl2 >= 0 ? lv.lcnt[sl2 * NL + l] : 0;
		}
		__syncthreads();
		// stage: value (NaN outside the grid, where distance() reads nothing) and list index
		// (0xFF: none, or a node on the tile's outer face, whose neighbours are not all staged)
		int po[D];
#pragma unroll
		for (int a = 0; a < D; a++) po[a] = P.porig[gp * 3 + a] - H;
		for (int t = threadIdx.x; t < ts.NT; t += blockDim.x) {
			int rem = t, ni = 0, leaf = 0;
			bool in = true, face = false;
#pragma unroll
			for (int a = 0; a < D; a++) {
				const int c = rem / ts.ts[a];
				rem -= c * ts.ts[a];
				const int p = po[a] + c;
				in = in && p >= g.off[a] && p < g.hi[a];
				face = face || c == 0 || c == ts.T[a] - 1;
				const int o = c < H ? -1 : (c >= H + P.csz[a] ? 1 : 0);
				ni = ni * 3 + o + 1;
				leaf += (c - H - o * P.csz[a]) * P.lstr[a];
			}
			float v = qnan;
			int m = 0xFF;
			if (in) {
				const int sl2 = nsl[ni];
				if (sl2 < 0) {
					v = nbg[ni];
				} else {
					const size_t i = (size_t)sl2 * P.BV + leaf;
					v = P.phi[i];
					const int lk = lv.lkp[i];
					if (!face && lk != NUL16)
						m = tiled_member<L>(lv, ncnt + ni * NL, sl2, P.BV, leaf, lk, v);
				}
			}
			ph[t] = v;
			mb[t] = (uint8_t)m;
		}
		__syncthreads();
		const size_t b0 = (size_t)sl * P.BV;
		for (int pm = 0; pm < 2 * L; pm++) {
			const int k = pm < L ? -(pm + 1) : pm - L + 1;
			const int li = k + L;
			const float dir = k < 0 ? -1.0f : 1.0f;
			// first loop: distance() of every member of the layer in the tile (Jacobi)
			for (int t = threadIdx.x; t < ts.NT; t += blockDim.x) {
				if (mb[t] != li) continue;
				float dist = __fmul_rn(ph[t], dir);
#pragma unroll
				for (int a = 0; a < D; a++) {
#pragma unroll
					for (int sg = -1; sg <= 1; sg += 2) {
						const float dn = __fmul_rn(ph[t + sg * ts.ts[a]], dir);
						if (dn < dist) dist = dn;
					}
				}
				nv[t] = __fadd_rn(__fmul_rn(dist, dir), dir);
			}
			__syncthreads();
			// second loop: commit
			for (int t = threadIdx.x; t < ts.NT; t += blockDim.x)
				if (mb[t] == li) ph[t] = nv[t];
			__syncthreads();
			// the brick's own leaves of the layer, in list order: result and status records
			const int pp = lv.ppos[gp * NL + li];
			if (pp < 0) continue;  // block-uniform: the partition is not in this layer's list
			const int n = ncnt[CTR * NL + li];
			const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
			unsigned flags = 0;
			bool any = false;
			StatusCache sc;
			for (int base = 0; base < n; base += blockDim.x) {
				const int j = base + threadIdx.x;
				int leaf = 0, to = k;
				if (j < n) {
					leaf = lst[j];
					int rem = leaf, ti = 0;
#pragma unroll
					for (int a = 0; a < D; a++) {
						const int c = rem / P.lstr[a];
						rem -= c * P.lstr[a];
						ti += (c + H) * ts.ts[a];
					}
					const float d = ph[ti];
					P.dlt[b0 + leaf] = d;
					to = layer_id(d, P.err);
				}
				status_round<L>(P, gp, sl, k, j < n && to != k, leaf, to, b, flags, any, cl, ct,
				                sc);
			}
			if (threadIdx.x < 32) {
				status_store<L>(P, sl, k, b, sc);
				flags = warp_or(flags);
				if (threadIdx.x == 0) {
					const int e = P.woffl[(size_t)li * (P.S + 1) + s] + pp;
					P.eflagl[(size_t)li * P.NP + e] = flags;
					if (any && !*(volatile int*)P.changed) atomicOr(P.changed, 1);
					done += n;
				}
			}
		}
	}
	block_add(&P.kstat[KS_DIST], done);
}

/// After k_dist_tiled: the first P.S blocks compact the records of the pending zero-layer update
/// (`stale`, if any) and of the 2L passes in pass order, one block per surface, a partition
/// joining a buffer list once (dedup: the passes recorded before any of these compactions ran);
/// the other blocks copy the passes' results from the delta grid into the isogrid, a warp per
/// (partition, layer). The last block to finish prepares the expansion (as k_compact's does) and
/// empties the partition queue.
template <int L>
__global__ void __launch_bounds__(256) k_dist_tiled_end(Dev P, ListView lv, int b, CompactArgs stale)
{
	constexpr int NL = 2 * L + 1;
	pdl_enter();
	if ((int)blockIdx.x < P.S) {
		const int s = blockIdx.x;
		if (stale.nblocks) compact_surface<L>(P, stale, s);
		for (int pm = 0; pm < 2 * L; pm++) {
			const int li = (pm < L ? -(pm + 1) : pm - L + 1) + L;
			CompactArgs a{P.S, P.woffl + (size_t)li * (P.S + 1), lv.plist, li, b,
			              P.eflagl + (size_t)li * P.NP};
			a.dedup = 1;
			compact_surface<L>(P, a, s);
		}
	} else {
		const int nq = P.counters[CNT_DQ];
		const int lane = lane_id();
		const int nw = ((gridDim.x - P.S) * blockDim.x) >> 5;
		for (int v = ((blockIdx.x - P.S) * blockDim.x + threadIdx.x) >> 5; v < nq * 2 * L;
		     v += nw) {
			const int q = v / (2 * L), pm = v - q * (2 * L);
			const int li = pm < L ? pm : pm + 1;  // every layer but the zero layer
			const int sl = P.slot[P.dq[q]];
			const int n = lv.lcnt[sl * NL + li];
			const uint16_t* lst = lv.lst + ((size_t)sl * NL + li) * P.BV;
			const size_t b0 = (size_t)sl * P.BV;
			for (int j = lane; j < n; j += 32) {
				const int leaf = lst[j];
				P.phi[b0 + leaf] = P.dlt[b0 + leaf];
			}
		}
	}
	__shared__ int last;
	__syncthreads();
	if (threadIdx.x == 0) {
		__threadfence();
		last = atomicAdd(&P.counters[CNT_CDONE], 1) == (int)gridDim.x - 1;
	}
	__syncthreads();
	if (!last) return;
	__threadfence();
	d_scan_counts(P.spcnt, NL, 0, 1, P.S, P.woff, P.sfrozen, true);
	if (threadIdx.x == 0) {
		P.counters[CNT_ACT] = 0;
		P.counters[CNT_TOUCH] = 0;
		P.counters[CNT_CAND] = 0;
		P.counters[CNT_CDONE] = 0;
		P.counters[CNT_DQ] = 0;
	}
}

// ---------------------------------------------------------------------------------------------
// flush_status_change (Surface.hpp:1183-1244) with Untrack::retrack / untrack
// (PartitionedMixin.hpp:489-558), leaf level: each partition with status changes replays its
// own edits in the reference's order (from-layer ascending, status list order), one thread per
// partition, and records the children-level events for k_flush_plist.
// ---------------------------------------------------------------------------------------------
template <int D, int L>
__device__ void d_flush_leaf(const Dev& P, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	const int n = P.counters[CNT_SUNION];
	unsigned long long done = 0;
	for (int e = G.bid * blockDim.x + threadIdx.x; e < n; e += G.nb * blockDim.x) {
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
			done += edits;
		}
		if (dead) {
			P.oslot[gp] = sl;
			P.slot[gp] = -1;
			P.q_retire[atomicAdd(&P.counters[CNT_RETIRE], 1)] = sl;
		}
	}
	block_add(&P.kstat[KS_FLUSH], done);
}
template <int D, int L>
__global__ void k_flush_leaf(Dev P)
{
	pdl_enter();
	d_flush_leaf<D, L>(P, hw_grid());
}

/// Shared-memory bytes k_flush_smem needs for a brick of BV leaves.
__host__ __device__ inline size_t flush_smem_bytes(int BV, int NL)
{
	(void)NL;
	return (size_t)4 * BV * sizeof(uint16_t) + (size_t)BV + 16;
}

/// k_flush_leaf for one block per partition, touching only what the edits touch. Same results.
///
/// The reference replays the edits one by one: from-layer phases in ascending order, each
/// removing its leaves from list `from` (swap-with-last) and appending the in-band ones to list
/// `to`. A leaf has one status entry, so list t only receives appends in the phases before and
/// after its own removal phase, and those appends land at positions that follow from counts.
/// So every list replays on its own warp: appends of earlier phases (ballot-ordered), its own
/// removal chain (one lane; each swap-with-last removal depends on the previous one), appends of
/// later phases. A list of length n losing m leaves only ever takes its moved entries from its
/// last m slots (the removal window), so only that window is staged in shared memory; every
/// other write goes straight to the brick's list. Leaves appended before the removals are tagged
/// (bit 15) while in the window so that their positions go to a separate lookup (the warp of
/// their old list may still read the old one). A leaf whose status ends where it started
/// (to == from: it changed twice in one iteration) is removed and re-appended within its own
/// phase by the removal lane.
template <int D, int L>
__device__ void d_flush_smem(const Dev& P, GridPos G, unsigned char* fsm)
{
	constexpr int NL = 2 * L + 1;
	constexpr uint16_t TAG = 0x8000u;
	const int BV = P.BV;
	uint16_t* slkp = (uint16_t*)fsm;       // [BV] positions of the leaves the removals touch
	uint16_t* schg = slkp + BV;            // [BV] status entries, phase-major
	uint16_t* snew = schg + BV;            // [BV] positions of leaves appended to another list
	uint16_t* swin = snew + BV;            // [BV] removal window of list t at coff[t]
	int8_t* ssto = (int8_t*)(swin + BV);   // [BV] status "to" of each entry
	__shared__ int cnt[NL], coff[NL + 1], nbef[NL], live0, nout, lastout;
	__shared__ unsigned appb[NL], remb;
	const int n = P.counters[CNT_SUNION];
	const size_t bv = (size_t)BV;
	const int lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	const unsigned lt = (1u << lane) - 1u;
	// The kernel lasts as long as its longest removal chain. Partitions with a long chain go in
	// a first sweep, so that they all start at once; the rest follow.
	constexpr int LONG_CHAIN = 64;
	__shared__ int take;
	unsigned long long done = 0;  // leaf edits replayed (thread 0)
	for (int sweep = 0; sweep < 2; sweep++)
	for (int e = G.bid; e < n; e += G.nb) {
		const int gp = P.q_sunion[e];
		const int sl = P.slot[gp];
		if (threadIdx.x == 0) {
			// sweep 1 finds a partition of sweep 0 already done: skipped by its chain length,
			// or, when it deactivated, by its slot (the status counts are not changed here)
			int mx = 0;
			if (sl >= 0)
				for (int l = 0; l < NL; l++) mx = max(mx, P.ccnt[sl * NL + l]);
			take = sl >= 0 && (mx >= LONG_CHAIN) == (sweep == 0);
		}
		__syncthreads();
		if (!take) {
			__syncthreads();
			continue;
		}
		uint16_t* lkp = P.lkp + sl * bv;
		if (threadIdx.x == 0) {
			int c = 0, lv = 0;
			for (int l = 0; l < NL; l++) {
				cnt[l] = P.lcnt[sl * NL + l];
				lv += cnt[l];
				coff[l] = c;
				c += P.ccnt[sl * NL + l];
			}
			coff[NL] = c;
			live0 = lv;
			nout = 0;
			lastout = -1;
			remb = 0;
		}
		if (threadIdx.x < NL) {
			appb[threadIdx.x] = 0;
			nbef[threadIdx.x] = 0;
		}
		__syncthreads();
		// status entries, the removed leaves' positions, and how many leaves each list receives
		// from earlier phases
		for (int fi = 0; fi < NL; fi++) {
			const uint16_t* src = P.chg + ((size_t)sl * NL + fi) * bv;
			const int nc = coff[fi + 1] - coff[fi];
			for (int c = threadIdx.x; c < nc; c += blockDim.x) {
				const int leaf = src[c];
				const int to = P.sto[sl * bv + leaf];
				schg[coff[fi] + c] = (uint16_t)leaf;
				ssto[coff[fi] + c] = (int8_t)to;
				slkp[leaf] = lkp[leaf];
				if (!inside_band(to, L)) {
					// Untrack (PartitionedMixin.hpp:530-558): the node leaves the band
					P.phi[sl * bv + leaf] = (float)to;
					atomicAdd(&nout, 1);
					atomicMax(&lastout, coff[fi] + c);
				} else if (to + L > fi) {
					atomicAdd(&nbef[to + L], 1);
				}
			}
		}
		__syncthreads();
		// each list's removal window: its original entries there
		for (int t = warp; t < NL; t += nwarps) {
			const int m = coff[t + 1] - coff[t];
			const int w0 = cnt[t] + nbef[t] - m;
			const uint16_t* src = P.lst + ((size_t)sl * NL + t) * bv;
			for (int pos = w0 + lane; pos < cnt[t]; pos += 32) {
				const int x = src[pos];
				swin[coff[t] + pos - w0] = (uint16_t)x;
				slkp[x] = (uint16_t)pos;
			}
		}
		__syncthreads();
		const int total = coff[NL];
		for (int t = warp; t < NL; t += nwarps) {
			uint16_t* lf = P.lst + ((size_t)sl * NL + t) * bv;
			uint16_t* win = swin + coff[t];
			const int m = coff[t + 1] - coff[t];
			int len = cnt[t];
			const int w0 = len + nbef[t] - m;
			// appends to list t from the phases before t
			for (int base = 0; base < coff[t]; base += 32) {
				const int c = base + lane;
				const bool hit = c < coff[t] && ssto[c] + L == t;
				const unsigned msk = __ballot_sync(FULL, hit);
				if (hit) {
					const int pos = len + __popc(msk & lt);
					const int leaf = schg[c];
					if (pos >= w0)
						win[pos - w0] = (uint16_t)(leaf | TAG);
					else
						lf[pos] = (uint16_t)leaf;
					snew[leaf] = (uint16_t)pos;
					if (pos == 0) {
						int f = 0;
						while (c >= coff[f + 1]) f++;
						atomicOr(&appb[f], 1u << t);
					}
				}
				len += __popc(msk);
			}
			__syncwarp();
			// phase t: swap-with-last removals (LookupMixin.hpp:339-371), in order. The next
			// removal's leaf and position are read a step ahead (off the chain's critical path);
			// the position is fixed up when this step moves that very leaf.
			if (lane == 0) {
				const int c0 = coff[t], c1 = coff[t + 1];
				int leaf = c0 < c1 ? schg[c0] : 0;
				int pos = c0 < c1 ? slkp[leaf] : 0;
				for (int c = c0; c < c1; c++) {
					const bool more = c + 1 < c1;
					const int nleaf = more ? schg[c + 1] : 0;
					int npos = more ? slkp[nleaf] : 0;
					const int last = len - 1;
					if (pos < last) {
						const int moved = win[last - w0];
						if (pos >= w0)
							win[pos - w0] = (uint16_t)moved;
						else
							lf[pos] = (uint16_t)(moved & ~TAG);
						if (moved & TAG) {
							snew[moved & ~TAG] = (uint16_t)pos;
						} else {
							slkp[moved] = (uint16_t)pos;
							lkp[moved] = (uint16_t)pos;
							if (more && moved == nleaf) npos = pos;
						}
					}
					slkp[leaf] = NUL16;
					len = last;
					if (last == 0) atomicOr(&remb, 1u << t);
					if (ssto[c] + L == t) {  // back to its own list: re-appended at the end
						win[len - w0] = (uint16_t)leaf;
						slkp[leaf] = (uint16_t)len;
						if (len == 0) atomicOr(&appb[t], 1u << t);
						len++;
					}
					leaf = nleaf;
					pos = npos;
				}
			}
			len = __shfl_sync(FULL, len, 0);
			__syncwarp();
			// what is left of the window (re-appended leaves) joins the list
			for (int pos = w0 + lane; pos < len; pos += 32) lf[pos] = (uint16_t)(win[pos - w0] & ~TAG);
			// appends to list t from the phases after t
			for (int base = coff[t + 1]; base < total; base += 32) {
				const int c = base + lane;
				const bool hit = c < total && ssto[c] + L == t;
				const unsigned msk = __ballot_sync(FULL, hit);
				if (hit) {
					const int pos = len + __popc(msk & lt);
					const int leaf = schg[c];
					lf[pos] = (uint16_t)leaf;
					snew[leaf] = (uint16_t)pos;
					if (pos == 0) {
						int f = 0;
						while (c >= coff[f + 1]) f++;
						atomicOr(&appb[f], 1u << t);
					}
				}
				len += __popc(msk);
			}
			if (lane == 0) cnt[t] = len;
		}
		__syncthreads();
		// the final position of every leaf with a status entry
		for (int c = threadIdx.x; c < total; c += blockDim.x) {
			const int leaf = schg[c];
			const int to = ssto[c];
			int f = 0;
			while (c >= coff[f + 1]) f++;
			lkp[leaf] = !inside_band(to, L) ? NUL16 : (to + L != f ? snew[leaf] : slkp[leaf]);
		}
		if (threadIdx.x < NL) {
			P.app[gp * NL + threadIdx.x] = appb[threadIdx.x];
			P.lcnt[sl * NL + threadIdx.x] = cnt[threadIdx.x];
		}
		if (threadIdx.x == 0) {
			P.rem[gp] = remb;
			done += total;
			if (nout > 0 && nout == live0) {
				// the last leaf left the band: the partition deactivates with the background
				// of that leaf's side (PartitionedMixin.hpp:530-558)
				P.bg[gp] = (float)ssto[lastout];
				P.oslot[gp] = sl;
				P.slot[gp] = -1;
				P.q_retire[atomicAdd(&P.counters[CNT_RETIRE], 1)] = sl;
			}
		}
		__syncthreads();
	}
	block_add(&P.kstat[KS_FLUSH], done);
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_flush_smem(Dev P)
{
	pdl_enter();
	extern __shared__ __align__(16) unsigned char fsm[];
	d_flush_smem<D, L>(P, hw_grid(), fsm);
}

/// Children-level half of the flush, for list k of surface s: replays, in the reference's order
/// (from-layer ascending, then status partition list order), the appends to list k and the
/// swap-with-last removals from it (LookupMixin.hpp:483-556). The events only read the leaf
/// flush's records (app, rem), which this kernel does not change. This is the general path:
/// tiles of the status lists staged in shared memory, events replayed by one lane on the
/// global lists (used when a list has more events than flush_plist_fast stages).
template <int L, int ECAP>
__device__ void flush_plist_serial(const Dev& P, int s, int k, int* slp, unsigned char* sev)
{
	constexpr int NL = 2 * L + 1;
	const int lane = lane_id();
	const SurfGeom& g = P.geom[s];
	int* pl = P.plist + (size_t)k * P.NP + g.pbase;
	int cnt = P.pcnt[s * NL + k];  // kept by warp 0
	for (int fi = 0; fi < NL; fi++) {
		const int ns = P.spcnt[s * NL + fi];
		const int* sp = P.splist + (size_t)fi * P.NP + g.pbase;
		for (int t0 = 0; t0 < ns; t0 += ECAP) {
			const int nt = min(ECAP, ns - t0);
			__syncthreads();
			for (int i = threadIdx.x; i < nt; i += blockDim.x) {
				const int lp = sp[t0 + i];
				const int gp = g.pbase + lp;
				unsigned char ev;
				if (fi == k)
					ev = ((P.rem[gp] >> k) & 1u) ? 2 : 0;
				else
					ev = ((P.app[gp * NL + fi] >> k) & 1u) ? 1 : 0;
				slp[i] = lp;
				sev[i] = ev;
			}
			__syncthreads();
			if (threadIdx.x >= 32) continue;
			for (int base = 0; base < nt; base += 32) {
				const int i = base + lane;
				const int ev0 = i < nt ? sev[i] : 0;
				unsigned m = __ballot_sync(FULL, ev0 != 0);
				while (m) {
					const int src = __ffs(m) - 1;
					m &= m - 1;
					if (lane == 0) {
						const int lp = slp[base + src];
						const int ev = sev[base + src];
						const int gp = g.pbase + lp;
						int* at = &P.ppos[gp * NL + k];
						if (ev == 1) {
							if (*at < 0) {
								pl[cnt] = lp;
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
	}
	if (threadIdx.x == 0) P.pcnt[s * NL + k] = cnt;
	__syncthreads();
}

/// Open-addressing map in shared memory from a partition's local index to its position in the
/// list being replayed (-1: not in it); keys -1 = empty slot. Returns the key's slot, or the
/// empty slot that ends its probe when it is absent (the map is never full).
template <int HCAP>
__device__ __forceinline__ int plist_slot(const int* hkey, int lp)
{
	int h = (int)(((unsigned)lp * 2654435761u) >> 20) & (HCAP - 1);
	while (hkey[h] != lp && hkey[h] != -1) h = (h + 1) & (HCAP - 1);
	return h;
}

/// flush_plist_serial with every event's lookups in shared memory. A list of length n that
/// loses at most R entries only ever moves entries from positions >= n - R (each swap-with-last
/// removal takes the current last entry, and the list is longer than n - R before each of its
/// removals), so only that window and the appended entries are staged; entries below it are
/// overwritten at most, never read. The positions of the window's and the events' partitions
/// live in a map in shared memory while one lane replays the events in order; the window and
/// the positions are written back after. Returns false, having changed nothing, when the list
/// has more than ECAP events (flush_plist_serial replays it then).
template <int L, int ECAP, int HCAP>
__device__ bool flush_plist_fast(const Dev& P, int s, int k, int* ev_lp, unsigned char* ev_kind,
                                 int* wnd, int* hkey, int* hval)
{
	constexpr int NL = 2 * L + 1;
	constexpr int PER = 8;  // status entries per thread per round, loaded together
	__shared__ int fo[NL + 1], nev_s, nrem_s;
	const SurfGeom& g = P.geom[s];
	int* pl = P.plist + (size_t)k * P.NP + g.pbase;
	const int cnt0 = P.pcnt[s * NL + k];
	if (threadIdx.x == 0) {
		int c = 0;
		for (int fi = 0; fi < NL; fi++) {
			fo[fi] = c;
			c += P.spcnt[s * NL + fi];
		}
		fo[NL] = c;
		nev_s = 0;
		nrem_s = 0;
	}
	for (int h = threadIdx.x; h < HCAP; h += blockDim.x) hkey[h] = -1;
	__syncthreads();
	// 1. the events in replay order: the status lists concatenated in from-layer order
	const int T = fo[NL];
	for (int base = 0; base < T; base += blockDim.x * PER) {
		int lp[PER];
		unsigned char ev[PER];
		int c = 0;
#pragma unroll
		for (int q = 0; q < PER; q++) {
			const int t = base + threadIdx.x * PER + q;
			ev[q] = 0;
			lp[q] = 0;
			if (t < T) {
				int fi = 0;
				while (t >= fo[fi + 1]) fi++;
				lp[q] = P.splist[(size_t)fi * P.NP + g.pbase + (t - fo[fi])];
				const int gp = g.pbase + lp[q];
				if (fi == k)
					ev[q] = ((P.rem[gp] >> k) & 1u) ? 2 : 0;
				else
					ev[q] = ((P.app[gp * NL + fi] >> k) & 1u) ? 1 : 0;
				c += ev[q] != 0;
			}
		}
		int tot;
		const int off = nev_s + block_excl_scan(c, &tot);
		int r = 0;
#pragma unroll
		for (int q = 0; q < PER; q++)
			if (ev[q]) {
				if (off + r < ECAP) {
					ev_lp[off + r] = lp[q];
					ev_kind[off + r] = ev[q];
				}
				r++;
				if (ev[q] == 2) atomicAdd(&nrem_s, 1);
			}
		__syncthreads();
		if (threadIdx.x == 0) nev_s += tot;
		__syncthreads();
	}
	const int nev = nev_s;
	if (nev > ECAP) return false;
	if (nev == 0) return true;
	// 2. the removal window and the positions of its and the events' partitions
	const int w0 = max(0, cnt0 - nrem_s);
	for (int i = threadIdx.x; i < cnt0 - w0; i += blockDim.x) {
		const int lp = pl[w0 + i];
		wnd[i] = lp;
		int h = (int)(((unsigned)lp * 2654435761u) >> 20) & (HCAP - 1);
		while (true) {
			const int prev = atomicCAS(&hkey[h], -1, lp);
			if (prev == -1) {
				hval[h] = w0 + i;
				break;
			}
			if (prev == lp) break;
			h = (h + 1) & (HCAP - 1);
		}
	}
	__syncthreads();
	for (int j = threadIdx.x; j < nev; j += blockDim.x) {
		const int lp = ev_lp[j];
		int h = (int)(((unsigned)lp * 2654435761u) >> 20) & (HCAP - 1);
		while (true) {
			const int prev = atomicCAS(&hkey[h], -1, lp);
			if (prev == -1) {
				hval[h] = P.ppos[(g.pbase + lp) * NL + k];
				break;
			}
			if (prev == lp) break;  // a window entry, or another event of the same partition
			h = (h + 1) & (HCAP - 1);
		}
	}
	__syncthreads();
	// 3. the replay, in order, on one lane
	if (threadIdx.x == 0) {
		int len = cnt0;
		for (int j = 0; j < nev; j++) {
			const int lp = ev_lp[j];
			const int h = plist_slot<HCAP>(hkey, lp);
			if (hkey[h] != lp) {  // every event's partition was entered above
				atomicOr(P.err, EB_CAPACITY);
				continue;
			}
			const int pos = hval[h];
			if (ev_kind[j] == 1) {
				if (pos < 0) {
					wnd[len - w0] = lp;
					hval[h] = len;
					len++;
				}
			} else if (pos >= 0) {
				const int last = len - 1;
				if (pos < last) {
					const int mv = wnd[last - w0];
					if (pos >= w0)
						wnd[pos - w0] = mv;
					else
						pl[pos] = mv;
					const int hm = plist_slot<HCAP>(hkey, mv);
					if (hkey[hm] == mv)  // window and appended entries are all in the map
						hval[hm] = pos;
					else
						atomicOr(P.err, EB_CAPACITY);
				}
				hval[h] = -1;
				len = last;
			}
		}
		nev_s = len;
	}
	__syncthreads();
	// 4. the window back, and the positions of every partition the replay saw
	const int len = nev_s;
	for (int i = threadIdx.x; i < len - w0; i += blockDim.x) pl[w0 + i] = wnd[i];
	for (int h = threadIdx.x; h < HCAP; h += blockDim.x)
		if (hkey[h] >= 0) P.ppos[(g.pbase + hkey[h]) * NL + k] = hval[h];
	if (threadIdx.x == 0) P.pcnt[s * NL + k] = len;
	__syncthreads();
	return true;
}

/// Children-level half of the flush: a block per (surface, list k), looping over pairs
/// w = bid, bid + nb, ... Warp 0 first checks 32 of the block's pairs at once for events (the
/// surface's status lists non-empty); the block then replays only those, so that the pairs of a
/// large batch's converged surfaces cost one load each.
template <int L>
__device__ void d_flush_plist(const Dev& P, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	constexpr int ECAP = 1024, HCAP = 4096;
	__shared__ int ev_lp[ECAP];
	__shared__ unsigned char ev_kind[ECAP];
	__shared__ int wnd[ECAP];
	__shared__ int hkey[HCAP];
	__shared__ int hval[HCAP];
	__shared__ unsigned busy_s;
	const int npairs = P.S * NL;
	for (int j0 = 0; G.bid + j0 * G.nb < npairs; j0 += 32) {
		if (threadIdx.x < 32) {
			const int w = G.bid + (j0 + (int)threadIdx.x) * G.nb;
			int T = 0;
			if (w < npairs) {
				const int s = w / NL;
				for (int fi = 0; fi < NL; fi++) T += P.spcnt[s * NL + fi];
			}
			const unsigned m = __ballot_sync(FULL, T != 0);
			if (threadIdx.x == 0) busy_s = m;
		}
		__syncthreads();
		unsigned m = busy_s;
		__syncthreads();
		while (m) {
			const int i = __ffs(m) - 1;
			m &= m - 1;
			const int w = G.bid + (j0 + i) * G.nb;
			const int s = w / NL, k = w - s * NL;
			if (!flush_plist_fast<L, ECAP, HCAP>(P, s, k, ev_lp, ev_kind, wnd, hkey, hval))
				flush_plist_serial<L, ECAP>(P, s, k, ev_lp, ev_kind);
		}
	}
}
template <int L>
__global__ void __launch_bounds__(1024) k_flush_plist(Dev P)
{
	pdl_enter();
	d_flush_plist<L>(P, hw_grid());
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
__device__ void d_expand_gen(const Dev& P, int mode, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	// Modes 1 and 2 take the candidates that mode 0 recorded, one thread each, unless there
	// were more than the buffer holds: then they walk the status lists like mode 0.
	const int ncand = P.counters[CNT_CAND];
	if (mode > 0 && ncand <= P.cand_cap) {
		for (int i = G.bid * blockDim.x + threadIdx.x; i < ncand; i += G.nb * blockDim.x) {
			const unsigned long long key = P.cand_key[i];
			const int gpn = P.cand_gp[i], leafn = P.cand_leaf[i];
			const int sn = P.slot[gpn];
			if (sn < 0) {
				atomicOr(P.err, EB_POOL);
				continue;
			}
			unsigned long long* cl = &P.claim[(size_t)sn * P.BV + leafn];
			if (mode == 1) {
				// the first claim of a leaf lists it for the append
				if (atomicMin(cl, key) == NOCLAIM)
					P.ccl[(size_t)sn * P.BV + atomicAdd(&P.ccln[sn], 1)] = (uint16_t)leafn;
				// most candidates of a brick find it touched already: a read first keeps them
				// off the one word's atomic queue
				if (*(volatile int*)&P.touched[sn] == 0 && atomicExch(&P.touched[sn], 1) == 0)
					P.q_touch[atomicAdd(&P.counters[CNT_TOUCH], 1)] = sn;
			} else if (*cl == key) {
				const SurfGeom& g = P.geom[P.surf_of[gpn]];
				const float side = ((key >> 43) & 1ull) ? 1.0f : -1.0f;
				const float v = P.phi[(size_t)sn * P.BV + leafn];
				P.dlt[(size_t)sn * P.BV + leafn] =
				    distance<D, L>(P, g, leaf_pos<D>(P, gpn, leafn), v, side);
			}
		}
		return;
	}
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
		const unsigned lt = (1u << lane) - 1u;
		// whole-warp rounds, so that the candidate slots are taken with one atomic per warp
		for (int c0 = 0; c0 < nc; c0 += 32) {
			const int c = c0 + lane;
			const int leaf = c < nc ? ch[c] : 0;
			const bool src = c < nc && P.sto[(size_t)sl * P.BV + leaf] == want;
			int qd[D];
			Vec<D> pos;
			{
				int rem = leaf;
#pragma unroll
				for (int a = 0; a < D; a++) {
					qd[a] = rem / P.lstr[a];
					rem -= qd[a] * P.lstr[a];
					pos[a] = P.porig[gp * 3 + a] + qd[a];
				}
			}
#pragma unroll
			for (int nb = 0; nb < 2 * D; nb++) {
				const int ax = nb >> 1, sg = (nb & 1) ? 1 : -1;
				Vec<D> q = pos;
				q[ax] += sg;
				bool cand = false;
				int gpn = 0, leafn = 0;
				float v = 0.0f;
				if (src && in_grid<D>(g, q)) {
					// the neighbour in this partition or the next one along the axis; the value
					// get_phi reads there
					const int qa = qd[ax] + sg;
					if (qa >= 0 && qa < P.csz[ax]) {
						gpn = gp;
						leafn = leaf + sg * P.lstr[ax];
					} else {
						next_partition<D>(P, g, gp, leaf, ax, sg, gpn, leafn);
					}
					const int sv = P.slot[gpn];
					v = sv < 0 ? P.bg[gpn] : P.phi[(size_t)sv * P.BV + leafn];
					cand = !inside_band(layer_id(v, P.err), L);
				}
				// key: phase (1 bit) | rank (24) | position in status list (16) | neighbour (3)
				const unsigned long long key = ((unsigned long long)phase << 43) |
				                               ((unsigned long long)rank << 19) |
				                               ((unsigned long long)c << 3) | (unsigned long long)nb;
				if (mode == 0) {
					const unsigned m = __ballot_sync(FULL, cand);
					if (!m) continue;
					const int ldr = __ffs(m) - 1;
					int base = 0;
					if (lane == ldr) base = atomicAdd(&P.counters[CNT_CAND], __popc(m));
					base = __shfl_sync(FULL, base, ldr);
					if (cand) {
						if (P.slot[gpn] < 0 && atomicExch(&P.actflag[gpn], 1) == 0)
							P.q_act[atomicAdd(&P.counters[CNT_ACT], 1)] = gpn;
						const int ci = base + __popc(m & lt);
						if (ci < P.cand_cap) {
							P.cand_key[ci] = key;
							P.cand_gp[ci] = gpn;
							P.cand_leaf[ci] = leafn;
						}
					}
				} else if (cand) {
					const int sn = P.slot[gpn];
					if (sn < 0) {
						atomicOr(P.err, EB_POOL);
						continue;
					}
					unsigned long long* cl = &P.claim[(size_t)sn * P.BV + leafn];
					if (mode == 1) {
						if (atomicMin(cl, key) == NOCLAIM)
							P.ccl[(size_t)sn * P.BV + atomicAdd(&P.ccln[sn], 1)] =
							    (uint16_t)leafn;
						if (*(volatile int*)&P.touched[sn] == 0 &&
						    atomicExch(&P.touched[sn], 1) == 0)
							P.q_touch[atomicAdd(&P.counters[CNT_TOUCH], 1)] = sn;
					} else if (*cl == key) {
						P.dlt[(size_t)sn * P.BV + leafn] = distance<D, L>(P, g, q, v, (float)side);
					}
				}
			}
		}
	}
}
template <int D, int L>
__global__ void __launch_bounds__(256) k_expand_gen(Dev P, int mode)
{
	pdl_enter();
	d_expand_gen<D, L>(P, mode, hw_grid());
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
	if (tid == 0) P.ccln[sl] = 0;
}

/// Child activation (TrackedMixin.hpp:37-41) of queued partitions: one block per partition.
template <int L>
__device__ void d_activate(const Dev& P, GridPos G)
{
	__shared__ int sl;
	const int n = P.counters[CNT_ACT];
	for (int q = G.bid; q < n; q += G.nb) {
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
template <int L>
__global__ void k_activate(Dev P)
{
	pdl_enter();
	d_activate<L>(P, hw_grid());
}

/// Appends each touched brick's claimed nodes to its outermost lists in claim-key order (the
/// reference's sequential track order) and records the partition's first key per side for the
/// children-level append. One block per touched brick; keys sorted in shared memory.
template <int L>
__device__ void d_expand_append(const Dev& P, GridPos G, unsigned long long* sk)
{
	constexpr int NL = 2 * L + 1;
	__shared__ int n0, base0, base1;
	const int n = P.counters[CNT_TOUCH];
	const size_t bv = (size_t)P.BV;
	for (int q = G.bid; q < n; q += G.nb) {
		const int sl = P.q_touch[q];
		const int gp = P.slot_gp[sl];
		// the brick's claimed leaves, listed by their first claims (no scan of every claim key)
		const int m = P.ccln[sl];
		for (int i = threadIdx.x; i < m; i += blockDim.x) {
			const int leaf = P.ccl[sl * bv + i];
			const unsigned long long k = P.claim[sl * bv + leaf];
			// keys use 44 bits; the leaf is packed below them.
			sk[i] = (k << 16) | (unsigned long long)leaf;
			P.claim[sl * bv + leaf] = NOCLAIM;
		}
		__syncthreads();
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
			P.ccln[sl] = 0;
		}
		__syncthreads();
	}
}
template <int L>
__global__ void k_expand_append(Dev P)
{
	pdl_enter();
	extern __shared__ unsigned long long sk[];
	d_expand_append<L>(P, hw_grid(), sk);
}

/// Children-level appends of the expansion (track_child of PartitionedMixin.hpp:201-213, in
/// first-claim order). One block per surface; entries ranked by key.
template <int L>
__device__ void d_expand_plist(const Dev& P, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	for (int s = G.bid; s < P.S; s += G.nb) {
	const int m = P.papn[s];
	if (m == 0) continue;
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
	__syncthreads();
	}
}
template <int L>
__global__ void k_expand_plist(Dev P)
{
	pdl_enter();
	d_expand_plist<L>(P, hw_grid());
}

// ---------------------------------------------------------------------------------------------
// Resets between iterations
// ---------------------------------------------------------------------------------------------

/// status_change grid reset (Reset::MultiList::reset, PartitionedMixin.hpp:336-360).
template <int L>
__device__ void d_clear_status(const Dev& P, GridPos G)
{
	constexpr int NL = 2 * L + 1;
	const int n = P.counters[CNT_SUNION];
	const int lane = lane_id();
	const int nwarps = (G.nb * blockDim.x) >> 5;
	for (int e = (G.bid * blockDim.x + threadIdx.x) >> 5; e < n; e += nwarps) {
		const int gp = P.q_sunion[e];
		const int sl = P.slot[gp];
		if (sl >= 0) {
			// every from-layer's count at once (lane fi), then the status lists' leaves as one
			// flat range, so that the loads of all the lists are in flight together
			const int c = lane < NL ? P.ccnt[sl * NL + lane] : 0;
			int inc = c;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const int y = __shfl_up_sync(FULL, inc, o);
				if (lane >= o) inc += y;
			}
			const int tot = __shfl_sync(FULL, inc, NL - 1);
			int exf[NL];  // first flat index of from-layer f
#pragma unroll
			for (int f = 0; f < NL; f++) exf[f] = __shfl_sync(FULL, inc - c, f);
			for (int i = lane; i < tot; i += 32) {
				int fi = 0;
#pragma unroll
				for (int f = 1; f < NL; f++)
					if (exf[f] <= i) fi = f;
				const uint16_t* ch = P.chg + ((size_t)sl * NL + fi) * P.BV;
				P.sto[(size_t)sl * P.BV + ch[i - exf[fi]]] = (int8_t)(L + 1);
			}
			__syncwarp();
			if (lane < NL) P.ccnt[sl * NL + lane] = 0;
		}
		if (lane < NL) P.sppos[gp * NL + lane] = -1;
		if (lane == 0) P.sflag[gp] = 0;
	}
}
template <int L>
__global__ void k_clear_status(Dev P)
{
	constexpr int NL = 2 * L + 1;
	pdl_enter();
	d_clear_status<L>(P, hw_grid());
	if (!last_block(&P.counters[CNT_LDONE])) return;
	for (int i = threadIdx.x; i < P.S * NL; i += blockDim.x) P.spcnt[i] = 0;
	if (threadIdx.x == 0) P.counters[CNT_SUNION] = 0;
}

/// The entries of the distance passes decoded once per iteration, and Dev::changed cleared for
/// the passes: for every layer but the zero layer and every entry e of its list (entry offsets
/// woffl), {partition, brick slot, surface, leaves in the brick's list} at etab[l*NP + e]. The
/// passes then start from one 16-byte load instead of the chain entry offsets -> partition
/// list -> slot -> list count.
///
/// pcnt given (a pool of at most kScanHereMax surfaces): the entry offsets are scanned here too,
/// every block for itself into dynamic shared memory (NL*(S+1) ints) and block 0 for the passes
/// (Dev::woffl), in place of k_scan_layers.
///
/// clear_status: the iteration's status reset (k_clear_status's work, the status lists of the
/// previous iteration) runs here too; nothing this kernel reads is status data.
///
/// dq given (tiled distance passes, ppos the lists' partition positions): every partition of the
/// passes is queued once, at its entry in the lowest layer index whose list holds it, and every
/// entry's flags (Dev::eflagl) start at zero.
template <int L>
__global__ void k_entry_table(Dev P, const int* plist, const int* lcnt, const int* pcnt,
                              const int* ppos, int* dq, int clear_status)
{
	constexpr int NL = 2 * L + 1;
	extern __shared__ int swoff[];  // the offsets, when scanned here
	__shared__ int lo[NL + 1];      // the layers' entries concatenated: layer l from lo[l]
	pdl_enter();
	// the passes' status-change flag starts at zero (nothing before the passes reads it)
	if (blockIdx.x == 0 && threadIdx.x == 0) *P.changed = 0;
	if (clear_status) d_clear_status<L>(P, hw_grid());
	const int* woffl = P.woffl;
	if (pcnt) {
		d_scan_layers(pcnt, NL, P.S, swoff, P.sfrozen);
		if (blockIdx.x == 0)
			for (int i = threadIdx.x; i < NL * (P.S + 1); i += blockDim.x) P.woffl[i] = swoff[i];
		woffl = swoff;
	}
	if (threadIdx.x == 0) {
		int c = 0;
		for (int l = 0; l < NL; l++) {
			lo[l] = c;
			if (l != L) c += woffl[(size_t)l * (P.S + 1) + P.S];
		}
		lo[NL] = c;
	}
	__syncthreads();
	const int total = lo[NL];
	for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
		int l = 0;
		while (t >= lo[l + 1]) l++;
		const int e = t - lo[l];
		const int* woff = woffl + (size_t)l * (P.S + 1);
		const int s = entry_surface(woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		const int gp = g.pbase + plist[(size_t)l * P.NP + g.pbase + (e - woff[s])];
		const int sl = P.slot[gp];
		P.etab[(size_t)l * P.NP + e] = make_int4(gp, sl, s, lcnt[sl * NL + l]);
		if (dq) {
			P.eflagl[(size_t)l * P.NP + e] = 0;
			bool first = true;
			for (int l2 = 0; l2 < l; l2++)
				if (l2 != L && ppos[gp * NL + l2] >= 0) first = false;
			if (first) dq[atomicAdd(&P.counters[CNT_DQ], 1)] = gp;
		}
	}
	if (clear_status && last_block(&P.counters[CNT_LDONE])) {
		for (int i = threadIdx.x; i < P.S * NL; i += blockDim.x) P.spcnt[i] = 0;
		if (threadIdx.x == 0) P.counters[CNT_SUNION] = 0;
	}
}

/// Affected buffer reset: clears the leaf lookups and lists of buffer b.
template <int L>
__device__ void d_clear_buffer(const Dev& P, int b, GridPos G, const int* woff)
{
	constexpr int NL = 2 * L + 1;
	FG_WARP_LOOP(woff)
	{
		const int s = entry_surface(woff, P.S, e);
		const SurfGeom& g = P.geom[s];
		// the list t of entry e: the surface's list counts loaded at once (lane t) and summed
		// with shuffles, instead of one dependent load per list passed
		const int i0 = e - woff[s];
		const int cl = lane < NL ? P.apcnt[b][s * NL + lane] : 0;
		int inc = cl;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(FULL, inc, o);
			if (lane >= o) inc += y;
		}
		const unsigned past = __ballot_sync(FULL, lane < NL && inc <= i0);
		const int t = __popc(past);  // lists that end at or before i0
		const int i = i0 - __shfl_sync(FULL, inc - cl, t < NL ? t : NL - 1);
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
static __device__ __forceinline__ void d_retire(const Dev& P, GridPos G)
{
	const int n = P.counters[CNT_RETIRE];
	for (int e = G.bid * blockDim.x + threadIdx.x; e < n; e += G.nb * blockDim.x) {
		const int sl = P.q_retire[e];
		const int gp = P.slot_gp[sl];
		if (P.oslot[gp] == sl) P.oslot[gp] = -1;
		P.slot_gp[sl] = -1;
		P.free_stack[atomicAdd(&P.counters[CNT_FREE_TOP], 1)] = sl;
	}
}
/// The tail of an iteration after the expansion: its partition-list appends (d_expand_plist,
/// which touch no brick of the retire queue) and the brick retirement, in one launch.
template <int L>
__global__ void k_retire(Dev P)
{
	pdl_enter();
	d_expand_plist<L>(P, hw_grid());
	d_retire(P, hw_grid());
	if (last_block(&P.counters[CNT_LDONE]) && threadIdx.x == 0) P.counters[CNT_RETIRE] = 0;
}

/// The affected buffer reset (d_clear_buffer). scan_here (a pool of at most kScanHereMax
/// surfaces): every block scans the buffer's entry offsets itself into dynamic shared memory
/// (S+1 ints), in place of a k_scan_counts launch before. retire_too: the iteration's
/// expansion partition appends and brick retirement (k_retire's work, which touches no buffer
/// data) run here too. The last block resets the buffer's partition counts (and the retire
/// queue).
template <int L>
__global__ void k_clear_buffer(Dev P, int b, int scan_here, int retire_too)
{
	constexpr int NL = 2 * L + 1;
	extern __shared__ int swoff[];
	pdl_enter();
	if (retire_too) {
		d_expand_plist<L>(P, hw_grid());
		d_retire(P, hw_grid());
	}
	const int* woff = P.woff;
	if (scan_here) {
		d_scan_counts(P.apcnt[b], NL, 0, 2, P.S, swoff, P.sfrozen);
		woff = swoff;
	}
	d_clear_buffer<L>(P, b, hw_grid(), woff);
	if (!last_block(&P.counters[CNT_LDONE])) return;
	for (int i = threadIdx.x; i < P.S * NL; i += blockDim.x) P.apcnt[b][i] = 0;
	if (retire_too && threadIdx.x == 0) P.counters[CNT_RETIRE] = 0;
}

/// Copies the isogrid partition lists to the delta partition lists (track_children of the
/// delta grid at update start, Surface.hpp:261 / PartitionedMixin.hpp:319-334, which mirrors
/// the isogrid lists into the freshly reset delta lists). Grid y = s*NL + l.
static __device__ __forceinline__ void d_copy_plists(const Dev& P, int NL, GridPos G)
{
	for (int w = G.bid; w < P.S * NL; w += G.nb) {
		const int s = w / NL, l = w % NL;
		const SurfGeom& g = P.geom[s];
		const int n = P.pcnt[s * NL + l];
		const size_t o = (size_t)l * P.NP + g.pbase;
		for (int i = threadIdx.x; i < n; i += blockDim.x) P.dplist[o + i] = P.plist[o + i];
		if (threadIdx.x == 0) P.dpcnt[s * NL + l] = n;
	}
}
static __global__ void k_copy_plists(Dev P, int NL)
{
	pdl_enter();
	// one block per (surface, list): grid (1, S*NL)
	d_copy_plists(P, NL, GridPos{(int)blockIdx.y, (int)gridDim.y});
}

/// Narrow-band size: sum over all isogrid lists of the leaf counts (64-bit accumulator).
template <int L>
__device__ void d_band_size(const Dev& P, unsigned long long* acc, GridPos G)
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
		if (lane == 0) {
			const unsigned long long n = (unsigned long long)P.lcnt[P.slot[gp] * NL + t];
			local += n;
			if (n) atomicAdd(&P.snu[s], n);
		}
	}
	if (lane_id() == 0 && local) atomicAdd(acc, local);
}
template <int L>
__global__ void k_band_size(Dev P, unsigned long long* acc)
{
	pdl_enter();
	d_band_size<L>(P, acc, hw_grid());
}

/// Makes surface s empty, with geometry ng (its partition range at pbase holds npcap
/// partitions, ng.np of them used): every brick it holds goes back to the pool's free stack and
/// every partition-level entry of the range returns to its state in a new pool (inactive,
/// background L+1, in no list), so that a seed then starts it exactly as a new Surface. The
/// world origins of the used partitions are recomputed for the new grid. Serving reuses a
/// finished request's surface this way for the next request.
template <int D, int L>
__global__ void k_reset_surface(Dev P, int s, SurfGeom ng, int npcap)
{
	constexpr int NL = 2 * L + 1;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npcap; i += gridDim.x * blockDim.x) {
		const int gp = ng.pbase + i;
		const int sl = P.slot[gp];
		if (sl >= 0) {
			P.slot_gp[sl] = -1;
			P.touched[sl] = 0;
			P.free_stack[atomicAdd(&P.counters[CNT_FREE_TOP], 1)] = sl;
		}
		P.slot[gp] = -1;
		P.bg[gp] = (float)(L + 1);
		P.oslot[gp] = -1;
		P.actflag[gp] = 0;
		P.sflag[gp] = 0;
		for (int l = 0; l < NL; l++) {
			const size_t k = (size_t)gp * NL + l;
			P.ppos[k] = -1;
			P.sppos[k] = -1;
			P.appos[0][k] = -1;
			P.appos[1][k] = -1;
			P.apkey[k] = NOCLAIM;
		}
		if (i < ng.np) {
			int r = i, c[3] = {0, 0, 0};
			for (int a = D - 1; a >= 0; a--) {
				c[a] = r % ng.ccount[a];
				r /= ng.ccount[a];
			}
			int* po = const_cast<int*>(P.porig) + (size_t)gp * 3;
			for (int a = 0; a < 3; a++) po[a] = a < D ? c[a] * P.csz[a] + ng.off[a] : 0;
		}
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		const_cast<SurfGeom*>(P.geom)[s] = ng;
		for (int l = 0; l < NL; l++) {
			P.pcnt[s * NL + l] = 0;
			P.dpcnt[s * NL + l] = 0;
			P.spcnt[s * NL + l] = 0;
			P.apcnt[0][s * NL + l] = 0;
			P.apcnt[1][s * NL + l] = 0;
		}
		P.papn[s] = 0;
		P.ndp[s] = 0;
		P.snu[s] = 0;
	}
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

template <int D, int L>
__device__ void seed_one(const Dev& P, int s, Vec<D> centre);

/// seed (Surface.hpp:207-241) executed by one thread: the window walk and its track calls are
/// sequential in the reference and set the initial list orders.
template <int D, int L>
__global__ void k_seed(Dev P, int s, Vec<D> centre)
{
	seed_one<D, L>(P, s, centre);
}

/// One seed per surface of the pool (centres[s*D..]), one thread per surface: surfaces share
/// no list state, only the brick allocator, which is atomic.
template <int D, int L>
__global__ void k_seed_all(Dev P, const int* centres)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= P.S) return;
	Vec<D> c;
	for (int a = 0; a < D; a++) c[a] = centres[s * D + a];
	seed_one<D, L>(P, s, c);
}

template <int D, int L>
__device__ void seed_one(const Dev& P, int s, Vec<D> centre)
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

// ---------------------------------------------------------------------------------------------
// Local update: update_start / delta / update_end (Surface.hpp:393-459, 404-430, 780-913).
// The delta() calls and calc_affected's ring growth are sequential in the reference and define
// list orders, so they run on one thread; everything after reuses the parallel passes.
// ---------------------------------------------------------------------------------------------

/// Partitioned::Lookup::track (PartitionedMixin.hpp:388-413) into affected buffer b: the
/// partition joins list t on first use, the leaf joins it unless already in a list.
template <int L>
__device__ void a_track(const Dev& P, int b, const SurfGeom& g, int s, int gp, int sl, int leaf,
                        int t)
{
	constexpr int NL = 2 * L + 1;
	if (P.appos[b][gp * NL + t] < 0) {
		const int c = P.apcnt[b][s * NL + t];
		P.aplist[b][(size_t)t * P.NP + g.pbase + c] = gp - g.pbase;
		P.appos[b][gp * NL + t] = c;
		P.apcnt[b][s * NL + t] = c + 1;
	}
	const size_t k = (size_t)sl * P.BV + leaf;
	if (P.alkp[b][k] == NUL16) {
		const int c = P.acnt[b][sl * NL + t];
		P.alst[b][((size_t)sl * NL + t) * P.BV + c] = (uint16_t)leaf;
		P.alkp[b][k] = (uint16_t)c;
		P.acnt[b][sl * NL + t] = c + 1;
	}
}

/// The delta(pos, val) calls (Surface.hpp:441-459) and the first step of calc_affected
/// (Surface.hpp:788-799), which tracks exactly those leaves, in call order, into affected buffer
/// 0's zero-layer lists: the delta grid's zero-layer lists are therefore the prefixes of the
/// affected zero-layer lists recorded in dlcnt / ndp. In parallel, with the call index as the
/// order key (see the ring kernels below): a leaf, and a partition's zero-layer list entry, are
/// claimed at their first call; k_ring_append / k_ring_plist then append them in call order.
/// Calls at positions outside the grid or in inactive partitions set the error bit and do
/// nothing, as the sequential loop does.
template <int D>
__device__ __forceinline__ bool seed_locate(const Dev& P, const SurfGeom& g, const int* pos, int i,
                                            int& gp, int& sl, int& leaf, bool flag)
{
	Vec<D> p;
	for (int a = 0; a < D; a++) p[a] = pos[i * D + a];
	if (!in_grid<D>(g, p)) {
		if (flag) atomicOr(P.err, EB_OUTSIDE);
		return false;
	}
	locate<D>(P, g, p, gp, leaf);
	sl = P.slot[gp];
	if (sl < 0) {
		if (flag) atomicOr(P.err, EB_INACTIVE);
		return false;
	}
	return true;
}

template <int D, int L>
__global__ void k_seed_claim(Dev P, int s, const int* pos, int n)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		int gp, sl, leaf;
		if (!seed_locate<D>(P, g, pos, i, gp, sl, leaf, true)) continue;
		const unsigned long long key = (unsigned long long)i;
		const int pe = gp * NL + L;
		if (P.appos[0][pe] < 0 && atomicMin(&P.apkey[pe], key) == NOCLAIM)
			P.aq[atomicAdd(&P.counters[CNT_AQ], 1)] = pe;
		const size_t k = (size_t)sl * P.BV + leaf;
		if (P.alkp[0][k] == NUL16 && atomicMin(&P.claim[k], key) == NOCLAIM &&
		    atomicExch(&P.touched[sl], 1) == 0)
			P.q_touch[atomicAdd(&P.counters[CNT_ATOUCH], 1)] = sl;
	}
}

/// The delta values: a later call at a leaf overwrites an earlier one, so each leaf takes the
/// value of its last call. Phases over the calls, using the leaf's claim word: 0 clears it, 1
/// keeps the largest call index + 1, 2 lets that call write its value, 3 restores the word.
template <int D, int L>
__global__ void k_seed_values(Dev P, int s, const int* pos, const float* val, int n, int phase)
{
	pdl_enter();
	const SurfGeom& g = P.geom[s];
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		int gp, sl, leaf;
		if (!seed_locate<D>(P, g, pos, i, gp, sl, leaf, false)) continue;
		const size_t k = (size_t)sl * P.BV + leaf;
		const unsigned long long me = (unsigned long long)i + 1;
		if (phase == 0) P.claim[k] = 0;
		else if (phase == 1) atomicMax(&P.claim[k], me);
		else if (phase == 2) { if (P.claim[k] == me) P.dlt[k] = val[i]; }
		else P.claim[k] = NOCLAIM;
	}
}

/// After the seed's appends: the delta grid's zero-layer prefix of each affected partition.
template <int L>
__global__ void k_seed_finish(Dev P, int s)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	const int np = P.apcnt[0][s * NL + L];
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
		const int gp = g.pbase + P.aplist[0][(size_t)L * P.NP + g.pbase + i];
		const int sl = P.slot[gp];
		P.dlcnt[sl] = P.acnt[0][sl * NL + L];
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) P.ndp[s] = np;
}

// ---------------------------------------------------------------------------------------------
// calc_affected rings (Surface.hpp:801-912), in parallel. L times, the in-band neighbours of the
// leaves added by the previous ring join affected buffer 0 under their current layer. The
// reference does this in one sequential loop: per list l, per partition entry of the affected
// list l (in list order, those present at the ring's start), per leaf added by the previous ring
// (in list order), per neighbour direction, a track call that appends the leaf to its list and,
// on the first call into a (partition, list), the partition to the affected partition list. Here
// every track call gets the key (l, entry, leaf position, direction) of its place in that loop:
// a leaf untracked at the ring's start goes to the smallest key that tracks it, a (partition,
// list) joins at the smallest key of any call into it, and both are appended in key order, which
// is the order the loop appends them in.
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long ring_key(int l, int entry, int pos, int nb)
{
	return ((unsigned long long)l << 47) | ((unsigned long long)entry << 19) |
	       ((unsigned long long)pos << 3) | (unsigned long long)nb;
}

/// Ring bounds (Surface.hpp:801-815): entries present at the previous ring's start expand the
/// leaves added since ([first, last) = [previous last, current count)); newer entries expand all
/// their leaves. Entries with leaves to expand are queued. One thread per (list, entry).
template <int L>
__global__ void k_ring_setup(Dev P, int s, int np, int cur)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	const int prev = cur ^ 1;
	for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < NL * np; t += gridDim.x * blockDim.x) {
		const int l = t / np, i = t % np;
		const int nc = P.apcnt[0][s * NL + l];
		if (i == 0) P.ring_n[cur * NL + l] = nc;
		if (i >= nc) continue;
		const size_t o = (size_t)l * P.NP + g.pbase + i;
		const int gp = g.pbase + P.aplist[0][o];
		const int first = i < P.ring_n[prev * NL + l] ? P.ring_last[o] : 0;
		const int last = P.acnt[0][P.slot[gp] * NL + l];
		P.ring_first[o] = first;
		P.ring_last[o] = last;
		if (last > first) P.ring_src[atomicAdd(&P.counters[CNT_ASRC], 1)] = (int)o;
	}
}

/// The track calls of one ring: one warp per queued entry, a lane per leaf; each call claims
/// its leaf (if untracked) and its (partition, list) (if not yet listed) with its key.
template <int D, int L>
__global__ void k_ring_claim(Dev P, int s)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	const int lane = threadIdx.x & 31;
	const int nw = (gridDim.x * blockDim.x) >> 5;
	const int n = P.counters[CNT_ASRC];
	for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += nw) {
		const size_t o = (size_t)P.ring_src[w];
		const int l = (int)((o - g.pbase) / P.NP), entry = (int)((o - g.pbase) % P.NP);
		const int gp = g.pbase + P.aplist[0][o];
		const int sl = P.slot[gp];
		const int first = P.ring_first[o], last = P.ring_last[o];
		for (int in = first + lane; in < last; in += 32) {
			const int leaf = P.alst[0][((size_t)sl * NL + l) * P.BV + in];
			const Vec<D> c = leaf_pos<D>(P, gp, leaf);
			for (int nb = 0; nb < 2 * D; nb++) {
				Vec<D> q = c;
				q[nb >> 1] += (nb & 1) ? 1 : -1;
				const int lid = layer_id(get_phi<D, L>(P, g, q), P.err);
				if (!inside_band(lid, L)) continue;
				int gpn, leafn;
				locate<D>(P, g, q, gpn, leafn);
				const int sln = P.slot[gpn];
				if (sln < 0) {
					atomicOr(P.err, EB_INACTIVE);
					continue;
				}
				const int t = lid + L;
				const unsigned long long key = ring_key(l, entry, in, nb);
				const int pe = gpn * NL + t;
				if (P.appos[0][pe] < 0 && atomicMin(&P.apkey[pe], key) == NOCLAIM)
					P.aq[atomicAdd(&P.counters[CNT_AQ], 1)] = pe;
				const size_t k = (size_t)sln * P.BV + leafn;
				if (P.alkp[0][k] == NUL16 && atomicMin(&P.claim[k], key) == NOCLAIM &&
				    atomicExch(&P.touched[sln], 1) == 0)
					P.q_touch[atomicAdd(&P.counters[CNT_ATOUCH], 1)] = sln;
			}
		}
	}
}

/// Appends each touched brick's claimed leaves to their lists (the list of the leaf's current
/// layer) in key order, and clears the claims. One block per brick; up to `cap` claimed leaves
/// are ranked in shared memory, more are ranked by scanning the brick's claims.
template <int L>
__global__ void k_ring_append(Dev P, int cap, int fixed_list)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	extern __shared__ unsigned char ring_smem[];
	unsigned long long* skey = (unsigned long long*)ring_smem;
	uint16_t* sleaf = (uint16_t*)(skey + cap);
	uint8_t* slist = (uint8_t*)(sleaf + cap);
	__shared__ int m, scnt[NL];
	const int nb = P.counters[CNT_ATOUCH];
	for (int b = blockIdx.x; b < nb; b += gridDim.x) {
		const int sl = P.q_touch[b];
		const size_t base = (size_t)sl * P.BV;
		if (threadIdx.x == 0) m = 0;
		if (threadIdx.x < NL) scnt[threadIdx.x] = 0;
		__syncthreads();
		for (int j = threadIdx.x; j < P.BV; j += blockDim.x) {
			const unsigned long long k = P.claim[base + j];
			if (k == NOCLAIM) continue;
			const int t = fixed_list >= 0 ? fixed_list : layer_id(P.phi[base + j], P.err) + L;
			atomicAdd(&scnt[t], 1);
			const int at = atomicAdd(&m, 1);
			if (at < cap) {
				skey[at] = k;
				sleaf[at] = (uint16_t)j;
				slist[at] = (uint8_t)t;
			}
		}
		__syncthreads();
		const int mm = m;
		if (mm <= cap) {
			for (int i = threadIdx.x; i < mm; i += blockDim.x) {
				const unsigned long long ki = skey[i];
				const int ti = slist[i];
				int r = 0;
				for (int j = 0; j < mm; j++) r += slist[j] == ti && skey[j] < ki;
				const int leaf = sleaf[i];
				const int c = P.acnt[0][sl * NL + ti] + r;
				P.alst[0][((size_t)sl * NL + ti) * P.BV + c] = (uint16_t)leaf;
				P.alkp[0][base + leaf] = (uint16_t)c;
			}
		} else {
			for (int i = threadIdx.x; i < P.BV; i += blockDim.x) {
				const unsigned long long ki = P.claim[base + i];
				if (ki == NOCLAIM) continue;
				const int ti = fixed_list >= 0 ? fixed_list : layer_id(P.phi[base + i], P.err) + L;
				int r = 0;
				for (int j = 0; j < P.BV; j++) {
					const unsigned long long kj = P.claim[base + j];
					if (kj < ki && (fixed_list >= 0 || layer_id(P.phi[base + j], P.err) + L == ti)) r++;
				}
				const int c = P.acnt[0][sl * NL + ti] + r;
				P.alst[0][((size_t)sl * NL + ti) * P.BV + c] = (uint16_t)i;
				P.alkp[0][base + i] = (uint16_t)c;
			}
		}
		__syncthreads();
		for (int j = threadIdx.x; j < P.BV; j += blockDim.x) P.claim[base + j] = NOCLAIM;
		if (threadIdx.x < NL) P.acnt[0][sl * NL + threadIdx.x] += scnt[threadIdx.x];
		if (threadIdx.x == 0) P.touched[sl] = 0;
		__syncthreads();
	}
}

/// Appends the (partition, list) entries that joined in this ring to the affected partition
/// lists in key order. One thread per entry.
template <int L>
__global__ void k_ring_plist(Dev P, int s)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	const int n = P.counters[CNT_AQ];
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const int pe = P.aq[i];
		const int t = pe % NL;
		const unsigned long long ki = P.apkey[pe];
		int r = 0;
		for (int j = 0; j < n; j++) {
			const int pj = P.aq[j];
			r += pj % NL == t && P.apkey[pj] < ki;
		}
		const int c = P.apcnt[0][s * NL + t] + r;
		P.aplist[0][(size_t)t * P.NP + g.pbase + c] = pe / NL - g.pbase;
		P.appos[0][pe] = c;
		atomicAdd(&P.counters[CNT_ATC + t], 1);
	}
}

/// Closes a ring: list lengths, key and queue reset.
template <int L>
__global__ void k_ring_finish(Dev P, int s)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const int n = P.counters[CNT_AQ];
	for (int i = threadIdx.x; i < n; i += blockDim.x) P.apkey[P.aq[i]] = NOCLAIM;
	__syncthreads();
	if (threadIdx.x < NL) {
		P.apcnt[0][s * NL + threadIdx.x] += P.counters[CNT_ATC + threadIdx.x];
		P.counters[CNT_ATC + threadIdx.x] = 0;
	}
	if (threadIdx.x == 0) {
		P.counters[CNT_AQ] = 0;
		P.counters[CNT_ATOUCH] = 0;
		P.counters[CNT_ASRC] = 0;
	}
}

/// Zero-layer leaves of surface s (the capacity a bounded update's deltas need).
template <int L>
__global__ void k_count_layer(Dev P, int s, int li, unsigned long long* out)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	const int np = P.pcnt[s * NL + li];
	unsigned long long c = 0;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
		const int gp = g.pbase + P.plist[(size_t)li * P.NP + g.pbase + i];
		c += P.lcnt[P.slot[gp] * NL + li];
	}
	if (c) atomicAdd(out, c);
}

/// isogrid.track_children(affected) and delta.track_children(affected) of update_end
/// (Surface.hpp:409-410; PartitionedMixin.hpp:319-334): per list, the affected partitions not
/// yet in the isogrid's partition list are appended to it in affected-list order, and the delta
/// partition lists (reset at update_start, holding the delta() partitions first) become equal to
/// the affected lists. One block per list; an ordered append by block-wide prefix sums.
template <int L>
__global__ void __launch_bounds__(1024) k_local_children(Dev P, int s)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	__shared__ int wsum[32];
	__shared__ int base;
	const SurfGeom& g = P.geom[s];
	const int l = blockIdx.x;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	const int na = P.apcnt[0][s * NL + l];
	if (threadIdx.x == 0) base = P.pcnt[s * NL + l];
	__syncthreads();
	for (int start = 0; start < na; start += blockDim.x) {
		const int i = start + threadIdx.x;
		int lp = 0, gp = 0;
		bool add = false;
		if (i < na) {
			const size_t o = (size_t)l * P.NP + g.pbase + i;
			lp = P.aplist[0][o];
			gp = g.pbase + lp;
			add = P.ppos[gp * NL + l] < 0;
			P.dplist[o] = lp;
		}
		const unsigned m = __ballot_sync(0xffffffffu, add);
		if (lane == 0) wsum[warp] = __popc(m);
		__syncthreads();
		int before = 0, total = 0;
		for (int w = 0; w < nwarp; w++) {
			if (w < warp) before += wsum[w];
			total += wsum[w];
		}
		if (add) {
			const int c = base + before + __popc(m & ((1u << lane) - 1u));
			P.plist[(size_t)l * P.NP + g.pbase + c] = lp;
			P.ppos[gp * NL + l] = c;
		}
		__syncthreads();
		if (threadIdx.x == 0) base += total;
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		P.pcnt[s * NL + l] = base;
		P.dpcnt[s * NL + l] = na;
	}
}

/// The partitions of a bounded update's box (Surface.hpp:313-330): box[a] children from cl[a]
/// along each axis, row-major; leaves with lo <= pos < lub are inside.
template <int D>
struct BoxParts {
	Vec<D> cl, box, lo, lub;
	int nb;
};

/// update(lo, hi, fn) (Surface.hpp:310-386), in three steps that keep the reference's order
/// (box partitions row-major, each partition's zero-layer list in order): count each
/// partition's leaves inside the box, scan the counts, write the positions at their offsets.
template <int D>
__device__ __forceinline__ int box_partition(const Dev& P, const SurfGeom& g, const BoxParts<D>& b,
                                             int ci)
{
	Vec<D> pc;
	int r = ci;
	for (int a = D - 1; a >= 0; a--) {
		pc[a] = r % b.box[a] + b.cl[a];
		r /= b.box[a];
	}
	int idx = 0;
	for (int a = 0; a < D; a++) idx = idx * g.ccount[a] + pc[a];
	return g.pbase + idx;
}

template <int D, int L>
__device__ __forceinline__ bool leaf_in_box(const Dev& P, const BoxParts<D>& b, int gp, int leaf,
                                            Vec<D>& p)
{
	p = leaf_pos<D>(P, gp, leaf);
	for (int a = 0; a < D; a++)
		if (p[a] < b.lo[a] || p[a] >= b.lub[a]) return false;
	return true;
}

/// One warp per box partition: its zero-layer leaves inside the box (counts[ci]).
template <int D, int L>
__global__ void k_bounded_count(Dev P, int s, BoxParts<D> b, int* counts)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	const int lane = threadIdx.x & 31, nw = (gridDim.x * blockDim.x) >> 5;
	for (int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < b.nb; ci += nw) {
		const int gp = box_partition<D>(P, g, b, ci);
		const int sl = P.slot[gp];
		int c = 0;
		if (sl >= 0) {
			const int nl = P.lcnt[sl * NL + L];
			const uint16_t* lst = P.lst + ((size_t)sl * NL + L) * P.BV;
			for (int j = lane; j < nl; j += 32) {
				Vec<D> p;
				c += leaf_in_box<D, L>(P, b, gp, lst[j], p);
			}
		}
		for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
		if (lane == 0) counts[ci] = c;
	}
}

/// Exclusive scan of n counts into offsets (one block, in order); the total into *total.
static __global__ void __launch_bounds__(1024) k_scan_offsets(const int* counts, int n, int* offsets,
                                                       int* total)
{
	pdl_enter();
	__shared__ int wsum[32];
	__shared__ int base;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	if (threadIdx.x == 0) base = 0;
	__syncthreads();
	for (int start = 0; start < n; start += blockDim.x) {
		const int i = start + threadIdx.x;
		const int v = i < n ? counts[i] : 0;
		int x = v;
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= o) x += y;
		}
		if (lane == 31) wsum[warp] = x;
		__syncthreads();
		int before = 0, tot = 0;
		for (int w = 0; w < nwarp; w++) {
			if (w < warp) before += wsum[w];
			tot += wsum[w];
		}
		if (i < n) offsets[i] = base + before + x - v;
		__syncthreads();
		if (threadIdx.x == 0) base += tot;
		__syncthreads();
	}
	if (threadIdx.x == 0) *total = base;
}

/// One warp per box partition: its inside leaves' positions at its offset, in list order (up to
/// cap positions in all).
template <int D, int L>
__global__ void k_bounded_write(Dev P, int s, BoxParts<D> b, const int* offsets, int* pos, int cap)
{
	pdl_enter();
	constexpr int NL = 2 * L + 1;
	const SurfGeom& g = P.geom[s];
	const int lane = threadIdx.x & 31, nw = (gridDim.x * blockDim.x) >> 5;
	for (int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < b.nb; ci += nw) {
		const int gp = box_partition<D>(P, g, b, ci);
		const int sl = P.slot[gp];
		if (sl < 0) continue;
		const int nl = P.lcnt[sl * NL + L];
		const uint16_t* lst = P.lst + ((size_t)sl * NL + L) * P.BV;
		int at = offsets[ci];
		for (int j0 = 0; j0 < nl; j0 += 32) {
			const int j = j0 + lane;
			Vec<D> p;
			const bool in = j < nl && leaf_in_box<D, L>(P, b, gp, lst[j], p);
			const unsigned m = __ballot_sync(0xffffffffu, in);
			const int c = at + __popc(m & ((1u << lane) - 1u));
			if (in && c < cap)
				for (int a = 0; a < D; a++) pos[c * D + a] = p[a];
			at += __popc(m);
		}
	}
}

/// The speed functor at each collected position, before any value changes.
template <int D, int L>
__global__ void k_bounded_speed(Dev P, int s, Speed sp, const int* pos, const int* n, float* val)
{
	pdl_enter();
	const SurfGeom& g = P.geom[s];
	const int m = *n;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
		Vec<D> p;
		for (int a = 0; a < D; a++) p[a] = pos[i * D + a];
		val[i] = speed_eval<D, L>(P, g, sp, p);
	}
}

}  // namespace fg
