// Device-side layout and helpers of the sparse-field level-set engine.
//
// One pool holds S surfaces that share D, L and the partition (brick) shape. Every partition of
// every surface has a global index gp = pbase[s] + local index, where the local index is the
// reference's row-major children-grid index (include/Felt/Impl/Util.hpp:23-40). An active
// partition owns one brick slot of the device pool; bricks hold the isogrid values, the ordered
// per-layer leaf lists and per-step scratch. All arithmetic on distances is FP32 and compiled
// with -fmad=false so that it rounds exactly as the reference's (-ffp-contract=off) CPU code.
#pragma once

#include <cstdint>

namespace fg {

constexpr uint16_t NUL16 = 0xFFFFu;

/// Programmatic dependent launch. The update's kernels are launched so that each may start
/// while the previous kernel of its stream drains; every such kernel calls this first: it
/// waits until the previous kernel has finished and its writes are visible (no wait for a
/// kernel launched the ordinary way), then lets the next kernel begin its launch.
__device__ __forceinline__ void pdl_enter()
{
	asm volatile("griddepcontrol.wait;" ::: "memory");
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
constexpr unsigned long long NOCLAIM = ~0ull;

// -------------------------------------------------------------------------------------------
// Bulk copies global -> shared memory through the tensor memory accelerator (untiled
// cp.async.bulk, no multicast), completed on a shared-memory mbarrier. Every wait is bounded.
// -------------------------------------------------------------------------------------------

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
	return (unsigned)__cvta_generic_to_shared(p);
}
/// One thread: the barrier expects one arrival per phase.
__device__ __forceinline__ void mbar_init(unsigned long long* bar)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
/// Orders the block's earlier generic accesses of shared memory before later bulk copies into
/// it (called by each issuing thread after a barrier).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
/// Any thread: `bytes` more to arrive on bar's current phase, then copies them from global src
/// to shared dst (both 16-byte aligned, bytes a multiple of 16), completing on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar)
{
	asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
	             "r"(bytes)
	             : "memory");
	asm volatile(
	    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
	        "r"(smem_u32(dst)),
	    "l"(src), "r"(bytes), "r"(smem_u32(bar))
	    : "memory");
}
/// One thread: the phase's single arrival (after every bulk_g2s of the phase was issued).
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
	asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
	                 smem_u32(bar))
	             : "memory");
}
/// Waits for the completion of phase `parity` of bar, at most `tries` polls (each poll may
/// suspend the thread for a short, hardware-chosen time). False if it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int tries)
{
	for (int i = 0; i < tries; i++) {
		unsigned ok;
		asm volatile("{\n\t.reg .pred p;\n\t"
		             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}"
		             : "=r"(ok)
		             : "r"(smem_u32(bar)), "r"(parity)
		             : "memory");
		if (ok) return true;
	}
	return false;
}

// error bits (Dev::err[0])
enum : int {
	EB_NONFINITE = 1,  // layer_id of NaN/inf
	EB_POOL = 2,       // brick pool exhausted
	EB_OUTSIDE = 4,    // band node tracked outside the grid
	EB_INACTIVE = 8,   // write to an inactive partition
	EB_CAPACITY = 16,  // a fixed-capacity buffer overflowed
	EB_TIMEOUT = 32    // a bounded wait gave up
};

/// Geometry of one surface of the pool.
struct SurfGeom {
	int size[3];
	int off[3];    // grid offset = -size/2 (Surface.hpp:1716-1719)
	int hi[3];     // off + size
	int ccount[3]; // children grid size (PartitionedMixin.hpp:131-141)
	int coff[3];   // children grid offset = off / part (truncating)
	int pbase;     // first global partition index
	int np;        // partitions of this surface
};

/// Pointers and sizes of the whole pool, passed by value to every kernel.
struct Dev {
	int S;        // surfaces
	int NP;       // partitions over all surfaces
	int BV;       // leaves per brick
	int nslots;   // brick capacity
	int csz[3];   // partition shape
	int lstr[3];  // leaf strides inside a brick (row-major, last axis fastest)

	const SurfGeom* geom;
	const int* surf_of;   // [NP] surface of a partition
	const int* porig;     // [NP*3] world position of a partition's first leaf

	// partition level
	int* slot;    // [NP] brick slot, -1 when inactive
	float* bg;    // [NP] background returned for an inactive partition
	int* oslot;   // [NP] slot of a partition deactivated in the current iteration, else -1
	int* ppos;    // [NP*NL] position in the isogrid partition list, -1 = untracked

	// partition lists, per layer a global array with per-surface segments at pbase:
	// list[l*NP + pbase + i], counts cnt[s*NL + l]
	int* plist; int* pcnt;      // isogrid children lookup lists
	int* dplist; int* dpcnt;    // delta partition lists (snapshot at update start)
	int* splist; int* spcnt;    // status-change partition lists (per from-layer)
	int* sppos;                 // [NP*NL] position in splist, -1
	int* aplist[2]; int* apcnt[2]; int* appos[2];  // affected lookups (two buffers)

	// bricks
	float* phi;       // [slot*BV + leaf]
	float* dlt;       // [slot*BV + leaf] delta / scratch
	uint16_t* lkp;    // [slot*BV + leaf] position in its isogrid layer list
	uint16_t* lst;    // [(slot*NL + l)*BV + i] ordered leaf lists
	int* lcnt;        // [slot*NL + l]
	int8_t* sto;      // [slot*BV + leaf] status "to" layer id, L+1 = none
	uint16_t* chg;    // [(slot*NL + f)*BV + i] status-change leaf list per from-layer
	int* ccnt;        // [slot*NL + f]
	uint16_t* alkp[2];  // affected buffer leaf lookups
	uint16_t* alst[2];  // affected buffer leaf lists
	int* acnt[2];
	unsigned long long* claim;  // [slot*BV + leaf] expansion claim keys
	uint16_t* ccl;    // [slot*BV + i] leaves of the brick with an expansion claim, first claim order
	int* ccln;        // [slot] their number
	// expansion candidates of the current iteration (key, partition, leaf), cand_cap at most
	unsigned long long* cand_key;
	int* cand_gp;
	int* cand_leaf;
	int cand_cap;
	int* slot_gp;     // [nslots] owner partition

	// allocator and queues
	int* free_stack;  // [nslots]
	int* counters;    // see CNT_* below
	int* q_act;       // [NP] partitions to activate
	int* actflag;     // [NP]
	int* q_touch;     // [nslots] bricks with expansion claims
	int* touched;     // [nslots]
	int* q_retire;    // [nslots] slots to release after the iteration
	int* q_sunion;    // [NP] partitions with status changes this iteration
	int* sflag;       // [NP] membership flag for q_sunion
	unsigned int* eflag;  // [NP] per-entry flags of the current pass
	unsigned int* eflag2; // [NP] the same for the odd passes of the fused distance passes
	unsigned* app;    // [NP*NL] flush: lists that went 0->1 during phase f (bitmask over to)
	unsigned* rem;    // [NP] flush: lists that went ->0 during their own phase (bitmask)
	unsigned long long* pap;  // [2*NP] expansion partition appends: first claim key per surface
	int* papg;        // [2*NP] the local partition index of each pap entry
	int* papn;        // [S]
	int* woff;        // [S+1] entry offsets of the current pass
	int* woffl;       // [NL*(S+1)] entry offsets of every layer's list, for the distance passes
	int4* etab;       // [NL*NP] the distance passes' entries decoded (k_entry_table)
	int* dq;          // [nslots] partitions of the tiled distance passes (k_entry_table)
	unsigned* eflagl; // [NL*NP] entry flags of every layer's pass (tiled distance passes)
	int* sfrozen;     // [S] surfaces stopped after a non-terminating update (no further work)
	int* err;         // [1] error bits
	int* changed;     // [1] status-change flag of the distance passes
	unsigned long long* kstat;  // [8] work units processed, see KS_* below
	unsigned long long* snu;    // [S] narrow-band node updates per surface (band size at the
	                            // start of each of its global updates, summed)

	// local update (update_start / delta / update_end)
	int* dlcnt;       // [nslots] delta leaves of a partition: a prefix of its affected list L
	int* ndp;         // [S] delta partitions: a prefix of the affected partition list L
	int* ring_first;  // [NL*NP] calc_affected ring bounds per (layer, partition entry)
	int* ring_last;   // [NL*NP]
	int* ring_src;    // [NL*NP] entries with leaves to expand in the current ring
	int* ring_n;      // [2*NL] partition-list lengths at the start of the last two rings
	unsigned long long* apkey;  // [NP*NL] first track key of (partition, list) in a ring
	int* aq;          // [NP*NL] (partition, list) entries that join the affected lists
};

enum {
	CNT_FREE_TOP = 0,
	CNT_ACT = 1,
	CNT_TOUCH = 2,
	CNT_RETIRE = 3,
	CNT_SUNION = 4,
	CNT_CAND = 5,  // expansion candidates recorded this iteration
	CNT_ASRC = 8,     // calc_affected: source entries of the ring
	CNT_AQ = 9,       // calc_affected: (partition, list) entries joining the lists
	CNT_ATOUCH = 10,  // calc_affected: bricks with claimed leaves
	CNT_ATC = 16,     // calc_affected: per list, partitions joining it (NL entries)
	CNT_CDONE = 26,   // blocks of the last compaction done (its last block prepares expansion)
	CNT_DQ = 27,      // partitions queued for the tiled distance passes
	CNT_LDONE = 28,   // blocks done of a launch whose last block resets counters (last_block)
	CNT_N = 32
};

/// Work-unit counters (Dev::kstat): band nodes through the distance passes, zero-layer nodes
/// through the speed functor, leaf edits replayed by the flush, cells marched by Polys.
enum { KS_DIST = 0, KS_ZERO = 1, KS_FLUSH = 2, KS_MARCH = 3, KS_N = 8 };

template <int D>
struct Vec {
	int v[D];
	__host__ __device__ int& operator[](int i) { return v[i]; }
	__host__ __device__ const int& operator[](int i) const { return v[i]; }
};

// -------------------------------------------------------------------------------------------
// Rounding and layers (include/Felt/Surface.hpp:1694-1709)
// -------------------------------------------------------------------------------------------

/// layer_id(v) = iround(v + FLT_EPSILON), half away from zero. Non-finite input sets the error
/// bit and yields an out-of-band id (the reference's boost::math::iround throws there).
__device__ __forceinline__ int layer_id(float v, int* err)
{
	const float x = __fadd_rn(v, 1.1920928955078125e-07f);
	if (!isfinite(x) || fabsf(x) >= 2147483648.0f) {
		atomicOr(err, EB_NONFINITE);
		return 1 << 20;
	}
	return (int)roundf(x);
}
__device__ __forceinline__ bool inside_band(int id, int L) { return (id < 0 ? -id : id) <= L; }

// -------------------------------------------------------------------------------------------
// Hashed noise, identical to the oracle's: MurmurHash3's fmix32 finaliser per axis, 24 bits
// mapped exactly to u * 2^-23 - 1.
// -------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t fmix32(uint32_t h)
{
	h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
	return h;
}
template <int D>
__device__ __forceinline__ float hash_noise(const Vec<D>& p, uint32_t seed)
{
	const uint32_t K[3] = {0x9e3779b1u, 0x7f4a7c15u, 0x94d049bbu};
	uint32_t h = fmix32(seed ^ 0x5eed5eedu);
#pragma unroll
	for (int a = 0; a < D; a++) h = fmix32(h ^ ((uint32_t)p[a] * K[a]));
	const uint32_t u = h >> 8;
	return __fsub_rn(__fmul_rn((float)u, 1.0f / 8388608.0f), 1.0f);
}

// -------------------------------------------------------------------------------------------
// Pool addressing
// -------------------------------------------------------------------------------------------

template <int D>
__device__ __forceinline__ bool in_grid(const SurfGeom& g, const Vec<D>& p)
{
#pragma unroll
	for (int a = 0; a < D; a++)
		if (p[a] < g.off[a] || p[a] >= g.hi[a]) return false;
	return true;
}

/// Global partition and leaf of an in-grid position (PartitionedMixin.hpp:221-245).
template <int D>
__device__ __forceinline__ void locate(const Dev& P, const SurfGeom& g, const Vec<D>& p, int& gp,
                                       int& leaf)
{
	int idx = 0, lf = 0;
#pragma unroll
	for (int a = 0; a < D; a++) {
		const int r = p[a] - g.off[a];
		const int c = r / P.csz[a];
		idx = idx * g.ccount[a] + c;
		lf += (r - c * P.csz[a]) * P.lstr[a];
	}
	gp = g.pbase + idx;
	leaf = lf;
}

/// Partitioned::Access::get (PartitionedMixin.hpp:594-601) with the lazy child get
/// (GridMixin.hpp:608-621): background L+1 outside the grid, the partition's background when
/// it is inactive.
template <int D, int L>
__device__ __forceinline__ float get_phi(const Dev& P, const SurfGeom& g, const Vec<D>& p)
{
	if (!in_grid<D>(g, p)) return (float)(L + 1);
	int gp, leaf;
	locate<D>(P, g, p, gp, leaf);
	const int sl = P.slot[gp];
	if (sl < 0) return P.bg[gp];
	return P.phi[(size_t)sl * P.BV + leaf];
}

/// World position of a leaf of partition gp.
template <int D>
__device__ __forceinline__ Vec<D> leaf_pos(const Dev& P, int gp, int leaf)
{
	Vec<D> p;
	int rem = leaf;
#pragma unroll
	for (int a = 0; a < D; a++) {
		const int q = rem / P.lstr[a];
		rem -= q * P.lstr[a];
		p[a] = P.porig[gp * 3 + a] + q;
	}
	return p;
}

// -------------------------------------------------------------------------------------------
// Stencils
// -------------------------------------------------------------------------------------------

/// Mean curvature by difference of normals (NumericMixin.hpp:72-156). The fixed-size Eigen sum
/// of the normal differences is unrolled by halving: x0 + (x1 + x2) in 3D. The position is a
/// node (Vec<D>) or a real position (any float D-vector with operator[], read through
/// interpolation by get); its coordinates step by +-1 in their own type, as the reference's
/// template on the position type does.
template <int D, class Get, class Pos>
__device__ float curv_g(const Get& get, const Pos& pos)
{
	const float centre = get(pos);
	Pos dir = pos;
	float nf[D], nb[D];
#pragma unroll
	for (int axis = 0; axis < D; axis++) {
		dir[axis] += 1;
		const float va = __fsub_rn(get(dir), centre);
		float sq = 0.0f;
#pragma unroll
		for (int an = 0; an < D; an++) {
			if (an == axis) continue;
			Pos dn = dir;
			dn[an] -= 1;
			const float lo = get(dn);
			dn[an] += 2;
			const float hi = get(dn);
			const float v = __fdiv_rn(__fsub_rn(hi, lo), 2.0f);
			sq = __fadd_rn(sq, __fmul_rn(v, v));
		}
		nf[axis] = __fdiv_rn(va, __fsqrt_rn(__fadd_rn(__fmul_rn(va, va), sq)));
		dir[axis] -= 1;
	}
#pragma unroll
	for (int axis = 0; axis < D; axis++) {
		dir[axis] -= 1;
		const float va = __fsub_rn(centre, get(dir));
		float sq = 0.0f;
#pragma unroll
		for (int an = 0; an < D; an++) {
			if (an == axis) continue;
			Pos dn = dir;
			dn[an] -= 1;
			const float lo = get(dn);
			dn[an] += 2;
			const float hi = get(dn);
			const float v = __fdiv_rn(__fsub_rn(hi, lo), 2.0f);
			sq = __fadd_rn(sq, __fmul_rn(v, v));
		}
		nb[axis] = __fdiv_rn(va, __fsqrt_rn(__fadd_rn(__fmul_rn(va, va), sq)));
		dir[axis] += 1;
	}
	float s;
	if (D == 2)
		s = __fadd_rn(__fsub_rn(nf[0], nb[0]), __fsub_rn(nf[D - 1], nb[D - 1]));
	else
		s = __fadd_rn(__fsub_rn(nf[0], nb[0]),
		              __fadd_rn(__fsub_rn(nf[1 % D], nb[1 % D]), __fsub_rn(nf[D - 1], nb[D - 1])));
	return __fdiv_rn(s, 2.0f);
}

/// Reads the isogrid through the pool (global memory).
template <int D, int L>
struct PoolGet {
	const Dev& P;
	const SurfGeom& g;
	__device__ float operator()(const Vec<D>& p) const { return get_phi<D, L>(P, g, p); }
};

/// Reads the isogrid around one brick: positions inside the brick's partition and the grid
/// straight from the brick (no partition lookup), the others through the pool. The same values
/// as PoolGet.
template <int D, int L>
struct BrickGet {
	const Dev& P;
	const SurfGeom& g;
	const float* brick;
	Vec<D> org;  // world position of the brick's leaf 0
	__device__ float operator()(const Vec<D>& p) const
	{
		int leaf = 0;
		bool in = true;
#pragma unroll
		for (int a = 0; a < D; a++) {
			const int q = p[a] - org[a];
			in = in && (unsigned)q < (unsigned)P.csz[a] && p[a] < g.hi[a];
			leaf += q * P.lstr[a];
		}
		return in ? brick[leaf] : get_phi<D, L>(P, g, p);
	}
};

template <int D, int L>
__device__ float curv(const Dev& P, const SurfGeom& g, const Vec<D>& pos)
{
	return curv_g<D>(PoolGet<D, L>{P, g}, pos);
}

/// City-block distance to the zero curve from the nearest in-grid neighbour on the way in
/// (Surface.hpp:1387-1440): d = side * min(side*phi_self, side*phi_n) + side.
template <int D, int L>
__device__ __forceinline__ float distance(const Dev& P, const SurfGeom& g, const Vec<D>& pos,
                                          float dist, float dir)
{
	dist = __fmul_rn(dist, dir);
	Vec<D> n = pos;
#pragma unroll
	for (int a = 0; a < D; a++) {
#pragma unroll
		for (int s = -1; s <= 1; s += 2) {
			n[a] = pos[a] + s;
			if (in_grid<D>(g, n)) {
				const float dn = __fmul_rn(get_phi<D, L>(P, g, n), dir);
				if (dn < dist) dist = dn;
			}
		}
		n[a] = pos[a];
	}
	return __fadd_rn(__fmul_rn(dist, dir), dir);
}

/// The partition next to gp along axis a (s = -1 or +1) and the leaf of it next to `leaf`, for
/// a neighbour that lies in the grid: the children grid is row-major with the last axis
/// fastest, so the partition index moves by the product of the later axes' counts, and the
/// leaf coordinate wraps to the neighbour's far face. No division (get_phi's locate).
template <int D>
__device__ __forceinline__ void next_partition(const Dev& P, const SurfGeom& g, int gp, int leaf,
                                               int a, int s, int& gp2, int& leaf2)
{
	int cst = 1;
#pragma unroll
	for (int b = D - 1; b > a; b--) cst *= g.ccount[b];
	gp2 = gp + s * cst;
	leaf2 = leaf + (s < 0 ? P.csz[a] - 1 : 1 - P.csz[a]) * P.lstr[a];
}

/// distance() for leaf `leaf` of partition gp (brick slot sl): neighbours inside the same
/// partition are read straight from the brick; the others from the next partition along the
/// axis (next_partition), its brick or its background. Same result as distance() at the
/// leaf's position (get_phi there).
template <int D, int L>
__device__ __forceinline__ float distance_leaf(const Dev& P, const SurfGeom& g, int gp, int sl,
                                               int leaf, float dist, float dir)
{
	dist = __fmul_rn(dist, dir);
	const float* brick = P.phi + (size_t)sl * P.BV;
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
					v = brick[leaf + s * P.lstr[a]];
				} else {
					int gp2, leaf2;
					next_partition<D>(P, g, gp, leaf, a, s, gp2, leaf2);
					const int sl2 = P.slot[gp2];
					v = sl2 < 0 ? P.bg[gp2] : P.phi[(size_t)sl2 * P.BV + leaf2];
				}
				const float dn = __fmul_rn(v, dir);
				if (dn < dist) dist = dn;
			}
		}
		n[a] = pos[a];
	}
	return __fadd_rn(__fmul_rn(dist, dir), dir);
}

/// Builtin speed: [a*curv] + [n*h] + [c] in that order (see include/felt_gpu.h).
struct Speed {
	int kind;
	float c, a, n;
	uint32_t seed;
};
template <int D, class Get>
__device__ __forceinline__ float speed_eval_g(const Get& get, const Speed& sp, const Vec<D>& pos)
{
	float acc = 0.0f;
	bool have = false;
	if (sp.kind & 2) {
		acc = __fmul_rn(sp.a, curv_g<D>(get, pos));
		have = true;
	}
	if (sp.kind & 4) {
		const float t = __fmul_rn(sp.n, hash_noise<D>(pos, sp.seed));
		acc = have ? __fadd_rn(acc, t) : t;
		have = true;
	}
	if (sp.kind & 1) acc = have ? __fadd_rn(acc, sp.c) : sp.c;
	return acc;
}

template <int D, int L>
__device__ __forceinline__ float speed_eval(const Dev& P, const SurfGeom& g, const Speed& sp,
                                            const Vec<D>& pos)
{
	float acc = 0.0f;
	bool have = false;
	if (sp.kind & 2) {
		acc = __fmul_rn(sp.a, curv<D, L>(P, g, pos));
		have = true;
	}
	if (sp.kind & 4) {
		const float t = __fmul_rn(sp.n, hash_noise<D>(pos, sp.seed));
		acc = have ? __fadd_rn(acc, t) : t;
		have = true;
	}
	if (sp.kind & 1) acc = have ? __fadd_rn(acc, sp.c) : sp.c;
	return acc;
}

/// Largest s with woff[s] <= e (entry -> surface of a flattened per-surface list).
__device__ __forceinline__ int entry_surface(const int* woff, int S, int e)
{
	int lo = 0, hi = S;
	while (hi - lo > 1) {
		const int mid = (lo + hi) >> 1;
		if (woff[mid] <= e)
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

}  // namespace fg
