// Raycasting to the zero curve: Felt's Surface::ray (include/Felt/Surface.hpp:468-616,
// 1450-1598) for a batch of rays.
//
// A ray follows the reference step by step: the partition holding the origin first; then, per
// axis, the partition planes the ray crosses, keeping the partitions that hold any of layers
// -1, 0, 1; those in order of squared distance from the origin (ties in the order found;
// std::sort leaves that order unspecified), consecutive repeats of a partition dropped; within
// each, samples every half unit along the ray until a zero-layer sample faces the ray, from
// which it converges onto the zero curve along the interpolated gradient (at most 100 steps).
// Arithmetic is FP32 in the reference's order (Eigen's ParametrizedLine / Hyperplane formulas;
// dot products and squared norms summed x0 + (x1 + x2)).
//
// Kernel shape, two passes so that each runs one uniform loop:
//  - k_ray_find: persistent threads, one ray per thread at a time, each thread taking its next
//    ray from a counter when it finishes one (warp-aggregated atomics), so a warp never waits
//    on its slowest ray. A ray is a small state machine (next candidate / march sample); when a
//    sample starts a convergence the ray is queued and the thread moves on.
//  - k_ray_conv: one queued ray per thread, the convergence steps (each one gradient: its
//    centre value is the next step's distance, the same interpolation).
// A convergence that leaves the grid is the partition's ray_miss; its ray goes back to
// k_ray_find, which replays the candidates it had consumed (deterministic) and goes on.
//
// Candidate order without a sort buffer: along one axis the walk's planes move away from the
// origin, so their crossings' squared distances never decrease, and the reference's stable
// sort of all candidates is the merge of the D per-axis walks, ties to the lower axis (its
// candidates were discovered first). Each axis keeps a cursor on its next candidate. Why the
// keys never decrease, in FP32 as computed: the crossing parameter t = (plane - o) / dir
// (rounded) is monotonic in the plane's position along the walk; every component
// p_i = o_i + dir_i t + dir_i TINY is monotonic in t with the sign of dir_i, so while t >= 0
// each |p_i - o_i| never decreases, and neither do the squares or their sum (rounding to
// nearest is monotonic). Every plane after the first lies at least a partition ahead of the
// origin (t > 0); the first may lie behind it by rounding only, and then its key is smaller
// than any later one. As a safety net the kernel also checks the keys it consumes; a decrease
// would make the ray restart its candidates in exact order (each next candidate by a full walk
// of the planes, the (distance, discovery index) after the previous one), the order
// fg_ray_device's mode 1 selects for every ray.
#include <cooperative_groups.h>

#include <algorithm>

#include <cfloat>
#include <cstdint>

#include "fg_engine.cuh"
#include "fg_field.cuh"
#include "fg_ray.cuh"

namespace fg {

namespace {

namespace cg = cooperative_groups;

constexpr float RAY_TINY = 0.00001f;     // Surface.hpp:67
constexpr int RAY_CONVERGE_STEPS = 100;  // Surface.hpp:1488
constexpr int RAY_MAX_MARCH = 1 << 16;   // bound on the reference's open loops
constexpr int RAY_THREADS = 128;

enum : int { PH_FETCH = 0, PH_NEXT = 1, PH_MARCH = 2, PH_CONV = 3 };

template <int D>
__device__ __forceinline__ bool inside_box(const float* p, const int* lo, const int* hi)
{
#pragma unroll
	for (int a = 0; a < D; a++) {
		if (p[a] >= (float)hi[a]) return false;
		if (p[a] < (float)lo[a]) return false;
	}
	return true;
}

template <int D>
__device__ __forceinline__ float dist2(const float* p, const float* o)
{
	float d[D];
#pragma unroll
	for (int a = 0; a < D; a++) d[a] = __fsub_rn(p[a], o[a]);
	return dot_e<D>(d, d);
}

__device__ __forceinline__ float sgnf(float v) { return (float)((0.0f < v) - (v < 0.0f)); }

/// The partition of an in-grid integer position (PartitionedMixin.hpp:221-245); a shift
/// instead of a division along axes whose partition size is a power of two.
template <int D>
__device__ __forceinline__ int part_of(const Dev& P, const SurfGeom& g, const Vec<D>& q)
{
	int idx = 0;
#pragma unroll
	for (int a = 0; a < D; a++) {
		const int r = q[a] - g.off[a];
		const int cs = P.csz[a];
		const int c = (cs & (cs - 1)) == 0 ? r >> (__ffs(cs) - 1) : r / cs;
		idx = idx * g.ccount[a] + c;
	}
	return g.pbase + idx;
}

/// interp at p through the partition lookup (any position): the general path, out of line so
/// that the kernels' code stays small.
template <int D, int L>
__device__ __noinline__ float interp_slow(const Dev& P, const SurfGeom& g, float x, float y,
                                          float z)
{
	const float p[3] = {x, y, z};
	return interp<D>(PoolGet<D, L>{P, g}, p);
}

/// The partition a march or convergence works in: corners of an interpolation are read
/// relative to it.
struct Home {
	int gp;          // global partition index
	int lo[3];       // its box origin
	int sl;          // its brick slot, -1 when inactive
	float bg;        // its background (when inactive)
};

template <int D>
__device__ __forceinline__ Home home_of(const Dev& P, int gp)
{
	Home h;
	h.gp = gp;
	h.sl = __ldg(P.slot + gp);
	h.bg = __ldg(P.bg + gp);
#pragma unroll
	for (int a = 0; a < 3; a++) h.lo[a] = a < D ? __ldg(P.porig + gp * 3 + a) : 0;
	return h;
}

/// interp (NumericMixin.hpp:403-481) with corners read relative to the home partition: along
/// each axis a corner lies in the home partition or one step away, located by children-grid
/// offsets (no division); a neighbour's slot is read only for corners that cross. Every lane
/// runs the same instructions. Corners further away (a convergence that wandered) take the
/// general path. The same values and arithmetic as interp over get_phi.
template <int D, int L>
struct HomeInterp {
	const Dev& P;
	const SurfGeom& g;
	const Home& h;
	__device__ __forceinline__ float operator()(const float* p) const
	{
		float pc[D];
		int step0[D], step1[D], r0[D], r1[D];
		bool in0[D], in1[D];
		bool far = false;
#pragma unroll
		for (int a = 0; a < D; a++) {
			const float f = floorf(p[a]);
			const int fl = (int)f;
			pc[a] = __fsub_rn(p[a], f);
			const int cs = P.csz[a];
			const int r = fl - h.lo[a];
			far = far || r < -cs || r + 1 >= 2 * cs;
			step0[a] = (r >= cs) - (r < 0);
			step1[a] = (r + 1 >= cs) - (r + 1 < 0);
			r0[a] = r - step0[a] * cs;
			r1[a] = r + 1 - step1[a] * cs;
			in0[a] = fl >= g.off[a] && fl < g.hi[a];
			in1[a] = fl + 1 >= g.off[a] && fl + 1 < g.hi[a];
		}
		if (far) return interp_slow<D, L>(P, g, p[0], p[1], D > 2 ? p[D - 1] : 0.0f);
		int cstride[D];
		cstride[D - 1] = 1;
#pragma unroll
		for (int a = D - 2; a >= 0; a--) cstride[a] = cstride[a + 1] * g.ccount[a + 1];
		float v[1 << D];
#pragma unroll
		for (int i = 0; i < (1 << D); i++) {
			int nb = h.gp, leaf = 0;
			bool in = true;
#pragma unroll
			for (int a = 0; a < D; a++) {
				const bool b = (i >> a) & 1;
				nb += (b ? step1[a] : step0[a]) * cstride[a];
				leaf += (b ? r1[a] : r0[a]) * P.lstr[a];
				in = in && (b ? in1[a] : in0[a]);
			}
			float val = (float)(L + 1);  // outside the grid
			if (in) {
				const bool home = nb == h.gp;
				const int sl = home ? h.sl : __ldg(P.slot + nb);
				if (sl >= 0)
					val = __ldg(P.phi + (size_t)sl * P.BV + leaf);
				else
					val = home ? h.bg : __ldg(P.bg + nb);
			}
			v[i] = val;
		}
		return interp_reduce<D>(v, pc);
	}
};

/// Whether all 2^D interpolation corners of p lie in the partition box from lo and in the grid.
template <int D>
__device__ __forceinline__ bool corners_inside(const Dev& P, const SurfGeom& g, const int* lo,
                                               const float* p)
{
	bool in = true;
#pragma unroll
	for (int a = 0; a < D; a++) {
		const int fl = (int)floorf(p[a]);
		in = in && fl >= lo[a] && fl + 1 < lo[a] + P.csz[a] && fl + 1 < g.hi[a];
	}
	return in;
}

/// round_to_next (Surface.hpp:1582-1599).
__device__ __forceinline__ float round_to_next(const Dev& P, const SurfGeom& g, int dim, float dd,
                                               float pos)
{
	float p = __fdiv_rn(__fsub_rn(pos, (float)g.off[dim]), (float)P.csz[dim]);
	p = dd == -1.0f ? floorf(p) : ceilf(p);
	p = __fmul_rn(p, (float)P.csz[dim]);
	return __fadd_rn(p, (float)g.off[dim]);
}

/// The crossing of the ray with the plane x[dim] = plane_pos, nudged by TINY along the ray
/// (Surface.hpp:1545-1552): Hyperplane(normal = -dd e_dim, offset = plane_pos * dd) met by
/// ParametrizedLine(o, dir). od, vd: o[dim], dir[dim].
template <int D>
__device__ __forceinline__ void crossing(const float* o, const float* dir, float od, float vd,
                                         float dd, float plane_pos, float* p)
{
	const float nd = -dd, off = __fmul_rn(plane_pos, dd);
	const float t = -__fdiv_rn(__fadd_rn(off, __fmul_rn(nd, od)), __fmul_rn(nd, vd));
#pragma unroll
	for (int i = 0; i < D; i++) p[i] = __fadd_rn(o[i], __fmul_rn(dir[i], t));
#pragma unroll
	for (int i = 0; i < D; i++) p[i] = __fadd_rn(p[i], __fmul_rn(dir[i], RAY_TINY));
}

/// ray_check_track_child (Surface.hpp:1539-1577): -1 when the crossing lies past the grid (the
/// reference's `false`, ending the axis), 1 when it is in a partition holding any of layers
/// -1, 0, 1 (a candidate: partition gp, squared distance key), else 0.
template <int D, int L>
__device__ __forceinline__ int check_track(const Dev& P, const SurfGeom& g, const float* o,
                                           const float* dir, float od, float vd, float dd,
                                           float plane_pos, int& gp, float& key)
{
	constexpr int NL = 2 * L + 1;
	float p[D];
	crossing<D>(o, dir, od, vd, dd, plane_pos, p);
	// the reference bounds the far side by the grid's size, not offset + size
#pragma unroll
	for (int i = 0; i < D; i++)
		if ((dir[i] > 0.0f && p[i] > (float)g.size[i]) ||
		    (dir[i] < 0.0f && p[i] < (float)g.off[i]))
			return -1;
	if (!inside_f<D, L>(g, p)) return 0;
	Vec<D> pf;
#pragma unroll
	for (int i = 0; i < D; i++) pf[i] = (int)floorf(p[i]);
	gp = part_of<D>(P, g, pf);
	const int sl = __ldg(P.slot + gp);
	if (sl < 0) return 0;
	const int* c = P.lcnt + sl * NL;
	if (!(__ldg(c + L) || __ldg(c + L + 1) || __ldg(c + L - 1))) return 0;
	key = dist2<D>(p, o);
	return 1;
}

/// The planes of one axis in the reference's order (Surface.hpp:527-600): plane 0 is p0 (the
/// next partition boundary, or the grid's edge when the origin is outside); then, when
/// round_to_next(p0) differs from p0, that boundary; then steps of dd * size_partition. The
/// positions are integers, so plane k is computed directly (the reference accumulates it).
struct AxisWalk {
	float dd, od, vd;  // direction sign, origin and direction along the axis
	float p0, b, step;
	int kend;          // planes the reference may test; 0 when the axis is skipped
};

template <int D>
__device__ __forceinline__ float pick(const float* v, int dim)
{
	float r = v[0];
#pragma unroll
	for (int a = 1; a < D; a++)
		if (a == dim) r = v[a];
	return r;
}

template <int D, int L>
__device__ __forceinline__ AxisWalk axis_walk(const Dev& P, const SurfGeom& g, const float* o,
                                              const float* dir, int dim)
{
	AxisWalk w;
	w.od = pick<D>(o, dim);
	w.vd = pick<D>(dir, dim);
	w.dd = sgnf(w.vd);
	w.kend = 0;
	if (w.dd == 0.0f) return w;
	float p0 = round_to_next(P, g, dim, w.dd, w.od);
	float plane[D];
#pragma unroll
	for (int a = 0; a < D; a++) plane[a] = a == dim ? p0 : 0.0f;
	if (!inside_f<D, L>(g, plane)) {
		float pg;
		if (w.dd == -1.0f) {
			pg = (float)(g.off[dim] + g.size[dim]);
			if (p0 < pg) return w;
		} else {
			pg = (float)g.off[dim];
			if (p0 > pg) return w;
		}
		p0 = pg;
	}
	const float p1 = round_to_next(P, g, dim, w.dd, p0);
	const bool has1 = p1 != p0;
	w.p0 = p0;
	w.step = __fmul_rn(w.dd, (float)P.csz[dim]);
	w.b = has1 ? p1 : __fadd_rn(p0, w.step);
	w.kend = (has1 ? 2 : 1) + RAY_MAX_MARCH;
	return w;
}

__device__ __forceinline__ float plane_at(const AxisWalk& w, int k)
{
	return k == 0 ? w.p0 : __fadd_rn(w.b, __fmul_rn((float)(k - 1), w.step));
}

/// Cursor of one axis: its next candidate (key = +inf once the walk has ended), and the key
/// it consumed last (to check that keys never decrease).
struct Cursor {
	float key, plane, last;
	int gp, kn;
	int stale;  // the head was consumed: advance before the next pick
};

/// Moves a cursor to the next candidate of its axis (the reference stops an axis at its first
/// crossing past the grid, except that plane 0's answer is ignored).
template <int D, int L>
__device__ __forceinline__ void advance(const Dev& P, const SurfGeom& g, const float* o,
                                        const float* dir, const AxisWalk& w, Cursor& c)
{
	while (c.kn < w.kend) {
		const int k = c.kn++;
		const float plane = plane_at(w, k);
		int gp = -1;
		float key = 0.0f;
		const int st = check_track<D, L>(P, g, o, dir, w.od, w.vd, w.dd, plane, gp, key);
		if (st == -1 && k >= 1) break;
		if (st == 1) {
			c.key = key;
			c.plane = plane;
			c.gp = gp;
			return;
		}
	}
	c.key = __int_as_float(0x7f800000);
	c.kn = w.kend;
}

struct NextCand {
	float key, plane;
	int disc, gp, axis;  // disc < 0: none
};

/// The candidate after (last_key, last_disc) in (squared distance, discovery index) order, by a
/// full walk of every axis.
template <int D, int L>
__device__ __noinline__ NextCand next_exact(const Dev& P, const SurfGeom& g, float o0, float o1,
                                            float o2, float d0, float d1, float d2,
                                            float last_key, int last_disc)
{
	const float o[3] = {o0, o1, o2}, dir[3] = {d0, d1, d2};
	NextCand b{0.0f, 0.0f, -1, -1, 0};
	int disc = 0;
#pragma unroll 1
	for (int dim = 0; dim < D; dim++) {
		const AxisWalk w = axis_walk<D, L>(P, g, o, dir, dim);
#pragma unroll 1
		for (int k = 0; k < w.kend; k++) {
			int gp = -1;
			float key = 0.0f;
			const int st = check_track<D, L>(P, g, o, dir, w.od, w.vd, w.dd, plane_at(w, k), gp, key);
			if (st == -1 && k >= 1) break;
			if (st != 1) continue;
			const bool after = key > last_key || (key == last_key && disc > last_disc);
			const bool better = b.disc < 0 || key < b.key || (key == b.key && disc < b.disc);
			if (after && better) b = NextCand{key, plane_at(w, k), disc, gp, dim};
			disc++;
		}
	}
	return b;
}

/// Whether the samples of a march in partition h may be stepped over where all their corners
/// lie in it: it is inactive and its background is at least 0.75 in magnitude, so that an
/// interpolation of it alone can never be layer 0.
__device__ __forceinline__ bool skippable(const Home& h)
{
	return h.sl < 0 && isfinite(h.bg) && fabsf(h.bg) >= 0.75f;
}

/// A ray whose march found the sample its convergence starts from (Surface.hpp:1484-1487).
struct ConvItem {
	float pos[3], nrm[3];
	float v;    // interp at pos
	int ray;
	int gp;     // partition whose march found it
	int m;      // candidates the ray had consumed (replayed if the convergence leaves the grid)
	int exact;  // candidates in exact order
	int pad;
};

/// A ray to continue after a convergence that left the grid (Surface.hpp:1491-1494): the
/// partition's ray_child returned ray_miss, so the next candidate follows.
struct ResumeItem {
	int ray;
	int m;       // candidates consumed before (replayed without marching)
	int exact;   // candidates in exact order
	int origin;  // the origin's partition is still to march
};

/// Queues of one pass. counters: [0] next input of k_ray_find, [1] queued convergences,
/// [2] rays resumed by k_ray_conv, [3] next convergence, [4] next ray of k_ray_march,
/// [5] rays k_ray_march leaves to k_ray_find.
struct RayQueues {
	int* counters;
	ConvItem* conv;
	const ResumeItem* find_in;  // input of k_ray_find
	const int* find_n_ptr;      // its length in device memory, or null: find_n
	int find_n;
	ResumeItem* resume_out;     // rays k_ray_conv sends back
	ResumeItem* slow;           // rays k_ray_march leaves to k_ray_find
};

/// Candidate lists of k_ray_walk, structure of arrays over the rays of a pass: entry j of ray
/// r at j * n + r (the runs of axes 0..D-1 one after another, each in its walk's order; a
/// candidate is its partition and plane, its key is recomputed from them), run lengths at
/// a * n + r; a first run length of -1 sends the ray to k_ray_find.
constexpr int RAY_LIST = 24;
struct RayLists {
	float* plane;
	int* gp;
	int* cnt;
	int n;
};

__device__ __forceinline__ int fetch_next(int* counter)
{
	cg::coalesced_group grp = cg::coalesced_threads();
	int base = 0;
	if (grp.thread_rank() == 0) base = atomicAdd(counter, (int)grp.size());
	return grp.shfl(base, 0) + (int)grp.thread_rank();
}

/// Surface::ray up to the sample where a convergence starts (Surface.hpp:468-616 with
/// ray_child, 1450-1487), for the rays k_ray_walk could not list and those resumed after a
/// convergence left the grid. Persistent threads, one ray at a time per thread: the origin's
/// partition, then candidates in order (merged from per-axis cursors, or in exact order),
/// marching each; a ray with a convergence to run is queued for k_ray_conv, a ray without
/// candidates left gets ray_miss.
template <int D, int L>
__global__ void __launch_bounds__(RAY_THREADS) k_ray_find(const __grid_constant__ Dev P,
                                                          const __grid_constant__ SurfGeom G,
                                                          const float* org, const float* dirs,
                                                          RayQueues Q, float* hit)
{
	__shared__ AxisWalk s_aw[RAY_THREADS][D];
	__shared__ Cursor s_cur[RAY_THREADS][D];
	AxisWalk* aw = s_aw[threadIdx.x];
	Cursor* cur = s_cur[threadIdx.x];
	const SurfGeom& g = G;
	const float INF = __int_as_float(0x7f800000);
	int ray = 0, phase = PH_FETCH;
	float o[D], dir[D];
	float pos[D];  // start of the partition's march
	Home hm;       // the partition marched
	bool bskip = false;
	int k = 0;           // march sample
	int prev = -1, consumed = 0, replay = 0;
	bool exact = false, ready = false;
	float last_key = -1.0f;
	int last_disc = -1;

	const int n_in = Q.find_n_ptr ? *Q.find_n_ptr : Q.find_n;
	for (;;) {
		if (phase == PH_FETCH) {
			const int idx = fetch_next(Q.counters);
			if (idx >= n_in) break;
			const ResumeItem r = Q.find_in[idx];
			ray = r.ray;
			replay = r.m;
			exact = r.exact != 0;
			const bool origin = r.origin != 0;
#pragma unroll
			for (int a = 0; a < D; a++) {
				o[a] = __ldg(org + (size_t)ray * D + a);
				dir[a] = __ldg(dirs + (size_t)ray * D + a);
			}
			ready = false;
			prev = -1;
			consumed = 0;
			last_key = -1.0f;
			last_disc = -1;
			phase = PH_NEXT;
			if (origin && inside_f<D, L>(g, o)) {
				// the origin's partition first; Eigen cast<int> truncates
				Vec<D> pc;
#pragma unroll
				for (int a = 0; a < D; a++) pc[a] = (int)o[a];
				hm = home_of<D>(P, part_of<D>(P, g, pc));
				bskip = skippable(hm);
#pragma unroll
				for (int a = 0; a < D; a++) pos[a] = o[a];
				k = 0;
				phase = PH_MARCH;
			}
		}
		while (phase == PH_NEXT) {
			int gp = -1, axis = 0;
			float plane = 0.0f;
			if (!exact) {
				if (!ready) {
#pragma unroll 1
					for (int a = 0; a < D; a++) {
						aw[a] = axis_walk<D, L>(P, g, o, dir, a);
						cur[a].kn = 0;
						cur[a].last = -1.0f;
						cur[a].stale = 1;
					}
					ready = true;
				}
				bool down = false;
				float bk = INF;
#pragma unroll 1
				for (int a = 0; a < D; a++) {
					if (cur[a].stale) {
						advance<D, L>(P, g, o, dir, aw[a], cur[a]);
						cur[a].stale = 0;
						down = down || cur[a].key < cur[a].last;
					}
					if (cur[a].key < bk) {  // ties go to the lower axis
						bk = cur[a].key;
						axis = a;
					}
				}
				if (down) {  // keys decreased along an axis: restart in exact order
					exact = true;
					prev = -1;
					consumed = 0;
					replay = 0;
					continue;
				}
				if (bk != INF) {
					gp = cur[axis].gp;
					plane = cur[axis].plane;
					cur[axis].last = bk;
					cur[axis].stale = 1;
				}
			} else {
				const NextCand c = next_exact<D, L>(P, g, o[0], o[1], D > 2 ? o[D - 1] : 0.0f,
				                                    dir[0], dir[1], D > 2 ? dir[D - 1] : 0.0f,
				                                    last_key, last_disc);
				if (c.disc >= 0) {
					last_key = c.key;
					last_disc = c.disc;
					gp = c.gp;
					axis = c.axis;
					plane = c.plane;
				}
			}
			if (gp < 0) {  // no candidate left: ray_miss
#pragma unroll
				for (int a = 0; a < D; a++) hit[(size_t)ray * D + a] = FLT_MAX;
				phase = PH_FETCH;
				break;
			}
			consumed++;
			if (gp == prev) continue;  // std::unique on the partition
			prev = gp;
			if (consumed <= replay) continue;  // marched before this resumed pass
			const float vd = pick<D>(dir, axis);
			crossing<D>(o, dir, pick<D>(o, axis), vd, sgnf(vd), plane, pos);
			hm = home_of<D>(P, gp);
			bskip = skippable(hm);
			k = 0;
			phase = PH_MARCH;
		}
		if (phase == PH_FETCH) continue;

		// one sample of the partition's march (ray_child, Surface.hpp:1463-1480)
		int blo[D], bhi[D];
#pragma unroll
		for (int a = 0; a < D; a++) {
			blo[a] = hm.lo[a];
			bhi[a] = blo[a] + P.csz[a];
		}
		float x[D];
		bool in;
		for (;;) {
			const float t = __fmul_rn(0.5f, (float)k);  // the reference's t += 0.5, exact
#pragma unroll
			for (int a = 0; a < D; a++)
				x[a] = k == 0 ? pos[a] : __fadd_rn(pos[a], __fmul_rn(dir[a], t));
			in = k < RAY_MAX_MARCH && inside_box<D>(x, blo, bhi);
			// In an inactive partition, a sample whose corners all lie in it interpolates its
			// background (to within 1e-6 relative), which is never layer 0 there: the reference
			// tests it and moves on, so step over it without reading.
			if (!in || !bskip || !corners_inside<D>(P, g, blo, x)) break;
			k++;
		}
		if (!in) {
			phase = PH_NEXT;  // left the partition: next candidate
			continue;
		}
		const HomeInterp<D, L> ip{P, g, hm};
		const float c = ip(x);
		if (layer_id(c, P.err) == 0) {
			float gr[D];
			grad_with<D, L>(ip, g, x, c, gr);
			normalize_d<D>(gr);
			if (dot_e<D>(gr, dir) < 0.0f) {
				const int qi = atomicAdd(Q.counters + 1, 1);
				ConvItem& it = Q.conv[qi];
#pragma unroll
				for (int a = 0; a < D; a++) {
					it.pos[a] = x[a];
					it.nrm[a] = gr[a];
				}
				it.v = c;
				it.ray = ray;
				it.gp = hm.gp;
				it.m = consumed;
				it.exact = exact ? 1 : 0;
				phase = PH_FETCH;
				continue;
			}
		}
		k++;
	}
}

/// The isogrid value at an integer position, read relative to home h as HomeInterp reads its
/// corners (positions more than one partition away through the partition lookup).
template <int D, int L>
__device__ __forceinline__ float home_get(const Dev& P, const SurfGeom& g, const Home& h,
                                          const Vec<D>& q)
{
	if (!in_grid<D>(g, q)) return (float)(L + 1);
	int nb = h.gp, leaf = 0, stride = 1;
#pragma unroll
	for (int a = D - 1; a >= 0; a--) {
		const int cs = P.csz[a];
		const int r = q[a] - h.lo[a];
		if (r < -cs || r >= 2 * cs) return get_phi<D, L>(P, g, q);
		const int st = (r >= cs) - (r < 0);
		nb += st * stride;
		leaf += (r - st * cs) * P.lstr[a];
		stride *= g.ccount[a];
	}
	const int sl = nb == h.gp ? h.sl : __ldg(P.slot + nb);
	if (sl >= 0) return __ldg(P.phi + (size_t)sl * P.BV + leaf);
	return nb == h.gp ? h.bg : __ldg(P.bg + nb);
}

/// Sub-blocks of RAY_SB^D nodes of an active brick, for the march: a sample whose floor lies in
/// sub-block b has its 2^D corners among the sub-block's nodes and the next node along each
/// axis. If all of those are >= 0.5001 (or all <= -0.5001), every interpolation there is too (a
/// convex combination, rounded), so its layer is not 0 and the sample can be stepped over.
constexpr int RAY_SB = 4;

__device__ __forceinline__ int sub_count(int cs) { return (cs + RAY_SB - 1) / RAY_SB; }

/// Flags of every sub-block of every active brick of surface s (1: all >= 0.5001, 2: all
/// <= -0.5001, else 0), brick slot major. One thread per (slot, sub-block).
template <int D, int L>
__global__ void __launch_bounds__(256) k_ray_ranges(const __grid_constant__ Dev P,
                                                    const __grid_constant__ SurfGeom G, int s,
                                                    uint8_t* flags, int nsub)
{
	const SurfGeom& g = G;
	const size_t total = (size_t)P.nslots * nsub;
	for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
	     t += (size_t)gridDim.x * blockDim.x) {
		const int slot = (int)(t / nsub);
		const int gp = __ldg(P.slot_gp + slot);
		uint8_t f = 0;
		if (gp >= 0 && __ldg(P.surf_of + gp) == s && __ldg(P.slot + gp) == slot) {
			const Home h = home_of<D>(P, gp);
			int b[D], rem = (int)(t % nsub);
#pragma unroll
			for (int a = D - 1; a >= 0; a--) {
				const int nb = sub_count(P.csz[a]);
				b[a] = rem % nb;
				rem /= nb;
			}
			float mn = __int_as_float(0x7f800000), mx = -mn;
			constexpr int E = RAY_SB + 1;
			int cnt = 1;
#pragma unroll
			for (int a = 0; a < D; a++) cnt *= E;
			for (int i = 0; i < cnt; i++) {
				Vec<D> q;
				int r = i;
#pragma unroll
				for (int a = D - 1; a >= 0; a--) {
					q[a] = h.lo[a] + b[a] * RAY_SB + r % E;
					r /= E;
				}
				const float v = home_get<D, L>(P, g, h, q);
				mn = fminf(mn, v);
				mx = fmaxf(mx, v);
			}
			f = mn >= 0.5001f ? 1 : (mx <= -0.5001f ? 2 : 0);
		}
		flags[t] = f;
	}
}

/// grad at x (value c) around home h, normalised: out of line for the march, which needs it only
/// at zero-layer samples.
template <int D, int L>
__device__ __noinline__ float3 march_grad(const Dev& P, const SurfGeom& g, Home h, float x0,
                                          float x1, float x2, float c)
{
	const float x[3] = {x0, x1, x2};
	float gr[3] = {0.0f, 0.0f, 0.0f};
	grad_with<D, L>(HomeInterp<D, L>{P, g, h}, g, x, c, gr);
	normalize_d<D>(gr);
	return make_float3(gr[0], gr[1], gr[2]);
}

/// The key (squared distance from the origin) of entry j of a ray's list, an axis-`dim` crossing:
/// the same arithmetic as when the walk found it.
template <int D>
__device__ __forceinline__ float list_key(const RayLists& R, int ray, int j, const float* o,
                                          const float* dir, int dim)
{
	const float plane = R.plane[(size_t)j * R.n + ray];
	const float vd = pick<D>(dir, dim);
	float p[D];
	crossing<D>(o, dir, pick<D>(o, dim), vd, sgnf(vd), plane, p);
	return dist2<D>(p, o);
}

/// The candidate walk of Surface::ray (Surface.hpp:520-600), one ray per thread: every
/// plane of every axis, the candidates of each axis stored in its walk's order. A ray with more
/// than RAY_LIST candidates, or whose keys decrease along an axis, is marked for k_ray_find.
template <int D, int L>
__global__ void __launch_bounds__(RAY_THREADS) k_ray_walk(const __grid_constant__ Dev P,
                                                          const __grid_constant__ SurfGeom G,
                                                          const float* org, const float* dirs,
                                                          RayLists R)
{
	const SurfGeom& g = G;
	const int n = R.n;
	for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
		float o[D], dir[D];
#pragma unroll
		for (int a = 0; a < D; a++) {
			o[a] = __ldg(org + (size_t)r * D + a);
			dir[a] = __ldg(dirs + (size_t)r * D + a);
		}
		int total = 0;
		bool ok = true;
#pragma unroll 1
		for (int dim = 0; dim < D; dim++) {
			const AxisWalk w = axis_walk<D, L>(P, g, o, dir, dim);
			int cnt = 0;
			float last = -1.0f;
#pragma unroll 1
			for (int k = 0; k < w.kend; k++) {
				const float plane = plane_at(w, k);
				int gp = -1;
				float key = 0.0f;
				const int st = check_track<D, L>(P, g, o, dir, w.od, w.vd, w.dd, plane, gp, key);
				if (st == -1 && k >= 1) break;
				if (st != 1) continue;
				ok = ok && key >= last;
				last = key;
				if (total < RAY_LIST) {
					const size_t j = (size_t)total * n + r;
					R.plane[j] = plane;
					R.gp[j] = gp;
				}
				total++;
				cnt++;
			}
			R.cnt[(size_t)dim * n + r] = cnt;
		}
		if (!ok || total > RAY_LIST) R.cnt[r] = -1;
	}
}

/// Surface::ray up to the sample where a convergence starts, over k_ray_walk's lists: the
/// origin's partition, then the candidates in order (the merge of the per-axis runs, ties to
/// the lower axis), consecutive repeats of a partition dropped, marching each. Persistent
/// threads; a ray with a convergence to run is queued for k_ray_conv, a ray without candidates
/// left gets ray_miss, an unlisted ray goes to k_ray_find.
template <int D, int L>
__global__ void __launch_bounds__(RAY_THREADS, 8) k_ray_march(const __grid_constant__ Dev P,
                                                           const __grid_constant__ SurfGeom G,
                                                           const float* org, const float* dirs,
                                                           int mode, RayLists R,
                                                           const uint8_t* ranges, int nsub,
                                                           RayQueues Q, float* hit)
{
	__shared__ int s_head[D][RAY_THREADS], s_end[D][RAY_THREADS];
	__shared__ float s_key[D][RAY_THREADS];  // key of each run's head
	const int tid = threadIdx.x;
	const SurfGeom& g = G;
	const int n = R.n;
	int ray = 0, phase = PH_FETCH;
	float o[D], dir[D];
	float pos[D];  // start of the partition's march
	Home hm;
	bool bskip = false;
	int k = 0;
	int stale = 0;  // runs whose head key is to be computed (bit per axis)
	int prev = -1, consumed = 0;
	for (;;) {
		if (phase == PH_FETCH) {
			ray = fetch_next(Q.counters + 4);
			if (ray >= n) break;
			if (mode != 0 || R.cnt[ray] < 0) {
				const int si = atomicAdd(Q.counters + 5, 1);
				Q.slow[si] = ResumeItem{ray, 0, mode == 1 ? 1 : 0, 1};
				continue;
			}
#pragma unroll
			for (int a = 0; a < D; a++) {
				o[a] = __ldg(org + (size_t)ray * D + a);
				dir[a] = __ldg(dirs + (size_t)ray * D + a);
			}
			int start = 0;
#pragma unroll
			for (int a = 0; a < D; a++) {
				s_head[a][tid] = start;
				start += R.cnt[(size_t)a * n + ray];
				s_end[a][tid] = start;
			}
			stale = (1 << D) - 1;
			prev = -1;
			consumed = 0;
			phase = PH_NEXT;
			if (inside_f<D, L>(g, o)) {
				// the origin's partition first; Eigen cast<int> truncates
				Vec<D> pc;
#pragma unroll
				for (int a = 0; a < D; a++) pc[a] = (int)o[a];
				hm = home_of<D>(P, part_of<D>(P, g, pc));
				bskip = skippable(hm);
#pragma unroll
				for (int a = 0; a < D; a++) pos[a] = o[a];
				k = 0;
				phase = PH_MARCH;
			}
		}
		while (phase == PH_NEXT) {
			int axis = -1;
			float bk = 0.0f;
#pragma unroll 1
			for (int a = 0; a < D; a++) {
				const int h = s_head[a][tid];
				if (h >= s_end[a][tid]) continue;
				if ((stale >> a) & 1) s_key[a][tid] = list_key<D>(R, ray, h, o, dir, a);
				const float ka = s_key[a][tid];
				if (axis < 0 || ka < bk) {  // ties go to the lower axis
					bk = ka;
					axis = a;
				}
			}
			stale = 0;
			if (axis < 0) {  // no candidate left: ray_miss
#pragma unroll
				for (int a = 0; a < D; a++) hit[(size_t)ray * D + a] = FLT_MAX;
				phase = PH_FETCH;
				break;
			}
			const int j = s_head[axis][tid]++;
			stale = 1 << axis;
			consumed++;
			const int gp = R.gp[(size_t)j * n + ray];
			if (gp == prev) continue;  // std::unique on the partition
			prev = gp;
			const float plane = R.plane[(size_t)j * n + ray];
			const float vd = pick<D>(dir, axis);
			crossing<D>(o, dir, pick<D>(o, axis), vd, sgnf(vd), plane, pos);
			hm = home_of<D>(P, gp);
			bskip = skippable(hm);
			k = 0;
			phase = PH_MARCH;
		}
		if (phase == PH_FETCH) continue;

		// one sample of the partition's march (ray_child, Surface.hpp:1463-1480)
		int blo[D], bhi[D];
#pragma unroll
		for (int a = 0; a < D; a++) {
			blo[a] = hm.lo[a];
			bhi[a] = blo[a] + P.csz[a];
		}
		float x[D];
		bool in;
		const uint8_t* rng = hm.sl >= 0 ? ranges + (size_t)hm.sl * nsub : nullptr;
		for (;;) {
			const float t = __fmul_rn(0.5f, (float)k);  // the reference's t += 0.5, exact
#pragma unroll
			for (int a = 0; a < D; a++)
				x[a] = k == 0 ? pos[a] : __fadd_rn(pos[a], __fmul_rn(dir[a], t));
			in = k < RAY_MAX_MARCH && inside_box<D>(x, blo, bhi);
			if (!in) break;
			// Samples that cannot be layer 0 are stepped over without interpolating: in an
			// inactive partition, those whose corners all lie in it (they interpolate its
			// background); in an active one, those in a sub-block of one sign, >= 0.5001 in
			// magnitude (k_ray_ranges).
			bool skip;
			if (rng) {
				int idx = 0;
#pragma unroll
				for (int a = 0; a < D; a++) {
					const int r = (int)floorf(x[a]) - blo[a];
					idx = idx * sub_count(P.csz[a]) + r / RAY_SB;
				}
				skip = __ldg(rng + idx) != 0;
			} else {
				skip = bskip && corners_inside<D>(P, g, blo, x);
			}
			if (!skip) break;
			k++;
		}
		if (!in) {
			phase = PH_NEXT;  // left the partition: next candidate
			continue;
		}
		const float c = HomeInterp<D, L>{P, g, hm}(x);
		if (layer_id(c, P.err) == 0) {
			const float3 g3 = march_grad<D, L>(P, g, hm, x[0], x[1], D > 2 ? x[D - 1] : 0.0f, c);
			const float gr[3] = {g3.x, g3.y, g3.z};
			if (dot_e<D>(gr, dir) < 0.0f) {
				const int qi = atomicAdd(Q.counters + 1, 1);
				ConvItem& it = Q.conv[qi];
#pragma unroll
				for (int a = 0; a < D; a++) {
					it.pos[a] = x[a];
					it.nrm[a] = gr[a];
				}
				it.v = c;
				it.ray = ray;
				it.gp = hm.gp;
				it.m = consumed;
				it.exact = 0;
				phase = PH_FETCH;
				continue;
			}
		}
		k++;
	}
}

/// The convergence of ray_child (Surface.hpp:1487-1510): step along the normal by the
/// interpolated distance until it is within TINY or the normal turns away, at most 100 steps.
/// A point that leaves the grid is ray_miss for that partition, and the ray is queued to
/// continue with its next candidate. Persistent threads: each loop iteration is one step of
/// the thread's current ray; a thread whose ray is done takes the next queued one.
template <int D, int L>
__global__ void __launch_bounds__(RAY_THREADS, 8) k_ray_conv(const __grid_constant__ Dev P,
                                                          const __grid_constant__ SurfGeom G,
                                                          const float* dirs, RayQueues Q,
                                                          float* hit)
{
	const SurfGeom& g = G;
	const int n = Q.counters[1];
	int i = -1, ray = 0, step = 0;
	float pos[D], nrm[D], dir[D], v = 0.0f;
	Home hm;
	for (;;) {
		if (i < 0) {
			i = fetch_next(Q.counters + 3);
			if (i >= n) break;
			const ConvItem& it = Q.conv[i];
			ray = it.ray;
#pragma unroll
			for (int a = 0; a < D; a++) {
				pos[a] = it.pos[a];
				nrm[a] = it.nrm[a];
				dir[a] = __ldg(dirs + (size_t)ray * D + a);
			}
			v = it.v;
			hm = home_of<D>(P, it.gp);
			step = 0;
		}
		const float dist = v;
#pragma unroll
		for (int a = 0; a < D; a++) pos[a] = __fsub_rn(pos[a], __fmul_rn(nrm[a], dist));
		if (!inside_f<D, L>(g, pos)) {
			const ConvItem& it = Q.conv[i];
			const int ri = atomicAdd(Q.counters + 2, 1);
			Q.resume_out[ri] = ResumeItem{ray, it.m, it.exact, 0};
			i = -1;
			continue;
		}
		bool done = fabsf(dist) <= RAY_TINY || dot_e<D>(nrm, dir) >= 0.0f;
		if (!done) {
			const HomeInterp<D, L> ip{P, g, hm};
			v = ip(pos);
			grad_with<D, L>(ip, g, pos, v, nrm);
			normalize_d<D>(nrm);
			done = ++step == RAY_CONVERGE_STEPS;
		}
		if (done) {
#pragma unroll
			for (int a = 0; a < D; a++) hit[(size_t)ray * D + a] = pos[a];
			i = -1;
		}
	}
}

/// Bytes of work memory for a pass over n rays.
size_t ray_work_bytes(size_t n, int D)
{
	const size_t b = 256 + n * sizeof(ConvItem) + 3 * n * sizeof(ResumeItem) +
	                 n * RAY_LIST * (sizeof(float) + sizeof(int)) + (size_t)D * n * sizeof(int);
	return (b + 255) & ~(size_t)255;
}

/// Sub-blocks per brick.
int ray_nsub(const EngineBase& eng)
{
	int nsub = 1;
	for (int a = 0; a < eng.dims(); a++) nsub *= (eng.part(a) + RAY_SB - 1) / RAY_SB;
	return nsub;
}

template <int D, int L>
void launch_rays(EngineBase& eng, int s, const float* o, const float* d, size_t n, int mode,
                 char* work, const uint8_t* ranges, float* h)
{
	struct Occ {
		int sms = 0, walk = 0, march = 0, find = 0, conv = 0;
	};
	static Occ occ;
	if (occ.sms == 0) {
		int dev = 0;
		FG_CUDA(cudaGetDevice(&dev));
		FG_CUDA(cudaDeviceGetAttribute(&occ.sms, cudaDevAttrMultiProcessorCount, dev));
		FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ.walk, k_ray_walk<D, L>, RAY_THREADS, 0));
		FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ.march, k_ray_march<D, L>, RAY_THREADS, 0));
		FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ.find, k_ray_find<D, L>, RAY_THREADS, 0));
		FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ.conv, k_ray_conv<D, L>, RAY_THREADS, 0));
		occ.walk = std::max(occ.walk, 1);
		occ.march = std::max(occ.march, 1);
		occ.find = std::max(occ.find, 1);
		occ.conv = std::max(occ.conv, 1);
	}
	auto grid = [&](int per_sm) {
		return (unsigned)std::min<size_t>((n + RAY_THREADS - 1) / RAY_THREADS, (size_t)occ.sms * per_sm);
	};
	cudaStream_t st = eng.stream();
	const Dev& P = eng.dev();
	const SurfGeom G = eng.geometry(s);
	int* counters = (int*)work;
	ConvItem* conv = (ConvItem*)(work + 256);
	ResumeItem* res[3] = {(ResumeItem*)(conv + n), (ResumeItem*)(conv + n) + n,
	                      (ResumeItem*)(conv + n) + 2 * n};
	float* lk = (float*)(res[2] + n);
	RayLists R{lk, (int*)(lk + n * RAY_LIST), (int*)(lk + 2 * n * RAY_LIST), (int)n};
	RayQueues Q{counters, conv, res[2], counters + 5, 0, res[0], res[2]};
	FG_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(int), st));
	if (mode == 0) {
		FG_RUN("k_ray_walk", st, k_ray_walk<D, L><<<grid(occ.walk), RAY_THREADS, 0, st>>>(P, G, o, d, R););
		FG_CUDA(cudaGetLastError());
	}
	FG_RUN("k_ray_march", st, k_ray_march<D, L><<<grid(occ.march), RAY_THREADS, 0, st>>>(P, G, o, d, mode, R, ranges, ray_nsub(eng), Q, h););
	FG_CUDA(cudaGetLastError());
	for (int pass = 0;; pass++) {
		if (pass > RAY_MAX_MARCH) throw Error(-13, "raycasting did not finish");
		FG_RUN("k_ray_find", st, k_ray_find<D, L><<<grid(occ.find), RAY_THREADS, 0, st>>>(P, G, o, d, Q, h););
		FG_CUDA(cudaGetLastError());
		FG_RUN("k_ray_conv", st, k_ray_conv<D, L><<<grid(occ.conv), RAY_THREADS, 0, st>>>(P, G, d, Q, h););
		FG_CUDA(cudaGetLastError());
		int resumed = 0;
		FG_CUDA(cudaMemcpyAsync(&resumed, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
		FG_CUDA(cudaStreamSynchronize(st));
		if (resumed == 0) break;
		// the rays whose convergence left the grid continue with their next candidates
		Q.find_in = Q.resume_out;
		Q.find_n_ptr = nullptr;
		Q.find_n = resumed;
		Q.resume_out = res[(pass + 1) & 1];
		FG_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(int), st));
	}
}

/// k_ray_ranges over the bricks of surface s.
void ranges_launch(EngineBase& eng, int s, uint8_t* ranges, int nsub)
{
	const Dev& P = eng.dev();
	const SurfGeom G = eng.geometry(s);
	const size_t total = (size_t)P.nslots * nsub;
	const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
	cudaStream_t st = eng.stream();
	const int D = eng.dims(), L = eng.layers();
#define FG_CASE(dd, ll) \
	if (D == dd && L == ll) FG_RUN("k_ray_ranges", st, k_ray_ranges<dd, ll><<<blocks, 256, 0, st>>>(P, G, s, ranges, nsub););
	FG_CASE(2, 1) FG_CASE(2, 2) FG_CASE(2, 3) FG_CASE(2, 4)
	FG_CASE(3, 1) FG_CASE(3, 2) FG_CASE(3, 3) FG_CASE(3, 4)
#undef FG_CASE
	FG_CUDA(cudaGetLastError());
}

}  // namespace

void ray_batch(EngineBase& eng, int s, const float* origins, const float* dirs, size_t n,
               float* hits, bool device_ptrs, int mode)
{
	if (s < 0 || s >= eng.surfaces()) throw Error(-1, "surface index out of range");
	if (mode < 0 || mode > 2) throw Error(-1, "candidate order mode is 0, 1 or 2");
	if (n == 0) return;
	const int D = eng.dims(), L = eng.layers();
	// passes of at most 2^21 rays bound the work memory (about 600 MB)
	const size_t chunk = std::min<size_t>(n, (size_t)1 << 21);
	const size_t cbytes = chunk * D * sizeof(float);
	const size_t work = ray_work_bytes(chunk, D);
	cudaStream_t st = eng.stream();
	// one stream-ordered allocation: the pass's work memory, then (host arrays) staging for
	// origins, dirs and hits
	const int nsub = ray_nsub(eng);
	const size_t rbytes = ((size_t)eng.dev().nslots * nsub + 255) & ~(size_t)255;
	char* dev = nullptr;
	FG_CUDA(cudaMallocAsync((void**)&dev, rbytes + work + (device_ptrs ? 0 : 3 * cbytes), st));
	uint8_t* ranges = (uint8_t*)dev;
	dev += rbytes;
	try {
		ranges_launch(eng, s, ranges, nsub);
		for (size_t b = 0; b < n; b += chunk) {
			const size_t m = std::min(chunk, n - b);
			const size_t bytes = m * D * sizeof(float);
			const float* dorg = origins + b * D;
			const float* ddir = dirs + b * D;
			float* dhit = hits + b * D;
			if (!device_ptrs) {
				float* f = (float*)(dev + work);
				FG_CUDA(cudaMemcpyAsync(f, origins + b * D, bytes, cudaMemcpyHostToDevice, st));
				FG_CUDA(cudaMemcpyAsync(f + chunk * D, dirs + b * D, bytes, cudaMemcpyHostToDevice, st));
				dorg = f;
				ddir = f + chunk * D;
				dhit = f + 2 * chunk * D;
			}
			bool launched = false;
#define FG_CASE(dd, ll)                                                              \
	if (D == dd && L == ll) {                                                        \
		launch_rays<dd, ll>(eng, s, dorg, ddir, m, mode, dev, ranges, dhit);         \
		launched = true;                                                             \
	}
			FG_CASE(2, 1) FG_CASE(2, 2) FG_CASE(2, 3) FG_CASE(2, 4)
			FG_CASE(3, 1) FG_CASE(3, 2) FG_CASE(3, 3) FG_CASE(3, 4)
#undef FG_CASE
			if (!launched) throw Error(-1, "unsupported dimension or layer count");
			if (!device_ptrs)
				FG_CUDA(cudaMemcpyAsync(hits + b * D, dhit, bytes, cudaMemcpyDeviceToHost, st));
		}
	} catch (...) {
		cudaFreeAsync(dev - rbytes, st);
		throw;
	}
	FG_CUDA(cudaFreeAsync(dev - rbytes, st));
	eng.sync();
	eng.check_errors();
}

}  // namespace fg
