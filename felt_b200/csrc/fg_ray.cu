// Raycasting to the zero curve: Felt's Surface::ray (include/Felt/Surface.hpp:468-616,
// 1450-1598) for a batch of rays, one thread per ray.
//
// Each thread follows the reference step by step: the partition holding the origin first;
// then, per axis, the partition planes the ray crosses, keeping the partitions that hold any of
// layers -1, 0, 1; those in order of squared distance from the origin (ties in the order found;
// std::sort leaves that order unspecified), consecutive repeats of a partition dropped; within
// each, samples every half unit along the ray until a zero-layer sample faces the ray, from
// which it converges onto the zero curve along the interpolated gradient. Arithmetic is FP32 in
// the reference's order (Eigen's ParametrizedLine / Hyperplane formulas; dot products and
// squared norms summed x0 + (x1 + x2)).
//
// The candidates of a ray are buffered per thread (up to `buffer` of them, at most RAY_BUFFER)
// and insertion-sorted there. A ray that finds more walks its planes again for each next
// candidate in (distance, discovery) order instead, which visits the same sequence without a
// buffer of unbounded size.
#include <cfloat>
#include <cstdint>

#include "fg_engine.cuh"
#include "fg_field.cuh"
#include "fg_ray.cuh"

namespace fg {

namespace {

constexpr float RAY_TINY = 0.00001f;     // Surface.hpp:67
constexpr int RAY_CONVERGE_STEPS = 100;  // Surface.hpp:1488
constexpr int RAY_MAX_MARCH = 1 << 16;   // bound on the reference's open loops
constexpr int RAY_BUFFER = 64;

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

/// The partition of an in-grid integer position (PartitionedMixin.hpp:221-245).
template <int D>
__device__ __forceinline__ int part_of(const Dev& P, const SurfGeom& g, const Vec<D>& q)
{
	int gp, leaf;
	locate<D>(P, g, q, gp, leaf);
	return gp;
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

/// ray within one partition (Surface.hpp:1450-1530); true with the hit in `out`.
template <int D, int L>
__device__ bool ray_child(const Dev& P, const SurfGeom& g, int gp, const float* start,
                          const float* dir, float* out)
{
	const PoolGet<D, L> get{P, g};
	int lo[D], hi[D];
#pragma unroll
	for (int a = 0; a < D; a++) {
		lo[a] = P.porig[gp * 3 + a];
		hi[a] = lo[a] + P.csz[a];
	}
	float pos[D];
#pragma unroll
	for (int a = 0; a < D; a++) pos[a] = start[a];
	float t = 0.0f;
	for (int it = 0; it < RAY_MAX_MARCH && inside_box<D>(pos, lo, hi); it++) {
		if (layer_id(interp<D>(get, pos), P.err) == 0) {
			float n[D];
			grad_f<D, L>(get, g, pos, n);
			normalize_d<D>(n);
			if (dot_e<D>(n, dir) < 0.0f) {
				for (int k = 0; k < RAY_CONVERGE_STEPS; k++) {
					const float dist = interp<D>(get, pos);
#pragma unroll
					for (int a = 0; a < D; a++) pos[a] = __fsub_rn(pos[a], __fmul_rn(n[a], dist));
					if (!inside_f<D, L>(g, pos)) return false;
					if (fabsf(dist) <= RAY_TINY || dot_e<D>(n, dir) >= 0.0f) break;
					grad_f<D, L>(get, g, pos, n);
					normalize_d<D>(n);
				}
#pragma unroll
				for (int a = 0; a < D; a++) out[a] = pos[a];
				return true;
			}
		}
		t = __fadd_rn(t, 0.5f);
#pragma unroll
		for (int a = 0; a < D; a++) pos[a] = __fadd_rn(start[a], __fmul_rn(dir[a], t));
	}
	return false;
}

/// ray_check_track_child (Surface.hpp:1539-1577) for the plane x[dim] = plane_pos: false when
/// the crossing lies past the grid (the walk along this axis ends); a candidate partition is
/// passed to emit(pos, gp).
template <int D, int L, class Emit>
__device__ __forceinline__ bool check_track(const Dev& P, const SurfGeom& g, const float* o,
                                            const float* dir, int dim, float dd, float plane_pos,
                                            Emit& emit)
{
	constexpr int NL = 2 * L + 1;
	// Hyperplane(normal = -dd e_dim, offset = plane_pos * dd); ParametrizedLine(o, dir)
	const float nd = -dd, off = __fmul_rn(plane_pos, dd);
	const float t = -__fdiv_rn(__fadd_rn(off, __fmul_rn(nd, o[dim])), __fmul_rn(nd, dir[dim]));
	float p[D];
#pragma unroll
	for (int i = 0; i < D; i++) p[i] = __fadd_rn(o[i], __fmul_rn(dir[i], t));
#pragma unroll
	for (int i = 0; i < D; i++) p[i] = __fadd_rn(p[i], __fmul_rn(dir[i], RAY_TINY));
	// the reference bounds the far side by the grid's size, not offset + size
#pragma unroll
	for (int i = 0; i < D; i++)
		if ((dir[i] > 0.0f && p[i] > (float)g.size[i]) ||
		    (dir[i] < 0.0f && p[i] < (float)g.off[i]))
			return false;
	if (!inside_f<D, L>(g, p)) return true;
	Vec<D> pf;
#pragma unroll
	for (int i = 0; i < D; i++) pf[i] = (int)floorf(p[i]);
	const int gp = part_of<D>(P, g, pf);
	const int sl = P.slot[gp];
	if (sl >= 0 && (P.lcnt[sl * NL + L] || P.lcnt[sl * NL + L + 1] || P.lcnt[sl * NL + L - 1]))
		emit(p, gp);
	return true;
}

/// The candidate walk of Surface::ray (Surface.hpp:520-600): every crossing of every axis, in
/// the reference's discovery order.
template <int D, int L, class Emit>
__device__ void walk_planes(const Dev& P, const SurfGeom& g, const float* o, const float* dir,
                            Emit& emit)
{
	for (int dim = 0; dim < D; dim++) {
		const float dd = (float)((0.0f < dir[dim]) - (dir[dim] < 0.0f));
		if (dd == 0.0f) continue;
		float pp = round_to_next(P, g, dim, dd, o[dim]);
		float plane[D];
#pragma unroll
		for (int a = 0; a < D; a++) plane[a] = 0.0f;
		plane[dim] = pp;
		if (!inside_f<D, L>(g, plane)) {
			float pg;
			if (dd == -1.0f) {
				pg = (float)(g.off[dim] + g.size[dim]);
				if (pp < pg) continue;
			} else {
				pg = (float)g.off[dim];
				if (pp > pg) continue;
			}
			plane[dim] = pg;
		}
		check_track<D, L>(P, g, o, dir, dim, dd, plane[dim], emit);
		pp = round_to_next(P, g, dim, dd, plane[dim]);
		if (pp != plane[dim]) {
			plane[dim] = pp;
			if (!check_track<D, L>(P, g, o, dir, dim, dd, plane[dim], emit)) continue;
		}
		const float cs = (float)P.csz[dim];
		for (int it = 0; it < RAY_MAX_MARCH; it++) {
			plane[dim] = __fadd_rn(plane[dim], __fmul_rn(dd, cs));
			if (!check_track<D, L>(P, g, o, dir, dim, dd, plane[dim], emit)) break;
		}
	}
}

/// Collects candidates in discovery order, up to cap of them; n counts them all.
template <int D>
struct Buffered {
	float (*pos)[D];
	int* gp;
	int cap;
	int n;
	__device__ void operator()(const float* p, int g)
	{
		if (n < cap) {
#pragma unroll
			for (int a = 0; a < D; a++) pos[n][a] = p[a];
			gp[n] = g;
		}
		n++;
	}
};

/// Finds the candidate that follows (key, idx) in (squared distance, discovery) order.
template <int D>
struct NextAfter {
	const float* o;
	float key;
	int idx;
	int i;  // discovery index of the current candidate
	float best_key;
	int best_idx;
	int best_gp;
	float best_pos[D];
	__device__ void operator()(const float* p, int g)
	{
		const float k = dist2<D>(p, o);
		const bool after = k > key || (k == key && i > idx);
		const bool before_best = best_idx < 0 || k < best_key || (k == best_key && i < best_idx);
		if (after && before_best) {
			best_key = k;
			best_idx = i;
			best_gp = g;
#pragma unroll
			for (int a = 0; a < D; a++) best_pos[a] = p[a];
		}
		i++;
	}
};

/// Surface::ray (Surface.hpp:468-616); false on a miss.
template <int D, int L>
__device__ bool ray_cast(const Dev& P, const SurfGeom& g, const float* o, const float* dir,
                         int buffer, float* out)
{
	if (inside_f<D, L>(g, o)) {
		Vec<D> pc;
#pragma unroll
		for (int a = 0; a < D; a++) pc[a] = (int)o[a];  // Eigen cast<int>: truncation
		if (ray_child<D, L>(P, g, part_of<D>(P, g, pc), o, dir, out)) return true;
	}
	float bpos[RAY_BUFFER][D];
	int bgp[RAY_BUFFER];
	Buffered<D> buf{bpos, bgp, buffer < RAY_BUFFER ? buffer : RAY_BUFFER, 0};
	walk_planes<D, L>(P, g, o, dir, buf);
	if (buf.n <= buf.cap) {
		// stable insertion sort by squared distance from the origin
		for (int i = 1; i < buf.n; i++) {
			float p[D];
#pragma unroll
			for (int a = 0; a < D; a++) p[a] = bpos[i][a];
			const int gp = bgp[i];
			const float k = dist2<D>(p, o);
			int j = i - 1;
			while (j >= 0 && dist2<D>(bpos[j], o) > k) {
#pragma unroll
				for (int a = 0; a < D; a++) bpos[j + 1][a] = bpos[j][a];
				bgp[j + 1] = bgp[j];
				j--;
			}
#pragma unroll
			for (int a = 0; a < D; a++) bpos[j + 1][a] = p[a];
			bgp[j + 1] = gp;
		}
		for (int i = 0; i < buf.n; i++) {
			if (i > 0 && bgp[i] == bgp[i - 1]) continue;  // std::unique on the partition
			if (ray_child<D, L>(P, g, bgp[i], bpos[i], dir, out)) return true;
		}
		return false;
	}
	// more candidates than the buffer holds: one walk per candidate, in the same order
	float key = -1.0f;
	int idx = -1, prev_gp = -1;
	for (int c = 0; c < buf.n; c++) {
		NextAfter<D> nx{o, key, idx, 0, 0.0f, -1, -1, {}};
		walk_planes<D, L>(P, g, o, dir, nx);
		if (nx.best_idx < 0) break;
		if (nx.best_gp != prev_gp && ray_child<D, L>(P, g, nx.best_gp, nx.best_pos, dir, out))
			return true;
		prev_gp = nx.best_gp;
		key = nx.best_key;
		idx = nx.best_idx;
	}
	return false;
}

template <int D, int L>
__global__ void __launch_bounds__(128) k_ray(Dev P, int s, const float* org, const float* dir,
                                             int n, int buffer, float* hit)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const SurfGeom& g = P.geom[s];
	float o[D], d[D], h[D];
#pragma unroll
	for (int a = 0; a < D; a++) {
		o[a] = org[(size_t)i * D + a];
		d[a] = dir[(size_t)i * D + a];
	}
	const bool ok = ray_cast<D, L>(P, g, o, d, buffer, h);
#pragma unroll
	for (int a = 0; a < D; a++) hit[(size_t)i * D + a] = ok ? h[a] : FLT_MAX;
}

template <int D, int L>
void launch_rays(EngineBase& eng, int s, const float* o, const float* d, size_t n, int buffer,
                 float* h)
{
	cudaStream_t st = eng.stream();
	FG_RUN("k_ray", st, k_ray<D, L><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(eng.dev(), s, o, d, (int)n, buffer, h););
	FG_CUDA(cudaGetLastError());
}

}  // namespace

int ray_buffer_max() { return RAY_BUFFER; }

void ray_batch(EngineBase& eng, int s, const float* origins, const float* dirs, size_t n,
               float* hits, bool device_ptrs, int buffer)
{
	if (s < 0 || s >= eng.surfaces()) throw Error(-1, "surface index out of range");
	if (buffer < 0) buffer = RAY_BUFFER;
	if (n == 0) return;
	if (n >= (size_t)1 << 30) throw Error(-1, "too many rays in one call (at most 2^30 - 1)");
	const int D = eng.dims(), L = eng.layers();
	const size_t bytes = n * D * sizeof(float);
	cudaStream_t st = eng.stream();
	float* dev = nullptr;
	const float* dorg = origins;
	const float* ddir = dirs;
	float* dhit = hits;
	if (!device_ptrs) {
		FG_CUDA(cudaMallocAsync((void**)&dev, 3 * bytes, st));
		FG_CUDA(cudaMemcpyAsync(dev, origins, bytes, cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(dev + n * D, dirs, bytes, cudaMemcpyHostToDevice, st));
		dorg = dev;
		ddir = dev + n * D;
		dhit = dev + 2 * n * D;
	}
	bool launched = false;
#define FG_CASE(dd, ll)                                            \
	if (D == dd && L == ll) {                                      \
		launch_rays<dd, ll>(eng, s, dorg, ddir, n, buffer, dhit); \
		launched = true;                                           \
	}
	FG_CASE(2, 1) FG_CASE(2, 2) FG_CASE(2, 3) FG_CASE(2, 4)
	FG_CASE(3, 1) FG_CASE(3, 2) FG_CASE(3, 3) FG_CASE(3, 4)
#undef FG_CASE
	if (!launched) throw Error(-1, "unsupported dimension or layer count");
	if (!device_ptrs) {
		FG_CUDA(cudaMemcpyAsync(hits, dhit, bytes, cudaMemcpyDeviceToHost, st));
		FG_CUDA(cudaFreeAsync(dev, st));
	}
	eng.sync();
	eng.check_errors();
}

}  // namespace fg
