// Device polygonisation: Felt::Polys (include/Felt/Polys.hpp) over Poly::Single children
// (include/Felt/Impl/Poly.hpp), for every surface of an engine's pool.
//
// The reference marches the leaves of a partition's 2L+1 layer lists in order and numbers the
// vertices in first-encounter order through a per-node edge cache. Here one block marches one
// pending partition: (1) classify every leaf's cell (corner mask) and claim each cut edge's
// cache slot with the smallest (cell, edge) sequence number; (2) a block scan over the cells
// numbers the first occurrences, which is exactly the reference's vertex order; (3) every cell
// emits its simplices from the ordering table, and every first occurrence leaves a descriptor in
// its vertex slot. A second, flat kernel then computes all vertices of the march (interpolated
// position and, in 3D, the normalised gradient of the interpolated field), one thread each, so
// the long gradient stencils do not hold a partition's block at its barriers.
#include <cstring>

#include "fg_field.cuh"
#include "fg_kernels.cuh"
#include "fg_polys.cuh"

#define FG_MC_QUAL static __device__ __constant__
#define FG_MC_FN static __device__ __forceinline__
#include "../include/felt_gpu/mc_tables.h"

namespace fg {

struct PolysDev {
	int* pend_lkp[2];   // [NP] position in the pending/done list, -1
	int* pend_list[2];  // [NP] per-surface segments at pbase
	int* pend_cnt[2];   // [S]
	int* pact;          // [NP] poly child active
	int* gvoff;         // [NP] vertex offset in the arena
	int* gnv;           // [NP] vertices
	int* gsoff;         // [NP] simplex offset
	int* gns;           // [NP] simplices
	float* vtx;         // arena: per vertex VF floats
	uint32_t* spx;      // arena: per simplex D indices
	unsigned long long* used;  // [2] vertices, simplices used
	long long vcap, scap;
	int* pendv;         // [S] which of the two lists is pending, per surface
	int* err;
	int* ovf;           // set when a march ran out of arena space
	unsigned long long* vstart;  // [1] vertex arena position when the current march began
	int* off;           // [S] 1 = notify leaves the surface out (serving: no polygons asked)
	int* sel;           // [S] surfaces a march works on (1), when it works on a selection
	int* cnt_sel;       // [S] pending counts of the surfaces a march works on
};

namespace {

constexpr float FEPS = 1.1920928955078125e-07f;

template <int D>
__device__ __forceinline__ int mc_edges()
{
	return D == 3 ? 12 : 4;
}
template <int D>
__device__ __forceinline__ int mc_order(int mask, int i)
{
	if (D == 3) return fg_mc3_order(mask, i);
	return fg_mc2_order_flat[mask * 4 + i];
}
template <int D>
__device__ __forceinline__ unsigned mc_edge_mask(int mask)
{
	if (D == 3) return fg_mc3_edge_mask(mask);
	return fg_mc2_edge_mask(mask);
}
template <int D>
__device__ __forceinline__ int mc_corner(int i, int a)
{
	if (D == 3) return fg_mc3_corner[i][a];
	return fg_mc2_corner[i][a];
}
template <int D>
__device__ __forceinline__ int mc_edge_off(int e, int a)
{
	if (D == 3) return fg_mc3_edge[e][a];
	return fg_mc2_edge[e][a];
}
template <int D>
__device__ __forceinline__ int mc_edge_axis(int e)
{
	if (D == 3) return fg_mc3_edge[e][3];
	return fg_mc2_edge[e][2];
}
/// Simplices of a corner mask: D-tuples read until -1 (Poly.hpp:259), flat in 2D.
template <int D>
__device__ __forceinline__ int mc_nspx(int mask)
{
	int n = 0;
	for (int o = 0; mc_order<D>(mask, o) != -1; o += D) n++;
	return n;
}

/// Poly::Single::idx vertex construction (Poly.hpp:296-346) for the edge at pa along axis.
template <int D, int L, class Get>
__device__ void make_vertex(const Get& get, const SurfGeom& g, const Vec<D>& pa, int axis,
                            float* out)
{
	Vec<D> pb = pa;
	pb[axis] += 1;
	const float va = get(pa);
	const float vb = get(pb);
	float pos[D];
	bool at_node = false;
	Vec<D> node;
	if (fabsf(va) <= FEPS) {
		at_node = true;
		node = pa;
	} else if (fabsf(vb) <= FEPS) {
		at_node = true;
		node = pb;
	}
	if (at_node) {
#pragma unroll
		for (int a = 0; a < D; a++) pos[a] = (float)node[a];
	} else {
		float mu;
		if (fabsf(__fsub_rn(va, vb)) <= FEPS)
			mu = 0.5f;
		else
			mu = __fdiv_rn(va, __fsub_rn(va, vb));
#pragma unroll
		for (int a = 0; a < D; a++) {
			const float fa = (float)pa[a], fb = (float)pb[a];
			pos[a] = __fadd_rn(fa, __fmul_rn(__fsub_rn(fb, fa), mu));
		}
	}
#pragma unroll
	for (int a = 0; a < D; a++) out[a] = pos[a];
	if (D == 3) {
		float n[D];
		if (at_node)
			grad_i<D>(get, g, node, n);
		else
			grad_f<D, L>(get, g, pos, n);
#pragma unroll
		for (int a = 0; a < D; a++) n[a] = __fdiv_rn(n[a], 1.0f);
		normalize3(n);
#pragma unroll
		for (int a = 0; a < D; a++) out[D + a] = n[a];
	}
}

/// Index, in a marched partition's staged box (origin = partition origin, extent bext,
/// row-major), of a leaf's cell origin: the leaf's node, moved one node along the last axis in
/// 3D (SpxGridPosOffset, PolyMixin.hpp:409), since the 3D cube's corners and edges step -z
/// from it (PolyMixin.hpp:377-406). The last axis has stride 1 in the box.
template <int D>
__device__ __forceinline__ int box_index(const Dev& P, const int* bext, int leaf)
{
	int bi = 0;
#pragma unroll
	for (int a = 0; a < D; a++) {
		const int q = leaf / P.lstr[a];
		leaf -= q * P.lstr[a];
		bi = bi * bext[a] + q;
	}
	return D == 3 ? bi + 1 : bi;
}

}  // namespace

/// Polys::notify (Polys.hpp:92-133), one block per surface. The reference walks the delta lists
/// of layers 0 and 2L tracking (appending) or untracking (swap-with-last removing) each
/// partition in the pending list, then tracks the poly-active partitions of the outermost
/// status lists. Within one list a partition appears once, so whether each entry is a real
/// append or removal depends only on the state before the list: the whole block decides a tile
/// of entries at once into shared memory, then one warp replays them in list order, appending
/// runs by ballot and replaying the (rare) removals one at a time.
template <int L>
__global__ void __launch_bounds__(256) k_polys_notify(Dev P, PolysDev Q)
{
	constexpr int NL = 2 * L + 1;
	constexpr int TILE = 1024;
	__shared__ int slp[TILE];
	__shared__ unsigned char sdec[TILE];  // bit 0 append, bit 1 remove
	__shared__ int cnt_s;
	const int s = blockIdx.x;
	if (s >= P.S || P.sfrozen[s] || Q.off[s]) return;
	const int lane = lane_id();
	const unsigned lt = (1u << lane) - 1u;
	const SurfGeom& g = P.geom[s];
	const int pd = Q.pendv[s];
	int* lkp = Q.pend_lkp[pd];
	int* lst = Q.pend_list[pd] + g.pbase;
	if (threadIdx.x == 0) cnt_s = Q.pend_cnt[pd][s];
	for (int pass = 0; pass < 4; pass++) {
		const bool status = pass >= 2;
		const int li = (pass & 1) ? NL - 1 : 0;
		const int n = status ? P.spcnt[s * NL + li] : P.dpcnt[s * NL + li];
		const int* src = (status ? P.splist : P.dplist) + (size_t)li * P.NP + g.pbase;
		for (int t0 = 0; t0 < n; t0 += TILE) {
			const int nt = min(TILE, n - t0);
			__syncthreads();  // the previous tile's edits are visible
			for (int i = threadIdx.x; i < nt; i += blockDim.x) {
				const int lp = src[t0 + i];
				const int gp = g.pbase + lp;
				const bool in = lkp[gp] >= 0;
				unsigned char dec = 0;
				if (status) {
					dec = (Q.pact[gp] && !in) ? 1 : 0;
				} else {
					bool act = Q.pact[gp] != 0;
					for (int lj = 0; !act && lj <= NL; lj += NL - 1)
						act = P.ppos[gp * NL + lj] >= 0;
					dec = (act && !in) ? 1 : (!act && in) ? 2 : 0;
				}
				slp[i] = lp;
				sdec[i] = dec;
			}
			__syncthreads();
			if (threadIdx.x < 32) {
				int cnt = cnt_s;
				for (int base = 0; base < nt; base += 32) {
					const int i = base + lane;
					const unsigned char dec = i < nt ? sdec[i] : 0;
					const int lp = i < nt ? slp[i] : 0;
					const int gp = g.pbase + lp;
					unsigned ma = __ballot_sync(FULL, dec & 1), mr = __ballot_sync(FULL, dec & 2);
					while (ma | mr) {
						const int r = mr ? __ffs(mr) - 1 : 32;
						const unsigned seg = ma & (r == 32 ? FULL : ((1u << r) - 1u));
						if (seg) {
							if ((seg >> lane) & 1u) {
								const int pos = cnt + __popc(seg & lt);
								lst[pos] = lp;
								lkp[gp] = pos;
							}
							cnt += __popc(seg);
							ma &= ~seg;
							__syncwarp();
						}
						if (r < 32) {
							if (lane == r) {
								const int at = lkp[gp], last = cnt - 1;
								if (at < last) {
									const int mv = lst[last];
									lst[at] = mv;
									lkp[g.pbase + mv] = at;
								}
								lkp[gp] = -1;
							}
							cnt -= 1;
							mr &= ~(1u << r);
							__syncwarp();
						}
					}
				}
				if (lane == 0) cnt_s = cnt;
			}
		}
	}
	__syncthreads();
	if (threadIdx.x == 0) Q.pend_cnt[pd][s] = cnt_s;
}

/// Polys::invalidate (Polys.hpp:171-191), one thread per surface.
template <int L>
__global__ void k_polys_invalidate(Dev P, PolysDev Q)
{
	constexpr int NL = 2 * L + 1;
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= P.S) return;
	const SurfGeom& g = P.geom[s];
	const int pd = Q.pendv[s];
	int* lkp = Q.pend_lkp[pd];
	int* lst = Q.pend_list[pd] + g.pbase;
	int cnt = Q.pend_cnt[pd][s];
	for (int i = 0; i < cnt; i++) lkp[g.pbase + lst[i]] = -1;
	cnt = 0;
	for (int li = 0; li <= NL; li += NL - 1) {
		const int n = P.pcnt[s * NL + li];
		const int* pl = P.plist + (size_t)li * P.NP + g.pbase;
		for (int i = 0; i < n; i++) {
			const int gp = g.pbase + pl[i];
			if (lkp[gp] < 0) {
				lkp[gp] = cnt;
				lst[cnt++] = pl[i];
			}
		}
	}
	Q.pend_cnt[pd][s] = cnt;
}

/// Serving: surface s's polygon children all inactive and empty, both pending lists empty
/// (the state of a new Polys), over the npcap partitions of its range.
__global__ void k_polys_reset_surface(PolysDev Q, int s, int pbase, int npcap)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npcap; i += gridDim.x * blockDim.x) {
		const int gp = pbase + i;
		Q.pend_lkp[0][gp] = -1;
		Q.pend_lkp[1][gp] = -1;
		Q.pact[gp] = 0;
		Q.gnv[gp] = 0;
		Q.gns[gp] = 0;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		Q.pend_cnt[0][s] = 0;
		Q.pend_cnt[1][s] = 0;
		Q.pendv[s] = 0;
	}
}

/// The pending counts of the surfaces a march works on (all, or those with sel[s] set), for
/// the scan of its entries; the others contribute none.
__global__ void k_polys_counts(Dev P, PolysDev Q, int selected)
{
	for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P.S; s += gridDim.x * blockDim.x)
		Q.cnt_sel[s] = (!selected || Q.sel[s]) ? Q.pend_cnt[Q.pendv[s]][s] : 0;
}

/// After a march (Polys.hpp:163-164): for every surface it worked on, the pending list becomes
/// the done list and the other list, reset, the new pending one. One block per surface.
__global__ void k_polys_flip(Dev P, PolysDev Q, int selected)
{
	const int s = blockIdx.x;
	if (s >= P.S || (selected && !Q.sel[s])) return;
	const SurfGeom& g = P.geom[s];
	const int which = Q.pendv[s] ^ 1;
	const int n = Q.pend_cnt[which][s];
	for (int i = threadIdx.x; i < n; i += blockDim.x)
		Q.pend_lkp[which][g.pbase + Q.pend_list[which][g.pbase + i]] = -1;
	__syncthreads();
	if (threadIdx.x == 0) {
		Q.pend_cnt[which][s] = 0;
		Q.pendv[s] = which;
	}
}


/// Polys::march body (Polys.hpp:138-161) for every pending partition of every surface (woff
/// over the pending counts), or for a single partition when single >= 0: classification of the
/// partition's cells, the first-occurrence vertex numbering of Poly::Single::idx and the simplex
/// index triplets. Vertex positions and normals are left to k_polys_vertices: each new vertex's
/// arena slot receives an 8-byte descriptor (partition, cell leaf, edge) instead.
///
/// The partition's values plus the one-node halo its cell corners reach (above the partition on
/// every axis; in 3D the cells' -z corners stay inside) are staged in shared memory, so
/// classification reads no global memory per corner.
template <int D, int L>
__global__ void __launch_bounds__(256) k_polys_march(Dev P, PolysDev Q, const int* woff,
                                                       int single)
{
	constexpr int NL = 2 * L + 1;
	constexpr int VF = D == 3 ? 2 * D : D;
	extern __shared__ int smem[];
	int bext[3] = {1, 1, 1}, bvol = 1;
	for (int a = 0; a < D; a++) {
		bext[a] = P.csz[a] + 1;
		bvol *= bext[a];
	}
	int* first = smem;                                          // [bvol * D] edge slots
	float* box = (float*)(first + bvol * D);                    // [bvol] staged phi
	uint16_t* cmask = (uint16_t*)(box + bvol);                  // [BV]
	uint16_t* cnew = cmask + P.BV;                              // [BV]
	uint16_t* cleaf = cnew + P.BV;                              // [BV]
	__shared__ int lstart[NL + 1];
	__shared__ int tot_v, tot_s, vb, sb, ok;
	__shared__ int msl[8];    // slots of the partition and its upper neighbours (-1 inactive)
	__shared__ float mbg[8];  // their backgrounds
	const int nent = single >= 0 ? 1 : woff[P.S];
	for (int e = blockIdx.x; e < nent; e += gridDim.x) {
		int gp;
		if (single >= 0) {
			gp = single;
		} else {
			const int s = entry_surface(woff, P.S, e);
			const SurfGeom& gs = P.geom[s];
			gp = gs.pbase + Q.pend_list[Q.pendv[s]][gs.pbase + (e - woff[s])];
		}
		const SurfGeom& g = P.geom[P.surf_of[gp]];
		const int sl = P.slot[gp];
		if (sl < 0) {
			// isogrid child inactive: Poly::Single::deactivate (Poly.hpp:95-101).
			if (threadIdx.x == 0) {
				Q.pact[gp] = 0;
				Q.gnv[gp] = 0;
				Q.gns[gp] = 0;
			}
			continue;
		}
		if (threadIdx.x == 0) {
			int c = 0;
			for (int l = 0; l < NL; l++) {
				lstart[l] = c;
				c += P.lcnt[sl * NL + l];
			}
			lstart[NL] = c;
		}
		Vec<D> bo;  // world position of box index 0
		for (int a = 0; a < D; a++) bo[a] = P.porig[gp * 3 + a];
		// the slots (or backgrounds) of the partition and of its upper neighbours, looked up
		// once: every staged value is then one independent load, the value get_phi reads there
		if (threadIdx.x < (1 << D)) {
			Vec<D> p;
			for (int a = 0; a < D; a++)
				p[a] = bo[a] + (((threadIdx.x >> (D - 1 - a)) & 1) ? P.csz[a] : 0);
			int s2 = -1;
			float b2 = (float)(L + 1);
			if (in_grid<D>(g, p)) {
				int gp2, leaf2;
				locate<D>(P, g, p, gp2, leaf2);
				s2 = P.slot[gp2];
				b2 = P.bg[gp2];
			}
			msl[threadIdx.x] = s2;
			mbg[threadIdx.x] = b2;
		}
		__syncthreads();
		for (int i = threadIdx.x; i < bvol; i += blockDim.x) {
			first[i * D] = 0x7fffffff;
			for (int a = 1; a < D; a++) first[i * D + a] = 0x7fffffff;
			int r = i, leaf = 0, dir = 0;
			bool ing = true;
			for (int a = D - 1; a >= 0; a--) {
				const int c = r % bext[a];
				r /= bext[a];
				const int pa = bo[a] + c;
				const bool up = c >= P.csz[a];
				dir |= (up ? 1 : 0) << (D - 1 - a);
				leaf += (up ? 0 : c) * P.lstr[a];
				ing = ing && pa < g.hi[a];  // pa >= off: the partition starts inside the grid
			}
			float v = (float)(L + 1);
			if (ing) {
				const int s2 = msl[dir];
				v = s2 >= 0 ? P.phi[(size_t)s2 * P.BV + leaf] : mbg[dir];
			}
			box[i] = v;
		}
		__syncthreads();
		const int n = lstart[NL];
		if (threadIdx.x == 0) atomicAdd(&P.kstat[KS_MARCH], (unsigned long long)n);
		const int per = (n + blockDim.x - 1) / blockDim.x;
		const int j0 = threadIdx.x * per, j1 = min(n, j0 + per);
		// 1. classify cells and claim edge slots: the lowest (cell, edge) claims a slot
		for (int j = j0; j < j1; j++) {
			int l = 0;
			while (j >= lstart[l + 1]) l++;
			const int leaf = P.lst[((size_t)sl * NL + l) * P.BV + (j - lstart[l])];
			const int bi = box_index<D>(P, bext, leaf);  // the cell's lowest corner
			unsigned mask = 0;
			for (int i = 0; i < (1 << D); i++) {
				int o = 0;
				for (int a = 0; a < D; a++) o = o * bext[a] + mc_corner<D>(i, a);
				mask |= (box[bi + o] > 0.0f ? 1u : 0u) << i;
			}
			cmask[j] = (uint16_t)mask;
			cleaf[j] = (uint16_t)leaf;
			if (mc_order<D>(mask, 0) == -1) continue;
			const unsigned em = mc_edge_mask<D>(mask);
			for (int ed = 0; ed < mc_edges<D>(); ed++) {
				if (!((em >> ed) & 1u)) continue;
				int o = 0;
				for (int a = 0; a < D; a++) o = o * bext[a] + mc_edge_off<D>(ed, a);
				atomicMin(&first[(bi + o) * D + mc_edge_axis<D>(ed)], j * 16 + ed);
			}
		}
		__syncthreads();
		// 2. first occurrences and simplex counts, scanned in cell order
		int my_v = 0, my_s = 0;
		for (int j = j0; j < j1; j++) {
			const unsigned mask = cmask[j];
			unsigned nm = 0;
			if (mc_order<D>(mask, 0) != -1) {
				const int bi = box_index<D>(P, bext, cleaf[j]);
				const unsigned em = mc_edge_mask<D>(mask);
				for (int ed = 0; ed < mc_edges<D>(); ed++) {
					if (!((em >> ed) & 1u)) continue;
					int o = 0;
					for (int a = 0; a < D; a++) o = o * bext[a] + mc_edge_off<D>(ed, a);
					if (first[(bi + o) * D + mc_edge_axis<D>(ed)] == j * 16 + ed) nm |= 1u << ed;
				}
				my_s += mc_nspx<D>(mask);
			}
			cnew[j] = (uint16_t)nm;
			my_v += __popc(nm);
		}
		int tv, ts;
		const int bv0 = block_excl_scan(my_v, &tv);
		const int bs0 = block_excl_scan(my_s, &ts);
		if (threadIdx.x == 0) {
			tot_v = tv;
			tot_s = ts;
			const unsigned long long a = atomicAdd(&Q.used[0], (unsigned long long)tv);
			const unsigned long long b = atomicAdd(&Q.used[1], (unsigned long long)ts);
			ok = (long long)(a + tv) <= Q.vcap && (long long)(b + ts) <= Q.scap;
			vb = (int)a;
			sb = (int)b;
			if (!ok) atomicExch(Q.ovf, 1);
		}
		__syncthreads();
		if (ok) {
			// 3a. vertex descriptors, numbered in first-occurrence order
			int vi = bv0;
			for (int j = j0; j < j1; j++) {
				const unsigned nm = cnew[j];
				if (!nm) continue;
				const int bi = box_index<D>(P, bext, cleaf[j]);
				for (int ed = 0; ed < mc_edges<D>(); ed++) {
					if (!((nm >> ed) & 1u)) continue;
					int o = 0;
					for (int a = 0; a < D; a++) o = o * bext[a] + mc_edge_off<D>(ed, a);
					*(unsigned long long*)(Q.vtx + ((size_t)vb + vi) * VF) =
					    ((unsigned long long)gp << 21) | ((unsigned long long)cleaf[j] << 4) |
					    (unsigned long long)ed;
					first[(bi + o) * D + mc_edge_axis<D>(ed)] = vi;
					vi++;
				}
			}
			__syncthreads();
			// 3b. simplices
			int si = bs0;
			for (int j = j0; j < j1; j++) {
				const unsigned mask = cmask[j];
				if (mc_order<D>(mask, 0) == -1) continue;
				const int bi = box_index<D>(P, bext, cleaf[j]);
				for (int o = 0; mc_order<D>(mask, o) != -1; o += D) {
					uint32_t* dst = Q.spx + ((size_t)sb + si) * D;
					for (int k = 0; k < D; k++) {
						const int ed = mc_order<D>(mask, o + k);
						int eo = 0;
						for (int a = 0; a < D; a++) eo = eo * bext[a] + mc_edge_off<D>(ed, a);
						dst[k] = (uint32_t)first[(bi + eo) * D + mc_edge_axis<D>(ed)];
					}
					si++;
				}
			}
			if (threadIdx.x == 0) {
				Q.pact[gp] = 1;
				Q.gvoff[gp] = vb;
				Q.gnv[gp] = tot_v;
				Q.gsoff[gp] = sb;
				Q.gns[gp] = tot_s;
			}
		}
		__syncthreads();
	}
}

/// Poly::Single::idx vertex construction (Poly.hpp:296-346) for every vertex that the last
/// k_polys_march placed in the arena range [vstart, used): decodes the descriptor in the slot
/// and overwrites it with the position (and, in 3D, the normal). One thread per vertex.
template <int D, int L>
__global__ void __launch_bounds__(256) k_polys_vertices(Dev P, PolysDev Q)
{
	constexpr int VF = D == 3 ? 2 * D : D;
	const long long v0 = (long long)Q.vstart[0], v1 = (long long)Q.used[0];
	for (long long i = v0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < v1;
	     i += (long long)gridDim.x * blockDim.x) {
		float* slot = Q.vtx + (size_t)i * VF;
		const unsigned long long d = *(const unsigned long long*)slot;
		const int gp = (int)(d >> 21), leaf = (int)((d >> 4) & 0x1ffff), ed = (int)(d & 15);
		const SurfGeom& g = P.geom[P.surf_of[gp]];
		Vec<D> pa = leaf_pos<D>(P, gp, leaf);
		if (D == 3) pa[D - 1] += 1;  // SpxGridPosOffset (PolyMixin.hpp:409)
#pragma unroll
		for (int a = 0; a < D; a++) pa[a] += mc_edge_off<D>(ed, a);
		float out[VF];
		make_vertex<D, L>(PoolGet<D, L>{P, g}, g, pa, mc_edge_axis<D>(ed), out);
#pragma unroll
		for (int k = 0; k < VF; k++) slot[k] = out[k];
	}
}

/// Copies the geometry of the requested partitions (job: src vertex offset, vertex count, src
/// simplex offset, simplex count, index) to consecutive destination ranges. Block per job.
template <int D>
__global__ void k_polys_gather(PolysDev Q, const int* job, const long long* dst, int n, float* sv,
                               uint32_t* ss)
{
	constexpr int VF = D == 3 ? 2 * D : D;
	for (int i = blockIdx.x; i < n; i += gridDim.x) {
		const size_t vo = (size_t)job[5 * i] * VF, so = (size_t)job[5 * i + 2] * D;
		const int nv = job[5 * i + 1] * VF, ns = job[5 * i + 3] * D;
		const size_t vd = (size_t)dst[2 * i] * VF, sd = (size_t)dst[2 * i + 1] * D;
		for (int k = threadIdx.x; k < nv; k += blockDim.x) sv[vd + k] = Q.vtx[vo + k];
		for (int k = threadIdx.x; k < ns; k += blockDim.x) ss[sd + k] = Q.spx[so + k];
	}
}

/// Arena compaction offsets, step 1: per chunk of ARENA_CHUNK partitions, the sums of their
/// vertex and simplex counts.
constexpr int ARENA_CHUNK = 4096;
__global__ void __launch_bounds__(256) k_arena_chunk_sums(PolysDev Q, int NP,
                                                          unsigned long long* csum)
{
	const int c0 = blockIdx.x * ARENA_CHUNK, c1 = min(NP, c0 + ARENA_CHUNK);
	unsigned long long v = 0, s = 0;
	for (int i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
		v += (unsigned long long)Q.gnv[i];
		s += (unsigned long long)Q.gns[i];
	}
	__shared__ unsigned long long rv[256], rs[256];
	rv[threadIdx.x] = v;
	rs[threadIdx.x] = s;
	__syncthreads();
	for (int o = blockDim.x / 2; o > 0; o >>= 1) {
		if ((int)threadIdx.x < o) {
			rv[threadIdx.x] += rv[threadIdx.x + o];
			rs[threadIdx.x] += rs[threadIdx.x + o];
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		csum[2 * blockIdx.x] = rv[0];
		csum[2 * blockIdx.x + 1] = rs[0];
	}
}

/// Step 2: exclusive scan of the chunk sums in place (one thread; there are NP / 4096 chunks)
/// and the totals.
__global__ void k_arena_chunk_scan(unsigned long long* csum, int nchunks, unsigned long long* tot)
{
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	unsigned long long v = 0, s = 0;
	for (int c = 0; c < nchunks; c++) {
		const unsigned long long a = csum[2 * c], b = csum[2 * c + 1];
		csum[2 * c] = v;
		csum[2 * c + 1] = s;
		v += a;
		s += b;
	}
	tot[0] = v;
	tot[1] = s;
}

/// Step 3: every partition's new vertex and simplex offsets (exclusive scan of the counts in
/// partition order, the order the host-side compaction used).
__global__ void __launch_bounds__(256) k_arena_offsets(PolysDev Q, int NP,
                                                       const unsigned long long* csum,
                                                       int* noff, int* nsoff)
{
	constexpr int PER = ARENA_CHUNK / 256;
	const int c0 = blockIdx.x * ARENA_CHUNK;
	const int i0 = c0 + threadIdx.x * PER;
	int v = 0, s = 0;
	for (int k = 0; k < PER; k++) {
		const int i = i0 + k;
		if (i < NP) {
			v += Q.gnv[i];
			s += Q.gns[i];
		}
	}
	int tv, ts;
	const int ev = block_excl_scan(v, &tv);
	const int es = block_excl_scan(s, &ts);
	long long ov = (long long)csum[2 * blockIdx.x] + ev, os = (long long)csum[2 * blockIdx.x + 1] + es;
	for (int k = 0; k < PER; k++) {
		const int i = i0 + k;
		if (i >= NP) break;
		noff[i] = (int)ov;
		nsoff[i] = (int)os;
		ov += Q.gnv[i];
		os += Q.gns[i];
	}
}

/// Moves the live geometry of every partition to the front of a fresh arena.
template <int D>
__global__ void k_polys_compact(Dev P, PolysDev Q, const int* noff, const int* nsoff, float* vtx2,
                                uint32_t* spx2)
{
	constexpr int VF = D == 3 ? 2 * D : D;
	for (int gp = blockIdx.x; gp < P.NP; gp += gridDim.x) {
		const int nv = Q.gnv[gp], ns = Q.gns[gp];
		if (!nv && !ns) continue;
		const size_t vo = (size_t)Q.gvoff[gp] * VF, so = (size_t)Q.gsoff[gp] * D;
		const size_t vn = (size_t)noff[gp] * VF, sn = (size_t)nsoff[gp] * D;
		for (int i = threadIdx.x; i < nv * VF; i += blockDim.x) vtx2[vn + i] = Q.vtx[vo + i];
		for (int i = threadIdx.x; i < ns * D; i += blockDim.x) spx2[sn + i] = Q.spx[so + i];
	}
}

namespace {

template <int D, int L>
class PolysImpl final : public PolysBase {
public:
	static constexpr int VF = D == 3 ? 2 * D : D;

	PolysImpl(EngineBase& eng, int s, size_t vertex_capacity) : eng_(eng), s_(s)
	{
		const Dev& P = eng.dev();
		auto al = [&](size_t bytes) {
			void* p = nullptr;
			FG_CUDA(locked_malloc(&p, bytes ? bytes : 1));
			owned_.push_back(p);
			return p;
		};
		std::memset(&Q_, 0, sizeof(Q_));
		for (int b = 0; b < 2; b++) {
			Q_.pend_lkp[b] = (int*)al(P.NP * sizeof(int));
			Q_.pend_list[b] = (int*)al(P.NP * sizeof(int));
			Q_.pend_cnt[b] = (int*)al(P.S * sizeof(int));
			FG_CUDA(cudaMemset(Q_.pend_lkp[b], 0xff, P.NP * sizeof(int)));
			FG_CUDA(cudaMemset(Q_.pend_cnt[b], 0, P.S * sizeof(int)));
		}
		Q_.pact = (int*)al(P.NP * sizeof(int));
		Q_.gvoff = (int*)al(P.NP * sizeof(int));
		Q_.gnv = (int*)al(P.NP * sizeof(int));
		Q_.gsoff = (int*)al(P.NP * sizeof(int));
		Q_.gns = (int*)al(P.NP * sizeof(int));
		FG_CUDA(cudaMemset(Q_.pact, 0, P.NP * sizeof(int)));
		FG_CUDA(cudaMemset(Q_.gnv, 0, P.NP * sizeof(int)));
		FG_CUDA(cudaMemset(Q_.gns, 0, P.NP * sizeof(int)));
		FG_CUDA(cudaMemset(Q_.gvoff, 0, P.NP * sizeof(int)));
		FG_CUDA(cudaMemset(Q_.gsoff, 0, P.NP * sizeof(int)));
		Q_.off = (int*)al(P.S * sizeof(int));
		FG_CUDA(cudaMemset(Q_.off, 0, P.S * sizeof(int)));
		Q_.used = (unsigned long long*)al(2 * sizeof(unsigned long long));
		FG_CUDA(cudaMemset(Q_.used, 0, 2 * sizeof(unsigned long long)));
		woff_ = (int*)al((P.S + 1) * sizeof(int));
		Q_.err = P.err;
		Q_.ovf = (int*)al(sizeof(int));
		Q_.vstart = (unsigned long long*)al(sizeof(unsigned long long));
		nchunks_ = (P.NP + ARENA_CHUNK - 1) / ARENA_CHUNK;
		noff_ = (int*)al(P.NP * sizeof(int));
		nsoff_ = (int*)al(P.NP * sizeof(int));
		csum_ = (unsigned long long*)al(2 * (size_t)nchunks_ * sizeof(unsigned long long));
		ctot_ = (unsigned long long*)al(2 * sizeof(unsigned long long));
		Q_.pendv = (int*)al(P.S * sizeof(int));
		FG_CUDA(cudaMemset(Q_.pendv, 0, P.S * sizeof(int)));
		Q_.sel = (int*)al(P.S * sizeof(int));
		Q_.cnt_sel = (int*)al(P.S * sizeof(int));
		pend_host_.assign((size_t)P.S, 0);
		const long long vc = vertex_capacity ? std::max<long long>((long long)vertex_capacity, 64)
		                                     : (1LL << 20);
		if (vc >= (1LL << 30)) throw Error(-1, "vertex capacity too large");
		keep_pool_memory();
		alloc_arena(vc, 2 * vc);
		// the compaction's other arena up front: the first compaction then allocates nothing
		// (a pool that has to grow from the driver mid-march stalls the step)
		FG_CUDA(cudaMallocAsync((void**)&spare_v_, (size_t)vc * VF * sizeof(float), eng.stream()));
		FG_CUDA(cudaMallocAsync((void**)&spare_s_, (size_t)2 * vc * D * sizeof(uint32_t), eng.stream()));
		spare_vcap_ = vc;
		spare_scap_ = 2 * vc;
		// kernels that first run when the arena fills, possibly many steps later: loaded now
		// (with lazy module loading a kernel's first launch also loads it)
		cudaFuncAttributes fa;
		FG_CUDA(cudaFuncGetAttributes(&fa, k_arena_chunk_sums));
		FG_CUDA(cudaFuncGetAttributes(&fa, k_arena_chunk_scan));
		FG_CUDA(cudaFuncGetAttributes(&fa, k_arena_offsets));
		FG_CUDA(cudaFuncGetAttributes(&fa, k_polys_compact<D>));
		int bvol = 1;
		for (int a = 0; a < D; a++) bvol *= eng.part(a) + 1;
		smem_ = (size_t)bvol * (D * sizeof(int) + sizeof(float)) +
		        3 * (size_t)P.BV * sizeof(uint16_t);
		smem_ = (smem_ + 15) & ~(size_t)15;
		// threads per marched partition: a block per partition, sized to its cells (a 2D 16^2
		// brick has a few dozen band cells, a 3D 16^3 brick thousands)
		march_threads_ = P.BV >= 2048 ? 256 : P.BV >= 512 ? 128 : 64;
		if (smem_ > 48 * 1024)
			FG_CUDA(cudaFuncSetAttribute(k_polys_march<D, L>,
			                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_));
		std::lock_guard<std::recursive_mutex> lock(device_lock());
		FG_CUDA(cudaDeviceSynchronize());
	}

	~PolysImpl() override
	{
		cudaStream_t st = eng_.stream();
		cudaStreamSynchronize(st);
		free_arena();
		if (spare_v_) cudaFreeAsync(spare_v_, st);
		if (spare_s_) cudaFreeAsync(spare_s_, st);
		if (stage_) cudaFreeAsync(stage_, st);
		cudaStreamSynchronize(st);
		for (void* p : owned_) locked_free(p);
	}

	void notify() override
	{
		const Dev& P = eng_.dev();
		FG_RUN("k_polys_notify", eng_.stream(), k_polys_notify<L><<<P.S, 256, 0, eng_.stream()>>>(P, Q_););
		FG_CUDA(cudaGetLastError());
	}

	void invalidate() override
	{
		const Dev& P = eng_.dev();
		FG_RUN("k_polys_invalidate", eng_.stream(), k_polys_invalidate<L><<<(P.S + 127) / 128, 128, 0, eng_.stream()>>>(P, Q_););
		FG_CUDA(cudaGetLastError());
	}

	void march() override { march_sel(nullptr, 0); }

	void march_some(const int* surfaces, int n) override
	{
		if (n <= 0) return;
		const Dev& P = eng_.dev();
		sel_host_.assign((size_t)P.S, 0);
		for (int i = 0; i < n; i++) {
			if (surfaces[i] < 0 || surfaces[i] >= P.S) throw Error(-1, "surface index out of range");
			sel_host_[surfaces[i]] = 1;
		}
		FG_CUDA(cudaMemcpyAsync(Q_.sel, sel_host_.data(), sel_host_.size() * sizeof(int),
		                        cudaMemcpyHostToDevice, eng_.stream()));
		march_sel(surfaces, n);
	}

	/// Polys::march (Polys.hpp:138-165) of every surface of the pool (surfaces == nullptr) or
	/// of the listed ones only (Q_.sel set): the others keep their pending lists for their own
	/// march later.
	void march_sel(const int* surfaces, int n)
	{
		const Dev& P = eng_.dev();
		cudaStream_t st = eng_.stream();
		const int selected = surfaces ? 1 : 0;
		FG_RUN("k_polys_counts", st, k_polys_counts<<<(P.S + 255) / 256, 256, 0, st>>>(P, Q_, selected););
		FG_RUN("k_scan_counts", st, k_scan_counts<<<1, 1024, 0, st>>>(Q_.cnt_sel, 1, 0, 0, P.S, woff_, P.sfrozen););
		// Re-marching a partition recomputes it from the isogrid, so a march that ran out of
		// arena space is simply repeated after the arena has grown.
		for (int attempt = 0;; attempt++) {
			begin_attempt(attempt);
			FG_RUN("k_polys_march", st, k_polys_march<D, L><<<grid() * (256 / march_threads_), march_threads_, smem_, st>>>(P, Q_, woff_, -1););
			FG_CUDA(cudaGetLastError());
			if (!overflowed()) break;
			if (attempt > 8) throw Error(-13, "polygonisation arena cannot grow further");
		}
		vertices();
		// swap pending and done, then reset the new pending list
		FG_RUN("k_polys_flip", st, k_polys_flip<<<P.S, 256, 0, st>>>(P, Q_, selected););
		FG_CUDA(cudaGetLastError());
		if (surfaces)
			for (int i = 0; i < n; i++) pend_host_[surfaces[i]] ^= 1;
		else
			for (int& v : pend_host_) v ^= 1;
		eng_.check_errors();
	}

	void march_partition(size_t part) override
	{
		const Dev& P = eng_.dev();
		const int gp = check_part(part);
		for (int attempt = 0;; attempt++) {
			begin_attempt(attempt);
			FG_RUN("k_polys_march", eng_.stream(), k_polys_march<D, L><<<1, march_threads_, smem_, eng_.stream()>>>(P, Q_, woff_, gp););
			FG_CUDA(cudaGetLastError());
			if (!overflowed()) break;
			if (attempt > 8) throw Error(-13, "polygonisation arena cannot grow further");
		}
		vertices();
		eng_.check_errors();
	}

	/// Resets the overflow flag and records where this attempt's vertices begin in the arena.
	void begin_attempt(int attempt)
	{
		cudaStream_t st = eng_.stream();
		maybe_compact(attempt > 0);
		FG_CUDA(cudaMemsetAsync(Q_.ovf, 0, sizeof(int), st));
		FG_CUDA(cudaMemcpyAsync(Q_.vstart, Q_.used, sizeof(unsigned long long),
		                        cudaMemcpyDeviceToDevice, st));
	}

	/// Positions (and normals) of the vertices the last successful march attempt described.
	void vertices()
	{
		cudaStream_t st = eng_.stream();
		FG_RUN("k_polys_vertices", st, k_polys_vertices<D, L><<<grid() * 2, 256, 0, st>>>(eng_.dev(), Q_););
		FG_CUDA(cudaGetLastError());
	}

	bool overflowed()
	{
		int o = 0;
		FG_CUDA(cudaMemcpyAsync(&o, Q_.ovf, sizeof(int), cudaMemcpyDeviceToHost, eng_.stream()));
		eng_.sync();
		return o != 0;
	}

	std::vector<uint32_t> changes() override
	{
		const Dev& P = eng_.dev();
		eng_.sync();
		const int done = pend_host_[s_] ^ 1;
		int n = 0;
		int pbase = pbase_of();
		FG_CUDA(cudaMemcpy(&n, Q_.pend_cnt[done] + s_, sizeof(int), cudaMemcpyDeviceToHost));
		std::vector<int> tmp(n);
		if (n)
			FG_CUDA(cudaMemcpy(tmp.data(), Q_.pend_list[done] + pbase, n * sizeof(int),
			                   cudaMemcpyDeviceToHost));
		(void)P;
		return std::vector<uint32_t>(tmp.begin(), tmp.end());
	}

	void partition(size_t part, float* vtx, size_t vcap, uint32_t* spx, size_t scap, size_t* nv,
	               size_t* ns, int* active) override
	{
		const int gp = check_part(part);
		eng_.sync();
		int rec[5];
		FG_CUDA(cudaMemcpy(&rec[0], Q_.pact + gp, sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(&rec[1], Q_.gvoff + gp, sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(&rec[2], Q_.gnv + gp, sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(&rec[3], Q_.gsoff + gp, sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(&rec[4], Q_.gns + gp, sizeof(int), cudaMemcpyDeviceToHost));
		*active = rec[0];
		*nv = (size_t)rec[2];
		*ns = (size_t)rec[4];
		if (vtx && rec[2]) {
			const size_t k = std::min(vcap, (size_t)rec[2] * VF);
			FG_CUDA(cudaMemcpy(vtx, Q_.vtx + (size_t)rec[1] * VF, k * sizeof(float),
			                   cudaMemcpyDeviceToHost));
		}
		if (spx && rec[4]) {
			const size_t k = std::min(scap, (size_t)rec[4] * D);
			FG_CUDA(cudaMemcpy(spx, Q_.spx + (size_t)rec[3] * D, k * sizeof(uint32_t),
			                   cudaMemcpyDeviceToHost));
		}
	}

	/// Vertex and simplex totals over every partition of the pool, summed on the device (the
	/// compaction's chunk sums); 16 bytes come back.
	void totals(size_t* nv, size_t* ns) override
	{
		const Dev& P = eng_.dev();
		cudaStream_t st = eng_.stream();
		FG_RUN("k_arena_chunk_sums", st, k_arena_chunk_sums<<<nchunks_, 256, 0, st>>>(Q_, P.NP, csum_););
		FG_RUN("k_arena_chunk_scan", st, k_arena_chunk_scan<<<1, 32, 0, st>>>(csum_, nchunks_, ctot_););
		FG_CUDA(cudaGetLastError());
		unsigned long long tot[2];
		FG_CUDA(cudaMemcpyAsync(tot, ctot_, sizeof(tot), cudaMemcpyDeviceToHost, st));
		eng_.sync();
		if (nv) *nv = (size_t)tot[0];
		if (ns) *ns = (size_t)tot[1];
	}

private:
	/// First global partition index of the selected surface: its range in the pool, which
	/// holds its partition capacity (more than its grid's partitions on a serving pool).
	int pbase_of() { return eng_.geometry(s_).pbase; }
	int check_part(size_t part)
	{
		int cc[3], co[3];
		const size_t np = eng_.partitions(s_, cc, co);
		if (part >= np) throw Error(-1, "partition index out of range");
		return pbase_of() + (int)part;
	}
	int grid() const
	{
		int dev = 0, sms = 148;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		return sms * 4;
	}
	// The arenas and the gather staging come from the stream-ordered allocator: they are
	// regrown while marching (the geometry grows with the surfaces), and its pooled,
	// stream-ordered frees do not stall the device the way cudaFree does.
	void alloc_arena(long long vcap, long long scap)
	{
		cudaStream_t st = eng_.stream();
		FG_CUDA(cudaMallocAsync((void**)&Q_.vtx, (size_t)vcap * VF * sizeof(float), st));
		FG_CUDA(cudaMallocAsync((void**)&Q_.spx, (size_t)scap * D * sizeof(uint32_t), st));
		Q_.vcap = vcap;
		Q_.scap = scap;
	}
	void free_arena()
	{
		cudaStream_t st = eng_.stream();
		if (Q_.vtx) cudaFreeAsync(Q_.vtx, st);
		if (Q_.spx) cudaFreeAsync(Q_.spx, st);
		Q_.vtx = nullptr;
		Q_.spx = nullptr;
	}
	/// Keeps the bump-allocated arenas at most half full before a march by moving the live
	/// geometry to the front of the other arena (kept between compactions, regrown when the
	/// live part needs more than 1/16 of it). The new offsets are scanned on the device; the
	/// host only reads the two totals.
	void maybe_compact(bool grow)
	{
		const Dev& P = eng_.dev();
		cudaStream_t st = eng_.stream();
		unsigned long long used[2];
		FG_CUDA(cudaMemcpyAsync(used, Q_.used, sizeof(used), cudaMemcpyDeviceToHost, st));
		eng_.sync();
		if (!grow && (long long)used[0] * 2 < Q_.vcap && (long long)used[1] * 2 < Q_.scap) return;
		FG_RUN("k_arena_chunk_sums", st, k_arena_chunk_sums<<<nchunks_, 256, 0, st>>>(Q_, P.NP, csum_););
		FG_RUN("k_arena_chunk_scan", st, k_arena_chunk_scan<<<1, 32, 0, st>>>(csum_, nchunks_, ctot_););
		FG_RUN("k_arena_offsets", st, k_arena_offsets<<<nchunks_, 256, 0, st>>>(Q_, P.NP, csum_, noff_, nsoff_););
		FG_CUDA(cudaGetLastError());
		unsigned long long tot[2];
		FG_CUDA(cudaMemcpyAsync(tot, ctot_, sizeof(tot), cudaMemcpyDeviceToHost, st));
		eng_.sync();
		const long long tv = (long long)tot[0], ts = (long long)tot[1];
		// 16x headroom over the live geometry: a march re-emits the geometry of the partitions
		// it re-marches, so with less room a polygonisation every step compacts every step.
		// After an overflowed march, `used` holds everything that march asked for (every
		// partition reserves its range, fitting or not): sized from it, the retry fits.
		long long vcap = grow ? 2 * Q_.vcap : Q_.vcap, scap = grow ? 2 * Q_.scap : Q_.scap;
		if (grow) {
			while (vcap < 2 * (long long)used[0] + tv) vcap *= 2;
			while (scap < 2 * (long long)used[1] + ts) scap *= 2;
		}
		while (tv * 16 > vcap) vcap *= 2;
		while (ts * 16 > scap) scap *= 2;
		if (vcap >= (1LL << 31) || scap >= (1LL << 31))
			throw Error(-13, "polygonisation arena too large");
		if (spare_vcap_ < vcap) {
			if (spare_v_) FG_CUDA(cudaFreeAsync(spare_v_, st));
			spare_v_ = nullptr;
			spare_vcap_ = 0;
			FG_CUDA(cudaMallocAsync((void**)&spare_v_, (size_t)vcap * VF * sizeof(float), st));
			spare_vcap_ = vcap;
		}
		if (spare_scap_ < scap) {
			if (spare_s_) FG_CUDA(cudaFreeAsync(spare_s_, st));
			spare_s_ = nullptr;
			spare_scap_ = 0;
			FG_CUDA(cudaMallocAsync((void**)&spare_s_, (size_t)scap * D * sizeof(uint32_t), st));
			spare_scap_ = scap;
		}
		FG_RUN("k_polys_compact", st, k_polys_compact<D><<<grid(), 256, 0, st>>>(P, Q_, noff_, nsoff_, spare_v_, spare_s_););
		FG_CUDA(cudaGetLastError());
		FG_CUDA(cudaMemcpyAsync(Q_.gvoff, noff_, P.NP * sizeof(int), cudaMemcpyDeviceToDevice, st));
		FG_CUDA(cudaMemcpyAsync(Q_.gsoff, nsoff_, P.NP * sizeof(int), cudaMemcpyDeviceToDevice, st));
		FG_CUDA(cudaMemcpyAsync(Q_.used, ctot_, 2 * sizeof(unsigned long long),
		                        cudaMemcpyDeviceToDevice, st));
		// the old arena becomes the spare
		std::swap(Q_.vtx, spare_v_);
		std::swap(Q_.spx, spare_s_);
		std::swap(Q_.vcap, spare_vcap_);
		std::swap(Q_.scap, spare_scap_);
	}


public:
	void reset_surface(int s) override
	{
		if (s < 0 || s >= eng_.surfaces()) throw Error(-1, "surface index out of range");
		const int npcap = eng_.partition_capacity(s);
		const int blocks = std::max(1, std::min((npcap + 255) / 256, 1024));
		FG_RUN("k_polys_reset_surface", eng_.stream(), k_polys_reset_surface<<<blocks, 256, 0, eng_.stream()>>>(Q_, s, eng_.geometry(s).pbase, npcap););
		FG_CUDA(cudaGetLastError());
		pend_host_[s] = 0;
	}

	void set_enabled(int s, bool on) override
	{
		if (s < 0 || s >= eng_.surfaces()) throw Error(-1, "surface index out of range");
		if (off_host_.empty()) off_host_.assign((size_t)eng_.surfaces(), 0);
		off_host_[s] = on ? 0 : 1;
		FG_CUDA(cudaMemcpyAsync(Q_.off + s, &off_host_[s], sizeof(int), cudaMemcpyHostToDevice,
		                        eng_.stream()));
	}

	void select(int s) override
	{
		if (s < 0 || s >= eng_.surfaces()) throw Error(-1, "surface index out of range");
		s_ = s;
	}

	void gather(const uint32_t* parts, size_t n, float* vtx, size_t vcap, uint32_t* spx,
	            size_t scap, uint32_t* counts, size_t* nv, size_t* ns) override
	{
		int cc[3], co[3];
		const int np = (int)eng_.partitions(s_, cc, co);
		const int pb = pbase_of();
		eng_.sync();
		std::vector<int> gnv(np), gns(np), gvo(np), gso(np);
		FG_CUDA(cudaMemcpy(gnv.data(), Q_.gnv + pb, np * sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(gns.data(), Q_.gns + pb, np * sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(gvo.data(), Q_.gvoff + pb, np * sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(gso.data(), Q_.gsoff + pb, np * sizeof(int), cudaMemcpyDeviceToHost));
		// per requested partition: source offsets, counts and destination offsets
		std::vector<int> job(5 * n);
		long long tv = 0, ts = 0;
		for (size_t i = 0; i < n; i++) {
			if (parts[i] >= (uint32_t)np) throw Error(-1, "partition index out of range");
			const int p = (int)parts[i];
			job[5 * i + 0] = gvo[p];
			job[5 * i + 1] = gnv[p];
			job[5 * i + 2] = gso[p];
			job[5 * i + 3] = gns[p];
			job[5 * i + 4] = (int)i;
			if (counts) {
				counts[2 * i] = (uint32_t)gnv[p];
				counts[2 * i + 1] = (uint32_t)gns[p];
			}
			tv += gnv[p];
			ts += gns[p];
		}
		*nv = (size_t)tv;
		*ns = (size_t)ts;
		if (!n || (!vtx && !spx)) return;
		if ((size_t)tv * VF > vcap || (size_t)ts * D > scap)
			throw Error(-13, "gather buffers too small");
		std::vector<long long> dst(2 * n);
		long long av = 0, as = 0;
		for (size_t i = 0; i < n; i++) {
			dst[2 * i] = av;
			dst[2 * i + 1] = as;
			av += job[5 * i + 1];
			as += job[5 * i + 3];
		}
		const size_t need = (size_t)tv * VF * sizeof(float) + (size_t)ts * D * sizeof(uint32_t) +
		                    job.size() * sizeof(int) + dst.size() * sizeof(long long) + 64;
		if (need > stage_cap_) {
			if (stage_) FG_CUDA(cudaFreeAsync(stage_, eng_.stream()));
			stage_ = nullptr;
			stage_cap_ = std::max(need, (size_t)1 << 20);
			FG_CUDA(cudaMallocAsync(&stage_, stage_cap_, eng_.stream()));
		}
		char* base = static_cast<char*>(stage_);
		float* sv = reinterpret_cast<float*>(base);
		uint32_t* ss = reinterpret_cast<uint32_t*>(base + (size_t)tv * VF * sizeof(float));
		int* dj = reinterpret_cast<int*>(ss + (size_t)ts * D);
		long long* dd = reinterpret_cast<long long*>(
		    (reinterpret_cast<uintptr_t>(dj + job.size()) + 15) & ~(uintptr_t)15);
		cudaStream_t st = eng_.stream();
		FG_CUDA(cudaMemcpyAsync(dj, job.data(), job.size() * sizeof(int), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(dd, dst.data(), dst.size() * sizeof(long long),
		                        cudaMemcpyHostToDevice, st));
		FG_RUN("k_polys_gather", st, k_polys_gather<D><<<grid(), 256, 0, st>>>(Q_, dj, dd, (int)n, sv, ss););
		FG_CUDA(cudaGetLastError());
		if (vtx && tv)
			FG_CUDA(cudaMemcpyAsync(vtx, sv, (size_t)tv * VF * sizeof(float), cudaMemcpyDeviceToHost, st));
		if (spx && ts)
			FG_CUDA(cudaMemcpyAsync(spx, ss, (size_t)ts * D * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
		FG_CUDA(cudaStreamSynchronize(st));
	}

private:
	EngineBase& eng_;
	int s_;
	PolysDev Q_;
	int* woff_ = nullptr;
	void* stage_ = nullptr;  // gather staging buffer
	size_t stage_cap_ = 0;
	size_t smem_ = 0;
	int march_threads_ = 256;
	int nchunks_ = 0;                        // arena compaction: chunks of partitions
	int* noff_ = nullptr;                    // [NP] new vertex offsets
	int* nsoff_ = nullptr;                   // [NP] new simplex offsets
	unsigned long long* csum_ = nullptr;     // [2 * nchunks] chunk sums, then their scan
	unsigned long long* ctot_ = nullptr;     // [2] live vertices, simplices
	float* spare_v_ = nullptr;               // the other vertex arena
	uint32_t* spare_s_ = nullptr;            // the other simplex arena
	long long spare_vcap_ = 0, spare_scap_ = 0;
	std::vector<void*> owned_;
	std::vector<int> off_host_;  // host copy of Q_.off (sources of its updates)
	std::vector<int> pend_host_; // host copy of Q_.pendv
	std::vector<int> sel_host_;  // host copy of Q_.sel
};

}  // namespace

PolysBase* make_polys(EngineBase& eng, int s, size_t vertex_capacity)
{
	const int D = eng.dims(), L = eng.layers();
#define FG_CASE(d, l) \
	if (D == d && L == l) return new PolysImpl<d, l>(eng, s, vertex_capacity);
	FG_CASE(2, 1) FG_CASE(2, 2) FG_CASE(2, 3) FG_CASE(2, 4)
	FG_CASE(3, 1) FG_CASE(3, 2) FG_CASE(3, 3) FG_CASE(3, 4)
#undef FG_CASE
	throw Error(-1, "unsupported dims/layers");
}

}  // namespace fg
