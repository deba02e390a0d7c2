// Surface::save / Surface::load (include/Felt/Surface.hpp:180-196) for device surfaces: the
// isogrid of a surface in the reference's file format, read from and written to the brick pool.
//
// The reference writes its isogrid with cereal's BinaryOutputArchive (PartitionedMixin.hpp:
// 692-708): raw little-endian arithmetic values, std::vector as a uint64 count then its
// elements, no framing for classes (unversioned hooks); Eigen matrices through Felt's hook
// (PartitionedMixin.hpp:717-738) as int32 rows, int32 cols, then a std::vector of the
// coefficients; Felt's Tuple<T, N> is an Eigen column vector. In write order:
//
//   f32 background (L+1)                       Partitioned::Access, PartitionedMixin.hpp:581-586
//   VecDi child size                           Partitioned::Children, PartitionedMixin.hpp:93-97
//   children grid                              Tracked::MultiListMultiIdxByRef, Tracked.hpp:209-217
//     Child background (inactive, geometry never set by the reference: written as zeros)
//     u64 count, Child[count] (children grid order)
//     children lookup                          Lookup::MultiListMultiIdx, Lookup.hpp:228-236
//       IdxTuple null; u64 count, IdxTuple[count] (position in each partition list or null);
//       ListTuple partition lists; VecDi size, offset, offset + size
//     VecDi size, offset, offset + size (children grid)
//   VecDi size, offset, offset + size          Grid::Size, GridMixin.hpp:255-259
//   f32 dx (1), VecDi pos_min, pos_max         Numeric::Spatial, NumericMixin.hpp:55-60
//   Child                                      Tracked::LazyMultiListSingleIdxByValue, Tracked.hpp:53-60
//     f32 background; u64 count, f32[count] values (0 when inactive)
//     leaf lookup                              Lookup::LazyMultiListSingleIdx, Lookup.hpp:170-177
//       u64 null; u64 count, u64[count] (position of each leaf in its list, or null);
//       ListTuple leaf lists; VecDi size, offset, offset + size
//     VecDi size, offset, offset + size
//   VecDi = i32 D, i32 1, u64 D, i32[D];  IdxTuple = i32 N, i32 1, u64 N, u64[N];
//   ListTuple = i32 N, i32 1, u64 N, then per list u64 length and u64 entries. null = 2^64 - 1.
//
// Saving reads the surface's partition arrays and gathers its active bricks in one kernel;
// loading validates the file against the invariants the engine relies on and writes a freshly
// created surface's pool directly (active partitions in bricks 0..k-1).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "fg_dev.cuh"
#include "fg_engine.cuh"
#include "fg_image.cuh"

namespace fg {

namespace {

constexpr uint64_t NULL_IDX = ~0ull;

/// Copies the bricks of the given slots into contiguous staging, in the given order.
template <int L>
__global__ void k_gather_bricks(Dev P, const int* slots, int n, float* phi, uint16_t* lkp,
                                uint16_t* lst, int* lcnt)
{
	constexpr int NL = 2 * L + 1;
	for (int i = blockIdx.x; i < n; i += gridDim.x) {
		const int sl = slots[i];
		const size_t src = (size_t)sl * P.BV, dst = (size_t)i * P.BV;
		for (int j = threadIdx.x; j < P.BV; j += blockDim.x) {
			phi[dst + j] = P.phi[src + j];
			lkp[dst + j] = P.lkp[src + j];
		}
		for (int j = threadIdx.x; j < NL * P.BV; j += blockDim.x)
			lst[dst * NL + j] = P.lst[src * NL + j];
		for (int j = threadIdx.x; j < NL; j += blockDim.x) lcnt[i * NL + j] = P.lcnt[sl * NL + j];
	}
}

/// Writes staged bricks into their slots (the inverse of k_gather_bricks) and sets the rest of
/// each brick as activation leaves it (brick_init): no status, empty affected lists, no claims.
template <int L>
__global__ void k_scatter_bricks(Dev P, const int* slots, const int* gps, int n, const float* phi,
                                 const uint16_t* lkp, const uint16_t* lst, const int* lcnt)
{
	constexpr int NL = 2 * L + 1;
	for (int i = blockIdx.x; i < n; i += gridDim.x) {
		const int sl = slots[i];
		const size_t dst = (size_t)sl * P.BV, src = (size_t)i * P.BV;
		for (int j = threadIdx.x; j < P.BV; j += blockDim.x) {
			P.phi[dst + j] = phi[src + j];
			P.lkp[dst + j] = lkp[src + j];
			P.sto[dst + j] = (int8_t)(L + 1);
			P.alkp[0][dst + j] = NUL16;
			P.alkp[1][dst + j] = NUL16;
			P.claim[dst + j] = NOCLAIM;
		}
		for (int j = threadIdx.x; j < NL * P.BV; j += blockDim.x) P.lst[dst * NL + j] = lst[src * NL + j];
		for (int j = threadIdx.x; j < NL; j += blockDim.x) {
			P.lcnt[sl * NL + j] = lcnt[i * NL + j];
			P.ccnt[sl * NL + j] = 0;
			P.acnt[0][sl * NL + j] = 0;
			P.acnt[1][sl * NL + j] = 0;
		}
		if (threadIdx.x == 0) {
			P.slot_gp[sl] = gps[i];
			P.touched[sl] = 0;
		}
	}
}

template <class T>
T* dev_alloc(size_t n, cudaStream_t st)
{
	T* p = nullptr;
	FG_CUDA(cudaMallocAsync((void**)&p, (n ? n : 1) * sizeof(T), st));
	return p;
}

struct Out {
	std::vector<uint8_t>& b;
	template <class T>
	void raw(const T& v)
	{
		const uint8_t* p = reinterpret_cast<const uint8_t*>(&v);
		b.insert(b.end(), p, p + sizeof(T));
	}
	void vec(int D, const int* v)
	{
		raw<int32_t>(D);
		raw<int32_t>(1);
		raw<uint64_t>((uint64_t)D);
		for (int a = 0; a < D; a++) raw<int32_t>(v[a]);
	}
	void box(int D, const int* size, const int* off)
	{
		int hi[3];
		for (int a = 0; a < D; a++) hi[a] = off[a] + size[a];
		vec(D, size);
		vec(D, off);
		vec(D, hi);
	}
	void tuple_head(int N)
	{
		raw<int32_t>(N);
		raw<int32_t>(1);
		raw<uint64_t>((uint64_t)N);
	}
};

struct In {
	const uint8_t* p;
	size_t n, at;
	template <class T>
	T raw()
	{
		if (n - at < sizeof(T)) throw Error(-1, "truncated surface file");
		T v;
		std::memcpy(&v, p + at, sizeof(T));
		at += sizeof(T);
		return v;
	}
	void bad(const char* what) { throw Error(-1, std::string("surface file: ") + what); }
	void vec(int D, int* v)
	{
		if (raw<int32_t>() != D || raw<int32_t>() != 1 || raw<uint64_t>() != (uint64_t)D)
			bad("malformed vector");
		for (int a = 0; a < D; a++) v[a] = raw<int32_t>();
	}
	void box(int D, int* size, int* off)
	{
		int hi[3];
		vec(D, size);
		vec(D, off);
		vec(D, hi);
	}
	void tuple_head(int N)
	{
		if (raw<int32_t>() != N || raw<int32_t>() != 1 || raw<uint64_t>() != (uint64_t)N)
			bad("malformed tuple");
	}
};

/// Position of local child c in world space and its children-grid coordinates.
void child_origin(const SurfGeom& g, int D, const int* csz, int c, int* off)
{
	int rem = c;
	for (int a = D - 1; a >= 0; a--) {
		const int k = rem % g.ccount[a];
		rem /= g.ccount[a];
		off[a] = k * csz[a] + g.off[a];
	}
}

int layer_of(float v)
{
	const float x = v + 1.1920928955078125e-07f;
	return (int)roundf(x);
}

}  // namespace

void export_image(EngineBase& eng, int s, SurfaceImage& img)
{
	const int L = eng.layers(), NL = 2 * L + 1;
	const Dev& P = eng.dev();
	const SurfGeom& g = eng.geometry(s);
	cudaStream_t st = eng.stream();
	eng.sync();
	img.np = g.np;
	img.BV = P.BV;
	img.NL = NL;
	std::vector<int> slot(g.np);
	img.bg.resize(g.np);
	img.ppos.resize((size_t)g.np * NL);
	FG_CUDA(cudaMemcpy(slot.data(), P.slot + g.pbase, g.np * sizeof(int), cudaMemcpyDeviceToHost));
	FG_CUDA(cudaMemcpy(img.bg.data(), P.bg + g.pbase, g.np * sizeof(float), cudaMemcpyDeviceToHost));
	FG_CUDA(cudaMemcpy(img.ppos.data(), P.ppos + (size_t)g.pbase * NL, (size_t)g.np * NL * sizeof(int),
	                   cudaMemcpyDeviceToHost));
	std::vector<int> pcnt(NL);
	FG_CUDA(cudaMemcpy(pcnt.data(), P.pcnt + (size_t)s * NL, NL * sizeof(int), cudaMemcpyDeviceToHost));
	img.plist.assign(NL, {});
	for (int l = 0; l < NL; l++) {
		img.plist[l].resize(pcnt[l]);
		if (pcnt[l])
			FG_CUDA(cudaMemcpy(img.plist[l].data(), P.plist + (size_t)l * P.NP + g.pbase,
			                   pcnt[l] * sizeof(int), cudaMemcpyDeviceToHost));
	}
	img.active.clear();
	std::vector<int> slots;
	for (int c = 0; c < g.np; c++)
		if (slot[c] >= 0) {
			img.active.push_back(c);
			slots.push_back(slot[c]);
		}
	const int nact = (int)slots.size();
	const size_t bv = (size_t)P.BV;
	img.phi.resize(nact * bv);
	img.lkp.resize(nact * bv);
	img.lst.resize(nact * bv * NL);
	img.lcnt.resize((size_t)nact * NL);
	if (nact == 0) return;
	int* dslots = dev_alloc<int>(nact, st);
	float* dphi = dev_alloc<float>(nact * bv, st);
	uint16_t* dlkp = dev_alloc<uint16_t>(nact * bv, st);
	uint16_t* dlst = dev_alloc<uint16_t>(nact * bv * NL, st);
	int* dlcnt = dev_alloc<int>((size_t)nact * NL, st);
	FG_CUDA(cudaMemcpyAsync(dslots, slots.data(), nact * sizeof(int), cudaMemcpyHostToDevice, st));
	const unsigned blocks = (unsigned)std::min(nact, 148 * 8);
#define FG_CASE(ll) \
	if (L == ll) FG_RUN("k_gather_bricks", st, k_gather_bricks<ll><<<blocks, 256, 0, st>>>(P, dslots, nact, dphi, dlkp, dlst, dlcnt););
	FG_CASE(1) FG_CASE(2) FG_CASE(3) FG_CASE(4)
#undef FG_CASE
	FG_CUDA(cudaGetLastError());
	FG_CUDA(cudaMemcpyAsync(img.phi.data(), dphi, nact * bv * sizeof(float), cudaMemcpyDeviceToHost, st));
	FG_CUDA(cudaMemcpyAsync(img.lkp.data(), dlkp, nact * bv * sizeof(uint16_t), cudaMemcpyDeviceToHost, st));
	FG_CUDA(cudaMemcpyAsync(img.lst.data(), dlst, nact * bv * NL * sizeof(uint16_t), cudaMemcpyDeviceToHost, st));
	FG_CUDA(cudaMemcpyAsync(img.lcnt.data(), dlcnt, (size_t)nact * NL * sizeof(int), cudaMemcpyDeviceToHost, st));
	for (void* p : {(void*)dslots, (void*)dphi, (void*)dlkp, (void*)dlst, (void*)dlcnt})
		FG_CUDA(cudaFreeAsync(p, st));
	FG_CUDA(cudaStreamSynchronize(st));
	eng.check_errors();
}

void import_image(EngineBase& eng, const SurfaceImage& img)
{
	const int L = eng.layers(), NL = 2 * L + 1;
	const Dev& P = eng.dev();
	const SurfGeom& g = eng.geometry(0);
	if (eng.surfaces() != 1 || img.np != g.np || img.NL != NL || img.BV != P.BV)
		throw Error(-1, "surface image does not fit this surface");
	cudaStream_t st = eng.stream();
	eng.sync();
	int top = 0;
	FG_CUDA(cudaMemcpy(&top, P.counters + CNT_FREE_TOP, sizeof(int), cudaMemcpyDeviceToHost));
	if (top != P.nslots) throw Error(-15, "loading needs a newly created surface");
	const int nact = (int)img.active.size();
	if (nact > P.nslots) throw Error(-4, "brick pool too small for the loaded surface");
	const size_t bv = (size_t)P.BV;
	// a fresh pool hands out bricks 0, 1, 2, ... (its free stack holds n-1 .. 0)
	std::vector<int> slot(g.np, -1), slot_gp(nact);
	for (int i = 0; i < nact; i++) {
		slot[img.active[i]] = i;
		slot_gp[i] = g.pbase + img.active[i];
	}
	FG_CUDA(cudaMemcpyAsync(P.slot + g.pbase, slot.data(), g.np * sizeof(int), cudaMemcpyHostToDevice, st));
	FG_CUDA(cudaMemcpyAsync(P.bg + g.pbase, img.bg.data(), g.np * sizeof(float), cudaMemcpyHostToDevice, st));
	FG_CUDA(cudaMemcpyAsync(P.ppos + (size_t)g.pbase * NL, img.ppos.data(), (size_t)g.np * NL * sizeof(int),
	                        cudaMemcpyHostToDevice, st));
	std::vector<int> pcnt(NL);
	for (int l = 0; l < NL; l++) {
		pcnt[l] = (int)img.plist[l].size();
		if (pcnt[l])
			FG_CUDA(cudaMemcpyAsync(P.plist + (size_t)l * P.NP + g.pbase, img.plist[l].data(),
			                        pcnt[l] * sizeof(int), cudaMemcpyHostToDevice, st));
	}
	FG_CUDA(cudaMemcpyAsync(P.pcnt, pcnt.data(), NL * sizeof(int), cudaMemcpyHostToDevice, st));
	if (nact) {
		FG_CUDA(cudaMemcpyAsync(P.slot_gp, slot_gp.data(), nact * sizeof(int), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(P.phi, img.phi.data(), nact * bv * sizeof(float), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(P.lkp, img.lkp.data(), nact * bv * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(P.lst, img.lst.data(), nact * bv * NL * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(P.lcnt, img.lcnt.data(), (size_t)nact * NL * sizeof(int), cudaMemcpyHostToDevice, st));
		// the rest of each brick as activation leaves it (brick_init)
		FG_CUDA(cudaMemsetAsync(P.sto, L + 1, nact * bv, st));
		FG_CUDA(cudaMemsetAsync(P.alkp[0], 0xff, nact * bv * sizeof(uint16_t), st));
		FG_CUDA(cudaMemsetAsync(P.alkp[1], 0xff, nact * bv * sizeof(uint16_t), st));
		FG_CUDA(cudaMemsetAsync(P.claim, 0xff, nact * bv * sizeof(unsigned long long), st));
		FG_CUDA(cudaMemsetAsync(P.ccnt, 0, (size_t)nact * NL * sizeof(int), st));
		FG_CUDA(cudaMemsetAsync(P.acnt[0], 0, (size_t)nact * NL * sizeof(int), st));
		FG_CUDA(cudaMemsetAsync(P.acnt[1], 0, (size_t)nact * NL * sizeof(int), st));
	}
	const int ntop = P.nslots - nact;
	FG_CUDA(cudaMemcpyAsync(P.counters + CNT_FREE_TOP, &ntop, sizeof(int), cudaMemcpyHostToDevice, st));
	FG_CUDA(cudaStreamSynchronize(st));
	eng.check_errors();
}

void restore_image(EngineBase& eng, int s, const SurfaceImage& img)
{
	const int L = eng.layers(), NL = 2 * L + 1;
	const Dev& P = eng.dev();
	if (s < 0 || s >= eng.surfaces()) throw Error(-1, "surface index out of range");
	const SurfGeom& g = eng.geometry(s);
	if (img.np != g.np || img.NL != NL || img.BV != P.BV)
		throw Error(-1, "surface image does not fit this surface");
	if (eng.frozen(s)) throw Error(-15, "restoring into a stopped surface");
	cudaStream_t st = eng.stream();
	eng.sync();
	// the surface must be empty: no active partition, every list of it empty
	std::vector<int> slot(g.np);
	FG_CUDA(cudaMemcpy(slot.data(), P.slot + g.pbase, g.np * sizeof(int), cudaMemcpyDeviceToHost));
	for (int v : slot)
		if (v >= 0) throw Error(-15, "restoring needs an empty surface (no active partition)");
	const int* counts[] = {P.pcnt, P.dpcnt, P.spcnt, P.apcnt[0], P.apcnt[1]};
	for (const int* c : counts) {
		std::vector<int> n(NL);
		FG_CUDA(cudaMemcpy(n.data(), c + (size_t)s * NL, NL * sizeof(int), cudaMemcpyDeviceToHost));
		for (int v : n)
			if (v) throw Error(-15, "restoring needs an empty surface (a partition list is not empty)");
	}
	const int nact = (int)img.active.size();
	int top = 0;
	FG_CUDA(cudaMemcpy(&top, P.counters + CNT_FREE_TOP, sizeof(int), cudaMemcpyDeviceToHost));
	if (nact > top) throw Error(-4, "brick pool too small for the restored surface");
	// bricks from the top of the free stack, as activation takes them
	std::vector<int> slots(nact), gps(nact);
	if (nact)
		FG_CUDA(cudaMemcpy(slots.data(), P.free_stack + (top - nact), nact * sizeof(int),
		                   cudaMemcpyDeviceToHost));
	for (int i = 0; i < nact; i++) {
		gps[i] = g.pbase + img.active[i];
		slot[img.active[i]] = slots[i];
	}
	const int ntop = top - nact;
	FG_CUDA(cudaMemcpyAsync(P.counters + CNT_FREE_TOP, &ntop, sizeof(int), cudaMemcpyHostToDevice, st));
	FG_CUDA(cudaMemcpyAsync(P.slot + g.pbase, slot.data(), g.np * sizeof(int), cudaMemcpyHostToDevice, st));
	FG_CUDA(cudaMemcpyAsync(P.bg + g.pbase, img.bg.data(), g.np * sizeof(float), cudaMemcpyHostToDevice, st));
	FG_CUDA(cudaMemcpyAsync(P.ppos + (size_t)g.pbase * NL, img.ppos.data(), (size_t)g.np * NL * sizeof(int),
	                        cudaMemcpyHostToDevice, st));
	std::vector<int> pcnt(NL);
	for (int l = 0; l < NL; l++) {
		pcnt[l] = (int)img.plist[l].size();
		if (pcnt[l])
			FG_CUDA(cudaMemcpyAsync(P.plist + (size_t)l * P.NP + g.pbase, img.plist[l].data(),
			                        pcnt[l] * sizeof(int), cudaMemcpyHostToDevice, st));
	}
	FG_CUDA(cudaMemcpyAsync(P.pcnt + (size_t)s * NL, pcnt.data(), NL * sizeof(int), cudaMemcpyHostToDevice, st));
	if (nact) {
		const size_t bv = (size_t)P.BV;
		int* dslots = dev_alloc<int>(nact, st);
		int* dgps = dev_alloc<int>(nact, st);
		float* dphi = dev_alloc<float>(nact * bv, st);
		uint16_t* dlkp = dev_alloc<uint16_t>(nact * bv, st);
		uint16_t* dlst = dev_alloc<uint16_t>(nact * bv * NL, st);
		int* dlcnt = dev_alloc<int>((size_t)nact * NL, st);
		FG_CUDA(cudaMemcpyAsync(dslots, slots.data(), nact * sizeof(int), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(dgps, gps.data(), nact * sizeof(int), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(dphi, img.phi.data(), nact * bv * sizeof(float), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(dlkp, img.lkp.data(), nact * bv * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(dlst, img.lst.data(), nact * bv * NL * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
		FG_CUDA(cudaMemcpyAsync(dlcnt, img.lcnt.data(), (size_t)nact * NL * sizeof(int), cudaMemcpyHostToDevice, st));
		const unsigned blocks = (unsigned)std::min(nact, 148 * 8);
#define FG_CASE(ll) \
	if (L == ll) FG_RUN("k_scatter_bricks", st, k_scatter_bricks<ll><<<blocks, 256, 0, st>>>(P, dslots, dgps, nact, dphi, dlkp, dlst, dlcnt););
		FG_CASE(1) FG_CASE(2) FG_CASE(3) FG_CASE(4)
#undef FG_CASE
		FG_CUDA(cudaGetLastError());
		for (void* q : {(void*)dslots, (void*)dgps, (void*)dphi, (void*)dlkp, (void*)dlst, (void*)dlcnt})
			FG_CUDA(cudaFreeAsync(q, st));
	}
	FG_CUDA(cudaStreamSynchronize(st));
	eng.check_errors();
}

void write_surface_file(const SurfaceImage& img, const SurfGeom& g, int D, int L, const int* csz,
                        std::vector<uint8_t>& out)
{
	const int NL = 2 * L + 1;
	const size_t bv = (size_t)img.BV;
	Out w{out};
	const int zero[3] = {0, 0, 0};
	std::vector<int> act_of(img.np, -1);
	for (size_t i = 0; i < img.active.size(); i++) act_of[img.active[i]] = (int)i;
	auto child = [&](float bg, int a, const int* off) {
		w.raw<float>(bg);
		if (a < 0) {
			w.raw<uint64_t>(0);
		} else {
			w.raw<uint64_t>(bv);
			const float* v = img.phi.data() + (size_t)a * bv;
			const uint8_t* pv = reinterpret_cast<const uint8_t*>(v);
			out.insert(out.end(), pv, pv + bv * sizeof(float));
		}
		w.raw<uint64_t>(NULL_IDX);
		if (a < 0) {
			w.raw<uint64_t>(0);
		} else {
			w.raw<uint64_t>(bv);
			const uint16_t* k = img.lkp.data() + (size_t)a * bv;
			for (size_t j = 0; j < bv; j++) w.raw<uint64_t>(k[j] == NUL16 ? NULL_IDX : (uint64_t)k[j]);
		}
		w.tuple_head(NL);
		for (int l = 0; l < NL; l++) {
			const int n = a < 0 ? 0 : img.lcnt[(size_t)a * NL + l];
			w.raw<uint64_t>((uint64_t)n);
			const uint16_t* e = img.lst.data() + ((size_t)a * NL + l) * bv;
			for (int j = 0; j < n; j++) w.raw<uint64_t>(e[j]);
		}
		w.box(D, off ? csz : zero, off ? off : zero);
		w.box(D, off ? csz : zero, off ? off : zero);
	};
	w.raw<float>((float)(L + 1));
	w.vec(D, csz);
	child((float)(L + 1), -1, nullptr);
	w.raw<uint64_t>((uint64_t)img.np);
	for (int c = 0; c < img.np; c++) {
		int off[3];
		child_origin(g, D, csz, c, off);
		child(img.bg[c], act_of[c], off);
	}
	w.tuple_head(NL);
	for (int l = 0; l < NL; l++) w.raw<uint64_t>(NULL_IDX);
	w.raw<uint64_t>((uint64_t)img.np);
	for (int c = 0; c < img.np; c++) {
		w.tuple_head(NL);
		for (int l = 0; l < NL; l++) {
			const int p = img.ppos[(size_t)c * NL + l];
			w.raw<uint64_t>(p < 0 ? NULL_IDX : (uint64_t)p);
		}
	}
	w.tuple_head(NL);
	for (int l = 0; l < NL; l++) {
		w.raw<uint64_t>(img.plist[l].size());
		for (int c : img.plist[l]) w.raw<uint64_t>((uint64_t)c);
	}
	for (int k = 0; k < 2; k++) w.box(D, g.ccount, g.coff);
	w.box(D, g.size, g.off);
	w.raw<float>(1.0f);
	int hi[3];
	for (int a = 0; a < D; a++) hi[a] = g.off[a] + g.size[a];
	w.vec(D, g.off);
	w.vec(D, hi);
}

void peek_surface_file(const uint8_t* p, size_t n, int& D, int& L, int* size, int* csz)
{
	In r{p, n, 0};
	r.raw<float>();
	D = r.raw<int32_t>();
	if (D != 2 && D != 3) r.bad("dimension other than 2 or 3");
	if (r.raw<int32_t>() != 1 || r.raw<uint64_t>() != (uint64_t)D) r.bad("malformed vector");
	for (int a = 0; a < D; a++) csz[a] = r.raw<int32_t>();
	r.raw<float>();
	if (r.raw<uint64_t>() != 0) r.bad("active background child");
	r.raw<uint64_t>();
	if (r.raw<uint64_t>() != 0) r.bad("active background lookup");
	const int NL = r.raw<int32_t>();
	if (NL < 3 || NL > 9 || NL % 2 == 0) r.bad("list count other than 3, 5, 7 or 9");
	L = (NL - 1) / 2;
	const size_t vec = 16 + 4 * (size_t)D, tail = 5 * vec + 4;
	if (n < tail + r.at) r.bad("too short");
	In t{p, n, n - tail};
	t.vec(D, size);
	for (int a = 0; a < D; a++)
		if (size[a] <= 0 || csz[a] <= 0) r.bad("non-positive size");
}

void read_surface_file(const uint8_t* p, size_t n, const SurfGeom& g, int D, int L,
                       const int* csz, int BV, SurfaceImage& img)
{
	const int NL = 2 * L + 1;
	const size_t bv = (size_t)BV;
	In r{p, n, 0};
	img.np = g.np;
	img.BV = BV;
	img.NL = NL;
	img.bg.assign(g.np, 0.0f);
	img.ppos.assign((size_t)g.np * NL, -1);
	img.plist.assign(NL, {});
	img.active.clear();
	img.phi.clear();
	img.lkp.clear();
	img.lst.clear();
	img.lcnt.clear();
	if (r.raw<float>() != (float)(L + 1)) r.bad("background other than L+1");
	int v[3], w3[3];
	r.vec(D, v);
	for (int a = 0; a < D; a++)
		if (v[a] != csz[a]) r.bad("partition size differs");
	std::vector<uint64_t> scratch;
	auto child = [&](int c) {
		const float bg = r.raw<float>();
		const uint64_t nd = r.raw<uint64_t>();
		if (nd != 0 && nd != bv) r.bad("partition data size");
		if (c < 0 && nd) r.bad("active background child");
		const int a = nd ? (int)img.active.size() : -1;
		if (c >= 0) img.bg[c] = bg;
		if (nd) {
			img.active.push_back(c);
			const size_t base = img.phi.size();
			img.phi.resize(base + bv);
			if (n - r.at < bv * sizeof(float)) r.bad("truncated");
			std::memcpy(img.phi.data() + base, p + r.at, bv * sizeof(float));
			r.at += bv * sizeof(float);
			for (size_t j = 0; j < bv; j++)
				if (!std::isfinite(img.phi[base + j])) r.bad("non-finite value");
		}
		if (r.raw<uint64_t>() != NULL_IDX) r.bad("leaf lookup background");
		if (r.raw<uint64_t>() != nd) r.bad("leaf lookup size");
		if (nd) {
			const size_t base = img.lkp.size();
			img.lkp.resize(base + bv);
			for (size_t j = 0; j < bv; j++) {
				const uint64_t x = r.raw<uint64_t>();
				if (x != NULL_IDX && x >= bv) r.bad("leaf lookup entry");
				img.lkp[base + j] = x == NULL_IDX ? NUL16 : (uint16_t)x;
			}
			img.lst.resize(img.lst.size() + (size_t)NL * bv, 0);
			img.lcnt.resize(img.lcnt.size() + NL, 0);
		}
		r.tuple_head(NL);
		for (int l = 0; l < NL; l++) {
			const uint64_t len = r.raw<uint64_t>();
			if (len > bv || (!nd && len)) r.bad("leaf list length");
			for (uint64_t j = 0; j < len; j++) {
				const uint64_t x = r.raw<uint64_t>();
				if (x >= bv) r.bad("leaf list entry");
				const size_t k = (size_t)a * bv + x;
				if (img.lkp[k] != j) r.bad("leaf lookup and list disagree");
				if (layer_of(img.phi[k]) != l - L) r.bad("leaf listed in a layer other than its own");
				img.lst[((size_t)a * NL + l) * bv + j] = (uint16_t)x;
			}
			if (nd) img.lcnt[(size_t)a * NL + l] = (int)len;
		}
		for (int k = 0; k < 2; k++) {
			r.box(D, v, w3);
			if (c >= 0) {
				int off[3];
				child_origin(g, D, csz, c, off);
				for (int q = 0; q < D; q++)
					if (v[q] != csz[q] || w3[q] != off[q]) r.bad("partition geometry differs");
			}
		}
		if (nd) {  // every tracked leaf is in its list
			size_t tracked = 0;
			for (size_t j = 0; j < bv; j++) tracked += img.lkp[(size_t)a * bv + j] != NUL16;
			size_t listed = 0;
			for (int l = 0; l < NL; l++) listed += img.lcnt[(size_t)a * NL + l];
			if (tracked != listed) r.bad("leaf lookup entries outside the lists");
		}
	};
	child(-1);
	if (r.raw<uint64_t>() != (uint64_t)g.np) r.bad("partition count differs");
	for (int c = 0; c < g.np; c++) child(c);
	r.tuple_head(NL);
	for (int l = 0; l < NL; l++)
		if (r.raw<uint64_t>() != NULL_IDX) r.bad("children lookup background");
	if (r.raw<uint64_t>() != (uint64_t)g.np) r.bad("children lookup size");
	for (int c = 0; c < g.np; c++) {
		r.tuple_head(NL);
		for (int l = 0; l < NL; l++) {
			const uint64_t x = r.raw<uint64_t>();
			if (x != NULL_IDX && x >= (uint64_t)g.np) r.bad("children lookup entry");
			img.ppos[(size_t)c * NL + l] = x == NULL_IDX ? -1 : (int)x;
		}
	}
	std::vector<int> act_of(g.np, -1);
	for (size_t i = 0; i < img.active.size(); i++) act_of[img.active[i]] = (int)i;
	r.tuple_head(NL);
	for (int l = 0; l < NL; l++) {
		const uint64_t len = r.raw<uint64_t>();
		if (len > (uint64_t)g.np) r.bad("partition list length");
		img.plist[l].resize(len);
		for (uint64_t j = 0; j < len; j++) {
			const uint64_t c = r.raw<uint64_t>();
			if (c >= (uint64_t)g.np) r.bad("partition list entry");
			if (img.ppos[(size_t)c * NL + l] != (int)j) r.bad("children lookup and list disagree");
			img.plist[l][j] = (int)c;
		}
	}
	// a partition is in list l exactly when it is active and its leaf list l is not empty
	for (int c = 0; c < g.np; c++)
		for (int l = 0; l < NL; l++) {
			const int pp = img.ppos[(size_t)c * NL + l];
			if (pp >= 0 && (pp >= (int)img.plist[l].size() || img.plist[l][pp] != c))
				r.bad("children lookup entry not in its list");
			const bool nonempty = act_of[c] >= 0 && img.lcnt[(size_t)act_of[c] * NL + l] > 0;
			if ((pp >= 0) != nonempty) r.bad("partition list membership");
		}
	for (int k = 0; k < 2; k++) {
		r.box(D, v, w3);
		for (int q = 0; q < D; q++)
			if (v[q] != g.ccount[q] || w3[q] != g.coff[q]) r.bad("children grid differs");
	}
	r.box(D, v, w3);
	for (int q = 0; q < D; q++)
		if (v[q] != g.size[q] || w3[q] != g.off[q]) r.bad("grid differs");
	if (r.raw<float>() != 1.0f) r.bad("dx other than 1");
	r.vec(D, v);
	r.vec(D, w3);
	if (r.at != n) r.bad("trailing bytes");
}

}  // namespace fg
