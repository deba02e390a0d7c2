// Host orchestration of the device pool (see fg_engine.cuh).
#include <algorithm>
#include <cstring>

#include "fg_engine.cuh"
#include "fg_kernels.cuh"

namespace fg {

namespace {

template <class T>
T* dalloc(size_t n, std::vector<void*>& owned)
{
	void* p = nullptr;
	if (n == 0) n = 1;
	cudaError_t e = locked_malloc(&p, n * sizeof(T));
	if (e != cudaSuccess)
		throw Error(-3, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
	owned.push_back(p);
	return static_cast<T*>(p);
}

__global__ void k_fill_int(int* p, long long n, int v)
{
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
	     i += (long long)gridDim.x * blockDim.x)
		p[i] = v;
}
__global__ void k_fill_float(float* p, long long n, float v)
{
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
	     i += (long long)gridDim.x * blockDim.x)
		p[i] = v;
}
/// Start of the device-side convergence loop: the first flush and expansion count as iteration
/// 1; the loop body runs while a layer changed.
__global__ void k_loop_init(const int* changed, int* iters, cudaGraphConditionalHandle loop)
{
	pdl_enter();
	if (threadIdx.x == 0) {
		*iters = 1;
		cudaGraphSetConditional(loop, *changed ? 1u : 0u);
	}
}

/// End of one iteration of the device-side convergence loop: counts it and goes on while a
/// layer changed and the count is not a multiple of cap (where the host looks for surfaces to
/// stop, as the host loop does), so the loop ends after at most cap - 1 iterations. Sets both
/// handles (the loop's and the one of the body's second iteration) where two are given.
__global__ void k_loop_test(const int* changed, int* iters, int cap, cudaGraphConditionalHandle a,
                            cudaGraphConditionalHandle b, int both)
{
	pdl_enter();
	if (threadIdx.x == 0) {
		const int it = *iters + 1;
		*iters = it;
		const unsigned go = (*changed != 0 && it % cap != 0) ? 1u : 0u;
		cudaGraphSetConditional(a, go);
		if (both) cudaGraphSetConditional(b, go);
	}
}

__global__ void k_iota_rev(int* p, int n)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		p[i] = n - 1 - i;
}

int sm_count()
{
	static int n = 0;
	if (!n) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
		if (n <= 0) n = 148;
	}
	return n;
}

}  // namespace

std::recursive_mutex& device_lock()
{
	static std::recursive_mutex m;
	return m;
}

template <int D, int L>
class Engine final : public EngineBase {
public:
	static constexpr int NL = 2 * L + 1;

	Engine(const PoolDesc& desc, cudaStream_t st) : st_(st)
	{
		if (desc.D != D || desc.L != L) throw Error(-1, "engine dims mismatch");
		const int S = (int)desc.sizes.size();
		if (S <= 0) throw Error(-1, "pool needs at least one surface");
		int BV = 1;
		for (int a = 0; a < D; a++) {
			if (desc.part[a] <= 0) throw Error(-1, "partition size must be positive");
			csz_[a] = desc.part[a];
			BV *= desc.part[a];
		}
		if (BV > 65535) throw Error(-1, "partition volume must be < 65536");
		geom_.resize(S);
		np_cap_.resize(S);
		if (!desc.caps.empty() && desc.caps.size() != (size_t)S)
			throw Error(-1, "one capacity per surface");
		long long NP = 0;
		for (int s = 0; s < S; s++) {
			SurfGeom& g = geom_[s];
			g = grid_geom(desc.sizes[s].data(), 0);
			long long cap = g.np;
			if (!desc.caps.empty()) {
				// any grid up to caps[s] on every axis: a partial partition on one axis adds a
				// partition along every axis, so the most is prod(caps / part + 1)
				long long m = 1;
				for (int a = 0; a < D; a++) {
					if (desc.caps[s][a] <= 0) throw Error(-1, "capacity must be positive");
					m *= desc.caps[s][a] / csz_[a] + 1;
				}
				if (m >= (1 << 24)) throw Error(-1, "too many partitions in one surface");
				cap = std::max(cap, m);
			}
			g.pbase = (int)NP;
			np_cap_[s] = (int)cap;
			NP += cap;
		}
		if (NP >= (1LL << 31) / NL) throw Error(-1, "pool too large");
		size_t nslots = desc.brick_capacity;
		if (nslots == 0) nslots = (size_t)std::min<long long>(NP, 1LL << 20);
		if (nslots > (size_t)NP) nslots = (size_t)NP;

		Dev& P = P_;
		std::memset(&P, 0, sizeof(P));
		P.S = S;
		P.NP = (int)NP;
		P.BV = BV;
		P.nslots = (int)nslots;
		for (int a = 0; a < 3; a++) P.csz[a] = a < D ? csz_[a] : 1;
		{
			int str = 1;
			for (int a = D - 1; a >= 0; a--) {
				P.lstr[a] = str;
				str *= csz_[a];
			}
		}
		// host-side partition tables
		std::vector<int> surf_of(NP), porig(NP * 3);
		for (int s = 0; s < S; s++) {
			const SurfGeom& g = geom_[s];
			for (int i = g.np; i < np_cap_[s]; i++) surf_of[g.pbase + i] = s;
			for (int i = 0; i < g.np; i++) {
				int r = i;
				int c[3] = {0, 0, 0};
				for (int a = D - 1; a >= 0; a--) {
					c[a] = r % g.ccount[a];
					r /= g.ccount[a];
				}
				surf_of[g.pbase + i] = s;
				for (int a = 0; a < 3; a++)
					porig[(size_t)(g.pbase + i) * 3 + a] = a < D ? c[a] * csz_[a] + g.off[a] : 0;
			}
		}
		auto& o = owned_;
		SurfGeom* dgeom = dalloc<SurfGeom>(S, o);
		FG_CUDA(cudaMemcpy(dgeom, geom_.data(), S * sizeof(SurfGeom), cudaMemcpyHostToDevice));
		P.geom = dgeom;
		int* dso = dalloc<int>(NP, o);
		FG_CUDA(cudaMemcpy(dso, surf_of.data(), NP * sizeof(int), cudaMemcpyHostToDevice));
		P.surf_of = dso;
		int* dpo = dalloc<int>(NP * 3, o);
		FG_CUDA(cudaMemcpy(dpo, porig.data(), NP * 3 * sizeof(int), cudaMemcpyHostToDevice));
		P.porig = dpo;

		const size_t npl = (size_t)NP * NL, spl = (size_t)S * NL;
		P.slot = dalloc<int>(NP, o);
		P.bg = dalloc<float>(NP, o);
		P.oslot = dalloc<int>(NP, o);
		P.ppos = dalloc<int>(npl, o);
		P.plist = dalloc<int>(npl, o);
		P.pcnt = dalloc<int>(spl, o);
		P.dplist = dalloc<int>(npl, o);
		P.dpcnt = dalloc<int>(spl, o);
		P.splist = dalloc<int>(npl, o);
		P.spcnt = dalloc<int>(spl, o);
		P.sppos = dalloc<int>(npl, o);
		for (int b = 0; b < 2; b++) {
			P.aplist[b] = dalloc<int>(npl, o);
			P.apcnt[b] = dalloc<int>(spl, o);
			P.appos[b] = dalloc<int>(npl, o);
		}
		const size_t nb = nslots * (size_t)BV, nbl = nslots * (size_t)NL * BV;
		P.phi = dalloc<float>(nb, o);
		P.dlt = dalloc<float>(nb, o);
		P.lkp = dalloc<uint16_t>(nb, o);
		P.lst = dalloc<uint16_t>(nbl, o);
		P.lcnt = dalloc<int>(nslots * NL, o);
		P.sto = dalloc<int8_t>(nb, o);
		P.chg = dalloc<uint16_t>(nbl, o);
		P.ccnt = dalloc<int>(nslots * NL, o);
		for (int b = 0; b < 2; b++) {
			P.alkp[b] = dalloc<uint16_t>(nb, o);
			P.alst[b] = dalloc<uint16_t>(nbl, o);
			P.acnt[b] = dalloc<int>(nslots * NL, o);
		}
		P.claim = dalloc<unsigned long long>(nb, o);
		P.ccl = dalloc<uint16_t>(nb, o);
		P.ccln = dalloc<int>(nslots, o);
		FG_CUDA(cudaMemsetAsync(P.ccln, 0, nslots * sizeof(int), st_));
		// expansion candidates: most iterations need a few thousand; past the cap the claim
		// and compute phases walk the status lists again instead
		P.cand_cap = (int)std::min<size_t>(nb / 4 + 1024, (size_t)1 << 22);
		P.cand_key = dalloc<unsigned long long>((size_t)P.cand_cap, o);
		P.cand_gp = dalloc<int>((size_t)P.cand_cap, o);
		P.cand_leaf = dalloc<int>((size_t)P.cand_cap, o);
		P.slot_gp = dalloc<int>(nslots, o);
		P.free_stack = dalloc<int>(nslots, o);
		P.counters = dalloc<int>(CNT_N, o);
		P.q_act = dalloc<int>(NP, o);
		P.actflag = dalloc<int>(NP, o);
		P.q_touch = dalloc<int>(nslots, o);
		P.touched = dalloc<int>(nslots, o);
		P.q_retire = dalloc<int>(nslots, o);
		P.q_sunion = dalloc<int>(NP, o);
		P.sflag = dalloc<int>(NP, o);
		P.eflag = dalloc<unsigned>(NP, o);
		P.eflag2 = dalloc<unsigned>(NP, o);
		P.app = dalloc<unsigned>(npl, o);
		P.rem = dalloc<unsigned>(NP, o);
		P.pap = dalloc<unsigned long long>(2 * (size_t)NP, o);
		P.papg = dalloc<int>(2 * (size_t)NP, o);
		P.papn = dalloc<int>(S, o);
		P.woff = dalloc<int>(S + 1, o);
		P.woffl = dalloc<int>((size_t)NL * (S + 1), o);
		P.etab = dalloc<int4>((size_t)NL * NP, o);
		P.dq = dalloc<int>(nslots, o);
		P.eflagl = dalloc<unsigned>(npl, o);
		P.sfrozen = dalloc<int>(S, o);
		FG_CUDA(cudaMemsetAsync(P.sfrozen, 0, S * sizeof(int), st_));
		frozen_.assign(S, 0);
		paused_.assign(S, 0);
		P.err = dalloc<int>(1, o);
		P.changed = dalloc<int>(1, o);
		P.kstat = dalloc<unsigned long long>(KS_N, o);
		P.snu = dalloc<unsigned long long>(S, o);
		FG_CUDA(cudaMemsetAsync(P.snu, 0, S * sizeof(unsigned long long), st_));
		P.dlcnt = dalloc<int>(nslots, o);
		P.ndp = dalloc<int>(S, o);
		P.ring_first = dalloc<int>(npl, o);
		P.ring_last = dalloc<int>(npl, o);
		P.ring_src = dalloc<int>(npl, o);
		P.ring_n = dalloc<int>(2 * NL, o);
		P.apkey = dalloc<unsigned long long>(npl, o);
		P.aq = dalloc<int>(npl, o);
		FG_CUDA(cudaMemsetAsync(P.kstat, 0, KS_N * sizeof(unsigned long long), st_));
		acc_ = dalloc<unsigned long long>(1, o);
		zcount_ = dalloc<unsigned long long>(1, o);
		d_iters_ = dalloc<int>(1, o);
		d_speeds_ = dalloc<Speed>(S, o);
		FG_CUDA(cudaHostAlloc((void**)&h_speeds_, (size_t)S * sizeof(Speed), cudaHostAllocDefault));
		FG_CUDA(cudaHostAlloc((void**)&h_out_, 2 * sizeof(int), cudaHostAllocDefault));

		fill(P.slot, NP, -1);
		fillf(P.bg, NP, (float)(L + 1));
		fill(P.oslot, NP, -1);
		fill(P.ppos, npl, -1);
		FG_CUDA(cudaMemsetAsync(P.apkey, 0xff, npl * sizeof(unsigned long long), st_));
		fill(P.sppos, npl, -1);
		fill(P.appos[0], npl, -1);
		fill(P.appos[1], npl, -1);
		fill(P.actflag, NP, 0);
		fill(P.sflag, NP, 0);
		fill(P.touched, nslots, 0);
		fill(P.slot_gp, nslots, -1);
		FG_CUDA(cudaMemsetAsync(P.pcnt, 0, spl * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.dpcnt, 0, spl * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.spcnt, 0, spl * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.apcnt[0], 0, spl * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.apcnt[1], 0, spl * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.papn, 0, S * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.counters, 0, CNT_N * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P.changed, 0, sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(acc_, 0, sizeof(unsigned long long), st_));
		FG_RUN("k_iota_rev", st_, k_iota_rev<<<grid_for(nslots), 256, 0, st_>>>(P.free_stack, (int)nslots););
		const int top = (int)nslots;
		FG_CUDA(cudaMemcpyAsync(P.counters + CNT_FREE_TOP, &top, sizeof(int), cudaMemcpyHostToDevice,
		                        st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		FG_CUDA(cudaGetLastError());
		smem_sort_ = 8;
		while (smem_sort_ < (size_t)BV * 8) smem_sort_ <<= 1;
		if (smem_sort_ > 48 * 1024)
			FG_CUDA(cudaFuncSetAttribute(k_expand_append<L>,
			                             cudaFuncAttributeMaxDynamicSharedMemorySize,
			                             (int)smem_sort_));
		warp_grid_ = sm_count() * 8;
		smem_halo_ = halo_smem_bytes(D, csz_);
		if (smem_halo_ > 200 * 1024) {
			smem_halo_ = 0;  // partition too large to stage with its halo
		} else if (smem_halo_ > 48 * 1024) {
			FG_CUDA(cudaFuncSetAttribute(k_delta_smem<D, L>,
			                             cudaFuncAttributeMaxDynamicSharedMemorySize,
			                             (int)smem_halo_));
		}
		// staging pays off once a brick's zero layer is dense: measured on C2 (16^3 bricks) the
		// staged kernel took a third of the direct one's time per step over 40 steps
		delta_staged_ = smem_halo_ != 0;
		// warps per entry of the first distance pass: the extra warps of a short list exit after
		// one entry-table load, those of a long one share its leaves (C2, 16^3 bricks: 8 warps
		// 1.13-1.16 ms per step against 1.16-1.17 with 4)
		dist_split_ = BV >= 4096 ? 8 : BV >= 1024 ? 2 : 1;
		block_passes_ = BV >= 2048;
		smem_flush_ = flush_smem_bytes(BV, NL);
		if (smem_flush_ <= 200 * 1024) {
			if (smem_flush_ > 48 * 1024)
				FG_CUDA(cudaFuncSetAttribute(k_flush_smem<D, L>,
				                             cudaFuncAttributeMaxDynamicSharedMemorySize,
				                             (int)smem_flush_));
		} else {
			smem_flush_ = 0;  // brick too large to stage: replay in global memory
		}
		// tiled distance passes: the brick with a halo of 2L nodes per side in shared memory
		// (the halo may reach no further than the next partition along each axis)
		{
			TileShape t{};
			t.H = 2 * L;
			t.NT = 1;
			bool ok = true;
			for (int a = 2; a >= 0; a--) {
				t.T[a] = a < D ? csz_[a] + 2 * t.H : 1;
				t.ts[a] = t.NT;
				t.NT *= t.T[a];
				if (a < D && t.H > csz_[a]) ok = false;
			}
			tiled_threads_ = t.NT >= 4096 ? 1024 : 256;
			smem_tiled_ = tiled_smem_bytes(t.NT, tiled_threads_);
			if (ok && smem_tiled_ <= 220 * 1024) {
				if (smem_tiled_ > 48 * 1024)
					FG_CUDA(cudaFuncSetAttribute(k_dist_tiled<D, L>,
					                             cudaFuncAttributeMaxDynamicSharedMemorySize,
					                             (int)smem_tiled_));
				int per_sm = 0;
				FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
				    &per_sm, k_dist_tiled<D, L>, tiled_threads_, smem_tiled_));
				tiled_grid_ = sm_count() * std::max(1, per_sm);
				tile_ = t;
				// opt-in only: slower than the sparse passes on every measured workload (C2
				// 1.60 against 0.99 ms per step; batched 3D, 8^3 partitions, 2.28 against 1.71;
				// batched 2D, 16^2 partitions, 2.26 against 1.97), the staged tiles being
				// mostly off the band
			} else {
				smem_tiled_ = 0;
			}
		}
	}

public:
	/// Launch tuning (fg_config): how the global update launches (0 automatic = 1, 1 the
	/// whole update as one CUDA graph, 2 every kernel launched from the host, no graphs),
	/// warps per partition entry in the first distance pass (0 = automatic), warp (1) or block
	/// (2) per entry in the record passes (0 = automatic). Graphs captured under the previous
	/// tuning are dropped.
	void set_tuning(int launch_mode, int dist_split, int record_passes, int delta_kernel,
	                int fuse_passes) override
	{
		if (fuse_passes == 1) fused_ = tiled_ = false;
		if (fuse_passes == 2) {
			fused_ = true;
			tiled_ = false;
		}
		if (fuse_passes == 3) {
			fused_ = false;
			tiled_ = smem_tiled_ != 0;
		}
		launch_mode_ = launch_mode;
		if (dist_split > 0) dist_split_ = dist_split;
		if (record_passes == 1) block_passes_ = false;
		if (record_passes == 2) block_passes_ = true;
		if (delta_kernel == 1) delta_staged_ = false;
		if (delta_kernel == 2) delta_staged_ = smem_halo_ != 0;
		drop_graphs();
	}
	void tuning(int* out) const override
	{
		out[0] = launch_mode_ == 2 ? 2 : 1;
		out[1] = dist_split_;
		out[2] = block_passes_ ? 2 : 1;
		out[3] = delta_staged_ ? 2 : 1;
		out[4] = tiled_ ? 3 : fused_ ? 2 : 1;
	}

private:

	~Engine() override
	{
		cudaStreamSynchronize(st_);
		for (cudaGraphExec_t& ex : iter_exec_)
			if (ex) cudaGraphExecDestroy(ex);
		for (cudaGraphExec_t& ex : step_exec_)
			if (ex) cudaGraphExecDestroy(ex);
		if (loop_exec_) cudaGraphExecDestroy(loop_exec_);
		for (void* p : owned_) locked_free(p);
		if (d_lpos_) locked_free(d_lpos_);
		if (d_lval_) locked_free(d_lval_);
		if (d_lcount_) locked_free(d_lcount_);
		if (h_speeds_) cudaFreeHost(h_speeds_);
		if (h_out_) cudaFreeHost(h_out_);
	}

	int dims() const override { return D; }
	int layers() const override { return L; }
	int surfaces() const override { return P_.S; }
	cudaStream_t stream() const override { return st_; }
	StepStats& stats() override { return stats_; }
	unsigned long long node_updates() override
	{
		unsigned long long n = 0;
		FG_CUDA(cudaMemcpyAsync(&n, acc_, sizeof(n), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		return n;
	}
	const Dev& dev() const override { return P_; }
	const SurfGeom& geometry(int s) const override { return geom_[s]; }
	void sync() override { FG_CUDA(cudaStreamSynchronize(st_)); }
	int part(int a) const override { return csz_[a]; }

	/// Geometry of a grid of the given size (Surface ctor, Surface.hpp:163-173, and the
	/// children grid, PartitionedMixin.hpp:59-86, 131-141), its partitions from pbase.
	SurfGeom grid_geom(const int* size, int pbase) const
	{
		SurfGeom g;
		std::memset(&g, 0, sizeof(g));
		bool exact = true;
		long long np = 1;
		for (int a = 0; a < D; a++) {
			const int sz = size[a];
			if (sz <= 0) throw Error(-1, "grid size must be positive");
			g.size[a] = sz;
			g.off[a] = (-1 * sz) / 2;
			g.hi[a] = g.off[a] + sz;
			g.ccount[a] = sz / csz_[a];
			if (g.ccount[a] * csz_[a] != sz) exact = false;
			g.coff[a] = g.off[a] / csz_[a];
		}
		if (!exact)
			for (int a = 0; a < D; a++) g.ccount[a] += 1;
		for (int a = 0; a < D; a++) np *= g.ccount[a];
		if (np >= (1 << 24)) throw Error(-1, "too many partitions in one surface");
		g.pbase = pbase;
		g.np = (int)np;
		return g;
	}

	// ---- serving: reuse of a surface of the pool ----
	void reset_surface(int s, const int* size) override
	{
		check_surface(s);
		const SurfGeom ng = grid_geom(size, geom_[s].pbase);
		if (ng.np > np_cap_[s])
			throw Error(-1, "grid larger than the partition range of this surface");
		FG_RUN("k_reset_surface", st_, k_reset_surface<D, L><<<grid_for(np_cap_[s]), 256, 0, st_>>>(P_, s, ng, np_cap_[s]););
		FG_CUDA(cudaGetLastError());
		geom_[s] = ng;
		frozen_[s] = 0;
	}

	void seed_async(int s, const int* pos) override
	{
		check_surface(s);
		Vec<D> c;
		for (int a = 0; a < D; a++) c[a] = pos[a];
		FG_RUN("k_seed", st_, k_seed<D, L><<<1, 1, 0, st_>>>(P_, s, c););
		FG_CUDA(cudaGetLastError());
	}

	void set_paused_n(const int* surfaces, const int* on, int n) override
	{
		bool any = false;
		for (int i = 0; i < n; i++) {
			check_surface(surfaces[i]);
			const int v = on[i] ? 1 : 0;
			if (paused_[surfaces[i]] != v) {
				paused_[surfaces[i]] = v;
				any = true;
			}
		}
		if (any) push_stopped();
	}

	void surface_node_updates(unsigned long long* out) override
	{
		FG_CUDA(cudaMemcpyAsync(out, P_.snu, (size_t)P_.S * sizeof(unsigned long long),
		                        cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
	}

	long long free_bricks() override
	{
		int top = 0;
		FG_CUDA(cudaMemcpyAsync(&top, P_.counters + CNT_FREE_TOP, sizeof(int),
		                        cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		return top;
	}

	int partition_capacity(int s) const override
	{
		check_surface(s);
		return np_cap_[s];
	}

	// ---- seed ----
	void seed(int s, const int* pos) override
	{
		check_surface(s);
		Vec<D> c;
		for (int a = 0; a < D; a++) c[a] = pos[a];
		FG_RUN("k_seed", st_, k_seed<D, L><<<1, 1, 0, st_>>>(P_, s, c););
		FG_CUDA(cudaGetLastError());
		check_errors();
	}

	void seed_all(const int* centres) override
	{
		int* d = nullptr;
		FG_CUDA(locked_malloc(&d, (size_t)P_.S * D * sizeof(int)));
		cudaError_t e = cudaMemcpyAsync(d, centres, (size_t)P_.S * D * sizeof(int),
		                                cudaMemcpyHostToDevice, st_);
		if (e == cudaSuccess) {
			FG_RUN("k_seed_all", st_, k_seed_all<D, L><<<(P_.S + 63) / 64, 64, 0, st_>>>(P_, d););
			e = cudaStreamSynchronize(st_);
		}
		locked_free(d);
		if (e != cudaSuccess) throw Error(-2, cudaGetErrorString(e));
		check_errors();
	}

	// ---- global update ----
	void update_builtin(const Speed* speeds) override
	{
		check_not_frozen();
		// through pinned staging: the copy is a plain DMA, no driver bounce buffer (the previous
		// update synchronised, so the staging is free)
		std::memcpy(h_speeds_, speeds, P_.S * sizeof(Speed));
		FG_CUDA(cudaMemcpyAsync(d_speeds_, h_speeds_, P_.S * sizeof(Speed), cudaMemcpyHostToDevice,
		                        st_));
		bool any_curv = false;
		for (int s = 0; s < P_.S; s++) any_curv = any_curv || (speeds[s].kind & 2);
		// staging a brick with its halo pays only for the curvature stencil
		const bool staged = any_curv && smem_halo_ && delta_staged_;
		if (run_step_graph(staged)) return;
		update_begin_global();
		delta_builtin(staged);
		first_passes(true);
		converge();
	}

	void update_begin_global() override
	{
		check_not_frozen();
		update_start();
		// delta.track_children(isogrid) on freshly reset delta lists = a copy of the lists.
		copy_plists();
		count_band();
		// entry offsets over the zero-layer partitions, for the delta kernel that follows
		scan(P_.pcnt, L, 0);
	}

	void update_finish_global() override
	{
		first_passes(false);
		converge();
	}

private:
	/// The builtin speed functor over the zero layer (Surface.hpp:263-294): staged, over
	/// bricks staged with their halo in shared memory (one block each), else warps reading the
	/// pool directly.
	void delta_builtin(bool staged)
	{
		if (staged)
			FG_RUN("k_delta_smem", st_, launch_pdl((k_delta_smem<D, L>), sm_count() * 8, 128, smem_halo_, st_, P_, d_speeds_););
		else
			FG_RUN("k_delta_builtin", st_, launch_pdl((k_delta_builtin<D, L>), warp_grid_, 256, 0, st_, P_, d_speeds_, dist_split_););
	}

	/// update_end_global up to the convergence loop (Surface.hpp:739-751):
	/// update_zero_layer(&affected_buffer), the first distance passes recording into buffer B.
	/// woff_ready: the zero layer's entry offsets are still those update_begin_global scanned
	/// (a builtin speed changes no list in between).
	void first_passes(bool woff_ready)
	{
		const int B = 1;  // buffers: B = m_grid_affected_buffer, A = m_grid_affected
		if (!woff_ready) scan(P_.pcnt, L, 0);
		const ListView iso{P_.plist, P_.pcnt, P_.lst, P_.lcnt, P_.lkp, P_.ppos};
		zero_apply(iso, nullptr, B);
		defer_compact(P_.woff, P_.plist, L, B);
		distance_passes(iso, B);  // k_entry_table clears Dev::changed
	}

	/// The whole global update with a builtin speed as ONE CUDA graph: update_start's due
	/// resets, the delta track_children copy, the band count, the speed functor, the zero-layer
	/// update and first distance passes, flush, expansion and retirement, then the convergence
	/// loop's while node (the body of run_device_loop's graph). One graph per combination of
	/// due resets and delta kernel, captured on first use; a step is then one graph launch and
	/// one read-back of the loop's count. Returns false (the caller launches phase by phase)
	/// under launch mode 2, while per-launch profiling is on, or where the graph cannot be
	/// built.
	bool run_step_graph(bool staged)
	{
		if (launch_mode_ == 2 || !loop_ok_ || !graphs_ok_ || !step_ok_ || prof_on()) return false;
		const int key = (status_dirty_ ? 1 : 0) | (buf_dirty_[0] ? 2 : 0) |
		                (buf_dirty_[1] ? 4 : 0) | (staged ? 8 : 0);
		if (!step_exec_[key] && !build_step_graph(key, staged)) return false;
		// the update leaves one buffer or the other to reset, by the parity of its iterations:
		// the graph of the other parity is built now too, so that no later update of the same
		// kind captures one in the middle of a timed run
		const int sib = (key & ~6) | ((key & 2) << 1) | ((key & 4) >> 1);
		if (sib != key && !step_exec_[sib]) {
			const bool sd = status_dirty_, b0 = buf_dirty_[0], b1 = buf_dirty_[1];
			status_dirty_ = (sib & 1) != 0;
			buf_dirty_[0] = (sib & 2) != 0;
			buf_dirty_[1] = (sib & 4) != 0;
			build_step_graph(sib, staged);
			status_dirty_ = sd;
			buf_dirty_[0] = b0;
			buf_dirty_[1] = b1;
		}
		FG_CUDA(cudaGraphLaunch(step_exec_[key], st_));
		int* out = h_out_;  // pinned
		FG_CUDA(cudaMemcpyAsync(&out[0], d_iters_, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaMemcpyAsync(&out[1], P_.changed, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		const int iters = out[0], changed = out[1];
		const int n = iters - 1;
		add_launches(step_launches_[key] + (long long)(n / 2) * (loop_launches_[0] + loop_launches_[1]) +
		             (n % 2) * loop_launches_[0]);
		// what update_start left
		status_dirty_ = false;
		buf_dirty_[0] = buf_dirty_[1] = false;
		converge_after(false, true, changed, iters);
		return true;
	}

	bool build_step_graph(int key, bool staged)
	{
		std::lock_guard<std::recursive_mutex> lock(device_lock());
		cudaGraph_t g = nullptr;
		bool ok = false;
		const long long l0 = launch_count();
		// capturing runs the host side of update_start and the passes, which marks the grids
		// it clears as clean and leaves a compaction pending; nothing captured has run yet
		const bool sd = status_dirty_, bd0 = buf_dirty_[0], bd1 = buf_dirty_[1];
		long long prefix = 0;
		try {
			ok = build_loop_into(g, prefix, [&] {
				update_start();
				copy_plists();
				count_band();
				scan(P_.pcnt, L, 0);
				delta_builtin(staged);
				first_passes(true);
				flush();
				expand();
				retire();
			});
		} catch (...) {
			ok = false;
		}
		cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
		if (cudaStreamIsCapturing(st_, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
			cudaGraph_t dropped = nullptr;
			cudaStreamEndCapture(st_, &dropped);
			if (dropped) cudaGraphDestroy(dropped);
			ok = false;
		}
		add_launches(-(launch_count() - l0));  // counted when they run
		if (ok && cudaGraphInstantiate(&step_exec_[key], g, 0) != cudaSuccess) {
			step_exec_[key] = nullptr;
			ok = false;
		}
		if (g) cudaGraphDestroy(g);
		cudaGetLastError();
		pending_ = CompactArgs{0, nullptr, nullptr, 0, 0};
		status_dirty_ = sd;
		buf_dirty_[0] = bd0;
		buf_dirty_[1] = bd1;
		if (!ok) step_ok_ = false;
		step_launches_[key] = prefix;
		return ok;
	}

	/// Graphs captured with the current launch parameters.
	void drop_graphs()
	{
		cudaStreamSynchronize(st_);
		for (cudaGraphExec_t& ex : iter_exec_)
			if (ex) cudaGraphExecDestroy(ex), ex = nullptr;
		for (cudaGraphExec_t& ex : step_exec_)
			if (ex) cudaGraphExecDestroy(ex), ex = nullptr;
		if (loop_exec_) cudaGraphExecDestroy(loop_exec_), loop_exec_ = nullptr;
	}

	/// The rest of update_end_global / update_end after the first distance passes, which
	/// recorded their changes in buffer B: flush and expand, then repeat the distance passes on
	/// the changed nodes until no layer changes (Surface.hpp:744-761, 417-428).
	/// The global update resets the consumed buffer at the end of each iteration, the local one
	/// at the start of the next (Surface.hpp:752-760 vs 420-428); the difference shows in the
	/// affected() lookup a local update leaves behind.
	void converge(bool local = false)
	{
		flush();
		expand();
		retire();
		int changed = 0;
		int iters = 1;
		const bool dev = !local && run_device_loop(changed, iters);
		if (!dev) changed = read_changed();
		converge_after(local, dev, changed, iters);
	}

	/// converge() after the first flush and expansion, and after the device-side loop when it
	/// ran (dev): the host-side record of the buffers it left, the surfaces to stop when it
	/// stopped at a multiple of kMaxIterations, and the host loop for what is left.
	void converge_after(bool local, bool dev, int changed, int iters)
	{
		const int B = 1, A = 0;
		status_dirty_ = true;
		buf_dirty_[B] = true;
		int cur = B, oth = A;
		if (dev) {
			// iterations alternate the buffers; each global one clears the buffer it consumed
			if ((iters - 1) % 2) std::swap(cur, oth);
			if (iters > 1) {
				buf_dirty_[cur] = true;
				buf_dirty_[oth] = false;
			}
			if (changed) freeze_oscillating(cur);  // stopped at a multiple of kMaxIterations
		}
		while (changed) {
			if (local && buf_dirty_[oth]) clear_buffer(oth);
			if (local || !replay_iteration(cur, oth)) iteration(local, cur, oth);
			status_dirty_ = true;
			buf_dirty_[oth] = true;
			if (!local) buf_dirty_[cur] = false;
			std::swap(cur, oth);
			changed = read_changed();
			iters++;
			if (changed && iters % kMaxIterations == 0) freeze_oscillating(cur);
		}
		stats_.iterations = iters;
		check_errors();
		if (!newly_frozen_.empty() && throw_on_freeze_) {
			newly_frozen_.clear();
			throw Error(-14, "the convergence loop of the update did not terminate (layer "
			                 "changes keep oscillating, typically where the band meets the grid "
			                 "edge); the surface is stopped");
		}
		newly_frozen_.clear();
	}

	/// One iteration of the convergence loop after the first: the distance passes over the
	/// nodes that changed in the previous one (buffer cur), recording into buffer oth, then
	/// flush, expansion and, in the global update, the reset of buffer cur.
	void iteration(bool local, int cur, int oth)
	{
		// the fused passes (lookup given) on the global update's iterations only
		const ListView bv{P_.aplist[cur], P_.apcnt[cur], P_.alst[cur], P_.acnt[cur],
		                  local ? nullptr : P_.alkp[cur], P_.appos[cur]};
		distance_passes(bv, oth, true);  // with the status reset (clear_status)
		flush();
		expand();
		if (local)
			retire();
		else
			clear_buffer(cur, true);  // with the brick retirement (retire)
	}

	/// The global update's iteration as a CUDA graph, captured on first use (one per buffer
	/// parity) and replayed: one launch instead of ~30, all of whose launch parameters are
	/// fixed. Returns false (and the caller launches the kernels one by one) while per-launch
	/// profiling is on or if capture is not possible.
	bool replay_iteration(int cur, int oth)
	{
		if (launch_mode_ == 2 || !graphs_ok_ || prof_on()) return false;
		cudaGraphExec_t& ex = iter_exec_[cur];
		if (!ex) {
			cudaGraph_t gph = nullptr;
			std::lock_guard<std::recursive_mutex> lock(device_lock());
			if (cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
				cudaGetLastError();
				graphs_ok_ = false;
				return false;
			}
			const long long l0 = launch_count();
			bool threw = false;
			try {
				iteration(false, cur, oth);
			} catch (...) {
				threw = true;
			}
			const cudaError_t e = cudaStreamEndCapture(st_, &gph);
			const long long captured = launch_count() - l0;
			add_launches(-captured);  // counted when they run
			if (threw || e != cudaSuccess || !gph ||
			    cudaGraphInstantiate(&ex, gph, 0) != cudaSuccess) {
				if (gph) cudaGraphDestroy(gph);
				ex = nullptr;
				cudaGetLastError();
				// nothing captured has run: the caller launches the iteration's kernels one by
				// one, and a real fault shows there
				graphs_ok_ = false;
				return false;
			}
			cudaGraphDestroy(gph);
			iter_launches_[cur] = captured;
		}
		FG_CUDA(cudaGraphLaunch(ex, st_));
		add_launches(iter_launches_[cur]);
		return true;
	}

	/// The global update's convergence loop on the device: one graph whose while node runs two
	/// iterations per pass (buffer B then A, the second under an if node), each followed by a
	/// test kernel that counts it and sets the conditions. Replaces a host read-back per
	/// iteration with one per update. Returns false (the host loop runs instead) while
	/// per-launch profiling is on or where the graph cannot be built; otherwise sets changed
	/// and iters as the host loop leaves them when it stops at a multiple of kMaxIterations or
	/// runs out of changes.
	bool run_device_loop(int& changed, int& iters)
	{
		if (launch_mode_ == 2 || !loop_ok_ || !graphs_ok_ || prof_on()) return false;
		if (!loop_exec_ && !build_device_loop()) return false;
		FG_CUDA(cudaGraphLaunch(loop_exec_, st_));
		int* out = h_out_;  // pinned
		FG_CUDA(cudaMemcpyAsync(&out[0], d_iters_, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaMemcpyAsync(&out[1], P_.changed, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		iters = out[0];
		changed = out[1];
		const int n = iters - 1;  // iterations run: n / 2 full passes, one more if n is odd
		add_launches(1 + (long long)(n / 2) * (loop_launches_[0] + loop_launches_[1]) +
		             (n % 2) * loop_launches_[0]);
		return true;
	}

	bool build_device_loop()
	{
		std::lock_guard<std::recursive_mutex> lock(device_lock());
		cudaGraph_t g = nullptr;
		bool ok = false;
		const long long l0 = launch_count();
		// capturing the iterations runs their host side, which marks the grids it clears as
		// clean; nothing captured has run yet
		const bool sd = status_dirty_, bd0 = buf_dirty_[0], bd1 = buf_dirty_[1];
		long long prefix = 0;
		try {
			ok = build_loop_into(g, prefix, [] {});
		} catch (...) {
			ok = false;
		}
		cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
		if (cudaStreamIsCapturing(st_, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
			cudaGraph_t dropped = nullptr;
			cudaStreamEndCapture(st_, &dropped);
			ok = false;
		}
		add_launches(-(launch_count() - l0));  // counted when they run
		if (ok && cudaGraphInstantiate(&loop_exec_, g, 0) != cudaSuccess) {
			loop_exec_ = nullptr;
			ok = false;
		}
		if (g) cudaGraphDestroy(g);
		cudaGetLastError();
		if (!ok) loop_ok_ = false;
		status_dirty_ = sd;
		buf_dirty_[0] = bd0;
		buf_dirty_[1] = bd1;
		return ok;
	}

	/// Adds the node of a conditional of the given kind after the last node captured on the
	/// stream, ends the capture and returns the conditional's body graph.
	cudaGraph_t end_capture_with_conditional(cudaGraphConditionalHandle h, cudaGraphConditionalNodeType kind)
	{
		cudaStreamCaptureStatus cs;
		cudaGraph_t cg = nullptr;
		const cudaGraphNode_t* deps = nullptr;
		size_t nd = 0;
		FG_CUDA(cudaStreamGetCaptureInfo(st_, &cs, nullptr, &cg, &deps, &nd));
		std::vector<cudaGraphNode_t> last(deps, deps + nd);
		cudaGraph_t done = nullptr;
		FG_CUDA(cudaStreamEndCapture(st_, &done));
		cudaGraphNodeParams p = {};
		p.type = cudaGraphNodeTypeConditional;
		p.conditional.handle = h;
		p.conditional.type = kind;
		p.conditional.size = 1;
		cudaGraphNode_t node;
		FG_CUDA(cudaGraphAddNode(&node, done, last.data(), last.size(), &p));
		return p.conditional.phGraph_out[0];
	}

	/// Captures into g what `prefix` launches, then the convergence loop (k_loop_init and the
	/// while node); `launches` = the kernels before the while node.
	template <class Prefix>
	bool build_loop_into(cudaGraph_t& g, long long& launches, Prefix&& prefix)
	{
		const int B = 1, A = 0;
		const auto mode = cudaStreamCaptureModeThreadLocal;
		FG_CUDA(cudaGraphCreate(&g, 0));
		cudaGraphConditionalHandle hloop, hsecond;
		FG_CUDA(cudaGraphConditionalHandleCreate(&hloop, g, 0, cudaGraphCondAssignDefault));
		FG_CUDA(cudaStreamBeginCaptureToGraph(st_, g, nullptr, nullptr, 0, mode));
		const long long p0 = launch_count();
		prefix();
		FG_RUN("k_loop_init", st_, launch_pdl((k_loop_init), 1, 32, 0, st_, P_.changed, d_iters_, hloop););
		launches = launch_count() - p0;
		const cudaGraph_t body = end_capture_with_conditional(hloop, cudaGraphCondTypeWhile);
		FG_CUDA(cudaGraphConditionalHandleCreate(&hsecond, body, 0, cudaGraphCondAssignDefault));
		// first iteration of a pass: buffer B consumed, A recorded
		FG_CUDA(cudaStreamBeginCaptureToGraph(st_, body, nullptr, nullptr, 0, mode));
		long long l0 = launch_count();
		iteration(false, B, A);
		FG_RUN("k_loop_test", st_, launch_pdl((k_loop_test), 1, 32, 0, st_, P_.changed, d_iters_, kMaxIterations, hsecond, hloop, 1););
		loop_launches_[0] = launch_count() - l0;
		const cudaGraph_t second = end_capture_with_conditional(hsecond, cudaGraphCondTypeIf);
		// second iteration: A consumed, B recorded
		FG_CUDA(cudaStreamBeginCaptureToGraph(st_, second, nullptr, nullptr, 0, mode));
		l0 = launch_count();
		iteration(false, A, B);
		FG_RUN("k_loop_test", st_, launch_pdl((k_loop_test), 1, 32, 0, st_, P_.changed, d_iters_, kMaxIterations, hloop, hloop, 0););
		loop_launches_[1] = launch_count() - l0;
		cudaGraph_t done = nullptr;
		FG_CUDA(cudaStreamEndCapture(st_, &done));
		return true;
	}

	/// The reference loops `while (is_status_changed)` with no bound (Surface.hpp:752-760,
	/// 420-428); where the band reaches the grid edge its layer changes can oscillate forever.
	/// After kMaxIterations iterations the surfaces still changing are frozen: no kernel works
	/// on them again, so the loop ends for the rest of the pool.
	void freeze_oscillating(int cur)
	{
		std::vector<int> cnt((size_t)P_.S * NL);
		FG_CUDA(cudaMemcpyAsync(cnt.data(), P_.apcnt[cur], cnt.size() * sizeof(int),
		                        cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		for (int s = 0; s < P_.S; s++) {
			int tot = 0;
			for (int l = 0; l < NL; l++) tot += cnt[(size_t)s * NL + l];
			if (tot && !frozen_[s]) {
				frozen_[s] = 1;
				newly_frozen_.push_back(s);
			}
		}
		push_stopped();
	}

	/// Device copy of the per-surface skip flags: stopped (frozen) or paused.
	void push_stopped()
	{
		stopped_.resize(frozen_.size());
		for (size_t s = 0; s < frozen_.size(); s++) stopped_[s] = frozen_[s] | paused_[s];
		FG_CUDA(cudaMemcpyAsync(P_.sfrozen, stopped_.data(), stopped_.size() * sizeof(int),
		                        cudaMemcpyHostToDevice, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
	}

public:
	bool frozen(int s) const override { return frozen_[s] != 0; }
	void set_throw_on_freeze(bool on) override { throw_on_freeze_ = on; }
	void set_paused(int s, bool on) override
	{
		check_surface(s);
		if ((paused_[s] != 0) == on) return;
		paused_[s] = on ? 1 : 0;
		push_stopped();
	}
	bool paused(int s) const override { return paused_[s] != 0; }

private:
	void check_not_frozen()
	{
		for (int s = 0; s < P_.S; s++)
			if (!frozen_[s]) return;
		throw Error(-15, "every surface of the pool is stopped after a non-terminating update");
	}

public:

	/// update_start(); delta(pos, v)...; update_end() on surface 0 (Surface.hpp:393-459,
	/// 404-430).
	void update_local(const std::vector<int>& pos, const std::vector<float>& vals) override
	{
		const int n = (int)vals.size();
		if (pos.size() != vals.size() * D) throw Error(-1, "delta positions/values mismatch");
		check_not_frozen();
		update_start();
		ensure_local_staging(n);
		if (n) {
			FG_CUDA(cudaMemcpyAsync(d_lpos_, pos.data(), pos.size() * sizeof(int),
			                        cudaMemcpyHostToDevice, st_));
			FG_CUDA(cudaMemcpyAsync(d_lval_, vals.data(), n * sizeof(float),
			                        cudaMemcpyHostToDevice, st_));
		}
		local_seed(n);
		local_end();
	}

	/// update(lo, hi, fn) with a builtin speed on surface 0 (Surface.hpp:310-386): the speed at
	/// the zero-layer leaves inside the box becomes the deltas of a local update.
	void update_bounded(const int* lo, const int* hi, const Speed& sp) override
	{
		Vec<D> vlo, vhi;
		for (int a = 0; a < D; a++) {
			vlo[a] = lo[a];
			vhi[a] = hi[a];
		}
		check_not_frozen();
		// capacity: every zero-layer leaf of the surface
		FG_CUDA(cudaMemsetAsync(zcount_, 0, sizeof(unsigned long long), st_));
		FG_RUN("k_count_layer", st_, launch_pdl((k_count_layer<L>), sm_count() * 2, 256, 0, st_, P_, 0, L, zcount_););
		unsigned long long nz = 0;
		FG_CUDA(cudaMemcpyAsync(&nz, zcount_, sizeof(nz), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		ensure_local_staging((int)nz + 1);
		update_start();
		// the partitions covering the box: pos_child (truncating division) of the grid's and
		// the box's corners, zero-based (Surface.hpp:313-330)
		const SurfGeom& g = geom_[0];
		BoxParts<D> b;
		long long nb = 1;
		for (int a = 0; a < D; a++) {
			const int grid_hi = (g.hi[a] - 1 - g.off[a]) / csz_[a];
			b.cl[a] = std::max(0, (vlo[a] - g.off[a]) / csz_[a]);
			const int cu = std::min(grid_hi, (vhi[a] - g.off[a]) / csz_[a]);
			b.box[a] = cu - b.cl[a] + 1;
			b.lo[a] = vlo[a];
			b.lub[a] = std::min(g.hi[a], vhi[a] + 1);
			nb *= b.box[a] > 0 ? b.box[a] : 0;
		}
		b.nb = (int)nb;
		int* counts = P_.ring_src;  // idle until calc_affected's rings
		int* offsets = P_.ring_first;
		FG_RUN("k_bounded_count", st_, launch_pdl((k_bounded_count<D, L>), warp_grid_, 256, 0, st_, P_, 0, b, counts););
		FG_RUN("k_scan_offsets", st_, launch_pdl((k_scan_offsets), 1, 1024, 0, st_, counts, b.nb, offsets, d_lcount_););
		FG_RUN("k_bounded_write", st_, launch_pdl((k_bounded_write<D, L>), warp_grid_, 256, 0, st_, P_, 0, b, offsets, d_lpos_, lcap_););
		FG_RUN("k_bounded_speed", st_, launch_pdl((k_bounded_speed<D, L>), grid_for(nz + 1), 256, 0, st_, P_, 0, sp, d_lpos_, d_lcount_, d_lval_););
		int n = 0;
		FG_CUDA(cudaMemcpyAsync(&n, d_lcount_, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		local_seed(n);
		local_end();
	}

	/// The n staged delta calls of a local update on surface 0 (Surface.hpp:441-459) and the
	/// first step of calc_affected (788-799), in parallel (fg_kernels.cuh).
	void local_seed(int n)
	{
		constexpr int RING_CAP = 2048;
		const int gb = grid_for(n);
		FG_RUN("k_seed_claim", st_, launch_pdl((k_seed_claim<D, L>), gb, 256, 0, st_, P_, 0, d_lpos_, n););
		FG_RUN("k_ring_append", st_, launch_pdl((k_ring_append<L>), sm_count() * 4, 256, RING_CAP * 11, st_, P_, RING_CAP, L););
		FG_RUN("k_ring_plist", st_, launch_pdl((k_ring_plist<L>), sm_count() * 2, 256, 0, st_, P_, 0););
		FG_RUN("k_ring_finish", st_, launch_pdl((k_ring_finish<L>), 1, 256, 0, st_, P_, 0););
		for (int phase = 0; phase < 4; phase++)
			FG_RUN("k_seed_values", st_, launch_pdl((k_seed_values<D, L>), gb, 256, 0, st_, P_, 0, d_lpos_, d_lval_, n, phase););
		FG_RUN("k_seed_finish", st_, launch_pdl((k_seed_finish<L>), sm_count(), 256, 0, st_, P_, 0););
	}

	/// calc_affected's L rings (Surface.hpp:801-912) on surface 0, each a set of parallel
	/// kernels that append in the reference's sequential order (fg_kernels.cuh).
	void calc_affected()
	{
		constexpr int RING_CAP = 2048;  // claimed leaves a brick ranks in shared memory
		const int np = geom_[0].np;
		FG_CUDA(cudaMemsetAsync(P_.ring_n, 0, 2 * NL * sizeof(int), st_));
		for (int ring = 1; ring <= L; ring++) {
			const int cur = (ring - 1) & 1;
			FG_RUN("k_ring_setup", st_, launch_pdl((k_ring_setup<L>), grid_for((long long)NL * np), 256, 0, st_, P_, 0, np, cur););
			FG_RUN("k_ring_claim", st_, launch_pdl((k_ring_claim<D, L>), warp_grid_, 256, 0, st_, P_, 0););
			FG_RUN("k_ring_append", st_, launch_pdl((k_ring_append<L>), sm_count() * 4, 256, RING_CAP * 11, st_, P_, RING_CAP, -1););
			FG_RUN("k_ring_plist", st_, launch_pdl((k_ring_plist<L>), sm_count() * 2, 256, 0, st_, P_, 0););
			FG_RUN("k_ring_finish", st_, launch_pdl((k_ring_finish<L>), 1, 256, 0, st_, P_, 0););
		}
	}

	/// update_end after the deltas are tracked (Surface.hpp:404-430).
	void local_end()
	{
		const int A = 0, B = 1;
		buf_dirty_[A] = true;
		calc_affected();
		FG_RUN("k_local_children", st_, launch_pdl((k_local_children<L>), NL, 1024, 0, st_, P_, 0););
		count_band();
		// update_zero_layer(&affected_buffer) over the delta leaves, then the distance passes
		// over the affected lists (update_distance(plookup = affected, buffer))
		FG_RUN("k_scan_counts", st_, launch_pdl((k_scan_counts), 1, 1024, 0, st_, P_.ndp, 1, 0, 0, P_.S, P_.woff, P_.sfrozen););
		const ListView aff{P_.aplist[A], P_.apcnt[A], P_.alst[A], P_.acnt[A]};
		zero_apply(aff, P_.dlcnt, B);
		defer_compact(P_.woff, P_.aplist[A], L, B);
		distance_passes(aff, B);  // k_entry_table clears Dev::changed
		converge(true);
	}

	void ensure_local_staging(int n)
	{
		if (n <= lcap_ && d_lpos_) return;
		int cap = std::max(n, 1024);
		cudaStreamSynchronize(st_);
		if (d_lpos_) locked_free(d_lpos_);
		if (d_lval_) locked_free(d_lval_);
		d_lpos_ = nullptr;
		d_lval_ = nullptr;
		FG_CUDA(locked_malloc(&d_lpos_, (size_t)cap * D * sizeof(int)));
		FG_CUDA(locked_malloc(&d_lval_, (size_t)cap * sizeof(float)));
		if (!d_lcount_) FG_CUDA(locked_malloc(&d_lcount_, sizeof(int)));
		lcap_ = cap;
	}

	// ---- queries ----
	void snapshot(int s, float* dst, size_t n, bool dst_device) override
	{
		check_surface(s);
		long long tot = 1;
		for (int a = 0; a < D; a++) tot *= geom_[s].size[a];
		if ((long long)n < tot) throw Error(-13, "snapshot buffer too small");
		float* out = dst;
		float* tmp = nullptr;
		if (!dst_device) {
			FG_CUDA(locked_malloc(&tmp, tot * sizeof(float)));
			out = tmp;
		}
		FG_RUN("k_snapshot", st_, k_snapshot<D, L><<<grid_for(tot), 256, 0, st_>>>(P_, s, out, tot););
		cudaError_t e = cudaGetLastError();
		if (e == cudaSuccess && tmp)
			e = cudaMemcpyAsync(dst, tmp, tot * sizeof(float), cudaMemcpyDeviceToHost, st_);
		if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
		if (tmp) locked_free(tmp);
		if (e != cudaSuccess) throw Error(-2, cudaGetErrorString(e));
	}

	float get(int s, const int* pos) override
	{
		check_surface(s);
		const SurfGeom& g = geom_[s];
		for (int a = 0; a < D; a++)
			if (pos[a] < g.off[a] || pos[a] >= g.hi[a]) return (float)(L + 1);
		int idx = 0, leaf = 0;
		for (int a = 0; a < D; a++) {
			const int r = pos[a] - g.off[a];
			const int c = r / csz_[a];
			idx = idx * g.ccount[a] + c;
			leaf += (r - c * csz_[a]) * P_.lstr[a];
		}
		const int gp = g.pbase + idx;
		int sl;
		float v;
		FG_CUDA(cudaMemcpyAsync(&sl, P_.slot + gp, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		if (sl < 0)
			FG_CUDA(cudaMemcpy(&v, P_.bg + gp, sizeof(float), cudaMemcpyDeviceToHost));
		else
			FG_CUDA(cudaMemcpy(&v, P_.phi + (size_t)sl * P_.BV + leaf, sizeof(float),
			                   cudaMemcpyDeviceToHost));
		return v;
	}

	size_t partitions(int s, int* ccount, int* coff) override
	{
		check_surface(s);
		for (int a = 0; a < D; a++) {
			ccount[a] = geom_[s].ccount[a];
			coff[a] = geom_[s].coff[a];
		}
		return (size_t)geom_[s].np;
	}

	std::vector<uint32_t> layer_list(int s, size_t part, int li) override
	{
		check_surface(s);
		check_layer(li);
		if (part >= (size_t)geom_[s].np) throw Error(-1, "partition index out of range");
		sync();
		const int gp = geom_[s].pbase + (int)part;
		int sl;
		FG_CUDA(cudaMemcpy(&sl, P_.slot + gp, sizeof(int), cudaMemcpyDeviceToHost));
		if (sl < 0) return {};
		int n;
		FG_CUDA(cudaMemcpy(&n, P_.lcnt + (size_t)sl * NL + li, sizeof(int), cudaMemcpyDeviceToHost));
		std::vector<uint16_t> tmp(n);
		if (n)
			FG_CUDA(cudaMemcpy(tmp.data(), P_.lst + ((size_t)sl * NL + li) * P_.BV,
			                   n * sizeof(uint16_t), cudaMemcpyDeviceToHost));
		return std::vector<uint32_t>(tmp.begin(), tmp.end());
	}

	std::vector<uint32_t> partition_list(int s, int which, int li) override
	{
		check_surface(s);
		check_layer(li);
		sync();
		const int* list;
		const int* cnt;
		switch (which) {
		case 0: list = P_.plist; cnt = P_.pcnt; break;
		case 1: list = P_.dplist; cnt = P_.dpcnt; break;
		case 2: list = P_.splist; cnt = P_.spcnt; break;
		case 3: list = P_.aplist[0]; cnt = P_.apcnt[0]; break;
		default: throw Error(-1, "unknown partition list");
		}
		int n;
		FG_CUDA(cudaMemcpy(&n, cnt + s * NL + li, sizeof(int), cudaMemcpyDeviceToHost));
		std::vector<int> tmp(n);
		if (n)
			FG_CUDA(cudaMemcpy(tmp.data(), list + (size_t)li * P_.NP + geom_[s].pbase,
			                   n * sizeof(int), cudaMemcpyDeviceToHost));
		return std::vector<uint32_t>(tmp.begin(), tmp.end());
	}

	std::vector<uint32_t> affected_list(int s, size_t part, int li) override
	{
		check_surface(s);
		check_layer(li);
		if (part >= (size_t)geom_[s].np) throw Error(-1, "partition index out of range");
		sync();
		const int gp = geom_[s].pbase + (int)part;
		int sl, ap;
		FG_CUDA(cudaMemcpy(&ap, P_.appos[0] + (size_t)gp * NL + li, sizeof(int),
		                   cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(&sl, P_.slot + gp, sizeof(int), cudaMemcpyDeviceToHost));
		if (ap < 0 || sl < 0) return {};
		int n;
		FG_CUDA(cudaMemcpy(&n, P_.acnt[0] + (size_t)sl * NL + li, sizeof(int),
		                   cudaMemcpyDeviceToHost));
		std::vector<uint16_t> tmp(n);
		if (n)
			FG_CUDA(cudaMemcpy(tmp.data(), P_.alst[0] + ((size_t)sl * NL + li) * P_.BV,
			                   n * sizeof(uint16_t), cudaMemcpyDeviceToHost));
		return std::vector<uint32_t>(tmp.begin(), tmp.end());
	}

	void partition_state(int s, size_t part, int* active, float* bg) override
	{
		check_surface(s);
		if (part >= (size_t)geom_[s].np) throw Error(-1, "partition index out of range");
		sync();
		const int gp = geom_[s].pbase + (int)part;
		int sl;
		FG_CUDA(cudaMemcpy(&sl, P_.slot + gp, sizeof(int), cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(bg, P_.bg + gp, sizeof(float), cudaMemcpyDeviceToHost));
		*active = sl >= 0 ? 1 : 0;
	}

	std::vector<uint32_t> dump(int s) override
	{
		check_surface(s);
		sync();
		const SurfGeom& g = geom_[s];
		std::vector<int> slots(g.np);
		std::vector<float> bgs(g.np);
		FG_CUDA(cudaMemcpy(slots.data(), P_.slot + g.pbase, g.np * sizeof(int),
		                   cudaMemcpyDeviceToHost));
		FG_CUDA(cudaMemcpy(bgs.data(), P_.bg + g.pbase, g.np * sizeof(float),
		                   cudaMemcpyDeviceToHost));
		std::vector<int> lcnt((size_t)P_.nslots * NL);
		FG_CUDA(cudaMemcpy(lcnt.data(), P_.lcnt, lcnt.size() * sizeof(int),
		                   cudaMemcpyDeviceToHost));
		std::vector<uint32_t> out;
		out.push_back(D);
		out.push_back(L);
		out.push_back((uint32_t)g.np);
		std::vector<uint16_t> tmp;
		for (int i = 0; i < g.np; i++) {
			const int sl = slots[i];
			uint32_t bits;
			std::memcpy(&bits, &bgs[i], 4);
			out.push_back(sl >= 0 ? 1u : 0u);
			out.push_back(bits);
			for (int l = 0; l < NL; l++) {
				const int n = sl >= 0 ? lcnt[(size_t)sl * NL + l] : 0;
				out.push_back((uint32_t)n);
				if (n) {
					tmp.resize(n);
					FG_CUDA(cudaMemcpy(tmp.data(), P_.lst + ((size_t)sl * NL + l) * P_.BV,
					                   n * sizeof(uint16_t), cudaMemcpyDeviceToHost));
					for (uint16_t x : tmp) out.push_back(x);
				}
			}
		}
		for (int which = 0; which < 3; which++)
			for (int l = 0; l < NL; l++) {
				const std::vector<uint32_t> pl = partition_list(s, which, l);
				out.push_back((uint32_t)pl.size());
				out.insert(out.end(), pl.begin(), pl.end());
			}
		return out;
	}

	unsigned long long band_size(int s) override
	{
		check_surface(s);
		FG_CUDA(cudaMemsetAsync(zcount_, 0, sizeof(unsigned long long), st_));
		for (int l = 0; l < NL; l++)
			FG_RUN("k_count_layer", st_, launch_pdl((k_count_layer<L>), sm_count() * 2, 256, 0, st_, P_, s, l, zcount_););
		unsigned long long n = 0;
		FG_CUDA(cudaMemcpyAsync(&n, zcount_, sizeof(n), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		return n;
	}

	void check_errors() override
	{
		int e = 0;
		FG_CUDA(cudaMemcpyAsync(&e, P_.err, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		FG_CUDA(cudaGetLastError());
		if (e) {
			FG_CUDA(cudaMemsetAsync(P_.err, 0, sizeof(int), st_));
			if (e & EB_POOL) throw Error(-4, "brick pool exhausted");
			if (e & EB_NONFINITE) throw Error(-10, "layer id of a non-finite distance");
			if (e & EB_OUTSIDE) throw Error(-11, "band node outside the grid");
			if (e & EB_INACTIVE) throw Error(-12, "write to an inactive partition");
			if (e & EB_CAPACITY) throw Error(-13, "device buffer capacity exceeded");
			if (e & EB_TIMEOUT) throw Error(-14, "bounded device wait gave up");
			throw Error(-2, "device error");
		}
	}

private:
	void check_surface(int s) const
	{
		if (s < 0 || s >= P_.S) throw Error(-1, "surface index out of range");
	}
	static void check_layer(int li)
	{
		if (li < 0 || li >= NL) throw Error(-1, "layer index out of range");
	}
	static int grid_for(long long n)
	{
		long long b = (n + 255) / 256;
		if (b < 1) b = 1;
		const long long cap = (long long)sm_count() * 32;
		return (int)(b < cap ? b : cap);
	}
	void fill(int* p, size_t n, int v)
	{
		FG_RUN("k_fill_int", st_, k_fill_int<<<grid_for(n), 256, 0, st_>>>(p, (long long)n, v););
	}
	void fillf(float* p, size_t n, float v)
	{
		FG_RUN("k_fill_float", st_, k_fill_float<<<grid_for(n), 256, 0, st_>>>(p, (long long)n, v););
	}

	void scan(const int* cnt, int l, int mode)
	{
		FG_RUN("k_scan_counts", st_, launch_pdl((k_scan_counts), 1, 1024, 0, st_, cnt, NL, l, mode, P_.S, P_.woff, P_.sfrozen););
	}

	/// update_start (Surface.hpp:393-399): resets of the status and affected grids left by the
	/// previous update. The delta values need no reset: every read follows a write of the same
	/// step.
	void update_start()
	{
		if (status_dirty_) clear_status();
		for (int b = 0; b < 2; b++)
			if (buf_dirty_[b]) clear_buffer(b);
	}

	void copy_plists()
	{
		dim3 grid(1, std::min(P_.S * NL, sm_count() * 8));  // blocks loop over (surface, list)
		FG_RUN("k_copy_plists", st_, launch_pdl((k_copy_plists), grid, 256, 0, st_, P_, NL););
	}

	void count_band()
	{
		scan(P_.pcnt, 0, 2);
		FG_RUN("k_band_size", st_, launch_pdl((k_band_size<L>), warp_grid_, 256, 0, st_, P_, acc_););
	}

	/// The 2L layer passes of update_distance (Surface.hpp:989-1125). The pass lists do not
	/// change while the passes run (they append to the other buffer), so one launch scans the
	/// entry offsets of every layer up front.
	/// clear_status: the iteration's status reset runs in the entry-table launch (in place of
	/// k_clear_status).
	void distance_passes(const ListView& lv, int b, bool clear_status = false)
	{
		// entry offsets of every layer, then the entries decoded; one launch for pools of up to
		// kScanHereMax surfaces
		const bool here = P_.S <= kScanHereMax;
		if (!here)
			FG_RUN("k_scan_layers", st_, launch_pdl((k_scan_layers), 1, 1024, 0, st_, lv.pcnt, NL, P_.S, P_.woffl, P_.sfrozen););
		const bool tiled = tiled_ && lv.lkp && lv.ppos;
		const size_t sm = here ? (size_t)NL * (P_.S + 1) * sizeof(int) : 0;
		FG_RUN("k_entry_table", st_, launch_pdl((k_entry_table<L>), sm_count() * 4, 256, sm, st_, P_, lv.plist, lv.lcnt, here ? lv.pcnt : nullptr, lv.ppos, tiled ? P_.dq : nullptr, clear_status ? 1 : 0););
		if (clear_status) status_dirty_ = false;
		if (tiled) {
			tiled_passes(lv, b);
			return;
		}
		if (fused_ && lv.lkp) {
			fused_passes(lv, b);
			return;
		}
		for (int k = -1; k >= -L; k--) layer_pass(lv, k, -1.0f, b);
		for (int k = 1; k <= L; k++) layer_pass(lv, k, 1.0f, b);
		const CompactArgs ca = take_compact();
		if (ca.nblocks)
			FG_RUN("k_compact", st_, launch_pdl((k_compact<L>), ca.nblocks, 256, 0, st_, P_, ca, 1););
		else
			expand_prep();
	}

	/// What the last compaction's last block does before the expansion, for a pass sequence
	/// that left none (k_compact with expand_prep).
	void expand_prep()
	{
		scan(P_.spcnt, 0, 1);
		FG_CUDA(cudaMemsetAsync(P_.counters + CNT_ACT, 0, 2 * sizeof(int), st_));
		FG_CUDA(cudaMemsetAsync(P_.counters + CNT_CAND, 0, sizeof(int), st_));
	}

	/// The 2L layer passes as 2L+1 launches (k_dist_fused): launch j runs the second pass of
	/// layer j-1 and the first pass of layer j, with the compaction of layer j-2's records (or
	/// the zero-layer update's, pending from before the passes) in its first blocks. The
	/// passes' entry flags alternate between the two arrays by pass parity, so a compaction
	/// never reads flags the second pass beside it writes.
	void fused_passes(const ListView& lv, int b)
	{
		auto layer = [](int j) { return j < L ? -(j + 1) : j - L + 1; };
		auto woff_of = [&](int j) { return P_.woffl + (size_t)(layer(j) + L) * (P_.S + 1); };
		auto flags_of = [&](int j) { return (j & 1) ? P_.eflag : P_.eflag2; };
		CompactArgs ca = take_compact();  // the zero-layer update's, flags in Dev::eflag
		for (int j = 0; j <= 2 * L; j++) {
			const FusedPass p2 = j >= 1 ? FusedPass{woff_of(j - 1), layer(j - 1)} : FusedPass{nullptr, 0};
			const FusedPass p1 = j < 2 * L ? FusedPass{woff_of(j), layer(j)} : FusedPass{nullptr, 0};
			const float side = j < L ? -1.0f : 1.0f;
			unsigned* ef2 = j >= 1 ? flags_of(j - 1) : nullptr;
			const int grid = (p2.woff && p1.woff ? 2 : 1) * warp_grid_ + ca.nblocks;
			FG_RUN("k_dist_fused", st_, launch_pdl((k_dist_fused<D, L>), grid, 256, 0, st_, P_, lv, p2, p1, side, dist_split_, b, ef2, ca, block_passes_ ? 1 : 0););
			ca = j >= 1 ? CompactArgs{P_.S, woff_of(j - 1), lv.plist, layer(j - 1) + L, b, flags_of(j - 1)}
			            : CompactArgs{0, nullptr, nullptr, 0, 0};
		}
		// the last pass's records: compacted before the flush reads them
		FG_RUN("k_compact", st_, launch_pdl((k_compact<L>), ca.nblocks, 256, 0, st_, P_, ca, 1););
	}

	/// The 2L layer passes as two launches: k_dist_tiled runs every pass of a brick in shared
	/// memory (a block per brick of the passes' lists, queued by k_entry_table), then
	/// k_dist_tiled_end commits the results and compacts the records of the zero-layer update
	/// (pending from before the passes) and of the passes in pass order.
	void tiled_passes(const ListView& lv, int b)
	{
		const CompactArgs stale = take_compact();
		FG_RUN("k_dist_tiled", st_, launch_pdl((k_dist_tiled<D, L>), tiled_grid_, tiled_threads_, smem_tiled_, st_, P_, lv, b, tile_););
		FG_RUN("k_dist_tiled_end", st_, launch_pdl((k_dist_tiled_end<L>), P_.S + sm_count() * 4, 256, 0, st_, P_, lv, b, stale););
	}

	/// A pass's compaction waits to ride on the next first-pass launch (k_dist1).
	void defer_compact(const int* woff, const int* plist, int li, int b)
	{
		const CompactArgs stale = take_compact();  // none is left behind on the normal path
		if (stale.nblocks)
			FG_RUN("k_compact", st_, launch_pdl((k_compact<L>), stale.nblocks, 256, 0, st_, P_, stale, 0););
		pending_ = CompactArgs{P_.S, woff, plist, li, b};
	}
	CompactArgs take_compact()
	{
		const CompactArgs ca = pending_;
		pending_ = CompactArgs{0, nullptr, nullptr, 0, 0};
		return ca;
	}

	void layer_pass(const ListView& lv, int k, float side, int b)
	{
		const int* woff = P_.woffl + (size_t)(k + L) * (P_.S + 1);
		const CompactArgs ca = take_compact();
		FG_RUN("k_dist1", st_, launch_pdl((k_dist1<D, L>), warp_grid_ + ca.nblocks, 256, 0, st_, P_, woff, lv, k, side, dist_split_, ca););
		if (block_passes_)
			FG_RUN("k_dist2", st_, launch_pdl((k_dist2<D, L>), warp_grid_, 256, 0, st_, P_, woff, lv, k, b););
		else
			FG_RUN("k_dist2", st_, launch_pdl((k_dist2_warp<D, L>), warp_grid_, 256, 0, st_, P_, woff, lv, k, b););
		defer_compact(woff, lv.plist, k + L, b);
	}

	/// update_zero_layer: block-per-partition for large bricks, warp-per-partition for small ones.
	void zero_apply(const ListView& lv, const int* ncount, int b)
	{
		if (block_passes_)
			FG_RUN("k_zero_apply", st_, launch_pdl((k_zero_apply<D, L>), warp_grid_, 256, 0, st_, P_, lv, ncount, b););
		else
			FG_RUN("k_zero_apply", st_, launch_pdl((k_zero_apply_warp<D, L>), warp_grid_, 256, 0, st_, P_, lv, ncount, b););
	}

	void flush()
	{
		if (smem_flush_)
			FG_RUN("k_flush_smem", st_, launch_pdl((k_flush_smem<D, L>), sm_count() * 8, 256, smem_flush_, st_, P_););
		else
			FG_RUN("k_flush_leaf", st_, launch_pdl((k_flush_leaf<D, L>), grid_for(P_.NP), 128, 0, st_, P_););
		// a block per (surface, list), looping where there are more than two per SM: in a large
		// batch most have no events and leave at once, without a block launch each
		FG_RUN("k_flush_plist", st_, launch_pdl((k_flush_plist<L>), std::min(P_.S * NL, sm_count() * 2), 1024, 0, st_, P_););
	}

	/// The status lists' entry offsets and the counters were prepared by the last compaction
	/// of the distance passes (k_compact's last block).
	void expand()
	{
		FG_RUN("k_expand_gen", st_, launch_pdl((k_expand_gen<D, L>), warp_grid_, 256, 0, st_, P_, 0););
		FG_RUN("k_activate", st_, launch_pdl((k_activate<L>), sm_count() * 4, 256, 0, st_, P_););
		FG_RUN("k_expand_gen", st_, launch_pdl((k_expand_gen<D, L>), warp_grid_, 256, 0, st_, P_, 1););
		FG_RUN("k_expand_gen", st_, launch_pdl((k_expand_gen<D, L>), warp_grid_, 256, 0, st_, P_, 2););
		FG_RUN("k_expand_append", st_, launch_pdl((k_expand_append<L>), sm_count() * 4, 256, smem_sort_, st_, P_););
		// the partition-list appends (d_expand_plist) run in the launch after, which retires
		// bricks (k_retire, or k_clear_buffer with retire_too)
	}

	void retire()
	{
		// its last block resets the retire queue
		FG_RUN("k_retire", st_, launch_pdl((k_retire<L>), std::max(grid_for(P_.nslots), std::min(P_.S, sm_count() * 8)), 256, 0, st_, P_););
	}

	void clear_status()
	{
		// its last block resets the status partition counts and the status queue
		FG_RUN("k_clear_status", st_, launch_pdl((k_clear_status<L>), warp_grid_, 256, 0, st_, P_););
		status_dirty_ = false;
	}

	/// retire_too: the iteration's brick retirement runs in the same launch (in place of
	/// k_retire).
	void clear_buffer(int b, bool retire_too = false)
	{
		const bool here = P_.S <= kScanHereMax;
		if (!here) scan(P_.apcnt[b], 0, 2);
		const size_t sm = here ? (size_t)(P_.S + 1) * sizeof(int) : 0;
		// its last block resets the buffer's partition counts (and the retire queue)
		FG_RUN("k_clear_buffer", st_, launch_pdl((k_clear_buffer<L>), warp_grid_, 256, sm, st_, P_, b, here ? 1 : 0, retire_too ? 1 : 0););
		buf_dirty_[b] = false;
	}

	int read_changed()
	{
		int c = 0;
		FG_CUDA(cudaMemcpyAsync(&c, P_.changed, sizeof(int), cudaMemcpyDeviceToHost, st_));
		FG_CUDA(cudaStreamSynchronize(st_));
		FG_CUDA(cudaGetLastError());
		return c;
	}

	cudaStream_t st_;
	Dev P_;
	int csz_[3] = {1, 1, 1};
	std::vector<SurfGeom> geom_;
	std::vector<int> np_cap_;  // partitions reserved per surface (its range at geom_[s].pbase)
	std::vector<void*> owned_;
	unsigned long long* acc_ = nullptr;     // node updates of all global updates so far
	unsigned long long* zcount_ = nullptr;  // zero-layer leaf count of a bounded update
	int* d_iters_ = nullptr;                 // iteration count of the device-side loop
	int launch_mode_ = 0;  // 0 automatic (= 1), 1 the update as one graph, 2 phase by phase
	cudaGraphExec_t step_exec_[16] = {};  // the whole update, by due resets and delta kernel
	long long step_launches_[16] = {};    // kernels before its while node
	bool step_ok_ = true;
	Speed* h_speeds_ = nullptr;  // pinned staging of the builtin speeds
	int* h_out_ = nullptr;       // pinned read-back of the device loop's count and flag
	bool delta_staged_ = true;   // curvature speeds over staged bricks (k_delta_smem)
	// the global update's distance passes fused (k_dist_fused): the same results in 2L+1
	// launches instead of 4L, but no faster on C2 (1.33 against 1.28 ms per step), so off
	// unless asked for
	bool fused_ = false;
	// the 2L distance passes per brick in shared memory (k_dist_tiled); smem_tiled_ = 0 where
	// the brick with its halo does not fit
	bool tiled_ = false;
	TileShape tile_{};
	size_t smem_tiled_ = 0;
	int tiled_threads_ = 256;
	int tiled_grid_ = 0;
	Speed* d_speeds_ = nullptr;
	size_t smem_sort_ = 0;
	size_t smem_flush_ = 0;
	size_t smem_halo_ = 0;
	int* d_lpos_ = nullptr;    // local-update staging: delta positions
	float* d_lval_ = nullptr;  // delta values
	int* d_lcount_ = nullptr;
	int lcap_ = 0;
	int warp_grid_ = 0;
	int dist_split_ = 1;  // warps per partition entry in the first distance pass
	cudaGraphExec_t iter_exec_[2] = {nullptr, nullptr};  // global iteration, by buffer parity
	long long iter_launches_[2] = {0, 0};
	bool graphs_ok_ = true;
	cudaGraphExec_t loop_exec_ = nullptr;  // the global convergence loop (conditional nodes)
	long long loop_launches_[2] = {0, 0};  // kernels of the loop's first and second iteration
	bool loop_ok_ = true;
	CompactArgs pending_{0, nullptr, nullptr, 0, 0};  // compaction riding on the next k_dist1
	// whole blocks (not warps) per partition entry in the record-keeping passes: pays off when
	// a brick holds thousands of leaves, costs idle threads when it holds a few hundred
	bool block_passes_ = false;
	bool status_dirty_ = false;
	bool buf_dirty_[2] = {false, false};
	static constexpr int kMaxIterations = 64;
	std::vector<int> frozen_;
	std::vector<int> paused_;
	std::vector<int> stopped_;  // host staging of frozen_ | paused_
	std::vector<int> newly_frozen_;
	bool throw_on_freeze_ = true;
	StepStats stats_;
};

void keep_pool_memory()
{
	int dev = 0;
	cudaMemPool_t pool;
	if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
		uint64_t keep = UINT64_MAX;
		cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
	}
	cudaGetLastError();
}

EngineBase* make_engine(const PoolDesc& desc, cudaStream_t stream)
{
	keep_pool_memory();
#define FG_CASE(d, l) \
	if (desc.D == d && desc.L == l) return new Engine<d, l>(desc, stream);
	FG_CASE(2, 1) FG_CASE(2, 2) FG_CASE(2, 3) FG_CASE(2, 4)
	FG_CASE(3, 1) FG_CASE(3, 2) FG_CASE(3, 3) FG_CASE(3, 4)
#undef FG_CASE
	throw Error(-1, "unsupported dims/layers (D in {2,3}, L in 1..4)");
}

}  // namespace fg
