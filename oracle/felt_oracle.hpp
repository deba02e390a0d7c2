// Felt sparse-field level-set oracle: a single-threaded CPU restatement of the reference's
// Surface<D,L>::update / update_start / delta / update_end / seed / snapshot and Polys
// (marching squares/cubes) semantics.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product (felt_b200/) links, loads or calls this code;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only as the
// checker. Every function names the reference file:line it restates (paths relative to the
// feltech/Felt source tree). The reference itself needs Eigen3 and Boost, which are absent here,
// so this restatement is pinned against the golden vectors held by the reference's own tests
// (tests/golden/, tests/test_oracle_golden.py).
//
// Arithmetic is FP32 exactly as in the reference (compile with -ffp-contract=off): layer
// thresholds must flip exactly where the reference's flip. The template parameter `Real` allows
// an FP64 run of the same method for error estimates.
#pragma once

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>
#include <atomic>
#include <exception>
#include <thread>
#include <condition_variable>
#include <functional>
#include <mutex>

namespace fo {

/// Threads of the loops the reference runs in parallel (set through fo_set_threads; 1 = the
/// plain sequential order). Every threaded loop below only writes state owned by its item, or
/// records its shared edits per item and applies them afterwards in item order, so results and
/// list orders are the same for any thread count.
inline std::atomic<int> g_threads{1};

/// Set on the threads of a running parallel loop: a loop started from inside one runs inline.
inline thread_local bool t_in_loop = false;

/// A persistent pool of host threads for the parallel loops, started on first use (the
/// reference's OpenMP runtime keeps its threads between regions too; starting threads per loop
/// would cost more than these loops take).
class ThreadPool {
public:
	static ThreadPool& get()
	{
		static ThreadPool pool;
		return pool;
	}
	/// fn(i) for i in [0, n) on nt threads (the caller included), indices taken in turn.
	template <class Fn>
	void run(long n, int nt, Fn&& fn)
	{
		std::lock_guard<std::mutex> one(run_mu_);  // one parallel loop at a time
		ensure(nt - 1);
		std::atomic<long> next{0};
		std::exception_ptr err;
		std::atomic<bool> failed{false};
		std::mutex err_mu;
		auto body = [&] {
			t_in_loop = true;
			struct Clear {
				~Clear() { t_in_loop = false; }
			} clear;
			try {
				for (long i; (i = next.fetch_add(1)) < n && !failed.load();) fn(i);
			} catch (...) {
				std::lock_guard<std::mutex> g(err_mu);
				if (!failed.exchange(true)) err = std::current_exception();
			}
		};
		std::function<void()> job(body);
		{
			std::lock_guard<std::mutex> g(mu_);
			job_ = &job;
			want_ = nt - 1;
			taken_ = 0;
			done_ = 0;
			gen_++;
		}
		cv_.notify_all();
		body();
		{
			std::unique_lock<std::mutex> g(mu_);
			done_cv_.wait(g, [&] { return done_ == want_; });
			job_ = nullptr;
		}
		if (err) std::rethrow_exception(err);
	}
	~ThreadPool()
	{
		{
			std::lock_guard<std::mutex> g(mu_);
			stop_ = true;
			gen_++;
		}
		cv_.notify_all();
		for (auto& t : workers_) t.join();
	}

private:
	void ensure(int n)
	{
		while ((int)workers_.size() < n) workers_.emplace_back([this] { loop(); });
	}
	void loop()
	{
		unsigned long long seen = 0;
		std::unique_lock<std::mutex> g(mu_);
		for (;;) {
			cv_.wait(g, [&] { return stop_ || (gen_ != seen && taken_ < want_); });
			if (stop_) return;
			seen = gen_;
			taken_++;
			std::function<void()>* job = job_;
			g.unlock();
			(*job)();
			g.lock();
			if (++done_ == want_) done_cv_.notify_one();
		}
	}
	std::mutex run_mu_, mu_;
	std::condition_variable cv_, done_cv_;
	std::vector<std::thread> workers_;
	std::function<void()>* job_ = nullptr;
	unsigned long long gen_ = 0;
	int want_ = 0, taken_ = 0, done_ = 0;
	bool stop_ = false;
};

/// fn(i) for i in [0, n) across g_threads threads. min_items is the size below which the loop
/// runs inline: the reference's regions are parallel only from 32 active partitions
/// (Surface.hpp:19-27), Polys::march always (Polys.hpp:140). fn must only write state owned by
/// item i.
template <class Fn>
void parallel_items(long n, Fn&& fn, long min_items = 32)
{
	const int nt = (int)std::min<long>(g_threads.load(), n);
	if (nt <= 1 || n < min_items || t_in_loop) {
		for (long i = 0; i < n; i++) fn(i);
		return;
	}
	ThreadPool::get().run(n, nt, fn);
}

using PosIdx = std::size_t;
constexpr std::size_t NUL = std::numeric_limits<std::size_t>::max();

template <int D> using Vi = std::array<int, D>;

/// Error raised where the reference would throw (boost iround on NaN) or hit undefined
/// behaviour (tracking outside the grid, writing an inactive partition).
struct Error : std::runtime_error {
	int code;
	Error(int c, const char* m) : std::runtime_error(m), code(c) {}
};
enum { ERR_NONFINITE = -10, ERR_OUTSIDE = -11, ERR_INACTIVE = -12 };

// ---------------------------------------------------------------------------------------------
// Index helpers (include/Felt/Impl/Util.hpp)
// ---------------------------------------------------------------------------------------------

/// Row-major index, last axis fastest, accumulated in int (Util.hpp:23-40).
template <int D>
inline PosIdx index_of(const Vi<D>& pos, const Vi<D>& size, const Vi<D>& off)
{
	int acc = 0;
	for (int i = 0; i < D; i++) {
		int a = pos[i] - off[i];
		for (int j = i + 1; j < D; j++) a *= size[j];
		acc += a;
	}
	return PosIdx(acc);
}

/// Inverse of index_of (Util.hpp:56-83).
template <int D>
inline Vi<D> pos_of(PosIdx idx, const Vi<D>& size, const Vi<D>& off)
{
	Vi<D> p;
	for (int a = D - 1; a != 0; a--) {
		p[a] = int(idx) % size[a] + off[a];
		idx /= PosIdx(size[a]);
	}
	p[0] = int(idx) % size[0] + off[0];
	return p;
}

/// Bounds test done in float, half-open [lo, hi) (Util.hpp:94-106).
template <int D, class T>
inline bool inside(const std::array<T, D>& pos, const Vi<D>& lo, const Vi<D>& hi)
{
	for (int i = 0; i < D; i++) {
		if (static_cast<float>(pos[i]) >= static_cast<float>(hi[i])) return false;
		if (static_cast<float>(pos[i]) < static_cast<float>(lo[i])) return false;
	}
	return true;
}

/// Round half away from zero, raising on non-finite input: the contract of
/// boost::math::iround used by Surface::layer_id (Surface.hpp:1694-1697).
template <class Real>
inline int iround_away(Real v)
{
	if (!std::isfinite(v)) throw Error(ERR_NONFINITE, "layer_id of non-finite value");
	const Real r = std::round(v);
	if (r >= Real(2147483648.0) || r < Real(-2147483648.0))
		throw Error(ERR_NONFINITE, "layer_id out of int range");
	return int(r);
}

/// layer_id(v) = iround(v + FLT_EPSILON) (Surface.hpp:1694-1697). The epsilon is the float
/// epsilon even in an FP64 run, as Distance is hard-wired to float in the reference.
template <class Real>
inline int layer_id(Real v)
{
	return iround_away<Real>(v + Real(std::numeric_limits<float>::epsilon()));
}

/// |id| <= L (Surface.hpp:1705-1709).
inline bool inside_band(int id, int L) { return (id < 0 ? -id : id) <= L; }

inline int sgn(int v) { return (0 < v) - (v < 0); }

// ---------------------------------------------------------------------------------------------
// Hashed noise used by the noise speed kinds. A project-defined 32-bit integer hash of
// (pos, seed) to 24 bits, mapped to u * 2^-23 - 1 in [-1, 1): every step is integer or exact in
// FP32, so CPU and GPU produce identical values. Mixing is MurmurHash3's public-domain fmix32
// finaliser applied once per axis.
// ---------------------------------------------------------------------------------------------
inline uint32_t fmix32(uint32_t h)
{
	h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
	return h;
}
template <int D>
inline float hash_noise(const Vi<D>& pos, uint32_t seed)
{
	static const uint32_t K[3] = {0x9e3779b1u, 0x7f4a7c15u, 0x94d049bbu};
	uint32_t h = fmix32(seed ^ 0x5eed5eedu);
	for (int a = 0; a < D; a++) h = fmix32(h ^ (uint32_t(pos[a]) * K[a]));
	const uint32_t u = h >> 8;
	return float(u) * (1.0f / 8388608.0f) - 1.0f;
}

// ---------------------------------------------------------------------------------------------
// Partitioned two-level grid with per-child multi-list single-index leaf lookups and a
// multi-list multi-index children lookup. Restates Impl::Partitioned::{Lookup,Tracked::Simple,
// Tracked::Numeric} (Partitioned.hpp:17-193) built from Tracked::LazyMultiListSingleIdxByValue
// children (Tracked.hpp:16-79) and a Tracked::MultiListMultiIdxByRef children grid
// (Tracked.hpp:170-228).
// ---------------------------------------------------------------------------------------------
template <int D, int N, class T>
struct PGrid {
	Vi<D> size{}, off{}, hi{};        // grid size, offset and offset+size
	Vi<D> csize{}, ccount{}, coff{};  // child size, children-grid size and offset
	int bv = 1;                       // leaves per child
	T bg{};                           // value outside the grid (PartitionedMixin.hpp:596-597)

	struct Child {
		Vi<D> off{};
		T bg{};
		std::vector<T> data;       // empty when inactive
		std::vector<PosIdx> lkp;   // leaf -> position in its list, empty when inactive
		std::array<std::vector<PosIdx>, N> lists;
	};
	std::vector<Child> ch;
	std::vector<std::array<PosIdx, N>> cpos;  // children lookup: per child per list position
	std::array<std::vector<PosIdx>, N> clists;

	PGrid() = default;

	/// Children ctor (PartitionedMixin.hpp:59-86) and calc_children_size (131-141): a partial
	/// partition on any axis adds one child along every axis.
	PGrid(const Vi<D>& size_, const Vi<D>& off_, const Vi<D>& csize_, T bg_)
		: size(size_), off(off_), csize(csize_), bg(bg_)
	{
		bool exact = true;
		for (int a = 0; a < D; a++) {
			hi[a] = off[a] + size[a];
			ccount[a] = size[a] / csize[a];
			if (ccount[a] * csize[a] != size[a]) exact = false;
			coff[a] = off[a] / csize[a];
			bv *= csize[a];
		}
		if (!exact)
			for (int a = 0; a < D; a++) ccount[a] += 1;
		PosIdx n = 1;
		for (int a = 0; a < D; a++) n *= PosIdx(ccount[a]);
		ch.resize(n);
		cpos.assign(n, {});
		for (auto& c : cpos) c.fill(NUL);
		for (PosIdx i = 0; i < n; i++) {
			const Vi<D> pc = pos_of<D>(i, ccount, coff);
			for (int a = 0; a < D; a++) ch[i].off[a] = (pc[a] - coff[a]) * csize[a] + off[a];
			ch[i].bg = bg;
		}
	}

	PosIdx nchildren() const { return ch.size(); }
	bool active(PosIdx pc) const { return !ch[pc].lkp.empty(); }

	/// pos_child / pos_idx_child (PartitionedMixin.hpp:221-245).
	PosIdx pidx_child(const Vi<D>& pos) const
	{
		Vi<D> pc;
		for (int a = 0; a < D; a++) pc[a] = (pos[a] - off[a]) / csize[a] + coff[a];
		return index_of<D>(pc, ccount, coff);
	}
	PosIdx leaf_of(PosIdx pc, const Vi<D>& pos) const { return index_of<D>(pos, csize, ch[pc].off); }
	Vi<D> pos_leaf(PosIdx pc, PosIdx leaf) const { return pos_of<D>(leaf, csize, ch[pc].off); }
	bool in_grid(const Vi<D>& pos) const { return inside<D>(pos, off, hi); }

	/// Tracked::Activate::activate (TrackedMixin.hpp:37-41): data filled with the child's own
	/// background, lookup filled with null.
	void activate(PosIdx pc)
	{
		Child& c = ch[pc];
		c.data.assign(bv, c.bg);
		c.lkp.assign(bv, NUL);
	}
	/// Tracked::Activate::deactivate (TrackedMixin.hpp:48-62) and the lookup-only
	/// Lookup::MultiList::Activate::deactivate (LookupMixin.hpp:213-222).
	void deactivate(PosIdx pc)
	{
		Child& c = ch[pc];
		std::vector<T>().swap(c.data);
		std::vector<PosIdx>().swap(c.lkp);
		for (auto& l : c.lists) std::vector<PosIdx>().swap(l);
	}
	void deactivate(PosIdx pc, T bg_)
	{
		ch[pc].bg = bg_;
		deactivate(pc);
	}

	// --- children-level lookup (LookupMixin.hpp:457-570, MultiList::MultiIdx) ---
	bool ctracked(PosIdx pc, int l) const { return cpos[pc][l] != NUL; }
	bool ctracked_any(PosIdx pc) const
	{
		for (int l = 0; l < N; l++)
			if (cpos[pc][l] != NUL) return true;
		return false;
	}
	void ctrack(PosIdx pc, int l)
	{
		if (cpos[pc][l] != NUL) return;
		cpos[pc][l] = clists[l].size();
		clists[l].push_back(pc);
	}
	void cuntrack(PosIdx pc, int l)
	{
		PosIdx& at = cpos[pc][l];
		if (at == NUL) return;
		auto& lst = clists[l];
		const PosIdx last = lst.size() - 1;
		if (at < last) {
			const PosIdx moved = lst[last];
			lst[at] = moved;
			cpos[moved][l] = at;
		}
		at = NUL;
		lst.pop_back();
	}

	// --- leaf-level lookup (LookupMixin.hpp:298-386, MultiList::SingleIdx) ---
	bool ltrack(PosIdx pc, PosIdx leaf, int l)
	{
		Child& c = ch[pc];
		if (c.lkp.empty()) throw Error(ERR_INACTIVE, "leaf track on inactive partition");
		if (c.lkp[leaf] != NUL) return false;
		c.lkp[leaf] = c.lists[l].size();
		c.lists[l].push_back(leaf);
		return true;
	}
	void luntrack(PosIdx pc, PosIdx leaf, int l)
	{
		Child& c = ch[pc];
		PosIdx& at = c.lkp[leaf];
		if (at == NUL) return;
		auto& lst = c.lists[l];
		const PosIdx last = lst.size() - 1;
		if (at < last) {
			const PosIdx moved = lst[last];
			lst[at] = moved;
			c.lkp[moved] = at;
		}
		at = NUL;
		lst.pop_back();
	}

	/// Leafs::track_child (PartitionedMixin.hpp:201-213).
	void track_child(PosIdx pc, int l)
	{
		if (ctracked(pc, l)) return;
		if (!active(pc)) activate(pc);
		ctrack(pc, l);
	}

	/// Partitioned::Tracked::track (PartitionedMixin.hpp:441-469) with child
	/// Tracked::MultiList::ByValue::track (TrackedMixin.hpp:342-346): the value is written even
	/// when the leaf is already tracked.
	void track(T val, PosIdx pc, PosIdx leaf, int l)
	{
		track_child(pc, l);
		ch[pc].data[leaf] = val;
		ltrack(pc, leaf, l);
	}
	void track(T val, const Vi<D>& pos, int l)
	{
		if (!in_grid(pos)) throw Error(ERR_OUTSIDE, "track outside grid");
		const PosIdx pc = pidx_child(pos);
		track(val, pc, leaf_of(pc, pos), l);
	}
	/// Child-level track without touching the children lookup, as used by Surface::update's
	/// functor loop and update_distance's first pass (Surface.hpp:290-292, 1071).
	void child_track(T val, PosIdx pc, PosIdx leaf, int l)
	{
		if (!active(pc)) throw Error(ERR_INACTIVE, "child track on inactive partition");
		ch[pc].data[leaf] = val;
		ltrack(pc, leaf, l);
	}
	/// Partitioned::Lookup::track (PartitionedMixin.hpp:388-413) for lookup-only grids.
	void track_lookup(PosIdx pc, PosIdx leaf, int l)
	{
		track_child(pc, l);
		ltrack(pc, leaf, l);
	}
	void track_lookup(const Vi<D>& pos, int l)
	{
		if (!in_grid(pos)) throw Error(ERR_OUTSIDE, "track outside grid");
		const PosIdx pc = pidx_child(pos);
		track_lookup(pc, leaf_of(pc, pos), l);
	}

	/// Partitioned::Untrack::untrack (PartitionedMixin.hpp:489-517).
	void untrack(T bg_, PosIdx pc, PosIdx leaf, int l)
	{
		luntrack(pc, leaf, l);
		ch[pc].data[leaf] = bg_;
		if (ch[pc].lists[l].empty()) {
			cuntrack(pc, l);
			if (!ctracked_any(pc)) deactivate(pc, bg_);
		}
	}

	/// Partitioned::Untrack::retrack (PartitionedMixin.hpp:519-558).
	void retrack(PosIdx pc, PosIdx leaf, int from, int to)
	{
		luntrack(pc, leaf, from);
		ltrack(pc, leaf, to);
		if (!ctracked(pc, to) || ch[pc].lists[from].empty()) {
			ctrack(pc, to);
			if (ch[pc].lists[from].empty()) cuntrack(pc, from);
		}
	}

	/// Child reset: Tracked::MultiList::Reset::reset (TrackedMixin.hpp:420-428) writes the
	/// child background to every tracked leaf, then LookupMixin.hpp:377-386 clears the lists.
	void child_reset(PosIdx pc, bool valued)
	{
		Child& c = ch[pc];
		for (int l = 0; l < N; l++) {
			for (PosIdx leaf : c.lists[l]) {
				if (valued) c.data[leaf] = c.bg;
				c.lkp[leaf] = NUL;
			}
			c.lists[l].clear();
		}
	}

	/// Reset::MultiList::reset (PartitionedMixin.hpp:336-360). The reference iterates each
	/// children list while untracking from it; the swap-with-last removals never overwrite a
	/// slot ahead of the iterator, so each originally listed child is visited once, in the
	/// original order, which is what iterating a copy does here.
	template <class Mask>
	void reset(const Mask& mask, bool valued)
	{
		for (int l = 0; l < N; l++) {
			const std::vector<PosIdx> parts = clists[l];
			for (PosIdx pc : parts) {
				cuntrack(pc, l);
				if (!mask.ctracked_any(pc))
					deactivate(pc);
				else if (active(pc))
					child_reset(pc, valued);
			}
		}
	}

	/// Reset::MultiList::track_children (PartitionedMixin.hpp:319-334).
	template <class Mask>
	void track_children(const Mask& mask)
	{
		for (int l = 0; l < N; l++)
			for (PosIdx pc : mask.clists[l]) {
				if (ctracked(pc, l)) continue;
				if (!active(pc)) activate(pc);
				ctrack(pc, l);
			}
	}

	/// Lazy get by child and leaf (GridMixin.hpp:608-621).
	T cget(PosIdx pc, PosIdx leaf) const
	{
		const Child& c = ch[pc];
		return c.data.empty() ? c.bg : c.data[leaf];
	}
	void cset(PosIdx pc, PosIdx leaf, T v)
	{
		if (ch[pc].data.empty()) throw Error(ERR_INACTIVE, "set on inactive partition");
		ch[pc].data[leaf] = v;
	}
	/// Partitioned::Access::get (PartitionedMixin.hpp:594-601).
	T get(const Vi<D>& pos) const
	{
		if (!in_grid(pos)) return bg;
		const PosIdx pc = pidx_child(pos);
		return cget(pc, leaf_of(pc, pos));
	}
};

// ---------------------------------------------------------------------------------------------
// Numeric stencils (include/Felt/Impl/Mixin/NumericMixin.hpp)
// ---------------------------------------------------------------------------------------------

/// Eigen's fixed-size sum(): unrolled by halving, so 3 terms sum as x0 + (x1 + x2).
template <class Real, int D>
inline Real eigen_sum(const std::array<Real, D>& v)
{
	if (D == 1) return v[0];
	if (D == 2) return v[0] + v[1];
	return v[0] + (v[1] + v[2]);
}

/// Mean curvature by difference of normals (NumericMixin.hpp:72-156), over any grid read
/// through `get`. Normals use forward/backward differences along each axis and central
/// differences across the others; the result is sum(n_fwd - n_back) / 2. The position is a node
/// or a real position (read through interpolation by get), stepped in its own type.
template <int D, class Real, class Get, class Pos>
inline Real curv_at(Get&& get, const Pos& pos)
{
	const Real centre = get(pos);
	Pos dir = pos;
	std::array<Real, D> nf, nb;
	for (int axis = 0; axis < D; axis++) {
		dir[axis] += 1;
		const Real va = get(dir) - centre;
		Real sq = 0;
		for (int an = 0; an < D; an++) {
			if (an == axis) continue;
			Pos dn = dir;
			dn[an] -= 1;
			const Real lo = get(dn);
			dn[an] += 2;
			const Real hi = get(dn);
			const Real v = (hi - lo) / 2;
			sq += v * v;
		}
		nf[axis] = va / std::sqrt(va * va + sq);
		dir[axis] -= 1;
	}
	for (int axis = 0; axis < D; axis++) {
		dir[axis] -= 1;
		const Real va = centre - get(dir);
		Real sq = 0;
		for (int an = 0; an < D; an++) {
			if (an == axis) continue;
			Pos dn = dir;
			dn[an] -= 1;
			const Real lo = get(dn);
			dn[an] += 2;
			const Real hi = get(dn);
			const Real v = (hi - lo) / 2;
			sq += v * v;
		}
		nb[axis] = va / std::sqrt(va * va + sq);
		dir[axis] += 1;
	}
	std::array<Real, D> dn;
	for (int a = 0; a < D; a++) dn[a] = nf[a] - nb[a];
	return eigen_sum<Real, D>(dn) / 2;
}

/// The Numeric API at a node (NumericMixin.hpp:165-355, grid spacing 1) over any grid read
/// through get, with in_grid its bounds test, into out in this order: grad (189-231), gradF
/// (279-298), gradB (308-326), gradC (335-355), gradE (243-270), each D values, then divergence
/// (165-175). Whole-number steps are exact, so the functions share their samples.
template <int D, class Real, class Get, class In>
inline void numeric_at(Get&& get, In&& in_grid, const Vi<D>& pos, Real* out)
{
	const Real centre = get(pos);
	Vi<D> t = pos;
	Real* grad = out;
	Real* gf = out + D;
	Real* gb = out + 2 * D;
	Real* gc = out + 3 * D;
	Real* ge = out + 4 * D;
	for (int a = 0; a < D; a++) {
		t[a] -= 1;
		const Real back = get(t);
		const bool in_back = in_grid(t);
		t[a] += 2;
		const Real fwd = get(t);
		const bool in_fwd = in_grid(t);
		t[a] -= 1;
		int order = 0;
		Real b = centre, f = centre;
		if (in_back) {
			b = back;
			order++;
		}
		if (in_fwd) {
			f = fwd;
			order++;
		}
		grad[a] = order ? (f - b) / Real(order) : Real(0);
		gf[a] = fwd - centre;
		gb[a] = centre - back;
		gc[a] = (fwd - back) / Real(2);
		ge[a] = std::min(fwd - centre, Real(0)) + std::max(centre - back, Real(0));
	}
	std::array<Real, D> diff;
	for (int a = 0; a < D; a++) diff[a] = gf[a] - gb[a];
	out[5 * D] = eigen_sum<Real, D>(diff);
}

/// Neighbour enumeration order -x,+x,-y,+y,-z,+z (NumericMixin.hpp:489-500).
template <int D, class Fn>
inline void neighs(Vi<D> pos, Fn&& fn)
{
	for (int a = 0; a < D; a++) {
		pos[a] -= 1;
		fn(pos);
		pos[a] += 2;
		fn(pos);
		pos[a] -= 1;
	}
}

// ---------------------------------------------------------------------------------------------
// Speed functors. The three builtin terms are combined in a fixed order:
//   acc = a * curv(pos)         (if CURV)
//   acc = acc + n * h(pos,seed) (if NOISE; acc = n*h when first)
//   acc = acc + c               (if CONST; acc = c when first)
// ---------------------------------------------------------------------------------------------
enum { SPEED_CONST = 1, SPEED_CURV = 2, SPEED_NOISE = 4 };
struct Speed {
	int kind;
	float c, a, n;
	uint32_t seed;
};

template <int D, int L, class Real = float>
class Surface {
public:
	static constexpr int NL = 2 * L + 1;
	using Iso = PGrid<D, NL, Real>;
	using Delta = PGrid<D, NL, Real>;
	using Status = PGrid<D, NL, int>;
	using Affected = PGrid<D, NL, char>;

	Iso iso;
	Delta delta_;
	Status status;
	Affected aff, affb;

	static int lidx(int id) { return id + L; }  // layer_idx (Surface.hpp:672-675)

	static Vi<D> offset_of(const Vi<D>& size)  // Surface.hpp:1716-1719
	{
		Vi<D> o;
		for (int a = 0; a < D; a++) o[a] = (-1 * size[a]) / 2;
		return o;
	}

	/// Surface ctor (Surface.hpp:163-173).
	Surface(const Vi<D>& size, const Vi<D>& part)
		: iso(size, offset_of(size), part, Real(L + 1)),
		  delta_(size, offset_of(size), part, Real(0)),
		  status(size, offset_of(size), part, L + 1),
		  aff(size, offset_of(size), part, 0),
		  affb(size, offset_of(size), part, 0)
	{}

	int layer_of(Real v) const { return layer_id<Real>(v); }

	/// seed (Surface.hpp:207-241). The window loop visits index prod(window) too (`<=`), which
	/// maps back to the window's minimum corner, outside the band for D >= 2.
	void seed(const Vi<D>& centre)
	{
		Vi<D> pmin, win, zero{};
		for (int a = 0; a < D; a++) {
			pmin[a] = centre[a] - L;
			win[a] = 2 * L + 1;
		}
		PosIdx nmax = 1;
		for (int a = 0; a < D; a++) nmax *= PosIdx(win[a]);
		for (PosIdx i = 0; i <= nmax; i++) {
			Vi<D> pos = pos_of<D>(i, win, zero);
			int l1 = 0;
			for (int a = 0; a < D; a++) {
				pos[a] += pmin[a];
				l1 += std::abs(pos[a] - centre[a]);
			}
			const Real dist = Real(l1);
			const int lid = layer_of(dist);
			if (inside_band(lid, L)) iso.track(dist, pos, lidx(lid));
		}
	}

	// --- stencils on the isogrid ---
	Real get(const Vi<D>& pos) const { return iso.get(pos); }

	/// curv (NumericMixin.hpp:72-156) on the isogrid.
	Real curv(const Vi<D>& pos) const
	{
		return curv_at<D, Real>([this](const Vi<D>& p) { return get(p); }, pos);
	}

	/// The Numeric API at a node (NumericMixin.hpp:165-355, grid spacing 1): numeric_at on the
	/// isogrid.
	void numeric(const Vi<D>& pos, Real* out) const
	{
		numeric_at<D, Real>([this](const Vi<D>& p) { return get(p); },
		                    [this](const Vi<D>& p) { return iso.in_grid(p); }, pos, out);
	}

	Real speed(const Speed& s, const Vi<D>& pos) const
	{
		Real acc = 0;
		bool have = false;
		if (s.kind & SPEED_CURV) {
			acc = Real(s.a) * curv(pos);
			have = true;
		}
		if (s.kind & SPEED_NOISE) {
			const Real t = Real(s.n) * Real(hash_noise<D>(pos, s.seed));
			acc = have ? acc + t : t;
			have = true;
		}
		if (s.kind & SPEED_CONST) acc = have ? acc + Real(s.c) : Real(s.c);
		return acc;
	}

	// --- the global update ---

	/// update_start (Surface.hpp:393-399).
	void update_start()
	{
		delta_.reset(iso, true);
		aff.reset(iso, false);
		affb.reset(iso, false);
		status.reset(iso, true);
	}

	/// update(fn) (Surface.hpp:254-296) with a builtin speed.
	template <class Fn>
	void update_fn(Fn&& fn)
	{
		update_start();
		delta_.track_children(iso);
		const std::vector<PosIdx>& parts = iso.clists[lidx(0)];
		// The reference runs this loop across OpenMP threads (Surface.hpp:284-292); each
		// partition's leaves stay with one thread, so results and orders do not depend on the
		// thread count.
		parallel_items((long)parts.size(), [&](long i) {
			const PosIdx pc = parts[(size_t)i];
			for (PosIdx leaf : iso.ch[pc].lists[lidx(0)]) {
				const Vi<D> pos = iso.pos_leaf(pc, leaf);
				const Real d = fn(pos);
				delta_.child_track(d, pc, leaf, lidx(0));
			}
		});
		update_end_global();
	}
	void update(const Speed& s)
	{
		update_fn([&](const Vi<D>& pos) { return speed(s, pos); });
	}

	/// update(lo, hi, fn) bounded update (Surface.hpp:310-386).
	template <class Fn>
	void update_bounded_fn(const Vi<D>& lo, const Vi<D>& hi, Fn&& fn)
	{
		Vi<D> glo = iso.off, gup;
		for (int a = 0; a < D; a++) gup[a] = iso.off[a] + iso.size[a];
		auto pchild = [&](const Vi<D>& p) {
			Vi<D> pc;
			for (int a = 0; a < D; a++) pc[a] = (p[a] - iso.off[a]) / iso.csize[a] + iso.coff[a];
			return pc;
		};
		Vi<D> gm1;
		for (int a = 0; a < D; a++) gm1[a] = gup[a] - 1;
		const Vi<D> gcl = pchild(glo), gcu = pchild(gm1), plo = pchild(lo), phi = pchild(hi);
		Vi<D> cl, cu, box, lub, zero{};
		for (int a = 0; a < D; a++) {
			cl[a] = std::max(gcl[a], plo[a]);
			cu[a] = std::min(gcu[a], phi[a]);
			box[a] = cu[a] - cl[a] + 1;
			lub[a] = std::min(gup[a], hi[a] + 1);
		}
		PosIdx nb = 1;
		for (int a = 0; a < D; a++) nb *= PosIdx(box[a]);
		update_start();
		// The reference runs the box's partitions across OpenMP threads (Surface.hpp:336): the
		// functor values are taken per partition on one thread each, then tracked into the delta
		// grid in the sequential order.
		std::vector<PosIdx> pcs((size_t)nb);
		std::vector<std::vector<std::pair<PosIdx, Real>>> vals((size_t)nb);
		parallel_items((long)nb, [&](long ci) {
			Vi<D> pc = pos_of<D>(PosIdx(ci), box, zero);
			for (int a = 0; a < D; a++) pc[a] += cl[a];
			const PosIdx pci = index_of<D>(pc, iso.ccount, iso.coff);
			pcs[(size_t)ci] = pci;
			for (PosIdx leaf : iso.ch[pci].lists[lidx(0)]) {
				const Vi<D> pos = iso.pos_leaf(pci, leaf);
				if (inside<D>(pos, lo, lub)) vals[(size_t)ci].emplace_back(leaf, fn(pos));
			}
		});
		for (size_t ci = 0; ci < (size_t)nb; ci++)
			for (const auto& v : vals[ci]) delta_.track(v.second, pcs[ci], v.first, lidx(0));
		update_end();
	}
	void update_bounded(const Vi<D>& lo, const Vi<D>& hi, const Speed& s)
	{
		update_bounded_fn(lo, hi, [&](const Vi<D>& pos) { return speed(s, pos); });
	}

	/// delta(pos, val) (Surface.hpp:441-459).
	void delta(const Vi<D>& pos, Real v) { delta_.track(v, pos, lidx(0)); }

	/// update_end (Surface.hpp:404-430).
	void update_end()
	{
		calc_affected();
		iso.track_children(aff);
		delta_.track_children(aff);
		update_zero_layer(affb);
		Affected* pl = &aff;
		Affected* pb = &affb;
		bool changed = update_distance(*pl, *pb);
		flush_status_change();
		expand_narrow_band();
		int iters = 1;
		while (changed) {
			pl->reset(iso, false);
			std::swap(pl, pb);
			status.reset(aff, true);
			changed = update_distance(*pl, *pb);
			flush_status_change();
			expand_narrow_band();
			if (changed && ++iters % kMaxIterations == 0) throw_oscillation();
		}
	}

	/// The reference's convergence loops (Surface.hpp:420-428, 752-760) are unbounded; where
	/// the band meets the grid edge layer changes can oscillate forever. Both this oracle and
	/// the device engine stop after kMaxIterations iterations (this one by raising).
	static constexpr int kMaxIterations = 64;
	[[noreturn]] static void throw_oscillation()
	{
		throw Error(-14, "convergence loop did not terminate (oscillating layer changes)");
	}

	/// update_end_global (Surface.hpp:739-762).
	void update_end_global()
	{
		update_zero_layer(affb);
		bool changed = update_distance(iso, affb);
		flush_status_change();
		expand_narrow_band();
		if (changed) {
			Affected* pl = &affb;
			Affected* pb = &aff;
			int iters = 1;
			while (changed) {
				status.reset(iso, true);
				changed = update_distance(*pl, *pb);
				flush_status_change();
				expand_narrow_band();
				pl->reset(iso, false);
				std::swap(pl, pb);
				if (changed && ++iters % kMaxIterations == 0) throw_oscillation();
			}
		}
	}

	/// calc_affected (Surface.hpp:780-913).
	void calc_affected()
	{
		const int l0 = lidx(0);
		for (PosIdx pc : delta_.clists[l0])
			for (PosIdx leaf : delta_.ch[pc].lists[l0]) aff.track_lookup(pc, leaf, l0);

		std::array<std::vector<PosIdx>, NL> first, last;
		for (int ud = 1; ud <= L; ud++) {
			for (int l = 0; l < NL; l++) {
				const PosIdx nc = aff.clists[l].size();
				last[l].resize(nc);
				first[l].resize(nc, 0);
				for (PosIdx i = 0; i < nc; i++)
					last[l][i] = aff.ch[aff.clists[l][i]].lists[l].size();
			}
			for (int l = 0; l < NL; l++) {
				for (PosIdx ic = 0; ic < first[l].size(); ic++) {
					const PosIdx pc = aff.clists[l][ic];
					for (PosIdx in = first[l][ic]; in < last[l][ic]; in++) {
						const PosIdx leaf = aff.ch[pc].lists[l][in];
						const Vi<D> centre = aff.pos_leaf(pc, leaf);
						neighs<D>(centre, [&](const Vi<D>& pn) {
							const int lid = layer_of(iso.get(pn));
							if (inside_band(lid, L)) aff.track_lookup(pn, lidx(lid));
						});
					}
				}
			}
			for (int l = 0; l < NL; l++)
				for (PosIdx i = 0; i < first[l].size(); i++) first[l][i] = last[l][i];
		}
	}

	/// update_zero_layer (Surface.hpp:920-979). The reference runs the partitions across OpenMP
	/// threads (Surface.hpp:929); here each partition's new values are written by one thread and
	/// its layer changes recorded, then the status changes are made in the sequential order.
	void update_zero_layer(Affected& buf)
	{
		const int l0 = lidx(0);
		const std::vector<PosIdx> parts = delta_.clists[l0];
		std::vector<std::vector<std::pair<PosIdx, int>>> moved(parts.size());
		parallel_items((long)parts.size(), [&](long i) {
			const PosIdx pc = parts[(size_t)i];
			for (PosIdx leaf : delta_.ch[pc].lists[l0]) {
				const Real prev = iso.cget(pc, leaf);
				const Real d = delta_.cget(pc, leaf);
				const Real nw = prev + d;
				const int lid = layer_of(nw);
				iso.cset(pc, leaf, nw);
				if (lid != 0) moved[(size_t)i].emplace_back(leaf, lid);
			}
		});
		for (size_t i = 0; i < parts.size(); i++)
			for (const auto& m : moved[i]) status_change(parts[i], m.first, 0, m.second, buf);
	}

	/// update_distance over all layers (Surface.hpp:989-1003).
	template <class Grid>
	bool update_distance(const Grid& g, Affected& buf)
	{
		bool changed = false;
		for (int id = -1; id >= -L; id--) changed |= update_distance(id, -1, g, buf);
		for (int id = 1; id <= L; id++) changed |= update_distance(id, 1, g, buf);
		return changed;
	}

	/// update_distance for one layer (Surface.hpp:1015-1125): Jacobi within the layer.
	template <class Grid>
	bool update_distance(int id, int side, const Grid& g, Affected& buf)
	{
		bool changed = false;
		const int li = lidx(id);
		const std::vector<PosIdx> parts = g.clists[li];
		// first pass across threads, as the reference runs it (Surface.hpp:1028-1073):
		// partition-local writes only, so the thread count changes nothing
		parallel_items((long)parts.size(), [&](long i) {
			const PosIdx pc = parts[(size_t)i];
			for (PosIdx leaf : g.ch[pc].lists[li]) {
				const Real d = distance(pc, leaf, side);
				delta_.child_track(d, pc, leaf, li);
			}
		});
		// second pass, across threads as the reference runs it (Surface.hpp:1075-1121): values
		// written per partition, layer changes recorded and then made in the sequential order
		std::vector<std::vector<std::pair<PosIdx, int>>> moved(parts.size());
		parallel_items((long)parts.size(), [&](long i) {
			const PosIdx pc = parts[(size_t)i];
			for (PosIdx leaf : g.ch[pc].lists[li]) {
				const Real d = delta_.cget(pc, leaf);
				const int lid = layer_of(d);
				iso.cset(pc, leaf, d);
				if (lid != id) moved[(size_t)i].emplace_back(leaf, lid);
			}
		});
		for (size_t i = 0; i < parts.size(); i++)
			for (const auto& m : moved[i])
				changed |= status_change(parts[i], m.first, id, m.second, buf);
		return changed;
	}

	/// status_change (Surface.hpp:1138-1178).
	bool status_change(PosIdx pc, PosIdx leaf, int from, int to, Affected& buf)
	{
		if (from == to) return false;
		const int cur = status.cget(pc, leaf);
		if (cur != L + 1)
			status.cset(pc, leaf, to);
		else
			status.track(to, pc, leaf, lidx(from));
		if (inside_band(to, L)) buf.track_lookup(pc, leaf, lidx(to));
		return true;
	}

	/// flush_status_change (Surface.hpp:1183-1244). The reference runs each from-layer's
	/// partitions across OpenMP threads (Surface.hpp:1195), the children lookup edits under a
	/// mutex. Here each partition's leaf edits (PGrid::retrack / untrack) run on one thread
	/// against its own copy of its children-lookup membership, its children-lookup calls are
	/// recorded, and the calls are then made in the sequential order (from-layer, status list
	/// order, leaf order), so the children lists come out as the sequential loop leaves them.
	void flush_status_change()
	{
		constexpr int N = NL;
		for (int from = -L; from <= L; from++) {
			const int lf = lidx(from);
			const std::vector<PosIdx> parts = status.clists[lf];
			// recorded children-lookup calls: list index, +1 = ctrack, -1 = cuntrack
			std::vector<std::vector<std::pair<int, int>>> calls(parts.size());
			parallel_items((long)parts.size(), [&](long i) {
				const PosIdx pc = parts[(size_t)i];
				auto& rec = calls[(size_t)i];
				std::array<bool, N> tracked;
				for (int l = 0; l < N; l++) tracked[l] = iso.ctracked(pc, l);
				auto ctrack = [&](int l) {
					rec.emplace_back(l, 1);
					tracked[l] = true;
				};
				auto cuntrack = [&](int l) {
					rec.emplace_back(l, -1);
					tracked[l] = false;
				};
				for (PosIdx leaf : status.ch[pc].lists[lf]) {
					const int to = status.cget(pc, leaf);
					if (inside_band(to, L)) {
						// PGrid::retrack (PartitionedMixin.hpp:519-558)
						const int lt = lidx(to);
						iso.luntrack(pc, leaf, lf);
						iso.ltrack(pc, leaf, lt);
						const bool from_empty = iso.ch[pc].lists[lf].empty();
						if (!tracked[lt] || from_empty) {
							ctrack(lt);
							if (from_empty) cuntrack(lf);
						}
					} else {
						// PGrid::untrack (PartitionedMixin.hpp:489-517)
						const Real bgv = Real(to);
						iso.luntrack(pc, leaf, lf);
						iso.ch[pc].data[leaf] = bgv;
						if (iso.ch[pc].lists[lf].empty()) {
							cuntrack(lf);
							bool any = false;
							for (int l = 0; l < N; l++) any = any || tracked[l];
							if (!any) iso.deactivate(pc, bgv);
						}
					}
				}
			});
			for (size_t i = 0; i < parts.size(); i++)
				for (const auto& c : calls[i]) {
					if (c.second > 0)
						iso.ctrack(parts[i], c.first);
					else
						iso.cuntrack(parts[i], c.first);
				}
		}
	}

	/// expand_narrow_band (Surface.hpp:1249-1355).
	void expand_narrow_band()
	{
		for (int id : {-L, L}) {
			const int li = lidx(id);
			const int side = sgn(id);
			const std::vector<PosIdx> parts = status.clists[li];
			for (PosIdx pc : parts) {
				const std::vector<PosIdx> leaves = status.ch[pc].lists[li];
				for (PosIdx leaf : leaves) {
					if (status.cget(pc, leaf) != L * side - side) continue;
					const Vi<D> pos = status.pos_leaf(pc, leaf);
					neighs<D>(pos, [&](const Vi<D>& pn) {
						if (!iso.in_grid(pn)) return;
						Real dn = iso.get(pn);
						const int lf = layer_of(dn);
						if (inside_band(lf, L)) return;
						dn = distance(pn, dn, Real(side));
						iso.track(dn, pn, li);
					});
				}
			}
		}
	}

	/// distance (Surface.hpp:1364-1377, 1387-1440).
	Real distance(PosIdx pc, PosIdx leaf, int side) const
	{
		return distance(iso.pos_leaf(pc, leaf), iso.cget(pc, leaf), Real(side));
	}
	Real distance(const Vi<D>& pos, Real dist, Real dir) const
	{
		dist *= dir;
		neighs<D>(pos, [&](const Vi<D>& pn) {
			if (!iso.in_grid(pn)) return;
			const Real dn = iso.get(pn);
			if (dn * dir < dist) dist = dn * dir;
		});
		const Real dneigh = dist * dir;
		return dneigh + dir;
	}

	/// num_active_partitions (Surface.hpp:1733-1742).
	template <class G>
	static std::size_t num_active(const G& g)
	{
		std::size_t n = 0;
		for (int l = 0; l < NL; l++) n = std::max(n, g.clists[l].size());
		return n;
	}
};

// ---------------------------------------------------------------------------------------------
// Marching squares / cubes tables. These are the classic Lorensen-Cline tables in the corner,
// edge and vertex-ordering convention of the reference (PolyMixin.hpp:259-672); they must be
// identical for vertex indices and simplex index triplets to match. Shared with the device code
// through felt_b200/include/felt_gpu/mc_tables.h.
// ---------------------------------------------------------------------------------------------
}  // namespace fo

#include "../felt_b200/include/felt_gpu/mc_tables.h"

namespace fo {

template <int D> struct Geom;

template <> struct Geom<2> {
	static constexpr int num_edges = 4;
	static Vi<2> corner(int i) { return {fg_mc2_corner[i][0], fg_mc2_corner[i][1]}; }
	static Vi<2> edge_off(int e) { return {fg_mc2_edge[e][0], fg_mc2_edge[e][1]}; }
	static int edge_axis(int e) { return fg_mc2_edge[e][2]; }
	static unsigned edge_mask(int m) { return fg_mc2_edge_mask(m); }
	/// Simplex vertex order. Rows are 4 entries wide; the reference reads past a full row into
	/// the next one (Poly.hpp:259), so indexing is done in the flat table.
	static int order(int m, int i) { return fg_mc2_order_flat[m * 4 + i]; }
	static Vi<2> spx_offset() { return {0, 0}; }
};

template <> struct Geom<3> {
	static constexpr int num_edges = 12;
	static Vi<3> corner(int i) { return {fg_mc3_corner[i][0], fg_mc3_corner[i][1], fg_mc3_corner[i][2]}; }
	static Vi<3> edge_off(int e) { return {fg_mc3_edge[e][0], fg_mc3_edge[e][1], fg_mc3_edge[e][2]}; }
	static int edge_axis(int e) { return fg_mc3_edge[e][3]; }
	static unsigned edge_mask(int m) { return fg_mc3_edge_mask(m); }
	static int order(int m, int i) { return fg_mc3_order(m, i); }
	static Vi<3> spx_offset() { return {0, 0, -1}; }
};

/// interp (NumericMixin.hpp:403-481) of a grid at a real position: corners gathered in bit
/// order, reduced axis 0 first.
template <int D, class Grid, class Real>
Real field_interp(const Grid& iso, const std::array<Real, D>& p)
{
	Vi<D> fl;
	std::array<Real, D> pc;
	for (int ax = 0; ax < D; ax++) {
		const Real f = std::floor(p[ax]);
		fl[ax] = int(f);
		pc[ax] = p[ax] - f;
	}
	Real v[1 << D];
	for (int i = 0; i < (1 << D); i++) {
		Vi<D> q = fl;
		for (int ax = 0; ax < D; ax++) q[ax] += (i >> ax) & 1;
		v[i] = iso.get(q);
	}
	int n = 1 << D;
	while (n > 1) {
		const int axis = D - __builtin_ctz(unsigned(n));
		const Real t = pc[axis];
		for (int i = 0; i < n / 2; i++) {
			const Real lo = v[2 * i], hi = v[2 * i + 1];
			v[i] = t * hi + (Real(1) - t) * lo;
		}
		n >>= 1;
	}
	return v[0];
}

/// grad (NumericMixin.hpp:188-231) at a real position: the probe coordinate is stepped -1, +2,
/// -1 in float, so it can drift by rounding, exactly as in the reference.
template <int D, class Grid, class Real>
std::array<Real, D> field_grad_f(const Grid& iso, const std::array<Real, D>& p)
{
	std::array<Real, D> g;
	const Real centre = field_interp<D>(iso, p);
	std::array<Real, D> t = p;
	for (int ax = 0; ax < D; ax++) {
		Real back = centre, fwd = centre;
		int order = 0;
		t[ax] -= 1;
		if (inside<D>(t, iso.off, iso.hi)) {
			back = field_interp<D>(iso, t);
			order++;
		}
		t[ax] += 2;
		if (inside<D>(t, iso.off, iso.hi)) {
			fwd = field_interp<D>(iso, t);
			order++;
		}
		t[ax] -= 1;
		g[ax] = order != 0 ? (fwd - back) / Real(order) : Real(0);
	}
	for (int ax = 0; ax < D; ax++) g[ax] = g[ax] / Real(1);
	return g;
}

/// The Numeric API at a real position (NumericMixin.hpp:165-355 with Pos = float: get is interp,
/// inside the float bounds test), into out in this order: grad (189-231), gradF (279-298), gradB
/// (308-326), gradC (335-355), gradE (243-270), each D values, then divergence (165-175), curv
/// (72-156) and the interpolated value (403-481). Each function steps its own copy of the
/// position as the reference's does (grad, gradC, gradE: -1, +2, -1 per axis; gradF: +1, -1;
/// gradB: -1, +1): in float a step and its undo need not cancel, and the drift carries over to
/// the next axes, so the samples of one function are not those of another.
template <int D, class Grid>
void field_numeric(const Grid& iso, const std::array<float, D>& p, float* out)
{
	using P = std::array<float, D>;
	const auto get = [&](const P& q) { return field_interp<D>(iso, q); };
	const float centre = get(p);
	float* gf = out + D;
	float* gb = out + 2 * D;
	float* gc = out + 3 * D;
	float* ge = out + 4 * D;
	const std::array<float, D> g = field_grad_f<D>(iso, p);
	for (int a = 0; a < D; a++) out[a] = g[a];
	P t = p;
	for (int a = 0; a < D; a++) {
		t[a] += 1;
		gf[a] = get(t) - centre;
		t[a] -= 1;
	}
	t = p;
	for (int a = 0; a < D; a++) {
		t[a] -= 1;
		gb[a] = centre - get(t);
		t[a] += 1;
	}
	t = p;
	for (int a = 0; a < D; a++) {
		t[a] -= 1;
		const float back = get(t);
		t[a] += 2;
		const float fwd = get(t);
		t[a] -= 1;
		gc[a] = (fwd - back) / 2.0f;
	}
	t = p;
	for (int a = 0; a < D; a++) {
		t[a] -= 1;
		const float back = get(t);
		t[a] += 2;
		const float fwd = get(t);
		t[a] -= 1;
		ge[a] = std::min(fwd - centre, 0.0f) + std::max(centre - back, 0.0f);
	}
	std::array<float, D> diff;
	for (int a = 0; a < D; a++) diff[a] = gf[a] - gb[a];
	out[5 * D] = eigen_sum<float, D>(diff);
	out[5 * D + 1] = curv_at<D, float>(get, p);
	out[5 * D + 2] = centre;
}

/// Eigen normalize(): divide by sqrt(x0^2 + (x1^2 + x2^2)) when that is positive.
template <int D, class Real = float>
void eigen_normalize(std::array<Real, D>& v)
{
	std::array<Real, D> sq;
	for (int ax = 0; ax < D; ax++) sq[ax] = v[ax] * v[ax];
	const Real z = eigen_sum<Real, D>(sq);
	if (z > 0) {
		const Real r = std::sqrt(z);
		for (int ax = 0; ax < D; ax++) v[ax] = v[ax] / r;
	}
}

template <int D, class Real = float>
struct Vertex {
	std::array<Real, D> pos;
	std::array<Real, D> norm;  // 3D only
};

/// Polys<Surface> (Polys.hpp:1-229) over Poly::Single children (Poly.hpp:17-368). Real is
/// the surface's arithmetic type: float as in the reference, double for the FP64 run of the
/// same method that error figures are taken against.
template <int D, int L, class Real = float>
class Polys {
public:
	using Surf = Surface<D, L, Real>;
	using V = Vertex<D, Real>;
	static constexpr int NL = Surf::NL;
	using IdxTuple = std::array<std::size_t, D>;

	struct Single {
		Vi<D> off{}, size{};
		std::vector<IdxTuple> cache;  // empty when inactive
		std::vector<std::size_t> lkp;
		std::vector<std::size_t> list;
		std::vector<V> vtxs;
		std::vector<std::array<unsigned, D>> spxs;
		bool active() const { return !cache.empty(); }
	};

	/// SingleListSingleIdx lookup over partitions (Lookup.hpp:17-57, LookupMixin.hpp:97-185).
	struct Changes {
		std::vector<std::size_t> lkp;
		std::vector<std::size_t> list;
		void track(std::size_t i)
		{
			if (lkp[i] != NUL) return;
			lkp[i] = list.size();
			list.push_back(i);
		}
		void untrack(std::size_t i)
		{
			std::size_t& at = lkp[i];
			if (at == NUL) return;
			const std::size_t last = list.size() - 1;
			if (at < last) {
				list[at] = list[last];
				lkp[list[last]] = at;
			}
			at = NUL;
			list.pop_back();
		}
		void reset()
		{
			for (std::size_t i : list) lkp[i] = NUL;
			list.clear();
		}
	};

	const Surf* s;
	std::vector<Single> ch;
	Changes a, b;
	Changes* pend;
	Changes* done;

	/// Polys ctor (Polys.hpp:58-84); child geometry from Poly::Single::resize (Poly.hpp:124-133).
	explicit Polys(const Surf& surf) : s(&surf)
	{
		const std::size_t n = surf.iso.nchildren();
		ch.resize(n);
		for (std::size_t i = 0; i < n; i++)
			for (int ax = 0; ax < D; ax++) {
				ch[i].off[ax] = surf.iso.ch[i].off[ax] - 1;
				ch[i].size[ax] = surf.iso.csize[ax] + 2;
			}
		a.lkp.assign(n, NUL);
		b.lkp.assign(n, NUL);
		pend = &a;
		done = &b;
	}

	/// notify (Polys.hpp:92-133).
	void notify()
	{
		for (int li = 0; li <= NL; li += NL - 1) {
			for (std::size_t pc : s->delta_.clists[li]) {
				bool act = ch[pc].active();
				for (int lj = 0; !act && lj <= NL; lj += NL - 1) act = s->iso.ctracked(pc, lj);
				if (act)
					pend->track(pc);
				else
					pend->untrack(pc);
			}
		}
		for (int li = 0; li <= NL; li += NL - 1)
			for (std::size_t pc : s->status.clists[li])
				if (ch[pc].active()) pend->track(pc);
	}

	/// march (Polys.hpp:138-165).
	void march()
	{
		// across threads as in the reference (Polys.hpp:140): each pending partition's child is
		// its own state, and marching only reads the surface
		const std::vector<std::size_t>& todo = pend->list;
		parallel_items((long)todo.size(), [&](long i) {
			const std::size_t pc = todo[(size_t)i];
			Single& c = ch[pc];
			if (s->iso.active(pc)) {
				if (c.active())
					reset(c);
				else
					activate(c);
				march(pc);
			} else if (c.active()) {
				deactivate(c);
			}
		}, 1);
		std::swap(pend, done);
		pend->reset();
	}

	/// invalidate (Polys.hpp:171-191). The Polys children lookup is never populated by the
	/// reference, so only the isogrid's outermost partition lists contribute.
	void invalidate()
	{
		pend->reset();
		for (int li = 0; li <= NL; li += NL - 1)
			for (std::size_t pc : s->iso.clists[li]) pend->track(pc);
	}

	const std::vector<std::size_t>& changes() const { return done->list; }

	/// Poly::Single::march on one partition's child (Poly.hpp:138-147), activating or resetting
	/// it first as Polys::march does (Polys.hpp:149-154).
	void march_partition(std::size_t pc)
	{
		Single& c = ch[pc];
		if (c.active())
			reset(c);
		else
			activate(c);
		march(pc);
	}

	// --- Poly::Single ---
	std::size_t vol(const Single& c) const
	{
		std::size_t v = 1;
		for (int ax = 0; ax < D; ax++) v *= std::size_t(c.size[ax]);
		return v;
	}
	void activate(Single& c)
	{
		IdxTuple nul;
		nul.fill(NUL);
		c.cache.assign(vol(c), nul);
		c.lkp.assign(vol(c), NUL);
	}
	/// Poly::Single::reset (Poly.hpp:106-111).
	void reset(Single& c)
	{
		IdxTuple nul;
		nul.fill(NUL);
		for (std::size_t i : c.list) {
			c.cache[i] = nul;
			c.lkp[i] = NUL;
		}
		c.list.clear();
		c.vtxs.clear();
		c.spxs.clear();
	}
	/// Poly::Single::deactivate (Poly.hpp:95-101).
	void deactivate(Single& c)
	{
		std::vector<IdxTuple>().swap(c.cache);
		std::vector<std::size_t>().swap(c.lkp);
		std::vector<std::size_t>().swap(c.list);
		std::vector<V>().swap(c.vtxs);
		std::vector<std::array<unsigned, D>>().swap(c.spxs);
	}

	/// Poly::Single::march (Poly.hpp:138-147): all leaves of all layer lists, in list order.
	void march(std::size_t pc)
	{
		for (int l = 0; l < NL; l++)
			for (std::size_t leaf : s->iso.ch[pc].lists[l]) spx(pc, s->iso.pos_leaf(pc, leaf));
	}

	/// Poly::Single::spx (Poly.hpp:198-287).
	void spx(std::size_t pc, const Vi<D>& pos)
	{
		Single& c = ch[pc];
		Vi<D> pcalc;
		const Vi<D> so = Geom<D>::spx_offset();
		for (int ax = 0; ax < D; ax++) pcalc[ax] = pos[ax] - so[ax];
		unsigned mask = 0;
		for (int i = 0; i < (1 << D); i++) {
			const Vi<D> co = Geom<D>::corner(i);
			Vi<D> p;
			for (int ax = 0; ax < D; ax++) p[ax] = pcalc[ax] + co[ax];
			const Real v = s->iso.get(p);
			mask = mask | (unsigned(v > 0) << i);
		}
		const unsigned emask = Geom<D>::edge_mask(int(mask));
		if (Geom<D>::order(int(mask), 0) == -1) return;
		unsigned vidx[Geom<D>::num_edges];
		for (int e = 0; e < Geom<D>::num_edges; e++) {
			if ((emask >> e) & 1) {
				const Vi<D> eo = Geom<D>::edge_off(e);
				Vi<D> pa;
				for (int ax = 0; ax < D; ax++) pa[ax] = pcalc[ax] + eo[ax];
				vidx[e] = unsigned(idx(c, pa, Geom<D>::edge_axis(e)));
			}
		}
		for (int o = 0; Geom<D>::order(int(mask), o) != -1; o += D) {
			std::array<unsigned, D> sp;
			for (int k = 0; k < D; k++) sp[k] = vidx[Geom<D>::order(int(mask), o + k)];
			c.spxs.push_back(sp);
		}
	}

	/// Poly::Single::idx (Poly.hpp:296-346).
	std::size_t idx(Single& c, const Vi<D>& pa, int axis)
	{
		const std::size_t ci = index_of<D>(pa, c.size, c.off);
		const std::size_t cached = c.cache[ci][axis];
		if (cached != NUL) return cached;
		Vi<D> pb = pa;
		pb[axis] += 1;
		const Real va = s->iso.get(pa);
		const Real vb = s->iso.get(pb);
		const Real eps = Real(std::numeric_limits<float>::epsilon());
		V vtx;
		if (std::fabs(va) <= eps) {
			vtx = make_vertex_i(pa);
		} else if (std::fabs(vb) <= eps) {
			vtx = make_vertex_i(pb);
		} else {
			Real mu;
			if (std::fabs(va - vb) <= eps)
				mu = Real(0.5);
			else
				mu = va / (va - vb);
			std::array<Real, D> vc;
			for (int ax = 0; ax < D; ax++) {
				const Real fa = Real(pa[ax]);
				const Real fb = Real(pb[ax]);
				vc[ax] = fa + (fb - fa) * mu;
			}
			vtx = make_vertex_f(vc);
		}
		const std::size_t id = c.vtxs.size();
		c.vtxs.push_back(vtx);
		c.cache[ci][axis] = id;
		if (c.lkp[ci] == NUL) {
			c.lkp[ci] = c.list.size();
			c.list.push_back(ci);
		}
		return id;
	}

	// --- 3D vertex normals: Vertex ctor (PolyMixin.hpp:142-148) ---

	Real interp(const std::array<Real, D>& p) const { return field_interp<D>(s->iso, p); }

	/// grad (NumericMixin.hpp:188-231) at an integer position.
	std::array<Real, D> grad_i(const Vi<D>& p) const
	{
		std::array<Real, D> g;
		const Real centre = s->iso.get(p);
		Vi<D> t = p;
		for (int ax = 0; ax < D; ax++) {
			Real back = centre, fwd = centre;
			int order = 0;
			t[ax] -= 1;
			if (s->iso.in_grid(t)) {
				back = s->iso.get(t);
				order++;
			}
			t[ax] += 2;
			if (s->iso.in_grid(t)) {
				fwd = s->iso.get(t);
				order++;
			}
			t[ax] -= 1;
			g[ax] = order != 0 ? (fwd - back) / Real(order) : Real(0);
		}
		for (int ax = 0; ax < D; ax++) g[ax] = g[ax] / Real(1);
		return g;
	}
	std::array<Real, D> grad_f(const std::array<Real, D>& p) const
	{
		return field_grad_f<D>(s->iso, p);
	}
	static void normalize(std::array<Real, D>& v) { eigen_normalize<D, Real>(v); }
	V make_vertex_i(const Vi<D>& p) const
	{
		V v;
		for (int ax = 0; ax < D; ax++) v.pos[ax] = Real(p[ax]);
		if (D == 3) {
			v.norm = grad_i(p);
			normalize(v.norm);
		} else {
			v.norm.fill(Real(0));
		}
		return v;
	}
	V make_vertex_f(const std::array<Real, D>& p) const
	{
		V v;
		v.pos = p;
		if (D == 3) {
			v.norm = grad_f(p);
			normalize(v.norm);
		} else {
			v.norm.fill(Real(0));
		}
		return v;
	}
};


// ---------------------------------------------------------------------------------------------
// Raycasting (Surface.hpp:468-616, 1450-1598)
// ---------------------------------------------------------------------------------------------

/// Surface::ray: the zero-curve point a ray hits, or ray_miss (FLT_MAX in every component).
/// Eigen semantics restated in FP32: ParametrizedLine::intersectionPoint(Hyperplane(n, d)) =
/// o + t*dir with t = -(d + n.o) / (n.dir); pointAt(t) = o + dir*t; dot products and squared
/// norms sum as x0 + (x1 + x2). Candidate partitions are ordered by squared distance from the
/// origin, ties in the order they were found (std::sort leaves that order unspecified).
template <int D, int L>
class Raycast {
public:
	using Surf = Surface<D, L, float>;
	using Vf = std::array<float, D>;
	static constexpr int NL = Surf::NL;
	static constexpr float TINY = 0.00001f;  // Surface.hpp:67
	static constexpr int MAX_CONVERGE_STEPS = 100;
	// bounds on the reference's open loops (never reached with a unit-length direction)
	static constexpr int MAX_MARCH = 1 << 16;

	explicit Raycast(const Surf& s) : s(&s) {}

	static Vf miss()
	{
		Vf m;
		m.fill(std::numeric_limits<float>::max());
		return m;
	}

	Vf ray(const Vf& o, const Vf& dir) const
	{
		const auto& iso = s->iso;
		if (inside<D>(o, iso.off, iso.hi)) {
			Vi<D> pc;
			for (int a = 0; a < D; a++) pc[a] = int(o[a]);  // Eigen cast<int>: truncation
			const Vf h = ray_child(o, dir, iso.pidx_child(pc));
			if (h != miss()) return h;
		}
		std::vector<std::pair<Vf, PosIdx>> hits;
		for (int dim = 0; dim < D; dim++) {
			const float dd = float(sgn(dir[dim]));
			if (dd == 0) continue;
			float pp = round_to_next(dim, dd, o[dim]);
			Vf plane{};
			plane[dim] = pp;
			if (!inside<D>(plane, iso.off, iso.hi)) {
				float pg;
				if (dd == -1) {
					pg = float(iso.off[dim] + iso.size[dim]);
					if (pp < pg) continue;
				} else {
					pg = float(iso.off[dim]);
					if (pp > pg) continue;
				}
				plane[dim] = pg;
			}
			check_track(hits, o, dir, dim, dd, plane[dim]);
			pp = round_to_next(dim, dd, plane[dim]);
			if (pp != plane[dim]) {
				plane[dim] = pp;
				if (!check_track(hits, o, dir, dim, dd, plane[dim])) continue;
			}
			const float cs = float(iso.csize[dim]);
			for (int it = 0; it < MAX_MARCH; it++) {
				plane[dim] += dd * cs;
				if (!check_track(hits, o, dir, dim, dd, plane[dim])) break;
			}
		}
		std::stable_sort(hits.begin(), hits.end(), [&](const auto& a, const auto& b) {
			return dist2(a.first, o) < dist2(b.first, o);
		});
		hits.erase(std::unique(hits.begin(), hits.end(),
		                       [](const auto& a, const auto& b) { return a.second == b.second; }),
		           hits.end());
		for (const auto& h : hits) {
			const Vf p = ray_child(h.first, dir, h.second);
			if (p != miss()) return p;
		}
		return miss();
	}

private:
	const Surf* s;

	static float dot(const Vf& a, const Vf& b)
	{
		Vf m;
		for (int i = 0; i < D; i++) m[i] = a[i] * b[i];
		return eigen_sum<float, D>(m);
	}
	static float dist2(const Vf& p, const Vf& o)
	{
		Vf d;
		for (int i = 0; i < D; i++) d[i] = p[i] - o[i];
		return dot(d, d);
	}
	static int sgn(float v) { return (0.0f < v) - (v < 0.0f); }

	/// round_to_next (Surface.hpp:1582-1599).
	float round_to_next(int dim, float dd, float pos) const
	{
		const auto& iso = s->iso;
		float p = (pos - float(iso.off[dim])) / float(iso.csize[dim]);
		p = dd == -1.0f ? std::floor(p) : std::ceil(p);
		p *= float(iso.csize[dim]);
		p += float(iso.off[dim]);
		return p;
	}

	/// ray_check_track_child (Surface.hpp:1539-1577) for the plane x[dim] = plane_pos.
	bool check_track(std::vector<std::pair<Vf, PosIdx>>& hits, const Vf& o, const Vf& dir,
	                 int dim, float dd, float plane_pos) const
	{
		const auto& iso = s->iso;
		// Hyperplane(normal = -dd e_dim, offset = plane_pos * dd)
		const float nd = -dd, off = plane_pos * dd;
		const float t = -(off + nd * o[dim]) / (nd * dir[dim]);
		Vf p;
		for (int i = 0; i < D; i++) p[i] = o[i] + dir[i] * t;
		for (int i = 0; i < D; i++) p[i] = p[i] + dir[i] * TINY;
		for (int i = 0; i < D; i++)
			if ((dir[i] > 0 && p[i] > float(iso.size[i])) || (dir[i] < 0 && p[i] < float(iso.off[i])))
				return false;
		if (!inside<D>(p, iso.off, iso.hi)) return true;
		Vi<D> pf;
		for (int i = 0; i < D; i++) pf[i] = int(std::floor(p[i]));
		const PosIdx pc = iso.pidx_child(pf);
		const auto& lists = iso.ch[pc].lists;
		if (lists[Surf::lidx(0)].size() || lists[Surf::lidx(1)].size() || lists[Surf::lidx(-1)].size())
			hits.emplace_back(p, pc);
		return true;
	}

	/// ray within one partition (Surface.hpp:1450-1530).
	Vf ray_child(Vf pos, const Vf& dir, PosIdx pc) const
	{
		const auto& iso = s->iso;
		Vi<D> chi;
		for (int a = 0; a < D; a++) chi[a] = iso.ch[pc].off[a] + iso.csize[a];
		const Vf o = pos;
		float t = 0;
		for (int it = 0; it < MAX_MARCH && inside<D>(pos, iso.ch[pc].off, chi); it++) {
			if (s->layer_of(field_interp<D>(iso, pos)) == 0) {
				Vf n = field_grad_f<D>(iso, pos);
				eigen_normalize<D>(n);
				if (dot(n, dir) < 0) {
					for (int k = 0; k < MAX_CONVERGE_STEPS; k++) {
						const float dist = field_interp<D>(iso, pos);
						for (int a = 0; a < D; a++) pos[a] = pos[a] - n[a] * dist;
						if (!inside<D>(pos, iso.off, iso.hi)) return miss();
						if (std::abs(dist) <= TINY || dot(n, dir) >= 0) break;
						n = field_grad_f<D>(iso, pos);
						eigen_normalize<D>(n);
					}
					return pos;
				}
			}
			t += 0.5f;
			for (int a = 0; a < D; a++) pos[a] = o[a] + dir[a] * t;
		}
		return miss();
	}
};

}  // namespace fo
