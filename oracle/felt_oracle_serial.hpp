// TEST INFRASTRUCTURE ONLY (the oracle): Surface::save / Surface::load (Surface.hpp:180-196) in
// the reference's file format, restated for the oracle's grids.
//
// The reference writes its isogrid with cereal's BinaryOutputArchive (PartitionedMixin.hpp:
// 692-708; cereal as vendored under include/Felt/ThirdParty/cereal). That archive writes
// arithmetic values as their raw little-endian bytes, a std::vector as a uint64 element count
// followed by its elements (one raw block when they are arithmetic), and nothing for class
// boundaries (the serialize hooks are unversioned). Eigen matrices go through Felt's own hook
// (PartitionedMixin.hpp:717-738): int32 rows, int32 cols, then the coefficients as a
// std::vector. Felt's Tuple<T, N> is an Eigen column vector, so per-list tuples take that form
// too. The hooks, in the order they write:
//
//   IsoGrid (Partitioned::Tracked::Numeric, Partitioned.hpp:151-158)
//     f32 background                                (Partitioned::Access, PartitionedMixin.hpp:581-586)
//     VecDi child_size, Children children           (Partitioned::Children, PartitionedMixin.hpp:93-97)
//     VecDi size, offset, offset + size              (Grid::Size, GridMixin.hpp:255-259)
//     f32 dx, VecDi pos_min, VecDi pos_max           (Numeric::Spatial, NumericMixin.hpp:55-60)
//   Children (Tracked::MultiListMultiIdxByRef, Tracked.hpp:209-217)
//     Child background                               (Grid::Activate, GridMixin.hpp:46-50)
//     u64 count, Child[count]                        (Grid::Data, GridMixin.hpp:135-139)
//     ChildrenLookup                                 (Tracked::LookupInterface, TrackedMixin.hpp:119-123)
//     VecDi size, offset, offset + size (children grid)
//   ChildrenLookup (Lookup::MultiListMultiIdx, Lookup.hpp:228-236)
//     IdxTuple background (null in every list); u64 count, IdxTuple[count] (each child's position
//     in each children list); ListTuple children lists (LookupMixin.hpp:421-425); VecDi x3
//   Child (Tracked::LazyMultiListSingleIdxByValue, Tracked.hpp:53-60)
//     f32 background; u64 count, f32[count] values (0 when inactive); LeafLookup; VecDi x3
//   LeafLookup (Lookup::LazyMultiListSingleIdx, Lookup.hpp:170-177)
//     u64 background (null); u64 count, u64[count] (each leaf's position in its list, or null);
//     ListTuple leaf lists (LookupMixin.hpp:248-252); VecDi x3
//   VecDi     = i32 D, i32 1, u64 D, i32[D]
//   IdxTuple  = i32 N, i32 1, u64 N, u64[N]
//   ListTuple = i32 N, i32 1, u64 N, then N x (u64 len, u64[len])
//
// The children grid's background child is built from a background value alone (PartitionedMixin
// .hpp:59-68, Tracked.hpp:46-48), so the reference never sets its two sets of size/offset
// vectors and writes indeterminate bytes there; they are written here as zeros and ignored when
// read. Null is SIZE_MAX (Common.hpp:102).
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "felt_oracle.hpp"

namespace fo {

struct ByteOut {
	std::vector<uint8_t>& b;
	template <class T>
	void raw(const T& v)
	{
		const auto* p = reinterpret_cast<const uint8_t*>(&v);
		b.insert(b.end(), p, p + sizeof(T));
	}
	void i32(int32_t v) { raw(v); }
	void u64(uint64_t v) { raw(v); }
	void f32(float v) { raw(v); }
};

struct ByteIn {
	const uint8_t* p;
	size_t n, at = 0;
	template <class T>
	T raw()
	{
		if (n - at < sizeof(T)) throw Error(-1, "truncated surface file");
		T v;
		std::memcpy(&v, p + at, sizeof(T));
		at += sizeof(T);
		return v;
	}
	int32_t i32() { return raw<int32_t>(); }
	uint64_t u64() { return raw<uint64_t>(); }
	float f32() { return raw<float>(); }
	void expect_i32(int32_t v, const char* what)
	{
		if (i32() != v) throw Error(-1, (std::string("surface file: unexpected ") + what).c_str());
	}
	void expect_u64(uint64_t v, const char* what)
	{
		if (u64() != v) throw Error(-1, (std::string("surface file: unexpected ") + what).c_str());
	}
};

template <int D>
void put_vec(ByteOut& w, const Vi<D>& v)
{
	w.i32(D);
	w.i32(1);
	w.u64(D);
	for (int a = 0; a < D; a++) w.i32(v[a]);
}

template <int D>
Vi<D> get_vec(ByteIn& r)
{
	r.expect_i32(D, "vector rows");
	r.expect_i32(1, "vector cols");
	r.expect_u64(D, "vector length");
	Vi<D> v;
	for (int a = 0; a < D; a++) v[a] = r.i32();
	return v;
}

template <int D>
Vi<D> vsum(const Vi<D>& a, const Vi<D>& b)
{
	Vi<D> c;
	for (int i = 0; i < D; i++) c[i] = a[i] + b[i];
	return c;
}

template <int N>
void put_lists(ByteOut& w, const std::array<std::vector<PosIdx>, N>& lists)
{
	w.i32(N);
	w.i32(1);
	w.u64(N);
	for (int l = 0; l < N; l++) {
		w.u64(lists[l].size());
		for (PosIdx x : lists[l]) w.u64(x);
	}
}

template <int N>
std::array<std::vector<PosIdx>, N> get_lists(ByteIn& r, PosIdx bound)
{
	r.expect_i32(N, "list count");
	r.expect_i32(1, "list cols");
	r.expect_u64(N, "list count");
	std::array<std::vector<PosIdx>, N> lists;
	for (int l = 0; l < N; l++) {
		const uint64_t len = r.u64();
		if (len > bound) throw Error(-1, "surface file: list longer than its grid");
		lists[l].resize(len);
		for (auto& x : lists[l]) {
			x = r.u64();
			if (x >= bound) throw Error(-1, "surface file: list entry out of range");
		}
	}
	return lists;
}

/// Child::serialize and its LeafLookup (Tracked.hpp:53-60, Lookup.hpp:170-177).
template <int D, int N, class T>
void put_child(ByteOut& w, const typename PGrid<D, N, T>::Child& c, const Vi<D>& csize,
               bool sizes)
{
	const Vi<D> zero{};
	const Vi<D>& sz = sizes ? csize : zero;
	const Vi<D>& of = sizes ? c.off : zero;
	const Vi<D> hi = sizes ? vsum<D>(c.off, csize) : zero;
	w.f32(float(c.bg));
	w.u64(c.data.size());
	for (T v : c.data) w.f32(float(v));
	w.u64(NUL);
	w.u64(c.lkp.size());
	for (PosIdx x : c.lkp) w.u64(x);
	put_lists<N>(w, c.lists);
	put_vec<D>(w, sz);
	put_vec<D>(w, of);
	put_vec<D>(w, hi);
	put_vec<D>(w, sz);
	put_vec<D>(w, of);
	put_vec<D>(w, hi);
}

/// Surface::save (Surface.hpp:180-183): the isogrid in the reference's cereal binary layout.
template <int D, int L>
void save_surface(const Surface<D, L, float>& s, std::vector<uint8_t>& out)
{
	constexpr int N = 2 * L + 1;
	using G = PGrid<D, N, float>;
	const G& g = s.iso;
	ByteOut w{out};
	w.f32(g.bg);
	put_vec<D>(w, g.csize);
	// children grid: its background child, every child, its lookup, its size
	typename G::Child bgc;
	bgc.bg = g.bg;
	put_child<D, N, float>(w, bgc, g.csize, false);
	w.u64(g.ch.size());
	for (const auto& c : g.ch) put_child<D, N, float>(w, c, g.csize, true);
	w.i32(N);
	w.i32(1);
	w.u64(N);
	for (int l = 0; l < N; l++) w.u64(NUL);
	w.u64(g.cpos.size());
	for (const auto& t : g.cpos) {
		w.i32(N);
		w.i32(1);
		w.u64(N);
		for (int l = 0; l < N; l++) w.u64(t[l]);
	}
	put_lists<N>(w, g.clists);
	for (int k = 0; k < 2; k++) {
		put_vec<D>(w, g.ccount);
		put_vec<D>(w, g.coff);
		put_vec<D>(w, vsum<D>(g.coff, g.ccount));
	}
	put_vec<D>(w, g.size);
	put_vec<D>(w, g.off);
	put_vec<D>(w, g.hi);
	w.f32(1.0f);
	put_vec<D>(w, g.off);
	put_vec<D>(w, g.hi);
}

/// What a surface file holds before it is loaded: D from its first vector (the child size), N
/// from the background child's leaf lookup, the grid size from the fixed-size tail (grid size,
/// offset, offset + size, dx, pos_min, pos_max).
inline void peek_surface(const uint8_t* p, size_t n, int& dims, int& lists, int* size, int* part)
{
	ByteIn r{p, n};
	r.f32();
	dims = r.i32();
	if (dims != 2 && dims != 3) throw Error(-1, "surface file: dimension not 2 or 3");
	r.expect_i32(1, "vector cols");
	r.expect_u64((uint64_t)dims, "vector length");
	for (int a = 0; a < dims; a++) part[a] = r.i32();
	r.f32();                      // background child: background
	if (r.u64() != 0) throw Error(-1, "surface file: active background child");
	r.u64();                      // its lookup's background
	if (r.u64() != 0) throw Error(-1, "surface file: active background lookup");
	lists = r.i32();
	if (lists < 3 || lists > 9 || lists % 2 == 0) throw Error(-1, "surface file: bad list count");
	const size_t vec = 16 + 4 * (size_t)dims;
	const size_t tail = 5 * vec + 4;
	if (n < tail + r.at) throw Error(-1, "truncated surface file");
	ByteIn t{p, n, n - tail};
	t.expect_i32(dims, "vector rows");
	t.expect_i32(1, "vector cols");
	t.expect_u64((uint64_t)dims, "vector length");
	for (int a = 0; a < dims; a++) {
		size[a] = t.i32();
		if (size[a] <= 0 || part[a] <= 0) throw Error(-1, "surface file: bad sizes");
	}
}

/// Surface::load (Surface.hpp:185-196) into s, which must have been constructed with the
/// file's size and child size (the other grids start empty, as the reference's constructor
/// from an isogrid makes them).
template <int D, int L>
void load_surface(Surface<D, L, float>& s, const uint8_t* p, size_t n)
{
	constexpr int N = 2 * L + 1;
	using G = PGrid<D, N, float>;
	G& g = s.iso;
	ByteIn r{p, n};
	if (r.f32() != float(L + 1)) throw Error(-1, "surface file: background is not L+1");
	if (get_vec<D>(r) != g.csize) throw Error(-1, "surface file: child size differs");
	auto get_child = [&](typename G::Child& c, bool check_geom) {
		c.bg = r.f32();
		const uint64_t nd = r.u64();
		if (nd != 0 && nd != (uint64_t)g.bv) throw Error(-1, "surface file: child data size");
		c.data.resize(nd);
		for (auto& v : c.data) v = r.f32();
		r.expect_u64(NUL, "leaf lookup background");
		const uint64_t nl = r.u64();
		if (nl != nd) throw Error(-1, "surface file: leaf lookup size");
		c.lkp.resize(nl);
		for (auto& x : c.lkp) {
			x = r.u64();
			if (x != NUL && x >= (uint64_t)g.bv) throw Error(-1, "surface file: leaf lookup entry");
		}
		c.lists = get_lists<N>(r, (PosIdx)g.bv);
		for (int k = 0; k < 2; k++) {
			const Vi<D> sz = get_vec<D>(r), of = get_vec<D>(r);
			get_vec<D>(r);
			if (check_geom && (sz != g.csize || of != c.off))
				throw Error(-1, "surface file: child geometry differs");
		}
		if (nd == 0)
			for (const auto& l : c.lists)
				if (!l.empty()) throw Error(-1, "surface file: lists in an inactive child");
		for (int l = 0; l < N; l++)
			for (size_t i = 0; i < c.lists[l].size(); i++)
				if (c.lkp[c.lists[l][i]] != i) throw Error(-1, "surface file: lookup and list disagree");
	};
	typename G::Child bgc;
	get_child(bgc, false);
	if (r.u64() != g.ch.size()) throw Error(-1, "surface file: child count differs");
	for (auto& c : g.ch) get_child(c, true);
	r.expect_i32(N, "tuple rows");
	r.expect_i32(1, "tuple cols");
	r.expect_u64(N, "tuple length");
	for (int l = 0; l < N; l++) r.expect_u64(NUL, "children lookup background");
	r.expect_u64(g.cpos.size(), "children lookup size");
	for (auto& t : g.cpos) {
		r.expect_i32(N, "tuple rows");
		r.expect_i32(1, "tuple cols");
		r.expect_u64(N, "tuple length");
		for (int l = 0; l < N; l++) t[l] = r.u64();
	}
	g.clists = get_lists<N>(r, (PosIdx)g.ch.size());
	for (int l = 0; l < N; l++)
		for (size_t i = 0; i < g.clists[l].size(); i++)
			if (g.cpos[g.clists[l][i]][l] != i) throw Error(-1, "surface file: children lookup and list disagree");
	for (PosIdx pc = 0; pc < g.cpos.size(); pc++)
		for (int l = 0; l < N; l++) {
			const PosIdx i = g.cpos[pc][l];
			if (i != NUL && (i >= g.clists[l].size() || g.clists[l][i] != pc))
				throw Error(-1, "surface file: children lookup entry");
		}
	for (int k = 0; k < 2; k++) {
		if (get_vec<D>(r) != g.ccount || get_vec<D>(r) != g.coff) throw Error(-1, "surface file: children grid differs");
		get_vec<D>(r);
	}
	if (get_vec<D>(r) != g.size || get_vec<D>(r) != g.off) throw Error(-1, "surface file: grid differs");
	get_vec<D>(r);
	if (r.f32() != 1.0f) throw Error(-1, "surface file: dx other than 1");
	get_vec<D>(r);
	get_vec<D>(r);
	if (r.at != r.n) throw Error(-1, "surface file: trailing bytes");
}

}  // namespace fo
