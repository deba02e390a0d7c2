// C++ facade over the C ABI (include/felt_gpu.h) with the shape of Felt's template API:
// felt_gpu::Surface<D,L> for Felt::Surface<D,L> (include/Felt/Surface.hpp) and
// felt_gpu::Polys<D,L> for Felt::Polys<Surface> (include/Felt/Polys.hpp).
//
// Differences a caller of the reference meets:
//  - Positions are std::array<int, D> and ray points std::array<float, D> (the reference uses
//    Eigen VecDi / VecDf); index order is the same.
//  - update() takes either a builtin speed (Speed: constant, curvature, hashed noise and their
//    sum) or, in a translation unit compiled by nvcc that includes felt_gpu/device.cuh, any
//    __device__ functor with one of the reference's three signatures.
//  - isogrid() queries are member functions here (get, snapshot, layer_list, partition_list).
//  - Errors the reference leaves undefined (or asserts in debug builds) throw felt_gpu::Error
//    with the C ABI status code.
//  - Calls are asynchronous on the surface's CUDA stream; queries synchronise.
#pragma once

#include <array>
#include <cstdint>
#include <istream>
#include <iterator>
#include <ostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "felt_gpu.h"

#ifdef __CUDACC__
#include "device.cuh"
#define FELT_GPU_DEVICE_FUNCTORS 1
#endif

namespace felt_gpu {

struct Error : std::runtime_error {
	int code;
	Error(int c, const char* what) : std::runtime_error(what ? what : "felt_gpu error"), code(c)
	{
	}
};

inline void check(int rc)
{
	if (rc != FG_OK) throw Error(rc, fg_last_error());
}

template <int D>
using VecDi = std::array<int, D>;
template <int D>
using VecDf = std::array<float, D>;

/// Builtin speed: delta = [a * curv] + [n * h(pos, seed)] + [c], FP32, left to right.
struct Speed {
	fg_speed s{};
	static Speed constant(float c)
	{
		Speed r;
		r.s.kind = FG_SPEED_CONST;
		r.s.c = c;
		return r;
	}
	Speed& curvature(float a)
	{
		s.kind |= FG_SPEED_CURV;
		s.a = a;
		return *this;
	}
	Speed& noise(float n, uint32_t seed)
	{
		s.kind |= FG_SPEED_NOISE;
		s.n = n;
		s.seed = seed;
		return *this;
	}
	Speed& plus(float c)
	{
		s.kind |= FG_SPEED_CONST;
		s.c = c;
		return *this;
	}
};

template <int D, int L>
class Surface {
public:
	static constexpr int Dims = D;
	static constexpr int Layers = L;

	/// Surface(size, size_partition) (Surface.hpp:163-173).
	explicit Surface(const VecDi<D>& size, const VecDi<D>& part = filled(8),
	                 const fg_config* cfg = nullptr)
	    : size_(size)
	{
		check(fg_surface_create(D, L, size.data(), part.data(), cfg, &h_));
	}
	~Surface()
	{
		if (h_) fg_surface_destroy(h_);
	}
	Surface(const Surface&) = delete;
	Surface& operator=(const Surface&) = delete;
	Surface(Surface&& o) noexcept : h_(o.h_), size_(o.size_) { o.h_ = nullptr; }

	/// save(ostream) (Surface.hpp:180-183): the surface file, in the reference's format.
	void save(std::ostream& out) const
	{
		size_t n = 0;
		check(fg_save(h_, nullptr, 0, &n));
		std::vector<uint8_t> buf(n);
		check(fg_save(h_, buf.data(), buf.size(), &n));
		out.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)buf.size());
		out.flush();
	}

	/// load(istream) (Surface.hpp:185-196): a new surface from a surface file; its dimensions
	/// and layers must be this type's.
	static Surface load(std::istream& in, const fg_config* cfg = nullptr)
	{
		std::vector<uint8_t> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
		fg_surface* h = nullptr;
		check(fg_load(buf.data(), buf.size(), cfg, &h));
		int dims = 0, layers = 0;
		VecDi<D> size{}, part{};
		int sz[3], pt[3];
		const int rc = fg_surface_info(h, &dims, &layers, sz, pt);
		if (rc != FG_OK || dims != D || layers != L) {
			fg_surface_destroy(h);
			throw Error(FG_ERR_ARG, "surface file of another dimension or layer count");
		}
		for (int a = 0; a < D; a++) size[a] = sz[a];
		return Surface(h, size);
	}

	/// layer_idx(id) (Surface.hpp:672-675).
	static constexpr int layer_idx(int id) { return id + L; }

	/// seed(pos) (Surface.hpp:207-241).
	void seed(const VecDi<D>& pos) { check(fg_seed(h_, pos.data())); }

	/// update(fn) with a builtin speed (Surface.hpp:254-294).
	void update(const Speed& sp) { check(fg_update_builtin(h_, &sp.s)); }

#ifdef FELT_GPU_DEVICE_FUNCTORS
	/// update(fn) with a __device__ functor (felt_gpu/device.cuh).
	template <class Fn>
	void update(const Fn& fn)
	{
		check(update_device<D, L>(h_, fn));
	}
#endif

	/// update(lo, hi, fn) bounded update (Surface.hpp:310-386).
	void update(const VecDi<D>& lo, const VecDi<D>& hi, const Speed& sp)
	{
		check(fg_update_bounded(h_, lo.data(), hi.data(), &sp.s));
	}

	/// update_start / delta / update_end (Surface.hpp:393-459).
	void update_start() { check(fg_update_start(h_)); }
	void delta(const VecDi<D>& pos, float v) { check(fg_delta(h_, pos.data(), v)); }
	void update_end() { check(fg_update_end(h_)); }

	/// isogrid().get(pos).
	float get(const VecDi<D>& pos) const
	{
		float v = 0.0f;
		check(fg_get(h_, pos.data(), &v));
		return v;
	}

	/// ray(origin, dir) (Surface.hpp:468-616): the point where the ray meets the zero curve,
	/// or ray_miss.
	VecDf<D> ray(const VecDf<D>& origin, const VecDf<D>& dir) const
	{
		VecDf<D> hit{};
		check(fg_ray(h_, origin.data(), dir.data(), 1, hit.data()));
		return hit;
	}

	/// ray() for n rays in one launch: origins, dirs and hits hold n*D floats (host memory).
	void rays(const float* origins, const float* dirs, size_t n, float* hits) const
	{
		check(fg_ray(h_, origins, dirs, n, hits));
	}

	/// Surface::ray_miss (Surface.hpp:62-64): FLT_MAX in every component.
	static VecDf<D> ray_miss()
	{
		VecDf<D> m;
		m.fill(std::numeric_limits<float>::max());
		return m;
	}

	/// isogrid().snapshot()->data(): dense, row-major, last axis fastest.
	std::vector<float> snapshot() const
	{
		size_t n = 1;
		for (int a = 0; a < D; a++) n *= (size_t)size_[a];
		std::vector<float> out(n);
		check(fg_snapshot(h_, out.data(), n, 0));
		return out;
	}

	/// isogrid().children().get(part).lookup().list(layer_idx).
	std::vector<uint32_t> layer_list(size_t part, int layer) const
	{
		return fetch([&](uint32_t* o, size_t c, size_t* n) {
			return fg_layer_list(h_, part, layer, o, c, n);
		});
	}
	/// isogrid().children().lookup().list(layer_idx).
	std::vector<uint32_t> partition_list(int layer) const
	{
		return fetch([&](uint32_t* o, size_t c, size_t* n) {
			return fg_partition_list(h_, layer, o, c, n);
		});
	}
	/// delta(layer_idx), status_change(layer_idx), affected(): partition lists.
	std::vector<uint32_t> delta_partitions(int layer) const
	{
		return fetch([&](uint32_t* o, size_t c, size_t* n) {
			return fg_delta_partitions(h_, layer, o, c, n);
		});
	}
	std::vector<uint32_t> status_partitions(int layer) const
	{
		return fetch([&](uint32_t* o, size_t c, size_t* n) {
			return fg_status_partitions(h_, layer, o, c, n);
		});
	}
	std::vector<uint32_t> affected_partitions(int layer) const
	{
		return fetch([&](uint32_t* o, size_t c, size_t* n) {
			return fg_affected_partitions(h_, layer, o, c, n);
		});
	}

	/// stats() (Surface.hpp:623-629): active isogrid and delta partitions.
	std::pair<size_t, size_t> stats() const
	{
		size_t a = 0, b = 0;
		check(fg_stats(h_, &a, &b));
		return {a, b};
	}

	const VecDi<D>& size() const { return size_; }
	fg_surface* handle() const { return h_; }

private:
	static VecDi<D> filled(int v)
	{
		VecDi<D> r;
		r.fill(v);
		return r;
	}
	template <class F>
	static std::vector<uint32_t> fetch(F f)
	{
		size_t n = 0;
		check(f(nullptr, 0, &n));
		std::vector<uint32_t> out(n);
		if (n) check(f(out.data(), n, &n));
		return out;
	}

	Surface(fg_surface* h, const VecDi<D>& size) : h_(h), size_(size) {}

	fg_surface* h_ = nullptr;
	VecDi<D> size_;
};

/// Polys<Surface> (Polys.hpp:58-201). The surface must outlive it, as in the reference.
template <int D, int L>
class Polys {
public:
	struct Child {
		std::vector<float> vtxs;     // per vertex D position floats, then D normal floats in 3D
		std::vector<uint32_t> spxs;  // D local vertex indices per simplex
		bool active = false;
	};

	explicit Polys(const Surface<D, L>& s) { check(fg_polys_create(s.handle(), &h_)); }
	~Polys()
	{
		if (h_) fg_polys_destroy(h_);
	}
	Polys(const Polys&) = delete;
	Polys& operator=(const Polys&) = delete;

	void notify() { check(fg_polys_notify(h_)); }
	void march() { check(fg_polys_march(h_)); }
	void invalidate() { check(fg_polys_invalidate(h_)); }
	std::vector<uint32_t> changes() const
	{
		size_t n = 0;
		check(fg_polys_changes(h_, nullptr, 0, &n));
		std::vector<uint32_t> out(n);
		if (n) check(fg_polys_changes(h_, out.data(), n, &n));
		return out;
	}
	/// children().get(part).{vtxs(), spxs(), is_active()}.
	Child child(size_t part) const
	{
		Child c;
		size_t nv = 0, ns = 0;
		int active = 0;
		check(fg_polys_partition(h_, part, nullptr, 0, nullptr, 0, &nv, &ns, &active));
		constexpr int VF = D == 3 ? 2 * D : D;
		c.vtxs.resize(nv * VF);
		c.spxs.resize(ns * D);
		check(fg_polys_partition(h_, part, c.vtxs.data(), c.vtxs.size(), c.spxs.data(),
		                         c.spxs.size(), &nv, &ns, &active));
		c.active = active != 0;
		return c;
	}
	fg_polys* handle() const { return h_; }

private:
	fg_polys* h_ = nullptr;
};

}  // namespace felt_gpu
