// C ABI over the CPU oracle (felt_oracle.hpp), mirroring include/felt_gpu.h with an `fo_`
// prefix so that tests can drive the oracle and the device engine through identical call
// sequences and compare their dumps. TEST INFRASTRUCTURE ONLY.
#include "felt_oracle.hpp"
#include "felt_oracle_serial.hpp"

#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>

namespace {

thread_local std::string g_err;

struct SurfBase {
	int dims = 0, layers = 0;
	virtual ~SurfBase() = default;
	virtual void seed(const int* p) = 0;
	virtual void update(const fo::Speed& s) = 0;
	virtual void update_bounded(const int* lo, const int* hi, const fo::Speed& s) = 0;
	virtual void update_start() = 0;
	virtual void delta(const int* p, float v) = 0;
	virtual void update_end() = 0;
	virtual void snapshot(float* dst, size_t n) = 0;
	virtual float get(const int* p) = 0;
	virtual size_t nparts() = 0;
	virtual void partitions(int* csize, int* coff) = 0;
	virtual const std::vector<size_t>* leaf_list(size_t part, int l) = 0;
	virtual const std::vector<size_t>* plist(int which, int l) = 0;
	virtual const std::vector<size_t>* affected_list(size_t part, int l) = 0;
	virtual void pstate(size_t part, int* active, float* bg) = 0;
	virtual void stats(size_t* a, size_t* b) = 0;
	virtual size_t band_size() = 0;
	virtual void curv(const int* p, float* out) = 0;
	virtual void numeric(const int* p, float* out) = 0;
	virtual void numeric_f(const float* p, float* out) = 0;
	virtual void ray(const float* o, const float* d, float* out) = 0;
	virtual void save(std::vector<uint8_t>& out) = 0;
	virtual void geometry(int* size, int* part) = 0;
	virtual void load(const uint8_t* p, size_t n) = 0;
	/// The dense snapshot in the surface's own arithmetic type, widened to double.
	virtual void snapshot64(double* dst, size_t n) = 0;
	virtual bool fp64() const = 0;
};

struct PolysBase {
	virtual ~PolysBase() = default;
	virtual void notify() = 0;
	virtual void march() = 0;
	virtual void invalidate() = 0;
	virtual void march_partition(size_t pc) = 0;
	virtual const std::vector<size_t>& changes() = 0;
	virtual void part(size_t pc, float* vtx, size_t vcap, uint32_t* spx, size_t scap, size_t* nv,
	                  size_t* ns, int* active) = 0;
	virtual void totals(size_t* nv, size_t* ns) = 0;
	/// part() with the vertices in the surface's own arithmetic type, widened to double.
	virtual void part64(size_t pc, double* vtx, size_t vcap, size_t* nv) = 0;
};

/// One oracle surface. Real = float is the reference's arithmetic; Real = double is the FP64
/// run of the same method (the reference hard-wires float, Impl/Common.hpp:40), which error
/// figures are taken against. Raycasting, surface files and the real-position Numeric API exist
/// for float surfaces only.
template <int D, int L, class Real = float>
struct Surf : SurfBase {
	fo::Surface<D, L, Real> s;
	static constexpr bool F32 = std::is_same<Real, float>::value;
	[[noreturn]] static void f32_only() { throw fo::Error(-1, "not available in an FP64 run"); }
	static fo::Vi<D> v(const int* p)
	{
		fo::Vi<D> r;
		for (int a = 0; a < D; a++) r[a] = p[a];
		return r;
	}
	Surf(const int* size, const int* part) : s(v(size), v(part))
	{
		this->dims = D;
		this->layers = L;
	}
	void seed(const int* p) override { s.seed(v(p)); }
	void update(const fo::Speed& sp) override { s.update(sp); }
	void update_bounded(const int* lo, const int* hi, const fo::Speed& sp) override
	{
		s.update_bounded(v(lo), v(hi), sp);
	}
	void update_start() override { s.update_start(); }
	void delta(const int* p, float val) override { s.delta(v(p), val); }
	void update_end() override { s.update_end(); }
	void snapshot(float* dst, size_t n) override
	{
		// PartitionedMixin.hpp:642-660: row-major over the grid, each node via get().
		fo::Vi<D> size = s.iso.size, off = s.iso.off;
		size_t tot = 1;
		for (int a = 0; a < D; a++) tot *= size_t(size[a]);
		if (n < tot) throw fo::Error(-13, "snapshot buffer too small");
		for (size_t i = 0; i < tot; i++) dst[i] = float(s.iso.get(fo::pos_of<D>(i, size, off)));
	}
	void snapshot64(double* dst, size_t n) override
	{
		fo::Vi<D> size = s.iso.size, off = s.iso.off;
		size_t tot = 1;
		for (int a = 0; a < D; a++) tot *= size_t(size[a]);
		if (n < tot) throw fo::Error(-13, "snapshot buffer too small");
		for (size_t i = 0; i < tot; i++) dst[i] = double(s.iso.get(fo::pos_of<D>(i, size, off)));
	}
	bool fp64() const override { return !F32; }
	float get(const int* p) override { return float(s.iso.get(v(p))); }
	size_t nparts() override { return s.iso.nchildren(); }
	void partitions(int* csize, int* coff) override
	{
		for (int a = 0; a < D; a++) {
			csize[a] = s.iso.ccount[a];
			coff[a] = s.iso.coff[a];
		}
	}
	const std::vector<size_t>* leaf_list(size_t part, int l) override
	{
		return &s.iso.ch[part].lists[l];
	}
	const std::vector<size_t>* plist(int which, int l) override
	{
		switch (which) {
		case 0: return &s.iso.clists[l];
		case 1: return &s.delta_.clists[l];
		case 2: return &s.status.clists[l];
		case 3: return &s.aff.clists[l];
		default: return nullptr;
		}
	}
	const std::vector<size_t>* affected_list(size_t part, int l) override
	{
		return &s.aff.ch[part].lists[l];
	}
	void pstate(size_t part, int* active, float* bg) override
	{
		*active = s.iso.active(part) ? 1 : 0;
		*bg = float(s.iso.ch[part].bg);
	}
	void stats(size_t* a, size_t* b) override
	{
		*a = s.num_active(s.iso);
		*b = s.num_active(s.delta_);
	}
	size_t band_size() override
	{
		size_t n = 0;
		for (int l = 0; l < 2 * L + 1; l++)
			for (size_t pc : s.iso.clists[l]) n += s.iso.ch[pc].lists[l].size();
		return n;
	}
	void curv(const int* p, float* out) override { *out = float(s.curv(v(p))); }
	void numeric(const int* p, float* out) override
	{
		Real r[5 * D + 1];
		s.numeric(v(p), r);
		for (int i = 0; i < 5 * D + 1; i++) out[i] = float(r[i]);
	}
	void numeric_f(const float* p, float* out) override
	{
		if constexpr (F32) {
			std::array<float, D> q;
			for (int a = 0; a < D; a++) q[a] = p[a];
			fo::field_numeric<D>(s.iso, q, out);
		} else {
			f32_only();
		}
	}
	void save(std::vector<uint8_t>& out) override
	{
		if constexpr (F32)
			fo::save_surface<D, L>(s, out);
		else
			f32_only();
	}
	void geometry(int* size, int* part) override
	{
		for (int a = 0; a < D; a++) {
			size[a] = s.iso.size[a];
			part[a] = s.iso.csize[a];
		}
	}
	void load(const uint8_t* p, size_t n) override
	{
		if constexpr (F32)
			fo::load_surface<D, L>(s, p, n);
		else
			f32_only();
	}
	void ray(const float* o, const float* d, float* out) override
	{
		if constexpr (F32) {
			std::array<float, D> oo, dd;
			for (int a = 0; a < D; a++) {
				oo[a] = o[a];
				dd[a] = d[a];
			}
			const auto h = fo::Raycast<D, L>(s).ray(oo, dd);
			for (int a = 0; a < D; a++) out[a] = h[a];
		} else {
			f32_only();
		}
	}
};

template <int D, int L, class Real = float>
struct PolysImpl : PolysBase {
	fo::Polys<D, L, Real> p;
	explicit PolysImpl(const fo::Surface<D, L, Real>& s) : p(s) {}
	void notify() override { p.notify(); }
	void march() override { p.march(); }
	void invalidate() override { p.invalidate(); }
	void march_partition(size_t pc) override { p.march_partition(pc); }
	const std::vector<size_t>& changes() override { return p.changes(); }
	void part(size_t pc, float* vtx, size_t vcap, uint32_t* spx, size_t scap, size_t* nv,
	          size_t* ns, int* active) override
	{
		const auto& c = p.ch[pc];
		*nv = c.vtxs.size();
		*ns = c.spxs.size();
		*active = c.active() ? 1 : 0;
		const size_t per = (D == 3) ? 2 * D : D;
		for (size_t i = 0; i < c.vtxs.size() && (i + 1) * per <= vcap; i++) {
			for (int a = 0; a < D; a++) vtx[i * per + a] = float(c.vtxs[i].pos[a]);
			if (D == 3)
				for (int a = 0; a < D; a++) vtx[i * per + D + a] = float(c.vtxs[i].norm[a]);
		}
		for (size_t i = 0; i < c.spxs.size() && (i + 1) * D <= scap; i++)
			for (int a = 0; a < D; a++) spx[i * D + a] = c.spxs[i][a];
	}
	void part64(size_t pc, double* vtx, size_t vcap, size_t* nv) override
	{
		const auto& c = p.ch[pc];
		*nv = c.vtxs.size();
		const size_t per = (D == 3) ? 2 * D : D;
		for (size_t i = 0; i < c.vtxs.size() && (i + 1) * per <= vcap; i++) {
			for (int a = 0; a < D; a++) vtx[i * per + a] = double(c.vtxs[i].pos[a]);
			if (D == 3)
				for (int a = 0; a < D; a++) vtx[i * per + D + a] = double(c.vtxs[i].norm[a]);
		}
	}
	void totals(size_t* nv, size_t* ns) override
	{
		*nv = 0;
		*ns = 0;
		for (const auto& c : p.ch) {
			*nv += c.vtxs.size();
			*ns += c.spxs.size();
		}
	}
};

struct PolysHandle {
	std::unique_ptr<PolysBase> impl;
};

template <class F>
int guard(F&& f)
{
	try {
		f();
		return 0;
	} catch (const fo::Error& e) {
		g_err = e.what();
		return e.code;
	} catch (const std::exception& e) {
		g_err = e.what();
		return -1;
	}
}

SurfBase* make(int D, int L, const int* size, const int* part, bool fp64 = false)
{
#define FO_CASE(d, l)                                                          \
	if (D == d && L == l) {                                                    \
		if (fp64) return new Surf<d, l, double>(size, part);                   \
		return new Surf<d, l>(size, part);                                     \
	}
	FO_CASE(2, 1) FO_CASE(2, 2) FO_CASE(2, 3) FO_CASE(2, 4)
	FO_CASE(3, 1) FO_CASE(3, 2) FO_CASE(3, 3) FO_CASE(3, 4)
#undef FO_CASE
	return nullptr;
}

PolysBase* make_polys(SurfBase* s)
{
#define FO_CASE(d, l)                                                                         \
	if (s->dims == d && s->layers == l) {                                                     \
		if (s->fp64()) return new PolysImpl<d, l, double>(static_cast<Surf<d, l, double>*>(s)->s); \
		return new PolysImpl<d, l>(static_cast<Surf<d, l>*>(s)->s);                           \
	}
	FO_CASE(2, 1) FO_CASE(2, 2) FO_CASE(2, 3) FO_CASE(2, 4)
	FO_CASE(3, 1) FO_CASE(3, 2) FO_CASE(3, 3) FO_CASE(3, 4)
#undef FO_CASE
	return nullptr;
}

fo::Speed to_speed(const int kind, const float c, const float a, const float n, uint32_t seed)
{
	return fo::Speed{kind, c, a, n, seed};
}

void put_list(const std::vector<size_t>& l, uint32_t* out, size_t cap, size_t* n)
{
	*n = l.size();
	for (size_t i = 0; i < l.size() && i < cap; i++) out[i] = uint32_t(l[i]);
}

/// A standalone leaf lookup (LookupMixin.hpp:298-386, MultiList::SingleIdx, 3 lists): one
/// partition covering a 3D grid of the given size and offset, for the Lookup golden tests.
struct LeafLookup {
	fo::PGrid<3, 3, float> g;
	LeafLookup(const int* size, const int* off)
	    : g({size[0], size[1], size[2]}, {off[0], off[1], off[2]}, {size[0], size[1], size[2]}, 0.0f)
	{
		g.activate(0);
	}
	size_t leaf(const int* pos) const
	{
		const fo::Vi<3> p{pos[0], pos[1], pos[2]};
		if (!g.in_grid(p)) throw fo::Error(-1, "position outside the lookup grid");
		return g.leaf_of(0, p);
	}
};

/// A standalone partitioned lookup (Partitioned::Lookup: PartitionedMixin.hpp:388-413 over
/// LookupMixin's children and leaf lists), for the partitioned Lookup golden test.
struct PartLookup {
	fo::PGrid<3, 3, float> g;
	PartLookup(const int* size, const int* off, const int* part)
	    : g({size[0], size[1], size[2]}, {off[0], off[1], off[2]}, {part[0], part[1], part[2]}, 0.0f)
	{
	}
	size_t child(const int* cpos) const
	{
		const fo::Vi<3> c{cpos[0], cpos[1], cpos[2]};
		for (int a = 0; a < 3; a++)
			if (c[a] < g.coff[a] || c[a] >= g.coff[a] + g.ccount[a])
				throw fo::Error(-1, "partition outside the children grid");
		return fo::index_of<3>(c, g.ccount, g.coff);
	}
	fo::Vi<3> pos(const int* p) const
	{
		const fo::Vi<3> q{p[0], p[1], p[2]};
		if (!g.in_grid(q)) throw fo::Error(-1, "position outside the grid");
		return q;
	}
};

}  // namespace

extern "C" {

struct fo_speed {
	int kind;
	float c, a, n;
	uint32_t seed;
};

const char* fo_last_error(void) { return g_err.c_str(); }

/// Threads of the parallel loops (the reference's seven OpenMP loops); results do not
/// depend on it. Returns the count in effect.
int fo_set_threads(int n)
{
	if (n > 0) fo::g_threads.store(n);
	return fo::g_threads.load();
}

int fo_surface_create(int dims, int layers, const int* size, const int* part, void** out)
{
	return guard([&] {
		SurfBase* s = make(dims, layers, size, part);
		if (!s) throw fo::Error(-1, "unsupported dims/layers");
		*out = s;
	});
}
/* The same surface computed in FP64 (Real = double): the method's error figures are taken
 * against it. Lists, dumps and polygons work as for fo_surface_create; raycasting, surface
 * files and the real-position Numeric API do not. */
int fo_surface_create64(int dims, int layers, const int* size, const int* part, void** out)
{
	return guard([&] {
		SurfBase* s = make(dims, layers, size, part, true);
		if (!s) throw fo::Error(-1, "unsupported dims/layers");
		*out = s;
	});
}
int fo_snapshot64(void* s, double* dst, size_t n)
{
	return guard([&] { static_cast<SurfBase*>(s)->snapshot64(dst, n); });
}
/* Surface::save (Surface.hpp:180-183): the surface file, min(n, cap) bytes into buf, the
 * full length in *n. */
int fo_save(void* s, uint8_t* buf, size_t cap, size_t* n)
{
	return guard([&] {
		std::vector<uint8_t> out;
		static_cast<SurfBase*>(s)->save(out);
		*n = out.size();
		if (buf) std::memcpy(buf, out.data(), std::min(cap, out.size()));
	});
}

/* Surface::load (Surface.hpp:185-196): a new surface from a surface file. */
int fo_load(const uint8_t* p, size_t n, void** out)
{
	return guard([&] {
		int dims = 0, lists = 0, size[3] = {0, 0, 0}, part[3] = {0, 0, 0};
		fo::peek_surface(p, n, dims, lists, size, part);
		std::unique_ptr<SurfBase> s(make(dims, (lists - 1) / 2, size, part));
		if (!s) throw fo::Error(-1, "unsupported dims/layers");
		s->load(p, n);
		*out = s.release();
	});
}

/* Dimensions, layers, grid size and partition size of a surface. */
int fo_info(void* s, int* dims, int* layers, int* size, int* part)
{
	return guard([&] {
		SurfBase* b = static_cast<SurfBase*>(s);
		*dims = b->dims;
		*layers = b->layers;
		b->geometry(size, part);
	});
}

int fo_surface_destroy(void* s)
{
	delete static_cast<SurfBase*>(s);
	return 0;
}
int fo_seed(void* s, const int* pos)
{
	return guard([&] { static_cast<SurfBase*>(s)->seed(pos); });
}
int fo_update_builtin(void* s, const fo_speed* sp)
{
	return guard([&] {
		static_cast<SurfBase*>(s)->update(to_speed(sp->kind, sp->c, sp->a, sp->n, sp->seed));
	});
}
int fo_update_bounded(void* s, const int* lo, const int* hi, const fo_speed* sp)
{
	return guard([&] {
		static_cast<SurfBase*>(s)->update_bounded(lo, hi,
		                                         to_speed(sp->kind, sp->c, sp->a, sp->n, sp->seed));
	});
}
int fo_update_start(void* s)
{
	return guard([&] { static_cast<SurfBase*>(s)->update_start(); });
}
int fo_delta(void* s, const int* pos, float v)
{
	return guard([&] { static_cast<SurfBase*>(s)->delta(pos, v); });
}
int fo_delta_n(void* s, const int* pos, const float* v, size_t n)
{
	return guard([&] {
		SurfBase* b = static_cast<SurfBase*>(s);
		for (size_t i = 0; i < n; i++) b->delta(pos + i * size_t(b->dims), v[i]);
	});
}
int fo_update_end(void* s)
{
	return guard([&] { static_cast<SurfBase*>(s)->update_end(); });
}
int fo_snapshot(void* s, float* dst, size_t n)
{
	return guard([&] { static_cast<SurfBase*>(s)->snapshot(dst, n); });
}
int fo_get(void* s, const int* pos, float* out)
{
	return guard([&] { *out = static_cast<SurfBase*>(s)->get(pos); });
}
/* Surface::ray for n rays (origins, directions: n*D floats); hits n*D floats, FLT_MAX when
 * missed. */
int fo_ray(void* s, const float* origins, const float* dirs, size_t n, float* hits)
{
	return guard([&] {
		SurfBase* b = static_cast<SurfBase*>(s);
		const int D = b->dims;
		// rays are independent reads of the surface (Surface::ray is const): spread over the
		// configured threads, each writing only its own hit
		fo::parallel_items((long)n, [&](long i) {
			b->ray(origins + i * D, dirs + i * D, hits + i * D);
		});
	});
}

/* The Numeric API at a node: grad, gradF, gradB, gradC, gradE (dims values each), divergence. */
int fo_numeric(void* s, const int* pos, float* out)
{
	return guard([&] { static_cast<SurfBase*>(s)->numeric(pos, out); });
}

int fo_numeric_f(void* s, const float* pos, float* out)
{
	return guard([&] { static_cast<SurfBase*>(s)->numeric_f(pos, out); });
}

int fo_curv(void* s, const int* pos, float* out)
{
	return guard([&] { static_cast<SurfBase*>(s)->curv(pos, out); });
}
/* curv over a dense grid (values row-major, `bg` outside), for the stencil golden tests. */
int fo_curv_dense(int dims, const float* vals, const int* size, const int* off, float bg,
                  const int* pos, float* out)
{
	return guard([&] {
		auto run = [&](auto dtag) {
			constexpr int D = decltype(dtag)::value;
			fo::Vi<D> sz, of, hi, p;
			for (int a = 0; a < D; a++) {
				sz[a] = size[a];
				of[a] = off[a];
				hi[a] = off[a] + size[a];
				p[a] = pos[a];
			}
			auto get = [&](const fo::Vi<D>& q) {
				if (!fo::inside<D>(q, of, hi)) return bg;
				return vals[fo::index_of<D>(q, sz, of)];
			};
			*out = fo::curv_at<D, float>(get, p);
		};
		if (dims == 2)
			run(std::integral_constant<int, 2>{});
		else if (dims == 3)
			run(std::integral_constant<int, 3>{});
		else
			throw fo::Error(-1, "dims");
	});
}
/* The Numeric API over a dense grid (values row-major, `bg` outside) at a node (real = 0; pos
 * holds whole numbers) or a real position (real = 1), for the stencil golden tests: 5*dims + 3
 * values as fo_numeric_f returns them. */
int fo_numeric_dense(int dims, const float* vals, const int* size, const int* off, float bg,
                     const float* pos, int real, float* out)
{
	return guard([&] {
		auto run = [&](auto dtag) {
			constexpr int D = decltype(dtag)::value;
			struct Dense {
				const float* vals;
				fo::Vi<D> sz, off, hi;
				float bg;
				float get(const fo::Vi<D>& q) const
				{
					if (!fo::inside<D>(q, off, hi)) return bg;
					return vals[fo::index_of<D>(q, sz, off)];
				}
			} g{vals, {}, {}, {}, bg};
			for (int a = 0; a < D; a++) {
				g.sz[a] = size[a];
				g.off[a] = off[a];
				g.hi[a] = off[a] + size[a];
			}
			if (real) {
				std::array<float, D> p;
				for (int a = 0; a < D; a++) p[a] = pos[a];
				fo::field_numeric<D>(g, p, out);
				return;
			}
			fo::Vi<D> p;
			for (int a = 0; a < D; a++) p[a] = (int)pos[a];
			const auto get = [&](const fo::Vi<D>& q) { return g.get(q); };
			fo::numeric_at<D, float>(get, [&](const fo::Vi<D>& q) { return fo::inside<D>(q, g.off, g.hi); },
			                         p, out);
			out[5 * D + 1] = fo::curv_at<D, float>(get, p);
			out[5 * D + 2] = g.get(p);
		};
		if (dims == 2)
			run(std::integral_constant<int, 2>{});
		else if (dims == 3)
			run(std::integral_constant<int, 3>{});
		else
			throw fo::Error(-1, "dims");
	});
}
/* The standalone leaf lookup of the Lookup golden tests: track / untrack a position in list l
 * (0..2), reset, read list l, and read a position's index in its list (-1 for none). */
int fo_lookup_create(const int* size, const int* off, void** out)
{
	return guard([&] { *out = new LeafLookup(size, off); });
}
int fo_lookup_destroy(void* h)
{
	delete static_cast<LeafLookup*>(h);
	return 0;
}
int fo_lookup_index(void* h, const int* pos, size_t* out)
{
	return guard([&] { *out = static_cast<LeafLookup*>(h)->leaf(pos); });
}
int fo_lookup_track(void* h, const int* pos, int l)
{
	return guard([&] {
		auto* k = static_cast<LeafLookup*>(h);
		k->g.ltrack(0, k->leaf(pos), l);
	});
}
int fo_lookup_untrack(void* h, const int* pos, int l)
{
	return guard([&] {
		auto* k = static_cast<LeafLookup*>(h);
		k->g.luntrack(0, k->leaf(pos), l);
	});
}
int fo_lookup_reset(void* h)
{
	return guard([&] { static_cast<LeafLookup*>(h)->g.child_reset(0, false); });
}
int fo_lookup_list(void* h, int l, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] { put_list(static_cast<LeafLookup*>(h)->g.ch[0].lists[l], out, cap, n); });
}
int fo_lookup_get(void* h, const int* pos, long long* out)
{
	return guard([&] {
		auto* k = static_cast<LeafLookup*>(h);
		const size_t at = k->g.ch[0].lkp[k->leaf(pos)];
		*out = at == fo::NUL ? -1 : (long long)at;
	});
}
/* The standalone partitioned lookup: track a position in list l, the children list l, a
 * partition's index in children list l (-1 for none), a partition's leaf list l and a
 * position's index in its partition's list (-1 for none). Partitions are children-grid
 * positions. */
int fo_plookup_create(const int* size, const int* off, const int* part, void** out)
{
	return guard([&] { *out = new PartLookup(size, off, part); });
}
int fo_plookup_destroy(void* h)
{
	delete static_cast<PartLookup*>(h);
	return 0;
}
int fo_plookup_track(void* h, const int* pos, int l)
{
	return guard([&] {
		auto* k = static_cast<PartLookup*>(h);
		k->g.track_lookup(k->pos(pos), l);
	});
}
int fo_plookup_child_index(void* h, const int* part, size_t* out)
{
	return guard([&] { *out = static_cast<PartLookup*>(h)->child(part); });
}
int fo_plookup_children(void* h, int l, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] { put_list(static_cast<PartLookup*>(h)->g.clists[l], out, cap, n); });
}
int fo_plookup_child_get(void* h, const int* part, int l, long long* out)
{
	return guard([&] {
		auto* k = static_cast<PartLookup*>(h);
		const size_t at = k->g.cpos[k->child(part)][l];
		*out = at == fo::NUL ? -1 : (long long)at;
	});
}
int fo_plookup_leaves(void* h, const int* part, int l, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		auto* k = static_cast<PartLookup*>(h);
		put_list(k->g.ch[k->child(part)].lists[l], out, cap, n);
	});
}
int fo_plookup_leaf_get(void* h, const int* part, const int* pos, long long* out)
{
	return guard([&] {
		auto* k = static_cast<PartLookup*>(h);
		const size_t pc = k->child(part);
		const fo::Vi<3> q = k->pos(pos);
		if (k->g.pidx_child(q) != pc) throw fo::Error(-1, "position outside the partition");
		const auto& c = k->g.ch[pc];
		*out = -1;
		if (!c.lkp.empty()) {
			const size_t at = c.lkp[k->g.leaf_of(pc, q)];
			if (at != fo::NUL) *out = (long long)at;
		}
	});
}
/* The children-level lookup alone (LookupMixin.hpp:457-570, MultiList::MultiIdx: one index
 * per list), as a partitioned lookup with 1^3 partitions so that partitions are positions: for
 * the Lookup::Multi golden test. */
int fo_clookup_create(const int* size, const int* off, void** out)
{
	const int one[3] = {1, 1, 1};
	return guard([&] { *out = new PartLookup(size, off, one); });
}
int fo_clookup_track(void* h, const int* pos, int l)
{
	return guard([&] {
		auto* k = static_cast<PartLookup*>(h);
		k->g.ctrack(k->child(pos), l);
	});
}
int fo_clookup_untrack(void* h, const int* pos, int l)
{
	return guard([&] {
		auto* k = static_cast<PartLookup*>(h);
		k->g.cuntrack(k->child(pos), l);
	});
}
int fo_clookup_reset(void* h)
{
	return guard([&] {
		auto* k = static_cast<PartLookup*>(h);
		for (int l = 0; l < 3; l++) {
			const std::vector<size_t> listed = k->g.clists[l];
			for (size_t pc : listed) k->g.cuntrack(pc, l);
		}
	});
}
int fo_partitions(void* s, size_t* count, int* csize, int* coff)
{
	return guard([&] {
		*count = static_cast<SurfBase*>(s)->nparts();
		static_cast<SurfBase*>(s)->partitions(csize, coff);
	});
}
int fo_layer_list(void* s, size_t part, int l, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] { put_list(*static_cast<SurfBase*>(s)->leaf_list(part, l), out, cap, n); });
}
int fo_partition_list(void* s, int which, int l, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] { put_list(*static_cast<SurfBase*>(s)->plist(which, l), out, cap, n); });
}
int fo_affected_list(void* s, size_t part, int l, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] { put_list(*static_cast<SurfBase*>(s)->affected_list(part, l), out, cap, n); });
}
int fo_partition_state(void* s, size_t part, int* active, float* bg)
{
	return guard([&] { static_cast<SurfBase*>(s)->pstate(part, active, bg); });
}
int fo_stats(void* s, size_t* a, size_t* b)
{
	return guard([&] { static_cast<SurfBase*>(s)->stats(a, b); });
}
int fo_band_size(void* s, size_t* n)
{
	return guard([&] { *n = static_cast<SurfBase*>(s)->band_size(); });
}

/* Canonical dump; same encoding as fg_dump in include/felt_gpu.h. */
int fo_dump(void* sv, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		SurfBase* s = static_cast<SurfBase*>(sv);
		const int NL = 2 * s->layers + 1;
		size_t w = 0;
		auto put = [&](uint32_t x) {
			if (w < cap) out[w] = x;
			w++;
		};
		const size_t P = s->nparts();
		put(uint32_t(s->dims));
		put(uint32_t(s->layers));
		put(uint32_t(P));
		for (size_t pc = 0; pc < P; pc++) {
			int act;
			float bg;
			s->pstate(pc, &act, &bg);
			uint32_t bits;
			std::memcpy(&bits, &bg, 4);
			put(uint32_t(act));
			put(bits);
			for (int l = 0; l < NL; l++) {
				const auto& lst = *s->leaf_list(pc, l);
				put(uint32_t(lst.size()));
				for (size_t x : lst) put(uint32_t(x));
			}
		}
		for (int which = 0; which < 3; which++)
			for (int l = 0; l < NL; l++) {
				const auto& lst = *s->plist(which, l);
				put(uint32_t(lst.size()));
				for (size_t x : lst) put(uint32_t(x));
			}
		*n = w;
	});
}

int fo_polys_create(void* s, void** out)
{
	return guard([&] {
		PolysBase* p = make_polys(static_cast<SurfBase*>(s));
		if (!p) throw fo::Error(-1, "unsupported dims/layers");
		*out = p;
	});
}
int fo_polys_destroy(void* p)
{
	delete static_cast<PolysBase*>(p);
	return 0;
}
int fo_polys_notify(void* p)
{
	return guard([&] { static_cast<PolysBase*>(p)->notify(); });
}
int fo_polys_march(void* p)
{
	return guard([&] { static_cast<PolysBase*>(p)->march(); });
}
int fo_polys_invalidate(void* p)
{
	return guard([&] { static_cast<PolysBase*>(p)->invalidate(); });
}
int fo_polys_march_partition(void* p, size_t part)
{
	return guard([&] { static_cast<PolysBase*>(p)->march_partition(part); });
}
int fo_polys_changes(void* p, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] { put_list(static_cast<PolysBase*>(p)->changes(), out, cap, n); });
}
int fo_polys_partition(void* p, size_t part, float* vtx, size_t vcap, uint32_t* spx, size_t scap,
                       size_t* nv, size_t* ns, int* active)
{
	return guard(
	    [&] { static_cast<PolysBase*>(p)->part(part, vtx, vcap, spx, scap, nv, ns, active); });
}
/* fo_polys_partition's vertices (position then, in 3D, normal) as doubles, in the surface's own
 * arithmetic (FP64 for an fo_surface_create64 surface). */
int fo_polys_partition64(void* p, size_t part, double* vtx, size_t vcap, size_t* nv)
{
	return guard([&] { static_cast<PolysBase*>(p)->part64(part, vtx, vcap, nv); });
}
int fo_polys_totals(void* p, size_t* nv, size_t* ns)
{
	return guard([&] { static_cast<PolysBase*>(p)->totals(nv, ns); });
}

/* Timing helper for the CPU baseline: run `steps` global updates with a builtin speed and
 * return the node-updates processed (sum of band sizes at the start of each step) and the
 * wall seconds spent inside the updates. */
int fo_run_steps(void* sv, const fo_speed* sp, int steps, double* node_updates, double* seconds)
{
	return guard([&] {
		SurfBase* s = static_cast<SurfBase*>(sv);
		const fo::Speed speed = to_speed(sp->kind, sp->c, sp->a, sp->n, sp->seed);
		double nu = 0, secs = 0;
		for (int i = 0; i < steps; i++) {
			nu += double(s->band_size());
			const auto t0 = std::chrono::steady_clock::now();
			s->update(speed);
			const auto t1 = std::chrono::steady_clock::now();
			secs += std::chrono::duration<double>(t1 - t0).count();
		}
		*node_updates = nu;
		*seconds = secs;
	});
}

}  // extern "C"
