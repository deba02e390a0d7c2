// C ABI (include/felt_gpu.h) over the device engine. Exceptions never cross the boundary:
// every entry point maps them to a status code and keeps the message for fg_last_error().
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/felt_gpu.h"
#include "fg_engine.cuh"
#include "fg_polys.cuh"
#include "fg_ray.cuh"
#include "fg_image.cuh"
#include "fg_query.cuh"

#include "fg_handles.cuh"

namespace {

thread_local std::string g_err;

template <class F>
int guard(F&& f)
{
	try {
		f();
		return FG_OK;
	} catch (const fg::Error& e) {
		g_err = e.what();
		return e.code;
	} catch (const std::bad_alloc&) {
		g_err = "host allocation failed";
		return FG_ERR_NOMEM;
	} catch (const std::exception& e) {
		g_err = e.what();
		return FG_ERR_ARG;
	}
}

void need(const void* p, const char* what)
{
	if (!p) throw fg::Error(FG_ERR_ARG, std::string("null ") + what);
}

fg::Speed to_speed(const fg_speed* s)
{
	need(s, "speed");
	if (s->kind & ~7) throw fg::Error(FG_ERR_ARG, "unknown speed kind bits");
	return fg::Speed{s->kind, s->c, s->a, s->n, s->seed};
}

void apply_tuning(fg::EngineBase& eng, const fg_config* cfg)
{
	if (!cfg) return;
	if (cfg->launch_mode < 0 || cfg->launch_mode > 2)
		throw fg::Error(FG_ERR_ARG, "launch_mode must be 0, 1 or 2");
	if (cfg->dist_split != 0 && cfg->dist_split != 1 && cfg->dist_split != 2 &&
	    cfg->dist_split != 4 && cfg->dist_split != 8)
		throw fg::Error(FG_ERR_ARG, "dist_split must be 0, 1, 2, 4 or 8");
	if (cfg->record_passes < 0 || cfg->record_passes > 2)
		throw fg::Error(FG_ERR_ARG, "record_passes must be 0, 1 or 2");
	if (cfg->autotune < 0 || cfg->autotune > 1) throw fg::Error(FG_ERR_ARG, "autotune must be 0 or 1");
	int ds = cfg->dist_split, rp = cfg->record_passes;
	if (cfg->autotune && (ds == 0 || rp == 0)) {
		int part[3] = {1, 1, 1};
		for (int a = 0; a < eng.dims(); a++) part[a] = eng.part(a);
		int tds = 0, trp = 0;
		fg::autotune(eng.dims(), eng.layers(), part, tds, trp, nullptr, false);
		if (ds == 0) ds = tds;
		if (rp == 0) rp = trp;
	}
	if (cfg->delta_kernel < 0 || cfg->delta_kernel > 2)
		throw fg::Error(FG_ERR_ARG, "delta_kernel must be 0, 1 or 2");
	if (cfg->fuse_passes < 0 || cfg->fuse_passes > 3)
		throw fg::Error(FG_ERR_ARG, "fuse_passes must be 0, 1, 2 or 3");
	eng.set_tuning(cfg->launch_mode, ds, rp, cfg->delta_kernel, cfg->fuse_passes);
}

void put_list(const std::vector<uint32_t>& v, uint32_t* out, size_t cap, size_t* n)
{
	need(n, "count");
	*n = v.size();
	if (out)
		for (size_t i = 0; i < v.size() && i < cap; i++) out[i] = v[i];
}

}  // namespace

void fg::set_last_error(const std::string& msg) { g_err = msg; }

extern "C" {

const char* fg_last_error(void) { return g_err.c_str(); }

int fg_surface_create(int dims, int layers, const int* size, const int* part, const fg_config* cfg,
                      fg_surface** out)
{
	return guard([&] {
		need(size, "size");
		need(part, "part");
		need(out, "out");
		if (dims != 2 && dims != 3) throw fg::Error(FG_ERR_ARG, "dims must be 2 or 3");
		if (layers < 1 || layers > 4) throw fg::Error(FG_ERR_ARG, "layers must be in 1..4");
		int ndev = 0;
		if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
			throw fg::Error(FG_ERR_CUDA, "no CUDA device");
		fg::PoolDesc d;
		d.D = dims;
		d.L = layers;
		std::array<int, 3> sz = {1, 1, 1};
		for (int a = 0; a < dims; a++) {
			sz[a] = size[a];
			d.part[a] = part[a];
		}
		d.sizes.push_back(sz);
		if (cfg) d.brick_capacity = cfg->brick_capacity;
		auto s = std::make_unique<fg_surface>();
		if (cfg) s->vertex_capacity = cfg->vertex_capacity;
		FG_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
		s->eng.reset(fg::make_engine(d, s->st));
		apply_tuning(*s->eng, cfg);
		*out = s.release();
	});
}

int fg_save(fg_surface* s, uint8_t* buf, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		need(n, "length");
		fg::SurfaceImage img;
		fg::export_image(*s->eng, 0, img);
		std::vector<uint8_t> out;
		int csz[3];
		for (int a = 0; a < s->eng->dims(); a++) csz[a] = s->eng->part(a);
		fg::write_surface_file(img, s->eng->geometry(0), s->eng->dims(), s->eng->layers(), csz, out);
		*n = out.size();
		if (buf) std::memcpy(buf, out.data(), std::min(cap, out.size()));
	});
}

int fg_load(const uint8_t* data, size_t n, const fg_config* cfg, fg_surface** out)
{
	return guard([&] {
		need(data, "data");
		need(out, "out");
		int D = 0, L = 0, size[3] = {1, 1, 1}, csz[3] = {1, 1, 1};
		fg::peek_surface_file(data, n, D, L, size, csz);
		if (L > 4) throw fg::Error(FG_ERR_ARG, "surface file: more than 4 layers");
		fg_surface* s = nullptr;
		const int rc = fg_surface_create(D, L, size, csz, cfg, &s);
		if (rc != FG_OK) throw fg::Error(rc, g_err);
		std::unique_ptr<fg_surface> hold(s);
		const fg::SurfGeom& g = s->eng->geometry(0);
		for (int a = 0; a < D; a++)
			if (g.off[a] != -size[a] / 2) throw fg::Error(FG_ERR_ARG, "surface file: grid offset other than -size/2");
		fg::SurfaceImage img;
		fg::read_surface_file(data, n, g, D, L, csz, s->eng->dev().BV, img);
		fg::import_image(*s->eng, img);
		*out = hold.release();
	});
}

int fg_surface_destroy(fg_surface* s)
{
	return guard([&] { delete s; });
}

int fg_seed(fg_surface* s, const int* pos)
{
	return guard([&] {
		need(s, "surface");
		need(pos, "pos");
		s->eng->seed(0, pos);
	});
}

int fg_update_builtin(fg_surface* s, const fg_speed* speed)
{
	return guard([&] {
		need(s, "surface");
		const fg::Speed sp = to_speed(speed);
		s->eng->update_builtin(&sp);
	});
}

int fg_update_begin_global(fg_surface* s, const fg_device_view** view, void** stream)
{
	return guard([&] {
		need(s, "surface");
		s->eng->update_begin_global();
		if (view) *view = reinterpret_cast<const fg_device_view*>(&s->eng->dev());
		if (stream) *stream = (void*)s->eng->stream();
	});
}

int fg_update_finish_global(fg_surface* s)
{
	return guard([&] {
		need(s, "surface");
		s->eng->update_finish_global();
	});
}

int fg_update_bounded(fg_surface* s, const int* lo, const int* hi, const fg_speed* speed)
{
	return guard([&] {
		need(s, "surface");
		need(lo, "lo");
		need(hi, "hi");
		s->eng->update_bounded(lo, hi, to_speed(speed));
	});
}

int fg_update_start(fg_surface* s)
{
	return guard([&] {
		need(s, "surface");
		s->local_open = true;
		s->dpos.clear();
		s->dval.clear();
	});
}

int fg_delta(fg_surface* s, const int* pos, float val)
{
	return guard([&] {
		need(s, "surface");
		need(pos, "pos");
		if (!s->local_open) throw fg::Error(FG_ERR_STATE, "delta() outside update_start/end");
		for (int a = 0; a < s->eng->dims(); a++) s->dpos.push_back(pos[a]);
		s->dval.push_back(val);
	});
}

int fg_delta_n(fg_surface* s, const int* pos, const float* val, size_t n)
{
	return guard([&] {
		need(s, "surface");
		if (n && (!pos || !val)) throw fg::Error(FG_ERR_ARG, "null pos/val");
		if (!s->local_open) throw fg::Error(FG_ERR_STATE, "delta() outside update_start/end");
		const int D = s->eng->dims();
		s->dpos.insert(s->dpos.end(), pos, pos + n * D);
		s->dval.insert(s->dval.end(), val, val + n);
	});
}

int fg_update_end(fg_surface* s)
{
	return guard([&] {
		need(s, "surface");
		if (!s->local_open) throw fg::Error(FG_ERR_STATE, "update_end() without update_start()");
		s->local_open = false;
		s->eng->update_local(s->dpos, s->dval);
	});
}

int fg_snapshot(fg_surface* s, float* dst, size_t n, int dst_is_device)
{
	return guard([&] {
		need(s, "surface");
		need(dst, "dst");
		s->eng->snapshot(0, dst, n, dst_is_device != 0);
	});
}

int fg_get(fg_surface* s, const int* pos, float* out)
{
	return guard([&] {
		need(s, "surface");
		need(pos, "pos");
		need(out, "out");
		*out = s->eng->get(0, pos);
	});
}

static void query_args(size_t n, const void* pos, float* out)
{
	if (n) {
		need(pos, "positions");
		need(out, "out");
	}
}

int fg_query(fg_surface* s, int what, const float* pos, size_t n, float* out)
{
	return guard([&] {
		need(s, "surface");
		query_args(n, pos, out);
		fg::query(*s->eng, 0, what, pos, nullptr, n, out);
	});
}

int fg_query_nodes(fg_surface* s, int what, const int* pos, size_t n, float* out)
{
	return guard([&] {
		need(s, "surface");
		query_args(n, pos, out);
		fg::query(*s->eng, 0, what, nullptr, pos, n, out);
	});
}

int fg_ray(fg_surface* s, const float* origins, const float* dirs, size_t n, float* hits)
{
	return guard([&] {
		need(s, "surface");
		if (n) {
			need(origins, "origins");
			need(dirs, "dirs");
			need(hits, "hits");
		}
		fg::ray_batch(*s->eng, 0, origins, dirs, n, hits, false);
	});
}

int fg_ray_device(fg_surface* s, const float* origins, const float* dirs, size_t n, float* hits,
                  int order_mode)
{
	return guard([&] {
		need(s, "surface");
		if (n) {
			need(origins, "origins");
			need(dirs, "dirs");
			need(hits, "hits");
		}
		if (order_mode < 0 || order_mode > 2) throw fg::Error(FG_ERR_ARG, "order_mode is 0, 1 or 2");
		fg::ray_batch(*s->eng, 0, origins, dirs, n, hits, true, order_mode);
	});
}

int fg_partitions(fg_surface* s, size_t* count, int* ccount, int* coff)
{
	return guard([&] {
		need(s, "surface");
		int cc[3], co[3];
		const size_t n = s->eng->partitions(0, cc, co);
		if (count) *count = n;
		for (int a = 0; a < s->eng->dims(); a++) {
			if (ccount) ccount[a] = cc[a];
			if (coff) coff[a] = co[a];
		}
	});
}

int fg_layer_list(fg_surface* s, size_t part, int li, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		put_list(s->eng->layer_list(0, part, li), out, cap, n);
	});
}

int fg_partition_list(fg_surface* s, int li, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		put_list(s->eng->partition_list(0, 0, li), out, cap, n);
	});
}

int fg_delta_partitions(fg_surface* s, int li, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		put_list(s->eng->partition_list(0, 1, li), out, cap, n);
	});
}

int fg_status_partitions(fg_surface* s, int li, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		put_list(s->eng->partition_list(0, 2, li), out, cap, n);
	});
}

int fg_affected_partitions(fg_surface* s, int li, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		put_list(s->eng->partition_list(0, 3, li), out, cap, n);
	});
}

int fg_affected_list(fg_surface* s, size_t part, int li, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		put_list(s->eng->affected_list(0, part, li), out, cap, n);
	});
}

int fg_partition_state(fg_surface* s, size_t part, int* active, float* background)
{
	return guard([&] {
		need(s, "surface");
		need(active, "active");
		need(background, "background");
		s->eng->partition_state(0, part, active, background);
	});
}

int fg_update_iterations(fg_surface* s, int* iterations)
{
	return guard([&] {
		need(s, "surface");
		need(iterations, "iterations");
		*iterations = s->eng->stats().iterations;
	});
}

int fg_stats(fg_surface* s, size_t* iso, size_t* delta)
{
	return guard([&] {
		need(s, "surface");
		const int NL = 2 * s->eng->layers() + 1;
		size_t a = 0, b = 0;
		for (int l = 0; l < NL; l++) {
			a = std::max(a, s->eng->partition_list(0, 0, l).size());
			b = std::max(b, s->eng->partition_list(0, 1, l).size());
		}
		if (iso) *iso = a;
		if (delta) *delta = b;
	});
}

int fg_band_size(fg_surface* s, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		need(n, "n");
		*n = (size_t)s->eng->band_size(0);
	});
}

int fg_dump(fg_surface* s, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(s, "surface");
		put_list(s->eng->dump(0), out, cap, n);
	});
}

// ---- Polys ----

int fg_polys_create(fg_surface* s, fg_polys** out)
{
	return guard([&] {
		need(s, "surface");
		need(out, "out");
		auto p = std::make_unique<fg_polys>();
		p->surf = s;
		p->impl.reset(fg::make_polys(*s->eng, 0, s->vertex_capacity));
		*out = p.release();
	});
}

int fg_polys_destroy(fg_polys* p)
{
	return guard([&] { delete p; });
}

int fg_polys_notify(fg_polys* p)
{
	return guard([&] {
		need(p, "polys");
		p->impl->notify();
	});
}

int fg_polys_march(fg_polys* p)
{
	return guard([&] {
		need(p, "polys");
		p->impl->march();
	});
}

int fg_polys_invalidate(fg_polys* p)
{
	return guard([&] {
		need(p, "polys");
		p->impl->invalidate();
	});
}

int fg_polys_march_partition(fg_polys* p, size_t part)
{
	return guard([&] {
		need(p, "polys");
		p->impl->march_partition(part);
	});
}

int fg_polys_changes(fg_polys* p, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(p, "polys");
		put_list(p->impl->changes(), out, cap, n);
	});
}

int fg_polys_partition(fg_polys* p, size_t part, float* vtx, size_t vcap, uint32_t* spx,
                       size_t scap, size_t* nv, size_t* ns, int* active)
{
	return guard([&] {
		need(p, "polys");
		need(nv, "nv");
		need(ns, "ns");
		int act = 0;
		p->impl->partition(part, vtx, vcap, spx, scap, nv, ns, &act);
		if (active) *active = act;
	});
}

int fg_node_updates(fg_surface* s, unsigned long long* n)
{
	return guard([&] {
		need(s, "surface");
		need(n, "n");
		*n = s->eng->node_updates();
	});
}

// ---- batches ----

int fg_batch_create(int dims, int layers, const int* part, size_t n, const int* sizes,
                    const fg_config* cfg, fg_batch** out)
{
	return guard([&] {
		need(part, "part");
		need(sizes, "sizes");
		need(out, "out");
		if (dims != 2 && dims != 3) throw fg::Error(FG_ERR_ARG, "dims must be 2 or 3");
		if (layers < 1 || layers > 4) throw fg::Error(FG_ERR_ARG, "layers must be in 1..4");
		if (n == 0) throw fg::Error(FG_ERR_ARG, "a batch needs at least one surface");
		int ndev = 0;
		if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
			throw fg::Error(FG_ERR_CUDA, "no CUDA device");
		fg::PoolDesc d;
		d.D = dims;
		d.L = layers;
		for (int a = 0; a < dims; a++) d.part[a] = part[a];
		for (size_t i = 0; i < n; i++) {
			std::array<int, 3> sz = {1, 1, 1};
			for (int a = 0; a < dims; a++) sz[a] = sizes[i * dims + a];
			d.sizes.push_back(sz);
		}
		if (cfg) d.brick_capacity = cfg->brick_capacity;
		auto b = std::make_unique<fg_batch>();
		if (cfg) b->vertex_capacity = cfg->vertex_capacity;
		FG_CUDA(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
		b->eng.reset(fg::make_engine(d, b->st));
		apply_tuning(*b->eng, cfg);
		b->eng->set_throw_on_freeze(false);
		*out = b.release();
	});
}

int fg_batch_surface_stopped(fg_batch* b, size_t surface, int* stopped)
{
	return guard([&] {
		need(b, "batch");
		need(stopped, "stopped");
		if (surface >= (size_t)b->eng->surfaces()) throw fg::Error(FG_ERR_ARG, "surface index");
		*stopped = b->eng->frozen((int)surface) ? 1 : 0;
	});
}

int fg_batch_pause(fg_batch* b, size_t surface, int paused)
{
	return guard([&] {
		need(b, "batch");
		if (surface >= (size_t)b->eng->surfaces()) throw fg::Error(FG_ERR_ARG, "surface index");
		b->eng->set_paused((int)surface, paused != 0);
	});
}

int fg_batch_destroy(fg_batch* b)
{
	return guard([&] { delete b; });
}

int fg_batch_seed(fg_batch* b, const int* centres)
{
	return guard([&] {
		need(b, "batch");
		need(centres, "centres");
		b->eng->seed_all(centres);
	});
}

int fg_batch_update(fg_batch* b, const fg_speed* speeds)
{
	return guard([&] {
		need(b, "batch");
		need(speeds, "speeds");
		const int S = b->eng->surfaces();
		std::vector<fg::Speed> sp(S);
		for (int i = 0; i < S; i++) sp[i] = to_speed(&speeds[i]);
		b->eng->update_builtin(sp.data());
	});
}

static fg::PolysBase& batch_polys(fg_batch* b)
{
	if (!b->polys) b->polys.reset(fg::make_polys(*b->eng, 0, b->vertex_capacity));
	return *b->polys;
}

int fg_batch_polys_notify(fg_batch* b)
{
	return guard([&] {
		need(b, "batch");
		batch_polys(b).notify();
	});
}

int fg_batch_polys_march(fg_batch* b)
{
	return guard([&] {
		need(b, "batch");
		batch_polys(b).march();
	});
}

int fg_batch_polys_invalidate(fg_batch* b)
{
	return guard([&] {
		need(b, "batch");
		batch_polys(b).invalidate();
	});
}

int fg_batch_snapshot(fg_batch* b, size_t surface, float* dst, size_t n)
{
	return guard([&] {
		need(b, "batch");
		need(dst, "dst");
		b->eng->snapshot((int)surface, dst, n, false);
	});
}

int fg_batch_ray(fg_batch* b, size_t surface, const float* origins, const float* dirs, size_t n,
                 float* hits)
{
	return guard([&] {
		need(b, "batch");
		if (n) {
			need(origins, "origins");
			need(dirs, "dirs");
			need(hits, "hits");
		}
		if (surface >= (size_t)b->eng->surfaces()) throw fg::Error(FG_ERR_ARG, "surface index out of range");
		fg::ray_batch(*b->eng, (int)surface, origins, dirs, n, hits, false);
	});
}

int fg_batch_query(fg_batch* b, size_t surface, int what, const float* pos, size_t n, float* out)
{
	return guard([&] {
		need(b, "batch");
		query_args(n, pos, out);
		if (surface >= (size_t)b->eng->surfaces()) throw fg::Error(FG_ERR_ARG, "surface index out of range");
		fg::query(*b->eng, (int)surface, what, pos, nullptr, n, out);
	});
}

int fg_batch_query_nodes(fg_batch* b, size_t surface, int what, const int* pos, size_t n, float* out)
{
	return guard([&] {
		need(b, "batch");
		query_args(n, pos, out);
		if (surface >= (size_t)b->eng->surfaces()) throw fg::Error(FG_ERR_ARG, "surface index out of range");
		fg::query(*b->eng, (int)surface, what, nullptr, pos, n, out);
	});
}

int fg_batch_save(fg_batch* b, size_t surface, uint8_t* buf, size_t cap, size_t* n)
{
	return guard([&] {
		need(b, "batch");
		need(n, "length");
		if (surface >= (size_t)b->eng->surfaces()) throw fg::Error(FG_ERR_ARG, "surface index out of range");
		fg::SurfaceImage img;
		fg::export_image(*b->eng, (int)surface, img);
		std::vector<uint8_t> out;
		int csz[3];
		for (int a = 0; a < b->eng->dims(); a++) csz[a] = b->eng->part(a);
		fg::write_surface_file(img, b->eng->geometry((int)surface), b->eng->dims(), b->eng->layers(),
		                       csz, out);
		*n = out.size();
		if (buf) std::memcpy(buf, out.data(), std::min(cap, out.size()));
	});
}

int fg_batch_restore(fg_batch* b, size_t surface, const uint8_t* data, size_t n)
{
	return guard([&] {
		need(b, "batch");
		need(data, "data");
		if (surface >= (size_t)b->eng->surfaces()) throw fg::Error(FG_ERR_ARG, "surface index out of range");
		int D = 0, L = 0, size[3] = {1, 1, 1}, csz[3] = {1, 1, 1};
		fg::peek_surface_file(data, n, D, L, size, csz);
		const fg::SurfGeom& g = b->eng->geometry((int)surface);
		if (D != b->eng->dims() || L != b->eng->layers())
			throw fg::Error(FG_ERR_ARG, "surface file of another dimension or layer count");
		for (int a = 0; a < D; a++)
			if (size[a] != g.size[a] || csz[a] != b->eng->part(a))
				throw fg::Error(FG_ERR_ARG, "surface file of another grid or partition size");
		fg::SurfaceImage img;
		fg::read_surface_file(data, n, g, D, L, csz, b->eng->dev().BV, img);
		fg::restore_image(*b->eng, (int)surface, img);
	});
}

int fg_batch_dump(fg_batch* b, size_t surface, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(b, "batch");
		put_list(b->eng->dump((int)surface), out, cap, n);
	});
}

int fg_batch_polys_partition(fg_batch* b, size_t surface, size_t part, float* vtx, size_t vcap,
                             uint32_t* spx, size_t scap, size_t* nv, size_t* ns, int* active)
{
	return guard([&] {
		need(b, "batch");
		need(nv, "nv");
		need(ns, "ns");
		fg::PolysBase& p = batch_polys(b);
		p.select((int)surface);
		int act = 0;
		p.partition(part, vtx, vcap, spx, scap, nv, ns, &act);
		if (active) *active = act;
	});
}

int fg_batch_polys_changes(fg_batch* b, size_t surface, uint32_t* out, size_t cap, size_t* n)
{
	return guard([&] {
		need(b, "batch");
		fg::PolysBase& p = batch_polys(b);
		p.select((int)surface);
		put_list(p.changes(), out, cap, n);
	});
}

int fg_batch_polys_totals(fg_batch* b, size_t* nv, size_t* ns)
{
	return guard([&] {
		need(b, "batch");
		batch_polys(b).totals(nv, ns);
	});
}

int fg_batch_node_updates(fg_batch* b, unsigned long long* n)
{
	return guard([&] {
		need(b, "batch");
		need(n, "n");
		*n = b->eng->node_updates();
	});
}

int fg_batch_work_units(fg_batch* b, unsigned long long* out, size_t n)
{
	return guard([&] {
		need(b, "batch");
		need(out, "out");
		unsigned long long tmp[fg::KS_N];
		b->eng->sync();
		FG_CUDA(cudaMemcpy(tmp, b->eng->dev().kstat, sizeof(tmp), cudaMemcpyDeviceToHost));
		for (size_t i = 0; i < n && i < (size_t)fg::KS_N; i++) out[i] = tmp[i];
	});
}

int fg_batch_stream(fg_batch* b, void** stream)
{
	return guard([&] {
		need(b, "batch");
		need(stream, "stream");
		*stream = (void*)b->eng->stream();
	});
}

int fg_work_units(fg_surface* s, unsigned long long* out, size_t n)
{
	return guard([&] {
		need(s, "surface");
		need(out, "out");
		unsigned long long tmp[fg::KS_N];
		s->eng->sync();
		FG_CUDA(cudaMemcpy(tmp, s->eng->dev().kstat, sizeof(tmp), cudaMemcpyDeviceToHost));
		for (size_t i = 0; i < n && i < (size_t)fg::KS_N; i++) out[i] = tmp[i];
	});
}

int fg_surface_info(fg_surface* s, int* dims, int* layers, int* size, int* part)
{
	return guard([&] {
		need(s, "surface");
		need(dims, "dims");
		need(layers, "layers");
		*dims = s->eng->dims();
		*layers = s->eng->layers();
		for (int a = 0; a < *dims; a++) {
			if (size) size[a] = s->eng->geometry(0).size[a];
			if (part) part[a] = s->eng->part(a);
		}
	});
}

int fg_surface_stream(fg_surface* s, void** stream)
{
	return guard([&] {
		need(s, "surface");
		need(stream, "stream");
		*stream = (void*)s->eng->stream();
	});
}

int fg_launch_count(long long* n)
{
	return guard([&] {
		need(n, "n");
		*n = fg::launch_count();
	});
}

int fg_profile_enable(int on)
{
	return guard([&] { fg::prof_enable(on != 0); });
}

int fg_profile_reset(void)
{
	return guard([&] { fg::prof_reset(); });
}

int fg_autotune_candidates(int dims, const int* part, int* pairs, size_t cap, size_t* n)
{
	return guard([&] {
		need(part, "part");
		need(n, "n");
		if (dims != 2 && dims != 3) throw fg::Error(FG_ERR_ARG, "dims must be 2 or 3");
		std::vector<std::pair<int, int>> c;
		fg::tune_candidates(dims, part, c);
		*n = c.size();
		for (size_t i = 0; pairs && i < c.size() && i < cap / 2; i++) {
			pairs[2 * i] = c[i].first;
			pairs[2 * i + 1] = c[i].second;
		}
	});
}

int fg_autotune(int dims, int layers, const int* part, int force, fg_config* cfg, double* ms,
                size_t ms_cap, size_t* n)
{
	return guard([&] {
		need(part, "part");
		need(cfg, "config");
		if (dims != 2 && dims != 3) throw fg::Error(FG_ERR_ARG, "dims must be 2 or 3");
		if (layers < 1 || layers > 4) throw fg::Error(FG_ERR_ARG, "layers must be in 1..4");
		for (int a = 0; a < dims; a++)
			if (part[a] < 1 || part[a] > 32) throw fg::Error(FG_ERR_ARG, "partition edge must be in 1..32");
		int ndev = 0;
		if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
			throw fg::Error(FG_ERR_CUDA, "no CUDA device");
		std::vector<double> t;
		int ds = 0, rp = 0;
		fg::autotune(dims, layers, part, ds, rp, &t, force != 0);
		cfg->dist_split = ds;
		cfg->record_passes = rp;
		if (n) *n = t.size();
		for (size_t i = 0; ms && i < t.size() && i < ms_cap; i++) ms[i] = t[i];
	});
}

int fg_surface_tuning(fg_surface* s, int* out)
{
	return guard([&] {
		need(s, "surface");
		need(out, "out");
		s->eng->tuning(out);
	});
}

int fg_batch_tuning(fg_batch* b, int* out)
{
	return guard([&] {
		need(b, "batch");
		need(out, "out");
		b->eng->tuning(out);
	});
}

int fg_profile_only(const char* kernel)
{
	return guard([&] { fg::prof_only(kernel); });
}

static std::vector<fg::ProfEntry> g_prof_snapshot;

int fg_profile_count(size_t* n)
{
	return guard([&] {
		need(n, "n");
		g_prof_snapshot = fg::prof_read();
		*n = g_prof_snapshot.size();
	});
}

int fg_profile_entry(size_t i, char* name, size_t name_cap, double* ms, long long* launches)
{
	return guard([&] {
		if (i >= g_prof_snapshot.size()) throw fg::Error(FG_ERR_ARG, "profile entry out of range");
		const fg::ProfEntry& e = g_prof_snapshot[i];
		if (name && name_cap) {
			std::strncpy(name, e.name.c_str(), name_cap - 1);
			name[name_cap - 1] = 0;
		}
		if (ms) *ms = e.ms;
		if (launches) *launches = e.launches;
	});
}

int fg_polys_gather(fg_polys* p, const uint32_t* parts, size_t n, float* vtx, size_t vcap,
                    uint32_t* spx, size_t scap, uint32_t* counts, size_t* nv, size_t* ns)
{
	return guard([&] {
		need(p, "polys");
		need(nv, "nv");
		need(ns, "ns");
		if (n && !parts) throw fg::Error(FG_ERR_ARG, "null parts");
		p->impl->gather(parts, n, vtx, vcap, spx, scap, counts, nv, ns);
	});
}

int fg_polys_totals(fg_polys* p, size_t* nv, size_t* ns)
{
	return guard([&] {
		need(p, "polys");
		p->impl->totals(nv, ns);
	});
}

}  // extern "C"
