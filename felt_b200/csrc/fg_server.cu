// Continuous-batching server of level-set requests (fg_server_* in include/felt_gpu.h).
//
// The reference advances one Surface at a time and has no serving layer; this is the serving
// loop the B200 build adds around its batched engine. One long-lived pool holds `slots`
// surfaces, each with a partition range sized for the largest grid a request may ask for, and
// one brick pool that all of them share. A worker thread owns the pool and runs steps: every
// step is one batched Surface::update (include/Felt/Surface.hpp:254-296) of all surfaces in
// flight with their own builtin speeds, Polys::notify (include/Felt/Polys.hpp:92-133) for those
// that asked for polygons, and Polys::march (Polys.hpp:138-165) of each of those after its
// last update (of that surface only, so that its marches are those of the request alone).
// Between steps, requests that arrived meanwhile take the slots of finished ones: the slot's
// surface is reset (its bricks back to the pool) to the request's grid size and
// seeded, and from then on it advances in the same launches as the others. Finished slots are
// paused, so no kernel touches them, and their results are exactly those of a separate
// Surface given the same seed and updates.
//
// Admission: a request reserves an upper bound of the bricks its band can reach (every
// partition within reach of its seed after its steps, at one cell per update or its speed's
// largest |delta|, whichever is more), and is rejected at submission when the reservations in
// flight and queued would exceed the brick pool. Reservations return when a request finishes.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/felt_gpu.h"
#include "fg_engine.cuh"
#include "fg_handles.cuh"
#include "fg_polys.cuh"

namespace {

using Clock = std::chrono::steady_clock;

/// Device bytes of one brick as the engine allocates it: per leaf the value, delta, lookup,
/// 2L+1 ordered lists, status, status lists, two affected lookups and lists, expansion claim
/// and claimed-leaf list; per brick the list counts and the allocator's queues.
double brick_bytes(int D, int L, const int* part)
{
	const int NL = 2 * L + 1;
	double bv = 1;
	for (int a = 0; a < D; a++) bv *= part[a];
	const double leaf = 4 + 4 + 2 + 2.0 * NL + 1 + 2.0 * NL + 2 * 2 + 2 * 2.0 * NL + 8 + 2;
	return bv * leaf + 4.0 * (4 * NL + 7);
}

/// Largest |delta| a builtin speed can produce: |c| + |n| + |a| * D (a node's mean curvature
/// by difference of normals is at most D in magnitude: each axis adds a difference of two unit
/// normal components, halved).
double speed_bound(const fg_speed& sp, int D)
{
	double v = 0;
	if (sp.kind & FG_SPEED_CONST) v += std::fabs(sp.c);
	if (sp.kind & FG_SPEED_NOISE) v += std::fabs(sp.n);
	if (sp.kind & FG_SPEED_CURV) v += std::fabs(sp.a) * D;
	return v;
}

/// Bricks a request may hold at most: the partitions within reach of its seed. Over an
/// update with |delta| <= 1 the zero crossing moves at most one cell and the band follows it, so
/// after k steps the band lies within L + 1 + k cells of the seed (L + 2 + k taken here); a
/// speed that can exceed 1 per step is given its largest |delta| per step instead. Per axis the
/// reach spans at most ceil(span / part) + 1 partitions, and never more than the grid has.
long long request_bricks(int D, int L, const int* part, const fg_request& r)
{
	const double per_step = std::max(1.0, speed_bound(r.speed, D));
	const double reach = L + 2 + std::ceil(per_step * r.steps);
	long long nb = 1;
	for (int a = 0; a < D; a++) {
		const int p = part[a];
		const int size = r.size[a];
		const long long ccount = (size + p - 1) / p + 1;  // partial partitions add one
		const long long span = std::min<long long>(size, (long long)(2 * reach) + 1);
		nb *= std::min(ccount, (span + p - 1) / p + 1);
	}
	return nb;
}

struct Kept {
	std::vector<uint32_t> dump;
	std::vector<float> vtx;
	std::vector<uint32_t> spx;
	std::vector<uint32_t> counts;  // per partition: vertices, simplices
};

struct Slot {
	bool busy = false;
	fg_request req{};
	int remaining = 0;
	long long reserved = 0;
	double t_submit = 0, t_admit = 0;
};

struct Queued {
	fg_request req;
	long long reserved;
	double t_submit;
};

}  // namespace

struct fg_server {
	fg_server_config cfg{};
	int D = 3, L = 2;
	cudaStream_t st = nullptr;
	std::unique_ptr<fg::EngineBase> eng;
	std::unique_ptr<fg::PolysBase> polys;
	Clock::time_point t0 = Clock::now();

	std::mutex mu;
	std::condition_variable cv_work, cv_done;
	std::deque<Queued> queue;
	std::deque<fg_result> done;
	std::unordered_map<uint64_t, Kept> kept;
	bool stop = false;
	std::string fault;  // set when the worker hit an error it could not recover from
	int fault_code = 0;

	long long capacity = 0;  // bricks in the pool
	long long reserved = 0;  // bricks reserved by requests queued or in flight
	fg_server_stats stats{};

	std::vector<Slot> slots;
	std::vector<fg::Speed> speeds;
	std::vector<unsigned long long> snu;
	std::thread worker;

	double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
	long long bound(const fg_request& r) const { return request_bricks(D, L, cfg.part, r); }

	void run();
	void admit(std::vector<int>& fresh);
	void step();
	void finish(const std::vector<int>& fin, int status);
	void fail_all(int code, const std::string& msg);
};

void fg_server::admit(std::vector<int>& fresh)
{
	// the requests taken from the queue under the lock are in slots marked busy; reset, seed
	// and resume them here, outside the lock
	std::vector<int> on;
	for (int s : fresh) {
		Slot& sl = slots[s];
		eng->reset_surface(s, sl.req.size);
		polys->reset_surface(s);
		polys->set_enabled(s, sl.req.polygonise != 0);
		eng->seed_async(s, sl.req.centre);
		speeds[s] = fg::Speed{sl.req.speed.kind, sl.req.speed.c, sl.req.speed.a, sl.req.speed.n,
		                      sl.req.speed.seed};
		sl.remaining = sl.req.steps;
		sl.t_admit = now();
		on.push_back(0);
	}
	if (!fresh.empty()) {
		eng->set_paused_n(fresh.data(), on.data(), (int)fresh.size());
		eng->check_errors();
	}
}

void fg_server::step()
{
	eng->update_builtin(speeds.data());
	bool any_polys = false;
	for (size_t s = 0; s < slots.size(); s++)
		if (slots[s].busy && slots[s].req.polygonise) any_polys = true;
	if (any_polys) polys->notify();
	std::vector<int> fin, fin_polys;
	for (size_t s = 0; s < slots.size(); s++) {
		Slot& sl = slots[s];
		if (!sl.busy) continue;
		sl.remaining--;
		if (sl.remaining <= 0 || eng->frozen((int)s)) {
			fin.push_back((int)s);
			if (sl.req.polygonise) fin_polys.push_back((int)s);
		}
	}
	// only the finishing requests are marched: a request in flight keeps its pending
	// partitions for its own march, so its polygons are those of the same request alone
	if (!fin_polys.empty()) polys->march_some(fin_polys.data(), (int)fin_polys.size());
	const long long used = (long long)eng->dev().nslots - eng->free_bricks();
	{
		std::lock_guard<std::mutex> g(mu);
		stats.steps++;
		stats.peak_used_bricks =
		    std::max<unsigned long long>(stats.peak_used_bricks, (unsigned long long)used);
	}
	if (!fin.empty()) finish(fin, FG_OK);
}

void fg_server::finish(const std::vector<int>& fin, int status)
{
	eng->surface_node_updates(snu.data());
	const double t = now();
	std::vector<fg_result> out;
	std::vector<std::pair<uint64_t, Kept>> keep;
	for (int s : fin) {
		Slot& sl = slots[s];
		fg_result r{};
		r.tag = sl.req.tag;
		r.status = status != FG_OK ? status : eng->frozen(s) ? FG_ERR_TIMEOUT : FG_OK;
		r.steps_done = sl.req.steps - std::max(sl.remaining, 0);
		r.t_submit = sl.t_submit;
		r.t_admit = sl.t_admit;
		r.t_done = t;
		r.node_updates = snu[s];
		if (status == FG_OK && sl.req.polygonise) {
			polys->select(s);
			int cc[3], co[3];
			const size_t np = eng->partitions(s, cc, co);
			std::vector<uint32_t> parts(np);
			for (size_t i = 0; i < np; i++) parts[i] = (uint32_t)i;
			Kept k;
			size_t nv = 0, ns = 0;
			k.counts.resize(2 * np);
			polys->gather(parts.data(), np, nullptr, 0, nullptr, 0, k.counts.data(), &nv, &ns);
			r.vertices = nv;
			r.simplices = ns;
			if (cfg.keep_outputs) {
				const size_t vf = D == 3 ? 2 * D : D;
				k.vtx.resize(nv * vf);
				k.spx.resize(ns * D);
				polys->gather(parts.data(), np, k.vtx.data(), k.vtx.size(), k.spx.data(),
				              k.spx.size(), k.counts.data(), &nv, &ns);
				k.dump = eng->dump(s);
				keep.emplace_back(r.tag, std::move(k));
			}
		} else if (status == FG_OK && cfg.keep_outputs) {
			Kept k;
			k.dump = eng->dump(s);
			keep.emplace_back(r.tag, std::move(k));
		}
		out.push_back(r);
	}
	// the finished surfaces give their bricks back and stop being worked on
	std::vector<int> on(fin.size(), 1);
	eng->set_paused_n(fin.data(), on.data(), (int)fin.size());
	for (int s : fin) {
		eng->reset_surface(s, slots[s].req.size);
		polys->reset_surface(s);
	}
	std::lock_guard<std::mutex> g(mu);
	for (int s : fin) {
		reserved -= slots[s].reserved;
		slots[s].busy = false;
	}
	for (const fg_result& r : out) {
		stats.node_updates += r.node_updates;
		if (status == FG_OK)
			stats.completed++;  // stopped surfaces included (their status says so)
		else
			stats.failed++;
		done.push_back(r);
	}
	for (auto& k : keep) kept[k.first] = std::move(k.second);
	cv_done.notify_all();
}

void fg_server::fail_all(int code, const std::string& msg)
{
	std::vector<int> busy;
	for (size_t s = 0; s < slots.size(); s++)
		if (slots[s].busy) busy.push_back((int)s);
	{
		std::lock_guard<std::mutex> g(mu);
		fault = msg;
		fault_code = code;
	}
	try {
		if (!busy.empty()) finish(busy, code);
	} catch (const std::exception&) {
		// the pool is unusable: report the in-flight requests as failed without touching it
		std::lock_guard<std::mutex> g(mu);
		for (int s : busy) {
			fg_result r{};
			r.tag = slots[s].req.tag;
			r.status = code;
			r.t_submit = slots[s].t_submit;
			r.t_done = now();
			reserved -= slots[s].reserved;
			slots[s].busy = false;
			stats.failed++;
			done.push_back(r);
		}
		stop = true;
		cv_done.notify_all();
	}
}

void fg_server::run()
{
	for (;;) {
		std::vector<int> fresh;
		{
			std::unique_lock<std::mutex> lk(mu);
			auto busy = [&] {
				for (const Slot& s : slots)
					if (s.busy) return true;
				return false;
			};
			cv_work.wait(lk, [&] { return stop || !queue.empty() || busy(); });
			if (stop) break;
			// arrivals take free slots at the step boundary, in arrival order
			for (size_t s = 0; s < slots.size() && !queue.empty(); s++) {
				if (slots[s].busy) continue;
				Queued q = queue.front();
				queue.pop_front();
				slots[s].busy = true;
				slots[s].req = q.req;
				slots[s].reserved = q.reserved;
				slots[s].t_submit = q.t_submit;
				slots[s].remaining = -1;
				fresh.push_back((int)s);
				stats.started++;
			}
		}
		try {
			admit(fresh);
			step();
		} catch (const fg::Error& e) {
			fail_all(e.code, e.what());
		} catch (const std::exception& e) {
			fail_all(FG_ERR_CUDA, e.what());
		}
		std::lock_guard<std::mutex> g(mu);
		if (stop) break;
	}
}

namespace {

template <class F>
int sguard(F&& f)
{
	try {
		f();
		return FG_OK;
	} catch (const fg::Error& e) {
		fg::set_last_error(e.what());
		return e.code;
	} catch (const std::bad_alloc&) {
		fg::set_last_error("host allocation failed");
		return FG_ERR_NOMEM;
	} catch (const std::exception& e) {
		fg::set_last_error(e.what());
		return FG_ERR_ARG;
	}
}

void need(const void* p, const char* what)
{
	if (!p) throw fg::Error(FG_ERR_ARG, std::string("null ") + what);
}

}  // namespace

extern "C" {

int fg_server_create(const fg_server_config* cfg, fg_server** out)
{
	return sguard([&] {
		need(cfg, "config");
		need(out, "out");
		const int D = cfg->dims, L = cfg->layers;
		if (D != 2 && D != 3) throw fg::Error(FG_ERR_ARG, "dims must be 2 or 3");
		if (L < 1 || L > 4) throw fg::Error(FG_ERR_ARG, "layers must be in 1..4");
		if (cfg->slots == 0 || cfg->slots > 65535)
			throw fg::Error(FG_ERR_ARG, "slots must be in 1..65535");
		for (int a = 0; a < D; a++)
			if (cfg->part[a] <= 0 || cfg->max_size[a] <= 0)
				throw fg::Error(FG_ERR_ARG, "part and max_size must be positive");
		int ndev = 0;
		if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
			throw fg::Error(FG_ERR_CUDA, "no CUDA device");
		auto s = std::make_unique<fg_server>();
		s->cfg = *cfg;
		s->D = D;
		s->L = L;
		long long bricks = (long long)cfg->brick_capacity;
		if (!bricks) {
			if (!(cfg->budget_bytes > 0))
				throw fg::Error(FG_ERR_ARG, "give brick_capacity or budget_bytes");
			bricks = (long long)(cfg->budget_bytes / brick_bytes(D, L, cfg->part));
		}
		if (bricks < 1 || bricks >= (1LL << 31)) throw fg::Error(FG_ERR_ARG, "brick pool size");
		fg::PoolDesc d;
		d.D = D;
		d.L = L;
		std::array<int, 3> one = {1, 1, 1}, cap = {1, 1, 1};
		for (int a = 0; a < D; a++) {
			d.part[a] = cfg->part[a];
			one[a] = cfg->part[a];  // an idle slot: one partition
			cap[a] = cfg->max_size[a];
		}
		d.sizes.assign(cfg->slots, one);
		d.caps.assign(cfg->slots, cap);
		d.brick_capacity = (size_t)bricks;
		FG_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
		s->eng.reset(fg::make_engine(d, s->st));
		s->eng->set_throw_on_freeze(false);
		s->capacity = std::min<long long>(bricks, s->eng->dev().nslots);
		s->polys.reset(fg::make_polys(*s->eng, 0, cfg->vertex_capacity));
		s->slots.resize(cfg->slots);
		s->speeds.assign(cfg->slots, fg::Speed{FG_SPEED_CONST, 0.f, 0.f, 0.f, 0u});
		s->snu.assign(cfg->slots, 0);
		std::vector<int> all(cfg->slots), on(cfg->slots, 1);
		for (size_t i = 0; i < cfg->slots; i++) {
			all[i] = (int)i;
			s->polys->set_enabled((int)i, false);
		}
		s->eng->set_paused_n(all.data(), on.data(), (int)cfg->slots);
		s->stats.capacity_bricks = (unsigned long long)s->capacity;
		s->t0 = Clock::now();
		fg_server* raw = s.get();
		s->worker = std::thread([raw] { raw->run(); });
		*out = s.release();
	});
}

int fg_server_destroy(fg_server* s)
{
	return sguard([&] {
		if (!s) return;
		{
			std::lock_guard<std::mutex> g(s->mu);
			s->stop = true;
		}
		s->cv_work.notify_all();
		if (s->worker.joinable()) s->worker.join();
		s->polys.reset();
		s->eng.reset();
		if (s->st) cudaStreamDestroy(s->st);
		delete s;
	});
}

int fg_server_now(fg_server* s, double* t)
{
	return sguard([&] {
		need(s, "server");
		need(t, "time");
		*t = s->now();
	});
}

int fg_server_submit(fg_server* s, const fg_request* r)
{
	return sguard([&] {
		need(s, "server");
		need(r, "request");
		if (r->steps < 1) throw fg::Error(FG_ERR_ARG, "a request needs at least one step");
		if (r->speed.kind & ~7) throw fg::Error(FG_ERR_ARG, "unknown speed kind bits");
		bool too_large = false;
		for (int a = 0; a < s->D; a++) {
			if (r->size[a] <= 0) throw fg::Error(FG_ERR_ARG, "grid size must be positive");
			if (r->size[a] > s->cfg.max_size[a]) too_large = true;
			// the seed window must lie inside the grid (Surface::seed has no bounds guard)
			const int off = -r->size[a] / 2;
			if (r->centre[a] - s->L < off || r->centre[a] + s->L >= off + r->size[a])
				throw fg::Error(FG_ERR_ARG, "seed too close to the grid edge");
		}
		const long long need_bricks = s->bound(*r);
		const double t = s->now();
		{
			std::lock_guard<std::mutex> g(s->mu);
			s->stats.submitted++;
			if (s->stop) throw fg::Error(FG_ERR_STATE, "server stopped: " + s->fault);
			if (too_large) {
				s->stats.rejected++;
				throw fg::Error(FG_ERR_CAPACITY, "rejected: grid larger than the server's slots");
			}
			if (s->reserved + need_bricks > s->capacity) {
				s->stats.rejected++;
				throw fg::Error(FG_ERR_CAPACITY,
				                "rejected: the brick-pool budget is reserved by requests in flight");
			}
			s->reserved += need_bricks;
			s->stats.admitted++;
			s->stats.peak_reserved_bricks = std::max<unsigned long long>(
			    s->stats.peak_reserved_bricks, (unsigned long long)s->reserved);
			s->queue.push_back(Queued{*r, need_bricks, t});
		}
		s->cv_work.notify_one();
	});
}

int fg_server_poll(fg_server* s, fg_result* out, size_t cap, size_t* n, double wait_s)
{
	return sguard([&] {
		need(s, "server");
		need(n, "count");
		*n = 0;
		std::unique_lock<std::mutex> lk(s->mu);
		if (s->done.empty() && wait_s > 0)
			s->cv_done.wait_for(lk, std::chrono::duration<double>(wait_s),
			                    [&] { return !s->done.empty() || s->stop; });
		while (*n < cap && !s->done.empty()) {
			if (out) out[*n] = s->done.front();
			s->done.pop_front();
			(*n)++;
		}
	});
}

int fg_server_get_stats(fg_server* s, fg_server_stats* out)
{
	return sguard([&] {
		need(s, "server");
		need(out, "stats");
		std::lock_guard<std::mutex> g(s->mu);
		*out = s->stats;
		out->reserved_bricks = (unsigned long long)s->reserved;
		out->queued = s->queue.size();
		size_t busy = 0;
		for (const Slot& sl : s->slots) busy += sl.busy ? 1 : 0;
		out->in_flight = busy;
		out->fault_code = s->fault_code;
	});
}

int fg_server_result_dump(fg_server* s, uint64_t tag, uint32_t* out, size_t cap, size_t* n)
{
	return sguard([&] {
		need(s, "server");
		need(n, "count");
		std::lock_guard<std::mutex> g(s->mu);
		auto it = s->kept.find(tag);
		if (it == s->kept.end()) throw fg::Error(FG_ERR_ARG, "no kept output for this tag");
		*n = it->second.dump.size();
		if (out)
			std::memcpy(out, it->second.dump.data(), std::min(cap, *n) * sizeof(uint32_t));
	});
}

int fg_server_result_polys(fg_server* s, uint64_t tag, float* vtx, size_t vtx_cap, uint32_t* spx,
                           size_t spx_cap, uint32_t* counts, size_t counts_cap, size_t* nv,
                           size_t* ns, size_t* nparts)
{
	return sguard([&] {
		need(s, "server");
		need(nv, "vertex count");
		need(ns, "simplex count");
		need(nparts, "partition count");
		std::lock_guard<std::mutex> g(s->mu);
		auto it = s->kept.find(tag);
		if (it == s->kept.end()) throw fg::Error(FG_ERR_ARG, "no kept output for this tag");
		const Kept& k = it->second;
		const size_t vf = s->D == 3 ? 2 * s->D : s->D;
		*nv = k.vtx.size() / vf;
		*ns = k.spx.size() / s->D;
		*nparts = k.counts.size() / 2;
		if (vtx) std::memcpy(vtx, k.vtx.data(), std::min(vtx_cap, k.vtx.size()) * sizeof(float));
		if (spx) std::memcpy(spx, k.spx.data(), std::min(spx_cap, k.spx.size()) * sizeof(uint32_t));
		if (counts)
			std::memcpy(counts, k.counts.data(),
			            std::min(counts_cap, k.counts.size()) * sizeof(uint32_t));
	});
}

int fg_server_release(fg_server* s, uint64_t tag)
{
	return sguard([&] {
		need(s, "server");
		std::lock_guard<std::mutex> g(s->mu);
		s->kept.erase(tag);
	});
}

int fg_request_bricks(const fg_server_config* cfg, const fg_request* r, unsigned long long* bricks)
{
	return sguard([&] {
		need(cfg, "config");
		need(r, "request");
		need(bricks, "bricks");
		if (cfg->dims != 2 && cfg->dims != 3) throw fg::Error(FG_ERR_ARG, "dims must be 2 or 3");
		for (int a = 0; a < cfg->dims; a++)
			if (cfg->part[a] <= 0 || r->size[a] <= 0)
				throw fg::Error(FG_ERR_ARG, "part and size must be positive");
		*bricks = (unsigned long long)request_bricks(cfg->dims, cfg->layers, cfg->part, *r);
	});
}

int fg_brick_bytes(int dims, int layers, const int* part, double* bytes)
{
	return sguard([&] {
		need(part, "part");
		need(bytes, "bytes");
		if (dims != 2 && dims != 3) throw fg::Error(FG_ERR_ARG, "dims must be 2 or 3");
		*bytes = brick_bytes(dims, layers, part);
	});
}

}  // extern "C"
