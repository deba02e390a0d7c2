// Launch counting and optional per-kernel CUDA-event timing for every kernel of the library.
#include <atomic>
#include <map>
#include <string>
#include <mutex>

#include "fg_engine.cuh"

namespace fg {

namespace {

struct Pending {
	const char* name;
	cudaEvent_t a, b;
};

struct Prof {
	std::mutex mu;
	bool on = false;
	std::vector<Pending> pending;
	std::vector<cudaEvent_t> spare;
	std::map<std::string, std::pair<double, long long>> acc;
	const char* cur = nullptr;
	cudaEvent_t cur_a = nullptr;
	std::string only;  // when set, only launches of this kernel are bracketed
};

Prof& prof()
{
	static Prof p;
	return p;
}
std::atomic<long long> g_launches{0};

cudaEvent_t take(Prof& p)
{
	if (!p.spare.empty()) {
		cudaEvent_t e = p.spare.back();
		p.spare.pop_back();
		return e;
	}
	cudaEvent_t e;
	cudaEventCreate(&e);
	return e;
}

void drain(Prof& p)
{
	for (Pending& q : p.pending) {
		float ms = 0.0f;
		cudaEventSynchronize(q.b);
		cudaEventElapsedTime(&ms, q.a, q.b);
		auto& s = p.acc[q.name];
		s.first += ms;
		s.second += 1;
		p.spare.push_back(q.a);
		p.spare.push_back(q.b);
	}
	p.pending.clear();
}

}  // namespace

void prof_begin(const char* name, cudaStream_t st)
{
	g_launches.fetch_add(1, std::memory_order_relaxed);
	Prof& p = prof();
	if (!p.on) return;
	std::lock_guard<std::mutex> lk(p.mu);
	if (!p.only.empty() && p.only != name) return;
	p.cur = name;
	p.cur_a = take(p);
	cudaEventRecord(p.cur_a, st);
}

void prof_end(cudaStream_t st)
{
	Prof& p = prof();
	if (!p.on || !p.cur) return;
	std::lock_guard<std::mutex> lk(p.mu);
	cudaEvent_t b = take(p);
	cudaEventRecord(b, st);
	p.pending.push_back(Pending{p.cur, p.cur_a, b});
	p.cur = nullptr;
	if (p.pending.size() > 4096) drain(p);
}

long long launch_count() { return g_launches.load(); }

void add_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

bool prof_on()
{
	Prof& p = prof();
	std::lock_guard<std::mutex> lk(p.mu);
	return p.on;
}

void prof_enable(bool on)
{
	Prof& p = prof();
	std::lock_guard<std::mutex> lk(p.mu);
	p.on = on;
}

std::vector<ProfEntry> prof_read()
{
	Prof& p = prof();
	std::lock_guard<std::mutex> lk(p.mu);
	drain(p);
	std::vector<ProfEntry> out;
	for (auto& kv : p.acc) out.push_back(ProfEntry{kv.first, kv.second.first, kv.second.second});
	return out;
}

void prof_only(const char* name)
{
	Prof& p = prof();
	std::lock_guard<std::mutex> lk(p.mu);
	p.only = name ? name : "";
}

void prof_reset()
{
	Prof& p = prof();
	std::lock_guard<std::mutex> lk(p.mu);
	drain(p);
	p.acc.clear();
}

}  // namespace fg
