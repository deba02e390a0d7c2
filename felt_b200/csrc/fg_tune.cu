// Launch tuning by measurement (fg_autotune, fg_config.autotune).
//
// The global update's kernels have two shape knobs that depend on the brick (partition) size and
// the GPU: the warps given to each partition entry in the first distance pass (dist_split) and
// whether the passes that record status changes take a warp or a block per entry
// (record_passes). The automatic choice follows the brick size; the sweep here times each
// sensible pair on a scratch surface of this (D, L, partition) instead and keeps the fastest.
// Results are cached per (D, L, partition, device) for the life of the process and, when the
// environment variable FELT_TUNE_CACHE names a file, in that file (one line per key), so a
// later process skips the sweep. The knobs change launch shapes only: every list, order and
// value is the same whichever pair runs.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "fg_engine.cuh"

namespace fg {

namespace {

std::mutex g_tune_mu;
std::map<std::string, std::pair<int, int>> g_tuned;

std::string tune_key(int D, int L, const int* part)
{
	int dev = 0;
	cudaDeviceProp prop;
	std::memset(&prop, 0, sizeof(prop));
	if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
		cudaGetLastError();
		std::snprintf(prop.name, sizeof(prop.name), "unknown");
	}
	std::ostringstream k;
	k << "D" << D << "_L" << L << "_p";
	for (int a = 0; a < D; a++) k << (a ? "x" : "") << part[a];
	k << "_sm" << prop.major << prop.minor << "x" << prop.multiProcessorCount << "_";
	for (const char* c = prop.name; *c; c++) k << (*c == ' ' ? '-' : *c);
	return k.str();
}

bool file_lookup(const std::string& key, int& ds, int& rp)
{
	const char* path = std::getenv("FELT_TUNE_CACHE");
	if (!path || !*path) return false;
	std::ifstream f(path);
	std::string line;
	bool found = false;
	while (std::getline(f, line)) {
		std::istringstream in(line);
		std::string k;
		int a = 0, b = 0;
		if ((in >> k >> a >> b) && k == key) {
			ds = a;  // the last line for a key wins
			rp = b;
			found = true;
		}
	}
	return found;
}

void file_store(const std::string& key, int ds, int rp)
{
	const char* path = std::getenv("FELT_TUNE_CACHE");
	if (!path || !*path) return;
	std::ofstream f(path, std::ios::app);
	f << key << " " << ds << " " << rp << "\n";
}

/// Device time of `timed` updates of a scratch surface under one tuning, after the same
/// deterministic growth: a sphere seeded at the centre, grown by constant-speed updates to a
/// quarter of the grid's edge, then curvature-plus-constant updates timed.
double time_candidate(int D, int L, const int* part, int ds, int rp)
{
	PoolDesc d;
	d.D = D;
	d.L = L;
	std::array<int, 3> sz = {1, 1, 1};
	int edge = 0;
	for (int a = 0; a < D; a++) {
		d.part[a] = part[a];
		int e = std::max(64, 8 * part[a]);
		e = std::min(e, 256);
		e = (e + part[a] - 1) / part[a] * part[a];
		sz[a] = e;
		edge = a ? std::min(edge, e) : e;
	}
	d.sizes.push_back(sz);
	cudaStream_t st = nullptr;
	if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
		throw Error(-2, "autotune: stream creation failed");
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	double ms = 0;
	try {
		std::unique_ptr<EngineBase> eng(make_engine(d, st));
		eng->set_tuning(0, ds, rp, 0, 0);
		const int centre[3] = {0, 0, 0};
		eng->seed(0, centre);
		const Speed grow{1, -1.0f, 0.0f, 0.0f, 0u};
		const int steps = std::max(4, edge / 4 - L - 2);
		for (int i = 0; i < steps; i++) eng->update_builtin(&grow);
		const Speed flow{1 | 2, -0.4f, -0.2f, 0.0f, 0u};
		eng->update_builtin(&flow);  // the graphs this speed kind uses, captured untimed
		FG_CUDA(cudaEventCreate(&e0));
		FG_CUDA(cudaEventCreate(&e1));
		const int timed = 6;
		FG_CUDA(cudaEventRecord(e0, st));
		for (int i = 0; i < timed; i++) eng->update_builtin(&flow);
		FG_CUDA(cudaEventRecord(e1, st));
		FG_CUDA(cudaEventSynchronize(e1));
		float t = 0;
		FG_CUDA(cudaEventElapsedTime(&t, e0, e1));
		ms = t / timed;
	} catch (...) {
		if (e0) cudaEventDestroy(e0);
		if (e1) cudaEventDestroy(e1);
		cudaStreamDestroy(st);
		throw;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaStreamDestroy(st);
	return ms;
}

}  // namespace

void tune_candidates(int D, const int* part, std::vector<std::pair<int, int>>& out)
{
	long long bv = 1;
	for (int a = 0; a < D; a++) bv *= part[a];
	out.clear();
	for (int ds : {1, 2, 4, 8}) {
		if (ds > 1 && 32LL * ds > bv) continue;  // warps that would find no leaves
		for (int rp : {1, 2})
			if (rp == 1 || bv >= 256) out.push_back({ds, rp});
	}
}

void autotune(int D, int L, const int* part, int& ds, int& rp, std::vector<double>* ms,
              bool force)
{
	const std::string key = tune_key(D, L, part);
	{
		std::lock_guard<std::mutex> lk(g_tune_mu);
		if (!force) {
			auto it = g_tuned.find(key);
			if (it != g_tuned.end()) {
				ds = it->second.first;
				rp = it->second.second;
				if (ms) ms->clear();
				return;
			}
			if (file_lookup(key, ds, rp)) {
				g_tuned[key] = {ds, rp};
				if (ms) ms->clear();
				return;
			}
		}
	}
	std::vector<std::pair<int, int>> cand;
	tune_candidates(D, part, cand);
	std::vector<double> t(cand.size());
	size_t best = 0;
	for (size_t i = 0; i < cand.size(); i++) {
		t[i] = time_candidate(D, L, part, cand[i].first, cand[i].second);
		if (t[i] < t[best]) best = i;
	}
	ds = cand[best].first;
	rp = cand[best].second;
	if (ms) *ms = t;
	std::lock_guard<std::mutex> lk(g_tune_mu);
	g_tuned[key] = {ds, rp};
	file_store(key, ds, rp);
}

}  // namespace fg
