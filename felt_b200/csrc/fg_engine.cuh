// Host-side engine: owns one device pool of S surfaces (same D, L and partition shape) and
// drives the kernels of fg_kernels.cuh. A single Felt Surface is a pool with S = 1; the batched
// and serving paths use the same pool with many surfaces, so every kernel launch advances all of
// them together.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fg_dev.cuh"

namespace fg {

/// Error carrying a felt_gpu.h status code.
struct Error : std::runtime_error {
	int code;
	Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define FG_CUDA(x)                                                                       \
	do {                                                                                 \
		cudaError_t e_ = (x);                                                            \
		if (e_ != cudaSuccess)                                                           \
			throw ::fg::Error(-2, std::string(#x ": ") + cudaGetErrorString(e_));        \
	} while (0)

struct PoolDesc {
	int D = 3, L = 2;
	int part[3] = {8, 8, 8};
	std::vector<std::array<int, 3>> sizes;  // per surface grid size
	/// Per surface, the largest grid (per axis) it may be given later by reset_surface: its
	/// partition range is sized for any grid up to this and for its own size; empty = its own
	/// size only.
	std::vector<std::array<int, 3>> caps;
	size_t brick_capacity = 0;              // 0 = automatic
};

/// Per-step accounting the benchmarks and the serving loop read.
struct StepStats {
	unsigned long long node_updates = 0;  // band size at the start of each step, summed
	int iterations = 0;                   // distance/flush/expand iterations of the last step
};

class EngineBase {
public:
	virtual ~EngineBase() = default;
	virtual int dims() const = 0;
	virtual int layers() const = 0;
	virtual int surfaces() const = 0;
	virtual cudaStream_t stream() const = 0;

	virtual void seed(int s, const int* pos) = 0;
	/// One seed per surface, centres holding S*D ints.
	virtual void seed_all(const int* centres) = 0;
	/// Global update of every surface of the pool with one builtin speed per surface
	/// (host array of S speeds).
	virtual void update_builtin(const Speed* speeds) = 0;
	/// The two halves of update(fn) around a caller-supplied delta kernel.
	virtual void update_begin_global() = 0;
	virtual void update_finish_global() = 0;
	/// Local update of surface 0: update_start(), delta(pos,v)..., update_end().
	virtual void update_local(const std::vector<int>& pos, const std::vector<float>& vals) = 0;
	virtual void update_bounded(const int* lo, const int* hi, const Speed& sp) = 0;

	virtual void snapshot(int s, float* dst, size_t n, bool dst_device) = 0;
	virtual float get(int s, const int* pos) = 0;
	virtual size_t partitions(int s, int* ccount, int* coff) = 0;
	virtual std::vector<uint32_t> layer_list(int s, size_t part, int li) = 0;
	virtual std::vector<uint32_t> partition_list(int s, int which, int li) = 0;
	/// Leaf list of the affected lookup (Surface::affected(), Surface.hpp:693-696).
	virtual std::vector<uint32_t> affected_list(int s, size_t part, int li) = 0;
	virtual void partition_state(int s, size_t part, int* active, float* bg) = 0;
	virtual std::vector<uint32_t> dump(int s) = 0;
	virtual unsigned long long band_size(int s) = 0;
	virtual void check_errors() = 0;
	virtual StepStats& stats() = 0;
	/// Sum over all global updates so far of the band size at each update's start.
	virtual unsigned long long node_updates() = 0;
	/// True once surface s has been stopped after an update whose convergence loop did not
	/// terminate; no kernel works on it afterwards.
	virtual bool frozen(int s) const = 0;
	/// Whether an update that stops a surface raises (single surfaces) or only records it
	/// (batches, serving).
	virtual void set_throw_on_freeze(bool on) = 0;
	/// Pauses (or resumes) surface s: while paused no kernel works on it, so its state stays
	/// exactly as after its last update. Used to retire finished requests of a served batch.
	virtual void set_paused(int s, bool on) = 0;
	virtual bool paused(int s) const = 0;
	/// Serving: makes surface s empty (its bricks back to the pool, no partition active or
	/// listed, no status, no record of its stop) with grid `size`, whose partitions must fit
	/// the range the surface was created with. Its paused state is left as it is. Asynchronous.
	virtual void reset_surface(int s, const int* size) = 0;
	/// seed(pos) of surface s without waiting for it; errors show at the next check.
	virtual void seed_async(int s, const int* pos) = 0;
	/// set_paused for several surfaces at once (one device update).
	virtual void set_paused_n(const int* surfaces, const int* on, int n) = 0;
	/// Node updates per surface since it was created or last reset (S values; synchronises).
	virtual void surface_node_updates(unsigned long long* out) = 0;
	/// Bricks on the pool's free stack (synchronises).
	virtual long long free_bricks() = 0;
	/// Partitions reserved for surface s (the most any grid it is given may have).
	virtual int partition_capacity(int s) const = 0;
	/// Launch tuning: launch_mode 0 automatic (= 1), 1 the whole global update as one CUDA
	/// graph, 2 every kernel launched from the host, no graphs; dist_split warps per partition entry in the first distance pass (0 = automatic);
	/// record_passes 1 warp, 2 block per entry in the passes that record status changes (0 =
	/// automatic); delta_kernel of curvature speeds 1 direct, 2 staged brick + halo (0 =
	/// automatic); fuse_passes 1 the global update's distance passes as 4L launches, 2 as 2L+1
	/// fused ones (0 = automatic).
	virtual void set_tuning(int launch_mode, int dist_split, int record_passes, int delta_kernel,
	                        int fuse_passes) = 0;
	/// The tuning in effect (5 values): launch mode (1 one graph, 2 phase by phase),
	/// dist_split, record_passes (1 warp, 2 block), delta kernel (1 direct, 2 staged), distance
	/// passes (1 separate, 2 fused).
	virtual void tuning(int* out) const = 0;
	virtual const Dev& dev() const = 0;
	/// Host copy of surface s's geometry (the same as dev().geom[s]).
	virtual const SurfGeom& geometry(int s) const = 0;
	virtual void sync() = 0;
	virtual int part(int a) const = 0;
};

EngineBase* make_engine(const PoolDesc& desc, cudaStream_t stream);

/// Launch tuning by measurement (fg_tune.cu): the (dist_split, record_passes) pairs worth
/// timing for a partition shape, and the fastest of them for (D, L, part) on the current
/// device, timed on a scratch surface unless cached (ms: each candidate's device time per
/// update, empty when cached; force: time again).
void tune_candidates(int D, const int* part, std::vector<std::pair<int, int>>& out);
void autotune(int D, int L, const int* part, int& ds, int& rp, std::vector<double>* ms,
              bool force);

/// Makes memory freed by cudaFreeAsync stay in the current device's stream-ordered pool for
/// the next cudaMallocAsync (polygon arenas, ray queues) instead of going back to the driver
/// at every synchronisation.
void keep_pool_memory();

// ---- launch accounting and per-kernel timing ----
/// Called around every kernel launch of the library: counts launches and, when profiling is
/// enabled, brackets the launch with CUDA events on its stream.
void prof_begin(const char* name, cudaStream_t st);
void prof_end(cudaStream_t st);
long long launch_count();
/// Accounts for launches made by a graph replay (each captured launch counted once per replay).
void add_launches(long long n);
/// Whether per-launch profiling is on (launches then go one by one, not through graphs).
bool prof_on();
void prof_enable(bool on);
/// Brackets only the launches of the named kernel (NULL or "" = every kernel).
void prof_only(const char* name);
/// Synchronises pending events and returns (name, total ms, launches) per kernel name.
struct ProfEntry {
	std::string name;
	double ms;
	long long launches;
};
std::vector<ProfEntry> prof_read();

/// Launches a kernel that begins with pdl_enter() with programmatic stream serialisation: its
/// launch overlaps the end of the previous kernel on the stream instead of following it.
template <class... KArgs, class... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                Args&&... args)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = st;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
	if (e != cudaSuccess) throw Error(-2, std::string("kernel launch: ") + cudaGetErrorString(e));
}

/// Graph captures and the library's calls that synchronise the whole device (cudaMalloc,
/// cudaFree, cudaDeviceSynchronize) hold this lock: made from another thread while a stream is
/// being captured, such a call can invalidate the capture (engines of one process run in
/// several host threads when a server drives several batches).
std::recursive_mutex& device_lock();

template <class T>
inline cudaError_t locked_malloc(T** p, size_t bytes)
{
	std::lock_guard<std::recursive_mutex> g(device_lock());
	return cudaMalloc((void**)p, bytes);
}

inline cudaError_t locked_free(void* p)
{
	std::lock_guard<std::recursive_mutex> g(device_lock());
	return cudaFree(p);
}
void prof_reset();

#define FG_RUN(name, st, ...)            \
	do {                                 \
		::fg::prof_begin(name, st);      \
		__VA_ARGS__;                     \
		::fg::prof_end(st);              \
	} while (0)

}  // namespace fg
