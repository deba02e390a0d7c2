// fg_snapshot_noalloc: a dense isogrid snapshot into a caller's host buffer that allocates no
// memory at all.
//
// fg_snapshot with a host destination stages the dense grid in a device buffer that it
// allocates and frees on every call. Some callers cannot allow that: a host process whose
// device memory is owned and budgeted by another allocator (a framework's caching allocator,
// or a fixed reservation that leaves no room for the driver's allocations), or a real-time loop
// that must not enter the driver's allocator, whose cudaMalloc and cudaFree can stall or
// synchronise the whole device. This entry point stages through a fixed device array instead,
// declared below at file scope, so it never calls cudaMalloc, cudaFree or any allocating
// library routine.
//
// Limits and sharing:
//  - At most FG_NOALLOC_SNAPSHOT_MAX floats (2^21 = 2,097,152, e.g. a 128^3 or 1448^2 grid,
//    8 MiB) per call; larger grids are rejected with FG_ERR_CAPACITY.
//  - The array lives in every GPU that loads this library, for the life of the process.
//  - Every call shares it and it keeps the previous call's contents; the kernel writes every
//    element it later copies out, so nothing needs clearing. Calls that overlapped on the GPU
//    would race on the array, so calls are serialised by a process-wide lock and each call
//    waits for its copy to finish before returning.
//  - The call runs on the surface's own device (made current for the call when another device
//    is current). The first call on a device looks up the array's device address with that
//    device current (cudaGetSymbolAddress); that first call should come before any stream
//    capture.
#include <mutex>
#include <string>

#include "../../include/felt_gpu.h"
#include "fg_handles.cuh"
#include "fg_kernels.cuh"

/// Capacity of the fixed staging array, in floats (8 MiB).
#define FG_NOALLOC_SNAPSHOT_MAX (1u << 21)

namespace {

static __device__ __align__(256) float g_snapshot_scratch[FG_NOALLOC_SNAPSHOT_MAX];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_scratch_ptr[kMaxDevices] = {};

/// Device address of the scratch array on the current device, looked up once per device.
float* scratch_for_current_device()
{
	int dev = 0;
	FG_CUDA(cudaGetDevice(&dev));
	if (dev < 0 || dev >= kMaxDevices) throw fg::Error(FG_ERR_ARG, "device ordinal too large");
	if (!g_scratch_ptr[dev]) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_snapshot_scratch);
		if (e != cudaSuccess)
			throw fg::Error(FG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
			                                 cudaGetErrorString(e));
		g_scratch_ptr[dev] = static_cast<float*>(p);
	}
	return g_scratch_ptr[dev];
}

template <int D, int L>
__global__ void k_snapshot_scratch(fg::Dev P, float* scratch, long long total)
{
	const fg::SurfGeom& g = P.geom[0];
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
	     i += (long long)gridDim.x * blockDim.x) {
		fg::Vec<D> p;
		long long r = i;
		for (int a = D - 1; a >= 0; a--) {
			p[a] = (int)(r % g.size[a]) + g.off[a];
			r /= g.size[a];
		}
		scratch[i] = fg::get_phi<D, L>(P, g, p);
	}
}

void launch(int D, int L, const fg::Dev& P, float* scratch, long long total, cudaStream_t st)
{
	const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
#define FG_CASE(d, l)                                                                         \
	if (D == d && L == l) {                                                                   \
		FG_RUN("k_snapshot_scratch", st,                                                      \
		       k_snapshot_scratch<d, l><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(P, scratch, total)); \
		return;                                                                               \
	}
	FG_CASE(2, 1) FG_CASE(2, 2) FG_CASE(2, 3) FG_CASE(2, 4)
	FG_CASE(3, 1) FG_CASE(3, 2) FG_CASE(3, 3) FG_CASE(3, 4)
#undef FG_CASE
	throw fg::Error(FG_ERR_ARG, "unsupported dims/layers");
}

/// Makes `dev` the current device for the life of the guard, and restores the caller's.
struct DeviceGuard {
	int prev = -1;
	explicit DeviceGuard(int dev)
	{
		FG_CUDA(cudaGetDevice(&prev));
		if (prev != dev) FG_CUDA(cudaSetDevice(dev));
	}
	~DeviceGuard()
	{
		int cur = -1;
		if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
	}
};

/// The device whose memory holds the surface's pool (its geometry table lives there).
int surface_device(const fg::EngineBase& eng)
{
	cudaPointerAttributes at{};
	FG_CUDA(cudaPointerGetAttributes(&at, eng.dev().geom));
	if (at.type != cudaMemoryTypeDevice) throw fg::Error(FG_ERR_ARG, "surface not on a device");
	return at.device;
}

}  // namespace

extern "C" FG_API int fg_snapshot_noalloc(fg_surface* s, float* dst, size_t n)
{
	try {
		if (!s || !dst) throw fg::Error(FG_ERR_ARG, "null surface or destination");
		std::lock_guard<std::mutex> lk(g_mu);
		fg::EngineBase& eng = *s->eng;
		const DeviceGuard on(surface_device(eng));
		const fg::Dev& P = eng.dev();
		const fg::SurfGeom& g = eng.geometry(0);  // host copy of P.geom[0]
		long long total = 1;
		for (int a = 0; a < eng.dims(); a++) total *= g.size[a];
		if (total > (long long)FG_NOALLOC_SNAPSHOT_MAX)
			throw fg::Error(FG_ERR_CAPACITY,
			                "fg_snapshot_noalloc: grid of " + std::to_string(total) +
			                    " nodes exceeds the fixed staging array of " +
			                    std::to_string(FG_NOALLOC_SNAPSHOT_MAX) + " floats");
		if ((long long)n < total) throw fg::Error(FG_ERR_CAPACITY, "snapshot buffer too small");
		float* scratch = scratch_for_current_device();
		launch(eng.dims(), eng.layers(), P, scratch, total, eng.stream());
		FG_CUDA(cudaGetLastError());
		FG_CUDA(cudaMemcpyAsync(dst, scratch, (size_t)total * sizeof(float),
		                        cudaMemcpyDeviceToHost, eng.stream()));
		FG_CUDA(cudaStreamSynchronize(eng.stream()));
		return FG_OK;
	} catch (const fg::Error& e) {
		fg::set_last_error(e.what());
		return e.code;
	} catch (const std::exception& e) {
		fg::set_last_error(e.what());
		return FG_ERR_ARG;
	}
}
