// Device side of the C++ facade: Surface<D,L>::update(fn) with a caller-supplied __device__
// functor, the counterpart of Felt's `update(fn)` (include/Felt/Surface.hpp:254-294) and its
// functor dispatch (Surface.hpp:1754-1802).
//
// The reference accepts any callable returning float and taking (pos, isogrid), (pos) or ().
// Here the callable must be usable in device code (a struct with a __device__ operator(), or an
// nvcc extended lambda) and is called once per zero-layer node, concurrently, so it must be pure,
// exactly as the reference's OpenMP loop requires. The functor's translation unit is compiled by
// the caller's nvcc for sm_100a; this header launches its delta kernel between
// fg_update_begin_global and fg_update_finish_global on the surface's stream. Compile it with
// -fmad=false when the speed must round exactly like the CPU reference.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "../../csrc/fg_dev.cuh"
#include "../../csrc/fg_numeric.cuh"
#include "felt_gpu.h"

/// The device view handed out by fg_update_begin_global: the engine's pool description.
struct fg_device_view {
	fg::Dev dev;
};

namespace felt_gpu {

template <int D>
using DevVec = fg::Vec<D>;

/// A D-vector of floats: a real position, or what the gradient functions return.
template <int D>
using DevVecF = fg::VecF<D>;

/// Read access to the isogrid from a speed functor: get, curv, inside and the rest of the
/// reference's Numeric API (NumericMixin.hpp:72-481), each at a node (DevVec<D>) or a real
/// position (DevVecF<D>, read by interpolation); see fg::IsoView.
template <int D, int L>
using IsoGridView = fg::IsoView<D, L>;

namespace detail {

template <int D, int L, class Fn>
__device__ __forceinline__ float call_speed(const Fn& fn, const DevVec<D>& pos,
                                            const IsoGridView<D, L>& iso)
{
	if constexpr (std::is_invocable_v<const Fn&, const DevVec<D>&, const IsoGridView<D, L>&>)
		return fn(pos, iso);
	else if constexpr (std::is_invocable_v<const Fn&, const DevVec<D>&>)
		return fn(pos);
	else
		return fn();
}

/// One warp per zero-layer partition entry (entry offsets: the engine's zero-layer scan); each
/// lane evaluates the functor at its leaves and writes the delta grid.
template <int D, int L, class Fn>
__global__ void __launch_bounds__(256) k_user_delta(fg::Dev P, Fn fn)
{
	constexpr int NL = 2 * L + 1;
	const int lane = threadIdx.x & 31;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	const int total = P.woff[P.S];
	for (int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < total; e += nwarps) {
		const int s = fg::entry_surface(P.woff, P.S, e);
		const fg::SurfGeom& g = P.geom[s];
		const int gp = g.pbase + P.plist[(size_t)L * P.NP + g.pbase + (e - P.woff[s])];
		const int sl = P.slot[gp];
		const int n = P.lcnt[sl * NL + L];
		const uint16_t* lst = P.lst + ((size_t)sl * NL + L) * P.BV;
		const IsoGridView<D, L> iso{&P, &g};
		for (int j = lane; j < n; j += 32) {
			const int leaf = lst[j];
			P.dlt[(size_t)sl * P.BV + leaf] =
			    call_speed<D, L>(fn, fg::leaf_pos<D>(P, gp, leaf), iso);
		}
		if (lane == 0) atomicAdd(&P.kstat[fg::KS_ZERO], (unsigned long long)n);
	}
}

}  // namespace detail

/// update(fn) on a surface handle: update_start + delta.track_children, the functor over the
/// zero layer, then update_end_global. Returns the C ABI status (0 = OK).
template <int D, int L, class Fn>
int update_device(fg_surface* s, const Fn& fn)
{
	const fg_device_view* view = nullptr;
	void* stream = nullptr;
	int rc = fg_update_begin_global(s, &view, &stream);
	if (rc) return rc;
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	detail::k_user_delta<D, L, Fn><<<sms * 8, 256, 0, (cudaStream_t)stream>>>(view->dev, fn);
	if (cudaGetLastError() != cudaSuccess) return FG_ERR_CUDA;
	return fg_update_finish_global(s);
}

}  // namespace felt_gpu
