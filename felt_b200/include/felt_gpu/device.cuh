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
#include "../../csrc/fg_field.cuh"
#include "felt_gpu.h"

/// The device view handed out by fg_update_begin_global: the engine's pool description.
struct fg_device_view {
	fg::Dev dev;
};

namespace felt_gpu {

template <int D>
using DevVec = fg::Vec<D>;

/// A D-vector of floats returned by the gradient functions.
template <int D>
struct DevVecF {
	float v[D];
	__host__ __device__ float& operator[](int i) { return v[i]; }
	__host__ __device__ const float& operator[](int i) const { return v[i]; }
};

/// Read access to the isogrid from a speed functor: get (Access::get with the lazy child get,
/// PartitionedMixin.hpp:594-601), curv (NumericMixin.hpp:72-156), inside (GridMixin inside), and
/// the rest of the reference's Numeric API (NumericMixin.hpp:165-355): grad, gradF, gradB,
/// gradC, gradE, divergence. Like the reference's templates on the position type, each takes a
/// node (DevVec<D>) or a real position (DevVecF<D>); at a real position get is interp (linear
/// interpolation of the 2^D corners, NumericMixin.hpp:382-481), inside is the float test
/// offset <= p < offset + size, and the stencils step the coordinates by +-1 in float. FP32
/// rounded step by step as the reference's code (the grid spacing dx is 1, so its final
/// divisions by dx change nothing).
template <int D, int L>
struct IsoGridView {
	const fg::Dev* P;
	const fg::SurfGeom* g;
	__device__ float get(const DevVec<D>& p) const { return fg::get_phi<D, L>(*P, *g, p); }
	__device__ float get(const DevVecF<D>& p) const { return interp(p); }
	__device__ bool inside(const DevVec<D>& p) const { return fg::in_grid<D>(*g, p); }
	__device__ bool inside(const DevVecF<D>& p) const { return fg::inside_f<D, L>(*g, p.v); }
	/// interp (NumericMixin.hpp:403-481): corners in bit order, reduced along axis 0 first.
	__device__ float interp(const DevVecF<D>& p) const
	{
		return fg::interp<D>([this](const DevVec<D>& q) { return get(q); }, p.v);
	}
	template <class Pos>
	__device__ float curv(const Pos& p) const
	{
		return fg::curv_g<D>([this](const Pos& q) { return get(q); }, p);
	}

	/// grad (NumericMixin.hpp:189-231): central difference, one-sided at the grid's edge, 0
	/// where neither neighbour is inside.
	template <class Pos>
	__device__ DevVecF<D> grad(const Pos& p) const
	{
		DevVecF<D> r;
		const float centre = get(p);
		Pos t = p;
		for (int a = 0; a < D; a++) {
			float back = centre, fwd = centre;
			int order = 0;
			t[a] -= 1;
			if (inside(t)) {
				back = get(t);
				order++;
			}
			t[a] += 2;
			if (inside(t)) {
				fwd = get(t);
				order++;
			}
			t[a] -= 1;
			r[a] = order ? __fdiv_rn(__fsub_rn(fwd, back), (float)order) : 0.0f;
		}
		return r;
	}
	/// gradE (NumericMixin.hpp:243-270): the upwind (entropy-satisfying) gradient,
	/// max(centre - back, 0) + min(forward - centre, 0) per axis.
	template <class Pos>
	__device__ DevVecF<D> gradE(const Pos& p) const
	{
		DevVecF<D> r;
		const float centre = get(p);
		Pos t = p;
		for (int a = 0; a < D; a++) {
			t[a] -= 1;
			const float back = __fsub_rn(centre, get(t));
			t[a] += 2;
			const float fwd = __fsub_rn(get(t), centre);
			t[a] -= 1;
			const float b = back < 0.0f ? 0.0f : back;  // std::max(back, 0.0f)
			const float f = 0.0f < fwd ? 0.0f : fwd;    // std::min(fwd, 0.0f)
			r[a] = __fadd_rn(f, b);
		}
		return r;
	}
	/// gradF (NumericMixin.hpp:279-298): forward difference.
	template <class Pos>
	__device__ DevVecF<D> gradF(const Pos& p) const
	{
		DevVecF<D> r;
		const float centre = get(p);
		Pos t = p;
		for (int a = 0; a < D; a++) {
			t[a] += 1;
			r[a] = __fsub_rn(get(t), centre);
			t[a] -= 1;
		}
		return r;
	}
	/// gradB (NumericMixin.hpp:308-326): backward difference.
	template <class Pos>
	__device__ DevVecF<D> gradB(const Pos& p) const
	{
		DevVecF<D> r;
		const float centre = get(p);
		Pos t = p;
		for (int a = 0; a < D; a++) {
			t[a] -= 1;
			r[a] = __fsub_rn(centre, get(t));
			t[a] += 1;
		}
		return r;
	}
	/// gradC (NumericMixin.hpp:335-355): central difference.
	template <class Pos>
	__device__ DevVecF<D> gradC(const Pos& p) const
	{
		DevVecF<D> r;
		Pos t = p;
		for (int a = 0; a < D; a++) {
			t[a] -= 1;
			const float back = get(t);
			t[a] += 2;
			const float fwd = get(t);
			t[a] -= 1;
			r[a] = __fdiv_rn(__fsub_rn(fwd, back), 2.0f);
		}
		return r;
	}
	/// divergence (NumericMixin.hpp:165-175): the sum of gradF - gradB over the axes (Eigen's
	/// fixed-size sum: x0 + (x1 + x2) in 3D).
	template <class Pos>
	__device__ float divergence(const Pos& p) const
	{
		const DevVecF<D> f = gradF(p), b = gradB(p);
		float d[D];
		for (int a = 0; a < D; a++) d[a] = __fsub_rn(f[a], b[a]);
		return D == 2 ? __fadd_rn(d[0], d[1]) : __fadd_rn(d[0], __fadd_rn(d[1], d[D - 1]));
	}
};

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
