// Field sampling at real positions shared by the polygoniser and the raycaster: the isogrid's
// interpolation, gradients and Eigen's normalisation, in the reference's FP32 order.
#pragma once

#include "fg_dev.cuh"

namespace fg {

/// GridMixin inside() for a real position (Util.hpp:95-106): offset <= p < offset + size.
template <int D, int L>
__device__ __forceinline__ bool inside_f(const SurfGeom& g, const float* p)
{
	for (int a = 0; a < D; a++) {
		if (p[a] >= (float)g.hi[a]) return false;
		if (p[a] < (float)g.off[a]) return false;
	}
	return true;
}

/// The reduction of interp (NumericMixin.hpp:403-481): corner values v in bit order (bit a set
/// = +1 along axis a), reduced along axis 0 first with weights from the fractions pc.
template <int D>
__device__ __forceinline__ float interp_reduce(float* v, const float* pc)
{
#pragma unroll
	for (int r = 0; r < D; r++) {
		const float t = pc[r];
#pragma unroll
		for (int i = 0; i < (1 << (D - 1 - r)); i++)
			v[i] = __fadd_rn(__fmul_rn(t, v[2 * i + 1]), __fmul_rn(__fsub_rn(1.0f, t), v[2 * i]));
	}
	return v[0];
}

/// interp (NumericMixin.hpp:403-481): corners in bit order, reduced along axis 0 first.
template <int D, class Get>
__device__ __forceinline__ float interp(const Get& get, const float* p)
{
	Vec<D> fl;
	float pc[D];
#pragma unroll
	for (int a = 0; a < D; a++) {
		const float f = floorf(p[a]);
		fl[a] = (int)f;
		pc[a] = __fsub_rn(p[a], f);
	}
	float v[1 << D];
#pragma unroll
	for (int i = 0; i < (1 << D); i++) {
		Vec<D> q = fl;
#pragma unroll
		for (int a = 0; a < D; a++) q[a] += (i >> a) & 1;
		v[i] = get(q);
	}
	return interp_reduce<D>(v, pc);
}

/// grad (NumericMixin.hpp:188-231) at an integer node.
template <int D, class Get>
__device__ __forceinline__ void grad_i(const Get& get, const SurfGeom& g, const Vec<D>& p, float* out)
{
	const float centre = get(p);
	Vec<D> t = p;
#pragma unroll
	for (int a = 0; a < D; a++) {
		float back = centre, fwd = centre;
		int order = 0;
		t[a] -= 1;
		if (in_grid<D>(g, t)) {
			back = get(t);
			order++;
		}
		t[a] += 2;
		if (in_grid<D>(g, t)) {
			fwd = get(t);
			order++;
		}
		t[a] -= 1;
		out[a] = order ? __fdiv_rn(__fsub_rn(fwd, back), (float)order) : 0.0f;
	}
}

/// grad (NumericMixin.hpp:188-231) at a real position whose interpolated value `centre` is
/// known, over any interpolation ip(position): the probe coordinate steps -1, +2, -1 in FP32.
template <int D, int L, class Interp>
__device__ __forceinline__ void grad_with(const Interp& ip, const SurfGeom& g, const float* p,
                                          float centre, float* out)
{
	float t[D];
#pragma unroll
	for (int a = 0; a < D; a++) t[a] = p[a];
#pragma unroll
	for (int a = 0; a < D; a++) {
		float back = centre, fwd = centre;
		int order = 0;
		t[a] = __fsub_rn(t[a], 1.0f);
		if (inside_f<D, L>(g, t)) {
			back = ip(t);
			order++;
		}
		t[a] = __fadd_rn(t[a], 2.0f);
		if (inside_f<D, L>(g, t)) {
			fwd = ip(t);
			order++;
		}
		t[a] = __fsub_rn(t[a], 1.0f);
		out[a] = order ? __fdiv_rn(__fsub_rn(fwd, back), (float)order) : 0.0f;
	}
}

/// grad at a real position whose interpolated value `centre` is known.
template <int D, int L, class Get>
__device__ __forceinline__ void grad_fc(const Get& get, const SurfGeom& g, const float* p,
                                        float centre, float* out)
{
	grad_with<D, L>([&](const float* t) { return interp<D>(get, t); }, g, p, centre, out);
}

/// grad at a real position (NumericMixin.hpp:188-231 over interp).
template <int D, int L, class Get>
__device__ __forceinline__ void grad_f(const Get& get, const SurfGeom& g, const float* p, float* out)
{
	grad_fc<D, L>(get, g, p, interp<D>(get, p), out);
}

/// Eigen's fixed-size dot product: products summed x0 + x1 in 2D, x0 + (x1 + x2) in 3D.
template <int D>
__device__ __forceinline__ float dot_e(const float* a, const float* b)
{
	if (D == 2) return __fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1]));
	return __fadd_rn(__fmul_rn(a[0], b[0]),
	                 __fadd_rn(__fmul_rn(a[1], b[1]), __fmul_rn(a[2], b[2])));
}

/// Eigen normalize(): divide by sqrt(squaredNorm()) when positive.
template <int D>
__device__ __forceinline__ void normalize_d(float* v)
{
	const float z = dot_e<D>(v, v);
	if (z > 0.0f) {
		const float r = __fsqrt_rn(z);
#pragma unroll
		for (int a = 0; a < D; a++) v[a] = __fdiv_rn(v[a], r);
	}
}

__device__ __forceinline__ void normalize3(float* v) { normalize_d<3>(v); }


}  // namespace fg
