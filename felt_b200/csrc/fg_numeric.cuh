// The reference's Numeric API on the isogrid (NumericMixin.hpp:72-481) as device functions over
// the pool: shared by the facade's speed-functor view and the library's query kernel.
#pragma once

#include "fg_dev.cuh"
#include "fg_field.cuh"

namespace fg {

/// A D-vector of floats: a real position, or what the gradient functions return.
template <int D>
struct VecF {
	float v[D];
	__host__ __device__ float& operator[](int i) { return v[i]; }
	__host__ __device__ const float& operator[](int i) const { return v[i]; }
};

/// Read access to the isogrid (a speed functor's view, the query kernel's): get (Access::get with the lazy child get,
/// PartitionedMixin.hpp:594-601), curv (NumericMixin.hpp:72-156), inside (GridMixin inside), and
/// the rest of the reference's Numeric API (NumericMixin.hpp:165-355): grad, gradF, gradB,
/// gradC, gradE, divergence. Like the reference's templates on the position type, each takes a
/// node (Vec<D>) or a real position (VecF<D>); at a real position get is interp (linear
/// interpolation of the 2^D corners, NumericMixin.hpp:382-481), inside is the float test
/// offset <= p < offset + size, and the stencils step the coordinates by +-1 in float. FP32
/// rounded step by step as the reference's code (the grid spacing dx is 1, so its final
/// divisions by dx change nothing).
template <int D, int L>
struct IsoView {
	const Dev* P;
	const SurfGeom* g;
	__device__ float get(const Vec<D>& p) const { return get_phi<D, L>(*P, *g, p); }
	__device__ float get(const VecF<D>& p) const { return interp(p); }
	__device__ bool inside(const Vec<D>& p) const { return in_grid<D>(*g, p); }
	__device__ bool inside(const VecF<D>& p) const { return inside_f<D, L>(*g, p.v); }
	/// interp (NumericMixin.hpp:403-481): corners in bit order, reduced along axis 0 first.
	__device__ float interp(const VecF<D>& p) const
	{
		return ::fg::interp<D>([this](const Vec<D>& q) { return get(q); }, p.v);
	}
	template <class Pos>
	__device__ float curv(const Pos& p) const
	{
		return curv_g<D>([this](const Pos& q) { return get(q); }, p);
	}

	/// grad (NumericMixin.hpp:189-231): central difference, one-sided at the grid's edge, 0
	/// where neither neighbour is inside.
	template <class Pos>
	__device__ VecF<D> grad(const Pos& p) const
	{
		VecF<D> r;
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
	__device__ VecF<D> gradE(const Pos& p) const
	{
		VecF<D> r;
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
	__device__ VecF<D> gradF(const Pos& p) const
	{
		VecF<D> r;
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
	__device__ VecF<D> gradB(const Pos& p) const
	{
		VecF<D> r;
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
	__device__ VecF<D> gradC(const Pos& p) const
	{
		VecF<D> r;
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
		const VecF<D> f = gradF(p), b = gradB(p);
		float d[D];
		for (int a = 0; a < D; a++) d[a] = __fsub_rn(f[a], b[a]);
		return D == 2 ? __fadd_rn(d[0], d[1]) : __fadd_rn(d[0], __fadd_rn(d[1], d[D - 1]));
	}
};

}  // namespace fg
