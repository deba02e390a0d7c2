// The isogrid's Numeric API from the host: IsoGrid::get(VecDi | VecDf), curv, divergence,
// grad, gradF, gradB, gradC, gradE and inside (NumericMixin.hpp:72-481, GridMixin inside),
// evaluated at a batch of positions by one kernel on the surface's stream.
#include <algorithm>
#include <climits>

#include "../../include/felt_gpu.h"
#include "fg_engine.cuh"
#include "fg_numeric.cuh"
#include "fg_query.cuh"

namespace fg {
namespace {

template <int D, int L, class Pos>
__device__ __forceinline__ void query_one(const IsoView<D, L>& iso, int what, const Pos& p, float* o)
{
	switch (what) {
	case FG_Q_GET: o[0] = iso.get(p); return;
	case FG_Q_CURV: o[0] = iso.curv(p); return;
	case FG_Q_DIVERGENCE: o[0] = iso.divergence(p); return;
	case FG_Q_INSIDE: o[0] = iso.inside(p) ? 1.0f : 0.0f; return;
	default: break;
	}
	VecF<D> r;
	switch (what) {
	case FG_Q_GRAD: r = iso.grad(p); break;
	case FG_Q_GRADF: r = iso.gradF(p); break;
	case FG_Q_GRADB: r = iso.gradB(p); break;
	case FG_Q_GRADC: r = iso.gradC(p); break;
	default: r = iso.gradE(p); break;
	}
#pragma unroll
	for (int a = 0; a < D; a++) o[a] = r[a];
}

/// One thread per position: nodes from ipos (D ints each) or real positions from fpos (D floats
/// each). Any position is safe to read: the isogrid reads as L + 1 outside the grid.
template <int D, int L>
__global__ void __launch_bounds__(256) k_query(Dev P, int s, int what, const float* fpos,
                                               const int* ipos, int n, float* out)
{
	const IsoView<D, L> iso{&P, &P.geom[s]};
	const int w = what >= FG_Q_GRAD ? D : 1;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		if (ipos) {
			Vec<D> p;
#pragma unroll
			for (int a = 0; a < D; a++) p[a] = ipos[(size_t)i * D + a];
			query_one<D, L>(iso, what, p, out + (size_t)i * w);
		} else {
			VecF<D> p;
#pragma unroll
			for (int a = 0; a < D; a++) p[a] = fpos[(size_t)i * D + a];
			query_one<D, L>(iso, what, p, out + (size_t)i * w);
		}
	}
}

}  // namespace

void query(EngineBase& eng, int s, int what, const float* fpos, const int* ipos, size_t n, float* out)
{
	if (s < 0 || s >= eng.surfaces()) throw Error(-1, "surface index out of range");
	if (what < FG_Q_GET || what > FG_Q_GRADE) throw Error(-1, "unknown query");
	const int D = eng.dims(), L = eng.layers();
	if (n == 0) return;
	if (n > (size_t)(INT_MAX / 4)) throw Error(-1, "too many positions in one query");
	const int w = what >= FG_Q_GRAD ? D : 1;
	cudaStream_t st = eng.stream();
	const size_t in_bytes = n * D * 4, out_bytes = n * w * sizeof(float);
	void* din = nullptr;
	float* dout = nullptr;
	FG_CUDA(cudaMallocAsync(&din, in_bytes, st));
	cudaError_t e = cudaMallocAsync((void**)&dout, out_bytes, st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(din, ipos ? (const void*)ipos : (const void*)fpos, in_bytes,
		                    cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess) {
		const Dev& P = eng.dev();
		const int ni = (int)n;
		const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
		const float* fp = ipos ? nullptr : (const float*)din;
		const int* ip = ipos ? (const int*)din : nullptr;
#define FG_CASE(dd, ll) \
	if (D == dd && L == ll) FG_RUN("k_query", st, k_query<dd, ll><<<blocks, 256, 0, st>>>(P, s, what, fp, ip, ni, dout););
		FG_CASE(2, 1) FG_CASE(2, 2) FG_CASE(2, 3) FG_CASE(2, 4)
		FG_CASE(3, 1) FG_CASE(3, 2) FG_CASE(3, 3) FG_CASE(3, 4)
#undef FG_CASE
		e = cudaGetLastError();
	}
	if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, st);
	if (dout) cudaFreeAsync(dout, st);
	cudaFreeAsync(din, st);
	const cudaError_t e2 = cudaStreamSynchronize(st);
	if (e == cudaSuccess) e = e2;
	if (e != cudaSuccess) throw Error(-2, cudaGetErrorString(e));
}

}  // namespace fg
