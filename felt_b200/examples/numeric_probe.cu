// The Numeric API from a __device__ speed functor: grad, gradF, gradB, gradC, gradE and
// divergence (the reference's NumericMixin.hpp:165-355) evaluated at every zero-layer node during
// an update(fn), the way a speed functor calls them, and the same functions with curv and interp
// at the real position node + (0.3, -0.2, 0.45). The functor records the values into its own
// device buffer and returns a speed of 0, so the surface does not move; the program writes them
// out for comparison with the CPU restatement of the reference.
//
// Build (from the repository root):
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -fmad=false -Iinclude \
//        -Ifelt_b200/include felt_b200/examples/numeric_probe.cu -Lfelt_b200 -lfelt_gpu \
//        -Xlinker -rpath,$PWD/felt_b200 -o numeric_probe
// Run: ./numeric_probe out_file   (per grid node, row-major, 32^3 nodes: 16 values at the node,
//      a flag, 18 values at the real position)
#include <cstdio>
#include <vector>

#include "felt_gpu/surface.hpp"

using felt_gpu::DevVec;

constexpr int N = 32;     // grid edge
constexpr int VALS = 35;  // node: 5 gradients x 3, divergence, flag; real: the same, curv, interp

/// delta = a * curv(pos) + c.
struct CurvatureDrift {
	float a, c;
	template <class Iso>
	__device__ float operator()(const DevVec<3>& p, const Iso& iso) const
	{
		return a * iso.curv(p) + c;
	}
};

/// Records the Numeric API at each node it is called for; speed 0.
struct Recorder {
	float* out;
	template <class Iso>
	__device__ float operator()(const DevVec<3>& p, const Iso& iso) const
	{
		const int idx = ((p[0] + N / 2) * N + (p[1] + N / 2)) * N + (p[2] + N / 2);
		float* o = out + (size_t)idx * VALS;
		const felt_gpu::DevVecF<3> g[5] = {iso.grad(p), iso.gradF(p), iso.gradB(p), iso.gradC(p),
		                                   iso.gradE(p)};
		for (int k = 0; k < 5; k++)
			for (int a = 0; a < 3; a++) o[k * 3 + a] = g[k][a];
		o[15] = iso.divergence(p);
		o[16] = 1.0f;
		felt_gpu::DevVecF<3> q;
		const float off[3] = {0.3f, -0.2f, 0.45f};
		for (int a = 0; a < 3; a++) q[a] = __fadd_rn((float)p[a], off[a]);
		const felt_gpu::DevVecF<3> h[5] = {iso.grad(q), iso.gradF(q), iso.gradB(q), iso.gradC(q),
		                                   iso.gradE(q)};
		for (int k = 0; k < 5; k++)
			for (int a = 0; a < 3; a++) o[17 + k * 3 + a] = h[k][a];
		o[32] = iso.divergence(q);
		o[33] = iso.curv(q);
		o[34] = iso.get(q);
		return 0.0f;
	}
};

int main(int argc, char** argv)
{
	if (argc < 2) {
		std::fprintf(stderr, "usage: %s out_file\n", argv[0]);
		return 2;
	}
	const size_t n = (size_t)N * N * N * VALS;
	float* buf = nullptr;
	if (cudaMalloc(&buf, n * sizeof(float)) != cudaSuccess ||
	    cudaMemset(buf, 0, n * sizeof(float)) != cudaSuccess) {
		std::fprintf(stderr, "device allocation failed\n");
		return 1;
	}
	std::vector<float> host(n);
	try {
		felt_gpu::Surface<3, 2> s({N, N, N}, {8, 8, 8});
		s.seed({0, 0, 0});
		for (int i = 0; i < 6; i++) s.update(felt_gpu::Speed::constant(-1.0f));
		for (int i = 0; i < 4; i++) s.update(CurvatureDrift{-0.3f, -0.2f});
		s.update(Recorder{buf});
	} catch (const felt_gpu::Error& e) {
		std::fprintf(stderr, "felt_gpu error %d: %s\n", e.code, e.what());
		return 1;
	}
	if (cudaDeviceSynchronize() != cudaSuccess ||
	    cudaMemcpy(host.data(), buf, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
		std::fprintf(stderr, "copy failed\n");
		return 1;
	}
	cudaFree(buf);
	FILE* f = std::fopen(argv[1], "wb");
	if (!f) return 1;
	const bool ok = std::fwrite(host.data(), sizeof(float), n, f) == n;
	return std::fclose(f) == 0 && ok ? 0 : 1;
}
