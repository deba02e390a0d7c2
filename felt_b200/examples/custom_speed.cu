// update(fn) with caller-written __device__ functors through the C++ facade, one functor per
// signature the reference accepts: (pos, isogrid), (pos) and (). Each equals a builtin speed,
// so the result can be checked against the CPU restatement of the reference.
//
// Build (from the repository root):
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -fmad=false -Iinclude \
//        -Ifelt_b200/include felt_b200/examples/custom_speed.cu -Lfelt_b200 -lfelt_gpu \
//        -Xlinker -rpath,$PWD/felt_b200 -o custom_speed
// Run: ./custom_speed out_prefix   (writes out_prefix.dump and out_prefix.phi)
#include <cstdio>
#include <vector>

#include "felt_gpu/surface.hpp"

using felt_gpu::DevVec;

/// delta = a * curv(pos) + c: mean-curvature flow with a drift.
struct CurvatureDrift {
	float a, c;
	template <class Iso>
	__device__ float operator()(const DevVec<3>& p, const Iso& iso) const
	{
		return a * iso.curv(p) + c;
	}
};

/// delta = n * h(pos, seed) + c: hashed noise (the engine's hash, exact in FP32) with a drift.
struct NoisyDrift {
	float n, c;
	unsigned seed;
	__device__ float operator()(const DevVec<3>& p) const
	{
		return n * fg::hash_noise<3>(p, seed) + c;
	}
};

/// delta = c.
struct Constant {
	float c;
	__device__ float operator()() const { return c; }
};

static bool write_file(const char* path, const void* data, size_t bytes)
{
	FILE* f = std::fopen(path, "wb");
	if (!f) return false;
	const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
	return std::fclose(f) == 0 && ok;
}

int main(int argc, char** argv)
{
	if (argc < 2) {
		std::fprintf(stderr, "usage: %s out_prefix\n", argv[0]);
		return 2;
	}
	try {
		felt_gpu::Surface<3, 2> s({32, 32, 32}, {8, 8, 8});
		s.seed({0, 0, 0});
		for (int i = 0; i < 12; i++) s.update(CurvatureDrift{-0.3f, -0.2f});
		for (int i = 0; i < 4; i++) s.update(NoisyDrift{0.1f, -0.25f, 7u});
		for (int i = 0; i < 2; i++) s.update(Constant{0.2f});
		size_t n = 0;
		felt_gpu::check(fg_dump(s.handle(), nullptr, 0, &n));
		std::vector<uint32_t> words(n);
		felt_gpu::check(fg_dump(s.handle(), words.data(), n, &n));
		const std::vector<float> phi = s.snapshot();
		const std::string pre = argv[1];
		if (!write_file((pre + ".dump").c_str(), words.data(), n * sizeof(uint32_t)) ||
		    !write_file((pre + ".phi").c_str(), phi.data(), phi.size() * sizeof(float))) {
			std::fprintf(stderr, "cannot write %s.*\n", argv[1]);
			return 1;
		}
	} catch (const felt_gpu::Error& e) {
		std::fprintf(stderr, "felt_gpu error %d: %s\n", e.code, e.what());
		return 1;
	}
	return 0;
}
