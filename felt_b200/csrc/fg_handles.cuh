// Definitions of the opaque C-ABI handles (include/felt_gpu.h), shared by the translation units
// that implement entry points.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "fg_engine.cuh"
#include "fg_polys.cuh"

struct fg_surface {
	std::unique_ptr<fg::EngineBase> eng;
	size_t vertex_capacity = 0;  // initial polygonisation arena (fg_config)
	cudaStream_t st = nullptr;
	bool local_open = false;
	std::vector<int> dpos;
	std::vector<float> dval;
	~fg_surface()
	{
		eng.reset();
		if (st) cudaStreamDestroy(st);
	}
};

struct fg_polys {
	fg_surface* surf = nullptr;
	std::unique_ptr<fg::PolysBase> impl;
};

struct fg_batch {
	std::unique_ptr<fg::PolysBase> polys;  // destroyed before the engine it refers to
	size_t vertex_capacity = 0;            // initial polygonisation arena (fg_config)
	std::unique_ptr<fg::EngineBase> eng;
	cudaStream_t st = nullptr;
	~fg_batch()
	{
		polys.reset();
		eng.reset();
		if (st) cudaStreamDestroy(st);
	}
};

namespace fg {
/// Records the message fg_last_error() returns on the calling thread.
void set_last_error(const std::string& msg);
}  // namespace fg
