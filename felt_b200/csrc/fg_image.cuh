// Surface::save / Surface::load (include/Felt/Surface.hpp:180-196): host image of a surface's
// isogrid and its file in the reference's format.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "fg_engine.cuh"

namespace fg {

/// The isogrid of one surface, partition by partition (local children-grid order).
struct SurfaceImage {
	int np = 0, BV = 0, NL = 0;
	std::vector<float> bg;                 // [np] backgrounds
	std::vector<int> ppos;                 // [np * NL] position in each partition list, -1 none
	std::vector<std::vector<int>> plist;   // [NL] ordered partition lists
	std::vector<int> active;               // active partitions, increasing
	std::vector<float> phi;                // [active * BV] values
	std::vector<uint16_t> lkp;             // [active * BV] position in its leaf list, NUL16 none
	std::vector<uint16_t> lst;             // [active * NL * BV] ordered leaf lists
	std::vector<int> lcnt;                 // [active * NL] their lengths
};

/// Reads surface s of the engine's pool into img.
void export_image(EngineBase& eng, int s, SurfaceImage& img);
/// Writes img into a newly created single-surface engine of the same geometry.
void import_image(EngineBase& eng, const SurfaceImage& img);
/// Writes img into surface s of any pool, which must be empty (no active partition, every list
/// empty) and of the same geometry; its bricks come from the pool's free stack.
void restore_image(EngineBase& eng, int s, const SurfaceImage& img);

/// The surface file of img (geometry g, partition size csz) appended to out.
void write_surface_file(const SurfaceImage& img, const SurfGeom& g, int D, int L, const int* csz,
                        std::vector<uint8_t>& out);
/// Dimensions, layers, grid size and partition size of a surface file.
void peek_surface_file(const uint8_t* p, size_t n, int& D, int& L, int* size, int* csz);
/// Parses and validates a surface file for a surface of geometry g into img.
void read_surface_file(const uint8_t* p, size_t n, const SurfGeom& g, int D, int L,
                       const int* csz, int BV, SurfaceImage& img);

}  // namespace fg
