// Polys<Surface> on the device: per-partition marching squares/cubes (Poly::Single) and the
// incremental pending/done partition tracking of Felt::Polys (include/Felt/Polys.hpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "fg_engine.cuh"

namespace fg {

class PolysBase {
public:
	virtual ~PolysBase() = default;
	virtual void notify() = 0;
	virtual void march() = 0;
	/// march() of the listed surfaces of the pool only; the others keep their pending
	/// partitions for their own march (serving: a request is marched when it finishes, as it
	/// would be alone).
	virtual void march_some(const int* surfaces, int n) = 0;
	virtual void invalidate() = 0;
	virtual void march_partition(size_t part) = 0;
	virtual std::vector<uint32_t> changes() = 0;
	virtual void partition(size_t part, float* vtx, size_t vcap, uint32_t* spx, size_t scap,
	                       size_t* nv, size_t* ns, int* active) = 0;
	virtual void totals(size_t* nv, size_t* ns) = 0;
	/// Surface of the pool that changes(), partition() and march_partition() refer to.
	virtual void select(int s) = 0;
	/// Geometry of several partitions of the selected surface, concatenated in the given order
	/// (one gather kernel, two copies); counts receives (vertices, simplices) per partition.
	virtual void gather(const uint32_t* parts, size_t n, float* vtx, size_t vcap, uint32_t* spx,
	                    size_t scap, uint32_t* counts, size_t* nv, size_t* ns) = 0;
	/// Serving: forgets surface s's polygons and pending partitions (after the engine's
	/// reset_surface), as a new Polys of an empty surface has none.
	virtual void reset_surface(int s) = 0;
	/// Serving: whether notify tracks surface s's changes (a request that asks for no
	/// polygons is left out, so marches find nothing pending for it).
	virtual void set_enabled(int s, bool on) = 0;
};

/// Polygonisation of surface s of an engine's pool. vertex_capacity: initial vertex arena
/// (simplex arena twice that), 0 = 2^20; the arenas grow on demand.
PolysBase* make_polys(EngineBase& eng, int s, size_t vertex_capacity = 0);

}  // namespace fg
