// Declarations of the tile kernels (defined in tile_kernels_impl.cuh and
// instantiated in the tile_inst_*.cu translation units, so that the planner
// and the kernels compile in parallel).
#pragma once

#include "tile_plan.cuh"

namespace vqc {

// One pass of one state: the tiles of the pass strided over the grid.  GEN =
// false: every op is a one-qubit op; PACKED: the FP32 packed body
// (tile_f32.cuh) on a plan laid out for it.
template <class R, int M, bool ADJ, bool GEN, bool PACKED>
__global__ void k_tile(cplx<R>* psi, cplx<R>* lam, const DevPass* pass, const void* stages, const DevOp* ops,
                       const cplx<R>* pool, double* partials);
// One pass each of many states (the serving loop): item blockIdx.y.
template <class R, int M, bool ADJ>
__global__ void k_tile_batch(const TileItem* __restrict__ items);

}  // namespace vqc
