// Tile kernels: FP32 classic body and the serving batch kernel, forward passes.
#include "tile_kernels_impl.cuh"

VQC_INST_TILE(float, 9, false, true, false)
VQC_INST_TILE(float, 9, false, false, false)
VQC_INST_TILE(float, 10, false, true, false)
VQC_INST_TILE(float, 10, false, false, false)
VQC_INST_TILE(float, 11, false, true, false)
VQC_INST_TILE(float, 11, false, false, false)
VQC_INST_TILE(float, 12, false, true, false)
VQC_INST_TILE(float, 12, false, false, false)
VQC_INST_BATCH(float, 9, false)
VQC_INST_BATCH(float, 10, false)
VQC_INST_BATCH(float, 11, false)
VQC_INST_BATCH(float, 12, false)
