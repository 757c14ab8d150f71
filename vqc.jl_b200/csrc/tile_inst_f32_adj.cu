// Tile kernels: FP32 classic body and the serving batch kernel, reverse sweep.
#include "tile_kernels_impl.cuh"

VQC_INST_TILE(float, 9, true, true, false)
VQC_INST_TILE(float, 9, true, false, false)
VQC_INST_TILE(float, 10, true, true, false)
VQC_INST_TILE(float, 10, true, false, false)
VQC_INST_TILE(float, 11, true, true, false)
VQC_INST_TILE(float, 11, true, false, false)
VQC_INST_TILE(float, 12, true, true, false)
VQC_INST_TILE(float, 12, true, false, false)
VQC_INST_BATCH(float, 9, true)
VQC_INST_BATCH(float, 10, true)
VQC_INST_BATCH(float, 11, true)
VQC_INST_BATCH(float, 12, true)
