// Tile kernels: FP32 packed body (interpreted form of the compiled passes), reverse sweep.
#include "tile_kernels_impl.cuh"

VQC_INST_TILE(float, 9, true, true, true)
VQC_INST_TILE(float, 9, true, false, true)
VQC_INST_TILE(float, 10, true, true, true)
VQC_INST_TILE(float, 10, true, false, true)
VQC_INST_TILE(float, 11, true, true, true)
VQC_INST_TILE(float, 11, true, false, true)
VQC_INST_TILE(float, 12, true, true, true)
VQC_INST_TILE(float, 12, true, false, true)
