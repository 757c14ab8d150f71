// Tile kernels: FP32 packed body (interpreted form of the compiled passes), forward passes.
#include "tile_kernels_impl.cuh"

VQC_INST_TILE(float, 9, false, true, true)
VQC_INST_TILE(float, 9, false, false, true)
VQC_INST_TILE(float, 10, false, true, true)
VQC_INST_TILE(float, 10, false, false, true)
VQC_INST_TILE(float, 11, false, true, true)
VQC_INST_TILE(float, 11, false, false, true)
VQC_INST_TILE(float, 12, false, true, true)
VQC_INST_TILE(float, 12, false, false, true)
