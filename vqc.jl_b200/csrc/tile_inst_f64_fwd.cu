// Tile kernels: FP64 body and the serving batch kernel, forward passes.
#include "tile_kernels_impl.cuh"

VQC_INST_TILE(double, 9, false, true, false)
VQC_INST_TILE(double, 9, false, false, false)
VQC_INST_TILE(double, 10, false, true, false)
VQC_INST_TILE(double, 10, false, false, false)
VQC_INST_TILE(double, 11, false, true, false)
VQC_INST_TILE(double, 11, false, false, false)
VQC_INST_BATCH(double, 9, false)
VQC_INST_BATCH(double, 10, false)
VQC_INST_BATCH(double, 11, false)
