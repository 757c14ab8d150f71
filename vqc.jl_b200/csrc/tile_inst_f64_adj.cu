// Tile kernels: FP64 body and the serving batch kernel, reverse sweep.
#include "tile_kernels_impl.cuh"

VQC_INST_TILE(double, 9, true, true, false)
VQC_INST_TILE(double, 9, true, false, false)
VQC_INST_TILE(double, 10, true, true, false)
VQC_INST_TILE(double, 10, true, false, false)
VQC_INST_TILE(double, 11, true, true, false)
VQC_INST_TILE(double, 11, true, false, false)
VQC_INST_BATCH(double, 9, true)
VQC_INST_BATCH(double, 10, true)
VQC_INST_BATCH(double, 11, true)
