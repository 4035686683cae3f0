// Step and batch kernels for fp16 population storage (one translation unit per storage
// precision, so the build compiles the four in parallel).
#include "wt_kernels.cuh"

WT_INSTANTIATE(WT_F16)
