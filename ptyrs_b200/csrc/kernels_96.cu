// The per-frame cluster kernels for frames of side 96 (launch.cuh).
#include "side_kernels.cuh"

template struct ptyb::SideKernels<96>;
