// The per-frame cluster kernels for frames of side 64 (launch.cuh).
#include "side_kernels.cuh"

template struct ptyb::SideKernels<64>;
