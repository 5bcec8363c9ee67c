// The per-frame cluster kernels for frames of side 256 (launch.cuh).
#include "side_kernels.cuh"

template struct ptyb::SideKernels<256>;
