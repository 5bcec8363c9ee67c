// The per-frame cluster kernels for frames of side 192 (launch.cuh).
#include "side_kernels.cuh"

template struct ptyb::SideKernels<192>;
