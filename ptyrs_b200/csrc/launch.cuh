// Launches of the per-frame cluster kernels (frame, move, slice, line-search), one translation
// unit per frame side (kernels_<side>.cu), so the sides compile in parallel and the host
// sequencing compiles none of these kernels. Each function launches `nslot` frames, C CTAs per
// frame, on stream `s`; cudaErrorInvalidValue for a side, cluster size or mode not built.
#pragma once
#include "bh.cuh"
#include "frame.cuh"
#include "ml.cuh"
#include "multislice.cuh"
#include "position.cuh"

namespace ptyb {

cudaError_t launch_frame_side(int N, int C, int mode, const FrameArgs& a, int nslot, int K,
                              cudaStream_t s);
cudaError_t launch_move_side(int N, int C, int mode, const MoveArgs& a, int nslot, int K,
                             cudaStream_t s);
cudaError_t launch_slice_side(int N, int C, int mode, const SliceArgs& a, int nslot, int K,
                              cudaStream_t s);
// The line search's kernel at its one cluster size per side (gamma_cluster).
cudaError_t launch_gamma_side(int N, const GammaArgs& a, int nslot, cudaStream_t s);
// BH's bilinear Hessian at the line search's cluster size.
cudaError_t launch_bh_side(int N, const BhArgs& a, int nslot, cudaStream_t s);
// ML's line search through a multislice object at the line search's cluster size; K modes.
cudaError_t launch_slice_gamma_side(int N, const SliceGammaArgs& a, int nslot, int K,
                                    cudaStream_t s);
constexpr int gamma_cluster(int N) {
  return N == 64 ? 1 : N == 96 ? 2 : N == 128 ? 4 : N == 192 ? 8 : 16;
}

// The same, for one side (defined in that side's translation unit).
template <int N>
struct SideKernels {
  static cudaError_t frame(int C, int mode, const FrameArgs& a, int nslot, int K, cudaStream_t s);
  static cudaError_t move(int C, int mode, const MoveArgs& a, int nslot, int K, cudaStream_t s);
  static cudaError_t slice(int C, int mode, const SliceArgs& a, int nslot, int K, cudaStream_t s);
  static cudaError_t gamma(const GammaArgs& a, int nslot, cudaStream_t s);
  static cudaError_t bh(const BhArgs& a, int nslot, cudaStream_t s);
  static cudaError_t slice_gamma(const SliceGammaArgs& a, int nslot, int K, cudaStream_t s);
};
extern template struct SideKernels<64>;
extern template struct SideKernels<96>;
extern template struct SideKernels<128>;
extern template struct SideKernels<192>;
extern template struct SideKernels<256>;

}  // namespace ptyb
