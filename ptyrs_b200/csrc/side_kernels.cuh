// Definitions behind launch.cuh for one frame side, included only by kernels_<side>.cu: the
// cluster launch of each kernel template at the cluster sizes built for that side (one CTA at
// 64, two at 96, two or four at 128, eight at 192, eight or sixteen at 256).
#pragma once
#include "launch.cuh"

namespace ptyb {

// One launch of `kern` over nslot clusters of C CTAs with `smem` bytes of dynamic shared memory
// each; with `occupancy`, cudaErrorLaunchOutOfResources when no cluster of that shape fits.
template <int N, int C, typename Kern, typename Args>
cudaError_t launch_clusters(Kern kern, const Args& a, int nslot, size_t smem, cudaStream_t s,
                            bool occupancy = false) {
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (C > 8) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nslot * C);
  cfg.blockDim = dim3(FrameShape<N, C>::T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = C > 1 ? 1 : 0;
  if (occupancy && C > 1) {
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg);
    if (e != cudaSuccess) return e;
    if (clusters < 1) return cudaErrorLaunchOutOfResources;
  }
  return cudaLaunchKernelEx(&cfg, kern, a);
}

template <int N, int C>
cudaError_t frame_modes(int mode, const FrameArgs& a, int nslot, int K, cudaStream_t s) {
  const size_t smem = frame_smem_bytes<N, C>(K);
  switch (mode) {
    case kRpie: return launch_clusters<N, C>(frame_kernel<N, C, kRpie>, a, nslot, smem, s);
    case kLsqmlFused:
      return launch_clusters<N, C>(frame_kernel<N, C, kLsqmlFused>, a, nslot, smem, s);
    case kMlGrad: return launch_clusters<N, C>(frame_kernel<N, C, kMlGrad>, a, nslot, smem, s);
    case kBhGrad: return launch_clusters<N, C>(frame_kernel<N, C, kBhGrad>, a, nslot, smem, s);
    case kLlk: return launch_clusters<N, C>(frame_kernel<N, C, kLlk>, a, nslot, smem, s);
    case kStore: return launch_clusters<N, C>(frame_kernel<N, C, kStore>, a, nslot, smem, s);
    case kFromStore:
      return launch_clusters<N, C>(frame_kernel<N, C, kFromStore>, a, nslot, smem, s);
    case kProjectKept:
      return launch_clusters<N, C>(frame_kernel<N, C, kProjectKept>, a, nslot, smem, s);
    case kCarry: return launch_clusters<N, C>(frame_kernel<N, C, kCarry>, a, nslot, smem, s);
  }
  return cudaErrorInvalidValue;
}

template <int N, int C>
cudaError_t move_modes(int mode, const MoveArgs& a, int nslot, int K, cudaStream_t s) {
  const size_t smem = move_smem_bytes<N, C>(K);
  switch (mode) {
    case kMoveBack: return launch_clusters<N, C>(move_kernel<N, C, kMoveBack>, a, nslot, smem, s);
    case kDerivWindow:
      return launch_clusters<N, C>(move_kernel<N, C, kDerivWindow>, a, nslot, smem, s);
    case kSpectrum: return launch_clusters<N, C>(move_kernel<N, C, kSpectrum>, a, nslot, smem, s);
    case kFromSpectrum:
      return launch_clusters<N, C>(move_kernel<N, C, kFromSpectrum>, a, nslot, smem, s);
    case kDerivSums:
      return launch_clusters<N, C>(move_kernel<N, C, kDerivSums>, a, nslot, smem, s);
    case kBackSpectrum:
      return launch_clusters<N, C>(move_kernel<N, C, kBackSpectrum>, a, nslot, smem, s);
    case kPlainInverse:
      return launch_clusters<N, C>(move_kernel<N, C, kPlainInverse>, a, nslot, smem, s);
    case kMoveOwn: return launch_clusters<N, C>(move_kernel<N, C, kMoveOwn>, a, nslot, smem, s);
    case kDerivMove:
      return launch_clusters<N, C>(move_kernel<N, C, kDerivMove>, a, nslot, smem, s);
  }
  return cudaErrorInvalidValue;
}

template <int N, int C>
cudaError_t slice_modes(int mode, const SliceArgs& a, int nslot, int K, cudaStream_t s) {
  const size_t smem = frame_smem_bytes<N, C>(K);
  switch (mode) {
    case kSliceForward:
      return launch_clusters<N, C>(slice_kernel<N, C, kSliceForward>, a, nslot, smem, s);
    case kSliceBackward:
      return launch_clusters<N, C>(slice_kernel<N, C, kSliceBackward>, a, nslot, smem, s);
    case kSliceLlk: return launch_clusters<N, C>(slice_kernel<N, C, kSliceLlk>, a, nslot, smem, s);
    case kSliceGrad:
      return launch_clusters<N, C>(slice_kernel<N, C, kSliceGrad>, a, nslot, smem, s);
  }
  return cudaErrorInvalidValue;
}

// The cluster sizes built per side: C0 always, C1 too when nonzero.
template <int N>
struct SideClusters;
template <> struct SideClusters<64> { static constexpr int C0 = 1, C1 = 0; };
template <> struct SideClusters<96> { static constexpr int C0 = 2, C1 = 0; };
template <> struct SideClusters<128> { static constexpr int C0 = 2, C1 = 4; };
template <> struct SideClusters<192> { static constexpr int C0 = 8, C1 = 0; };
template <> struct SideClusters<256> { static constexpr int C0 = 8, C1 = 16; };

template <int N>
cudaError_t SideKernels<N>::frame(int C, int mode, const FrameArgs& a, int nslot, int K,
                                  cudaStream_t s) {
  constexpr int C0 = SideClusters<N>::C0, C1 = SideClusters<N>::C1;
  if (C == C0) return frame_modes<N, C0>(mode, a, nslot, K, s);
  if constexpr (C1 > 0)
    if (C == C1) return frame_modes<N, C1>(mode, a, nslot, K, s);
  return cudaErrorInvalidValue;
}

template <int N>
cudaError_t SideKernels<N>::move(int C, int mode, const MoveArgs& a, int nslot, int K,
                                 cudaStream_t s) {
  constexpr int C0 = SideClusters<N>::C0, C1 = SideClusters<N>::C1;
  if (C == C0) return move_modes<N, C0>(mode, a, nslot, K, s);
  if constexpr (C1 > 0)
    if (C == C1) return move_modes<N, C1>(mode, a, nslot, K, s);
  return cudaErrorInvalidValue;
}

template <int N>
cudaError_t SideKernels<N>::slice(int C, int mode, const SliceArgs& a, int nslot, int K,
                                  cudaStream_t s) {
  constexpr int C0 = SideClusters<N>::C0, C1 = SideClusters<N>::C1;
  if (C == C0) return slice_modes<N, C0>(mode, a, nslot, K, s);
  if constexpr (C1 > 0)
    if (C == C1) return slice_modes<N, C1>(mode, a, nslot, K, s);
  return cudaErrorInvalidValue;
}

template <int N>
cudaError_t SideKernels<N>::gamma(const GammaArgs& a, int nslot, cudaStream_t s) {
  constexpr int C = gamma_cluster(N);
  return launch_clusters<N, C>(gamma_kernel<N, C>, a, nslot, gamma_smem_bytes<N, C>(), s, true);
}

template <int N>
cudaError_t SideKernels<N>::slice_gamma(const SliceGammaArgs& a, int nslot, int K,
                                        cudaStream_t s) {
  constexpr int C = gamma_cluster(N);
  return launch_clusters<N, C>(slice_gamma_kernel<N, C>, a, nslot,
                               slice_gamma_smem_bytes<N, C>(K), s, true);
}

template <int N>
cudaError_t SideKernels<N>::bh(const BhArgs& a, int nslot, cudaStream_t s) {
  constexpr int C = gamma_cluster(N);
  return launch_clusters<N, C>(bh_hessian_kernel<N, C>, a, nslot, bh_smem_bytes<N, C>(), s,
                               true);
}

}  // namespace ptyb
