// The reconstruction engine behind the C ABI (include/ptyb200.h): the device state of one
// scan and the launch sequences of rPIE, LSQML and the LLK pass on one CUDA stream.
//
// Reference engine (physwkim/ptyrs): `GpuPtycho` (ptyrs/src/engine/gpu/mod.rs:533-881), rPIE
// (engine/gpu/rpie.rs:31-63, 198-529), LSQML (engine/gpu/lsqml.rs:75-126), the LLK pass
// (engine/gpu/device.rs:3379-3395).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <exception>
#include <mutex>
#include <set>
#include <thread>
#include <string>
#include <vector>

#include "../../include/ptyb200.h"
#include "frame.cuh"
#include "gather.cuh"
#include "lsqml.cuh"
#include "ml.cuh"
#include "position.cuh"
#include "multislice.cuh"
#include "opr.cuh"
#include "scan.h"

using namespace ptyb;

namespace ptyb {

// Counts of one frame per block, detector order in, FFT-shifted float out (engine/obs.rs:61-76):
// masked (u16 65535, or negative) becomes -1; per-frame photon sum and unmasked count; `bad`
// is set by a non-finite unmasked value.
template <typename T>
__global__ void __launch_bounds__(256) counts_kernel(const T* raw, int u16, float* iobs,
                                                     double* power, int* nobs, int* bad, int N) {
  __shared__ double shp[8];
  __shared__ int shc[8];
  const int f = blockIdx.x;
  const size_t plane = (size_t)N * N;
  double p = 0.0;
  int c = 0;
  for (int j = threadIdx.x; j < N * N; j += 256) {
    const int jy = j / N, jx = j % N;
    const double v = (double)raw[f * plane + (size_t)((jy + N / 2) % N) * N + (jx + N / 2) % N];
    const bool masked = u16 ? v == 65535.0 : v < 0.0;
    if (!masked && !isfinite(v)) *bad = 1;
    iobs[f * plane + j] = masked ? -1.f : (float)v;
    if (!masked) {
      p += v;
      ++c;
    }
  }
  p = warp_sum(p);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (threadIdx.x % 32 == 0) {
    shp[threadIdx.x / 32] = p;
    shc[threadIdx.x / 32] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sp = 0.0;
    int sc = 0;
    for (int w = 0; w < 8; ++w) {
      sp += shp[w];
      sc += shc[w];
    }
    power[f] = sp;
    nobs[f] = sc;
  }
}

__global__ void fill_kernel(float* x, float v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

}  // namespace ptyb

// Scratch of `ptyb_forward_intensity_noalloc`: a fixed 32 MiB per device that loads this
// library, held until the process exits. Host code must not pass `g_noalloc_scratch` itself
// to a kernel (on the host it names a stand-in, not the device array): it takes the device
// address from `noalloc_scratch()`.
constexpr size_t kNoallocScratchBytes = size_t(32) << 20;
// Object slices of a multislice handle, and the float scalars on the device (maxima, the
// batch's object and probe steps, one step per further slice).
constexpr int kMaxSlices = 16;
// Room for the kernel kinds of the per-kernel timing (the Kind enum below fits it).
constexpr int kMaxKinds = 48;
constexpr int kScalars = 8 + kMaxSlices + 2;
// The maxima of the AP / DM / RAAR blends' object and probe norms.
constexpr int kScalObjNorm = 8 + kMaxSlices, kScalProbeNorm = kScalObjNorm + 1;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

namespace {

constexpr int kAlgAp = 0, kAlgDm = 1, kAlgRaar = 2, kAlgRpie = 3, kAlgMl = 4, kAlgLsqml = 6;

// One device allocation, freed with the handle.
struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct ptyb_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  int P = 0, N = 0, nprobe = 0, nobj = 0, K = 0, nyo = 0, nxo = 0, C = 1, stack = 0;
  double nb_obs = 0, obs_total = 0, max_power = 0, pixel[2] = {0, 0};
  std::vector<int32_t> corners_h;
  // Resident state.
  float* iobs = nullptr;      // [P][N][N] shifted, < 0 masked
  int2* corners = nullptr;    // [P] (oy, ox)
  float2* object = nullptr;   // [nobj][nyo][nxo]
  float2* probe = nullptr;    // [nprobe][N][N]
  float2* quad = nullptr;     // [N][N]
  float2* tw = nullptr;       // [N]
  int* iota = nullptr;        // [P] 0..P-1
  int* order = nullptr;       // [P] frames of one launch (forward_intensity)
  int* order_all = nullptr;   // [order_cap] the call's epoch orders, concatenated
  size_t order_cap = 0;
  float* afar_all = nullptr;  // [P]
  // Scratch, sized for `slots` frames per launch.
  int slots = 0;
  float2* upd = nullptr;      // [slots][K][N][N]
  float2* field = nullptr;    // [slots][K][N][N]
  float* icalc = nullptr;     // [slots][N][N]
  float* omax = nullptr;      // [slots]
  double* llk = nullptr;      // [P][4]
  float* afar1 = nullptr;     // [slots]
  float* afar2 = nullptr;     // [slots]
  float2* partial = nullptr;  // [nchunk][K][N][N]
  int max_chunks = 0;
  float* scal = nullptr;      // [8]: pmax, pre max, object step, probe step
  float* pre = nullptr;       // [nyo][nxo]
  float2* d_obj = nullptr;    // [nyo][nxo]
  float2* d_probe = nullptr;  // [K][N][N]
  double* sums = nullptr;     // [slots][6]
  double* steplog = nullptr;  // [P][3]
  // ML: gradients (with compensation), the previous gradients, the CG directions, the line
  // search's per-frame sums and reduction partials.
  float2 *g_obj = nullptr, *g_obj_c = nullptr, *g_probe = nullptr, *g_probe_c = nullptr;
  float2 *last_obj = nullptr, *last_probe = nullptr, *dir_obj = nullptr, *dir_probe = nullptr;
  double* gamma_sums = nullptr;  // [P][2]
  // Position model (Patch sampling): per-frame offsets [P][2] (dy, dx object pixels) on the
  // device, whether they are refined, the batch's moved probes and its position sums.
  double* offsets = nullptr;
  bool have_offsets = false, refine_offsets = false;
  float2* wave = nullptr;        // [slots][K][N][N]
  double* pos_sums = nullptr;    // [slots][4]
  // Multislice (pty-chi's multislice object, LSQML only): slices, gap transfer functions, the
  // incident waves of slices 1.., every slice's χ, a plane of ones (slices without a phase).
  int C_sums = 1;                // CTAs per frame of the position-sums transform
  int nslice = 1;
  float2* tf = nullptr;          // [nslice-1][N][N]
  float2* incident = nullptr;    // [nslice-1][slots][K][N][N]
  float2* chi_slices = nullptr;  // [nslice][slots][K][N][N]
  float2* ones = nullptr;        // [N][N]
  double* slice_sums = nullptr;  // [slots][2]
  // ML under the position model: the moved probe direction per slot, each frame's position
  // sums (num_y, num_x, den_y, den_x).
  float2* wave2 = nullptr;       // [wave2_slots][K][N][N]
  int wave2_slots = 0;
  double* ml_pos_sums = nullptr; // [P][4]
  // The position model's spectra DFT(q·P) of the probe and of the ML probe direction, and
  // every frame's moved probe for one ML cycle.
  float2* spec = nullptr;        // [K][N][N]
  float2* spec_d = nullptr;      // [K][N][N]
  float2* wave_all = nullptr;    // [P][K][N][N]
  // ML: every frame's detector field of one cycle's gradient pass, [P][K][kx][ky], and the
  // probe gradient's summed spectrum under the position model.
  float2* psi_all = nullptr;
  float2* g_all = nullptr;         // [P][K][N][N] the gradient pass's exit-plane field g
  float2* g_probe_spec = nullptr; // [K][N][N]
  // Multislice gradients: every slice's 2·∂L/∂O_s* and its compensation.
  float2* g_slices = nullptr;     // [S][nyo][nxo]
  float2* g_slices_c = nullptr;
  // AP / DM / RAAR: every frame's carried exit waves and RAAR's iterate, [P][K][N][N]; the
  // probe blend's per-chunk norms and its norm plane.
  float2* carry = nullptr;
  float2* carry_it = nullptr;
  float* partial_den = nullptr;   // [max_den_chunks][N][N]
  int max_den_chunks = 0;
  float* probe_norm = nullptr;    // [N][N]
  float* blend_norm = nullptr;    // [nyo][nxo] the object blend's norm
  // OPR probe variation of LSQML (engine/opr.rs): k eigenmodes, the weights [P][k] and, when
  // modelled, the main mode's weights [P]; scratch for a batch's step.
  int opr_k = 0;
  int opr_slots = 0;             // slots the batch scratch below holds
  bool opr_on = false, opr_refine_w = true, opr_has_c = false, opr_refine_c = true;
  float2* opr_u = nullptr;       // [k][N][N]
  double* opr_w = nullptr;       // [P][k]
  double* opr_c = nullptr;       // [P]
  float* opr_vv = nullptr;       // [slots][N][N]
  float2* opr_r = nullptr;       // [slots][N][N]
  float2* opr_e = nullptr;       // [N][N]
  double* opr_sums = nullptr;    // [slots][3]
  double* opr_p = nullptr;       // [slots]
  double* opr_scal = nullptr;    // [4]
  // Their probe step under the position model: the residual's back-projection g, the step,
  // g's spectrum summed over frames with its compensation, each frame's ‖A·step‖² per mode
  // and the modes' slope and regulariser sums.
  float2 *pcg_g = nullptr, *pcg_step = nullptr, *pcg_spec = nullptr, *pcg_comp = nullptr;
  double* pcg_norms = nullptr;    // [P][K]
  double* pcg_modes = nullptr;    // [K][2]
  double* partials = nullptr;    // [kPartialBlocks][2]
  std::vector<Buf> bufs;
  // Per-kernel device timing (CUDA events on the engine's stream), when enabled.
  bool timing = false;
  std::vector<cudaEvent_t> event_pool;
  struct Pending {
    int kind;
    int64_t frames;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  double kind_ms[kMaxKinds] = {0};
  int64_t kind_n[kMaxKinds] = {0};
  int64_t kind_frames[kMaxKinds] = {0};  // frames the launches of each kind processed
  cudaEvent_t call_ev[2] = {nullptr, nullptr};
  float last_call_ms = 0.f;
  // Host state.
  int64_t cycle = 0;
  int64_t launches = 0;
  std::vector<ptyb_llk_record> history;
  std::vector<ptyb_lsqml_step> steps;
  std::vector<double> slice_steps;  // [frame of the last epoch][slice 1..]: a_obj
  int log_stride = 3;
  bool aborted = false;
  std::string err;
};

namespace {

thread_local std::string g_create_error;

// Device address of the no-alloc scratch on the current device, looked up once per device
// (with that device current) by cudaGetSymbolAddress.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

cudaError_t noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
  return cudaSuccess;
}

struct Fail {
  int code;
};

void check(ptyb_handle* h, cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    h->err = std::string(what) + ": " + cudaGetErrorString(e);
    h->aborted = true;
    throw Fail{PTYB_GPU};
  }
}

// Device memory comes from the device's stream-ordered pool, whose release threshold is set to
// its maximum once per device: memory a destroyed handle gave back stays with the pool, so the
// next handle on that device reuses it instead of the driver mapping new pages (as torch's
// caching allocator does). Each allocation is waited for, so any stream may use it at once.
std::mutex g_pool_mutex;
bool g_pool_kept[kMaxDevices] = {};

cudaError_t pool_alloc(ptyb_handle* h, void** p, size_t bytes) {
  if (h->device < 0 || h->device >= kMaxDevices) return cudaErrorInvalidDevice;
  {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pool_kept[h->device]) {
      cudaMemPool_t pool;
      cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, h->device);
      if (e != cudaSuccess) return e;
      uint64_t keep = UINT64_MAX;
      e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
      g_pool_kept[h->device] = true;
    }
  }
  cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(h->stream);
}

// Host↔device copies and fills on the handle's stream, waited for. The stream is
// non-blocking, so its kernels do not order after copies or fills on the legacy default
// stream: every transfer goes through it.
cudaError_t copy_sync(ptyb_handle* h, void* dst, const void* src, size_t bytes,
                      cudaMemcpyKind kind) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, h->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(h->stream);
}

cudaError_t fill_sync(ptyb_handle* h, void* dst, int value, size_t bytes) {
  cudaError_t e = cudaMemsetAsync(dst, value, bytes, h->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(h->stream);
}

template <typename T>
T* alloc(ptyb_handle* h, size_t count) {
  void* p = nullptr;
  check(h, pool_alloc(h, &p, count * sizeof(T) + 16), "cudaMallocAsync");
  h->bufs.push_back({p, count * sizeof(T)});
  return static_cast<T*>(p);
}

void launched(ptyb_handle* h, const char* what) {
  ++h->launches;
  check(h, cudaGetLastError(), what);
}

constexpr int kPartialBlocks = 296;

// Kernel kinds for the per-kernel timing (ptyb_kernel_name).
enum Kind : int {
  kKFrameRpie = 0, kKFrameLsqml, kKFrameMl, kKFrameLlk, kKFrameStore, kKFrameFromStore,
  kKObjRpie, kKObjOverlap, kKObjLsqml, kKObjMl, kKIllum, kKProbePartial, kKProbeFinal,
  kKAfar, kKDots, kKSolve, kKAxpy, kKMax, kKCounts, kKMisc, kKGamma, kKArraySums, kKMove,
  kKPositionSums, kKSliceForward, kKSliceBackward, kKSliceLlk, kKFrameProject, kKSpectrum,
  kKDerivSums, kKBackSpectrum, kKSliceGrad, kKFrameCarry, kKObjBlend, kKOprStep, kNumKinds
};
static_assert(kNumKinds <= kMaxKinds, "the timing arrays hold kMaxKinds kinds");
const char* const kKindNames[kNumKinds] = {
    "frame_rpie", "frame_lsqml", "frame_ml_grad", "frame_llk", "frame_store",
    "frame_from_store", "object_rpie", "object_overlap", "object_lsqml", "object_ml",
    "illumination", "probe_partial", "probe_finalize", "lsqml_afar", "lsqml_dots",
    "lsqml_solve", "axpy", "max", "counts", "misc", "ml_gamma", "array_sums", "move",
    "position_sums", "slice_forward", "slice_backward", "slice_llk", "frame_project", "spectrum",
    "deriv_sums", "back_spectrum", "slice_grad", "frame_carry", "object_blend", "opr_step"};

cudaEvent_t take_event(ptyb_handle* h) {
  if (!h->event_pool.empty()) {
    cudaEvent_t e = h->event_pool.back();
    h->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  check(h, cudaEventCreate(&e), "event");
  return e;
}

// Runs `launch` (which enqueues one kernel on the engine's stream), bracketed by events when
// timing is on.
template <typename F>
void timed(ptyb_handle* h, int kind, F&& launch, int64_t frames = 0) {
  if (!h->timing) {
    launch();
    return;
  }
  cudaEvent_t a = take_event(h), b = take_event(h);
  check(h, cudaEventRecord(a, h->stream), "event");
  launch();
  check(h, cudaEventRecord(b, h->stream), "event");
  h->pending.push_back({kind, frames, a, b});
}

// Folds the finished launches' times into the per-kind totals (after a stream sync).
void harvest(ptyb_handle* h) {
  for (auto& p : h->pending) {
    float ms = 0.f;
    check(h, cudaEventElapsedTime(&ms, p.a, p.b), "event time");
    h->kind_ms[p.kind] += ms;
    h->kind_n[p.kind] += 1;
    h->kind_frames[p.kind] += p.frames;
    h->event_pool.push_back(p.a);
    h->event_pool.push_back(p.b);
  }
  h->pending.clear();
}

// Brackets a whole algorithm call with events; `end_call` syncs and stores its device time.
void begin_call(ptyb_handle* h) {
  if (!h->call_ev[0]) {
    check(h, cudaEventCreate(&h->call_ev[0]), "event");
    check(h, cudaEventCreate(&h->call_ev[1]), "event");
  }
  check(h, cudaEventRecord(h->call_ev[0], h->stream), "event");
}

void end_call(ptyb_handle* h, const char* what) {
  check(h, cudaEventRecord(h->call_ev[1], h->stream), "event");
  check(h, cudaStreamSynchronize(h->stream), what);
  check(h, cudaEventElapsedTime(&h->last_call_ms, h->call_ev[0], h->call_ev[1]), "event time");
  harvest(h);
}

// Cluster size for frames of side N with K modes: `want` if it is built and fits shared
// memory, else the smallest that fits with at least two CTAs per SM, else the smallest that
// fits; 0 when none does.
int cluster_for(int N, int K, int want) {
  const size_t lim = 227 * 1024, two = 113 * 1024;
  struct Opt {
    int n, c;
    size_t bytes;
  };
  const Opt opts[] = {{64, 1, frame_smem_bytes<64, 1>(K)},   {96, 2, frame_smem_bytes<96, 2>(K)},
                      {128, 2, frame_smem_bytes<128, 2>(K)}, {128, 4, frame_smem_bytes<128, 4>(K)},
                      {192, 8, frame_smem_bytes<192, 8>(K)}, {256, 8, frame_smem_bytes<256, 8>(K)},
                      {256, 16, frame_smem_bytes<256, 16>(K)}};
  for (const Opt& o : opts)
    if (o.n == N && o.c == want && o.bytes <= lim) return o.c;
  for (const Opt& o : opts)
    if (o.n == N && o.bytes <= two) return o.c;
  for (const Opt& o : opts)
    if (o.n == N && o.bytes <= lim) return o.c;
  return 0;
}

template <int N, int C, int MODE>
cudaError_t launch_frame_nc(const FrameArgs& a, int nslot, int K, cudaStream_t s) {
  auto kern = frame_kernel<N, C, MODE>;
  const size_t smem = frame_smem_bytes<N, C>(K);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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
  return cudaLaunchKernelEx(&cfg, kern, a);
}

template <int MODE>
cudaError_t launch_frame_raw(ptyb_handle* h, const FrameArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  switch (h->N * 100 + h->C) {
    case 6401: return launch_frame_nc<64, 1, MODE>(a, nslot, h->K, h->stream);
    case 12802: return launch_frame_nc<128, 2, MODE>(a, nslot, h->K, h->stream);
    case 12804: return launch_frame_nc<128, 4, MODE>(a, nslot, h->K, h->stream);
    case 9602: return launch_frame_nc<96, 2, MODE>(a, nslot, h->K, h->stream);
    case 19208: return launch_frame_nc<192, 8, MODE>(a, nslot, h->K, h->stream);
    case 25608: return launch_frame_nc<256, 8, MODE>(a, nslot, h->K, h->stream);
    case 25616: return launch_frame_nc<256, 16, MODE>(a, nslot, h->K, h->stream);
  }
  return cudaErrorInvalidValue;
}

template <int MODE>
cudaError_t launch_frame(ptyb_handle* h, const FrameArgs& a, int nslot) {
  constexpr int kind = MODE == kRpie ? kKFrameRpie
                       : MODE == kLsqmlFused ? kKFrameLsqml
                       : MODE == kMlGrad ? kKFrameMl
                       : MODE == kLlk ? kKFrameLlk
                       : MODE == kStore ? kKFrameStore
                       : MODE == kProject || MODE == kProjectKept ? kKFrameProject
                       : MODE == kCarry ? kKFrameCarry
                                        : kKFrameFromStore;
  cudaError_t e = cudaSuccess;
  timed(h, kind, [&] { e = launch_frame_raw<MODE>(h, a, nslot); }, nslot);
  return e;
}

template <int N, int C, int MODE>
cudaError_t launch_move_nc(const MoveArgs& a, int nslot, int K, cudaStream_t s) {
  auto kern = move_kernel<N, C, MODE>;
  const size_t smem = move_smem_bytes<N, C>(K);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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
  return cudaLaunchKernelEx(&cfg, kern, a);
}

// Plane transforms of the position model over `nslot` frames (the frame kernel's cluster
// shape; window derivatives carry two planes).
template <int MODE>
cudaError_t launch_move(ptyb_handle* h, const MoveArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  const int K = MODE == kDerivWindow ? 2 : h->K;
  constexpr int kind = MODE == kDerivSums      ? kKDerivSums
                       : MODE == kSpectrum     ? kKSpectrum
                       : MODE == kBackSpectrum ? kKBackSpectrum
                                               : kKMove;
  const int C = MODE == kDerivSums ? h->C_sums : h->C;
  cudaError_t e = cudaErrorInvalidValue;
  timed(h, kind, [&] {
    switch (h->N * 100 + C) {
      case 6401: e = launch_move_nc<64, 1, MODE>(a, nslot, K, h->stream); break;
      case 12802: e = launch_move_nc<128, 2, MODE>(a, nslot, K, h->stream); break;
      case 12804: e = launch_move_nc<128, 4, MODE>(a, nslot, K, h->stream); break;
      case 9602: e = launch_move_nc<96, 2, MODE>(a, nslot, K, h->stream); break;
      case 19208: e = launch_move_nc<192, 8, MODE>(a, nslot, K, h->stream); break;
      case 25608: e = launch_move_nc<256, 8, MODE>(a, nslot, K, h->stream); break;
      case 25616: e = launch_move_nc<256, 16, MODE>(a, nslot, K, h->stream); break;
    }
 }, nslot);
  return e;
}

template <int N, int C, int MODE>
cudaError_t launch_slice_nc(const SliceArgs& a, int nslot, int K, cudaStream_t s) {
  auto kern = slice_kernel<N, C, MODE>;
  const size_t smem = frame_smem_bytes<N, C>(K);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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
  return cudaLaunchKernelEx(&cfg, kern, a);
}

template <int MODE>
cudaError_t launch_slice(ptyb_handle* h, const SliceArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  constexpr int kind = MODE == kSliceForward ? kKSliceForward
                       : MODE == kSliceBackward ? kKSliceBackward
                       : MODE == kSliceGrad     ? kKSliceGrad
                                                : kKSliceLlk;
  cudaError_t e = cudaErrorInvalidValue;
  timed(h, kind, [&] {
    switch (h->N * 100 + h->C) {
      case 6401: e = launch_slice_nc<64, 1, MODE>(a, nslot, h->K, h->stream); break;
      case 12802: e = launch_slice_nc<128, 2, MODE>(a, nslot, h->K, h->stream); break;
      case 12804: e = launch_slice_nc<128, 4, MODE>(a, nslot, h->K, h->stream); break;
      case 9602: e = launch_slice_nc<96, 2, MODE>(a, nslot, h->K, h->stream); break;
      case 19208: e = launch_slice_nc<192, 8, MODE>(a, nslot, h->K, h->stream); break;
      case 25608: e = launch_slice_nc<256, 8, MODE>(a, nslot, h->K, h->stream); break;
      case 25616: e = launch_slice_nc<256, 16, MODE>(a, nslot, h->K, h->stream); break;
    }
 }, nslot);
  return e;
}

MoveArgs move_args(ptyb_handle* h, const int* frames, float2* planes) {
  MoveArgs m = {};
  m.probe = h->probe;
  m.quad = h->quad;
  m.tw = h->tw;
  m.object = h->object;
  m.frames = frames;
  m.corners = h->corners;
  m.offsets = h->offsets;
  m.planes = planes;
  m.nxo = h->nxo;
  m.K = h->K;
  return m;
}

// DFT(q·P) of the K planes `probe` into `spec` (the probe spectra the moves start from,
// engine/features.rs:347-360).
void spectrum_of(ptyb_handle* h, const float2* probe, float2* spec) {
  MoveArgs m = move_args(h, h->iota, spec);
  m.probe = probe;
  check(h, launch_move<kSpectrum>(h, m, 1), "probe spectrum");
  ++h->launches;
}

// Each of `n` frames' moved probe conj(q)·T_d(q·P) from the spectrum `spec` into `out`
// ([slot][K][N][N]).
void move_frames(ptyb_handle* h, const int* frames, int n, const float2* spec, float2* out) {
  MoveArgs m = move_args(h, frames, out);
  m.spec = spec;
  check(h, launch_move<kFromSpectrum>(h, m, n), "probe move");
  ++h->launches;
}

void ensure_spec(ptyb_handle* h) {
  if (h->spec) return;
  const size_t np = (size_t)h->K * h->N * h->N;
  h->spec = alloc<float2>(h, np);
  h->spec_d = alloc<float2>(h, np);
}

FrameArgs frame_args(ptyb_handle* h, const int* frames) {
  FrameArgs a = {};
  a.object = h->object;
  a.probe = h->probe;
  a.quad = h->quad;
  a.tw = h->tw;
  a.iobs = h->iobs;
  a.frames = frames;
  a.corners = h->corners;
  a.out = h->upd;
  a.field = h->field;
  a.icalc = h->icalc;
  a.omax = h->omax;
  a.llk = h->llk;
  a.a_far = h->afar2;
  a.nyo = h->nyo;
  a.nxo = h->nxo;
  a.nprobe = h->nprobe;
  a.nobj = h->nobj;
  a.cost = kCostPoisson;
  return a;
}

GatherArgs gather_args(ptyb_handle* h, const int* frames, int nslot) {
  GatherArgs g = {};
  g.object = h->object;
  g.probe = h->probe;
  g.quad = h->quad;
  g.upd = h->upd;
  g.frames = frames;
  g.corners = h->corners;
  g.pmax = h->scal + 0;
  g.pre = h->pre;
  g.pre_max = h->scal + 1;
  g.out = h->d_obj;
  g.nslot = nslot;
  g.nyo = h->nyo;
  g.nxo = h->nxo;
  g.nprobe = h->nprobe;
  g.N = h->N;
  return g;
}

int ntiles(ptyb_handle* h) {
  return ((h->nyo + kTile - 1) / kTile) * ((h->nxo + kTile - 1) / kTile);
}

// Scratch for `n` frames per launch.
void ensure_slots(ptyb_handle* h, int n) {
  if (n <= h->slots) return;
  const size_t plane = (size_t)h->N * h->N;
  h->upd = alloc<float2>(h, (size_t)n * h->K * plane);
  h->field = alloc<float2>(h, (size_t)n * h->K * plane);
  h->icalc = alloc<float>(h, (size_t)n * plane);
  h->omax = alloc<float>(h, n);
  h->afar1 = alloc<float>(h, n);
  h->afar2 = alloc<float>(h, n);
  h->sums = alloc<double>(h, (size_t)n * 6 * kDotParts);
  if (h->have_offsets) {
    h->wave = alloc<float2>(h, (size_t)n * h->K * plane);
    h->pos_sums = alloc<double>(h, (size_t)n * 4);
  }
  if (h->nslice > 1) {
    h->incident = alloc<float2>(h, (size_t)(h->nslice - 1) * n * h->K * plane);
    h->chi_slices = alloc<float2>(h, (size_t)h->nslice * n * h->K * plane);
    h->slice_sums = alloc<double>(h, (size_t)n * 2);
  }
  h->slots = n;
}

// Probe-pass chunking: about 8 CTAs per SM over the probe pixels.
int probe_chunk(ptyb_handle* h, int nslot, int* nchunk) {
  const int pixblocks = (h->N * h->N + 255) / 256;
  int want = std::max(1, 148 * 8 / pixblocks);
  int chunk = std::min(kMaxProbeChunk, std::max(1, (nslot + want - 1) / want));
  *nchunk = (nslot + chunk - 1) / chunk;
  if (*nchunk > h->max_chunks) {
    h->partial = alloc<float2>(h, (size_t)(*nchunk) * h->K * h->N * h->N);
    h->max_chunks = *nchunk;
  }
  return chunk;
}

// Σ_frames (w·upd) into the probe (mode 0: P += coef·Σ with the rPIE weight; 1: d_probe =
// coef·Σ conj(q·O)·upd).
// Probe direction Σ w·upd over the batch; `quad` and `upd` default to the exit phase and the
// frame kernel's update planes.
void probe_pass(ptyb_handle* h, const int* frames, int nslot, int mode, float alpha, float coef,
                const float2* quad = nullptr, const float2* upd = nullptr) {
  int nchunk = 0;
  const int chunk = probe_chunk(h, nslot, &nchunk);
  ProbeArgs p = {};
  p.object = h->object;
  p.quad = quad ? quad : h->quad;
  p.upd = upd ? upd : h->upd;
  p.frames = frames;
  p.corners = h->corners;
  p.omax = h->omax;
  p.partial = h->partial;
  p.alpha = alpha;
  p.nslot = nslot;
  p.chunk = chunk;
  p.nxo = h->nxo;
  p.K = h->K;
  p.N = h->N;
  p.mode = mode == 0 ? 0 : 1;
  dim3 grid((h->N * h->N + 255) / 256, nchunk);
  timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(p); }, nslot);
  launched(h, "probe_partial");
  const int count = h->K * h->N * h->N;
  timed(h, kKProbeFinal, [&] {
  probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
      h->partial, nchunk, count, h->probe, h->d_probe, nullptr, coef, mode);
  });
  launched(h, "probe_finalize");
}

ptyb_llk llk_of_frames(ptyb_handle* h);

// The LLK of the current estimate over every frame: per-frame sums in frame order.
// `waves` (optional): every frame's moved probe, [P][K][N][N], when the caller has them.
ptyb_llk llk_pass(ptyb_handle* h, const float2* waves = nullptr) {
  const int stack = std::min(h->P, h->stack);
  const size_t pstride = (size_t)h->K * h->N * h->N;
  ensure_slots(h, stack);
  if (h->have_offsets && !waves && h->nslice == 1) {
    ensure_spec(h);
    spectrum_of(h, h->probe, h->spec);
  }
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    FrameArgs a = frame_args(h, h->iota + s0);
    a.llk = h->llk + (size_t)s0 * 4;
    if (h->nslice > 1) {
      SliceArgs sa = {};
      sa.f = a;
      sa.f.nslot = n;
      sa.tf = h->tf;
      sa.nslice = h->nslice;
      sa.obj_plane = (size_t)h->nyo * h->nxo;
      check(h, launch_slice<kSliceLlk>(h, sa, n), "llk pass");
      ++h->launches;
      continue;
    }
    if (waves) {
      // each frame's own (moved or varied) probe (engine/lsqml.rs:537-551)
      a.probe = waves + s0 * pstride;
      a.probe_stride = (int)pstride;
    } else if (h->have_offsets) {
      move_frames(h, h->iota + s0, n, h->spec, h->wave);
      a.probe = h->wave;
      a.probe_stride = (int)pstride;
    }
    check(h, launch_frame<kLlk>(h, a, n), "llk pass");
    ++h->launches;
  }
  return llk_of_frames(h);
}

// The normalised LLK from every frame's sums in h->llk, added in frame order on the host.
ptyb_llk llk_of_frames(ptyb_handle* h) {
  std::vector<double> v((size_t)h->P * 4);
  check(h, cudaMemcpyAsync(v.data(), h->llk, v.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream),
        "llk download");
  check(h, cudaStreamSynchronize(h->stream), "llk pass");
  double s[4] = {0, 0, 0, 0};
  for (int f = 0; f < h->P; ++f)
    for (int k = 0; k < 4; ++k) s[k] += v[(size_t)f * 4 + k];
  ptyb_llk l;
  l.poisson = s[0] / h->nb_obs;
  l.gaussian = s[1] / h->nb_obs;
  l.euclidian = s[2] / h->nb_obs;
  l.nb_photons_calc = s[3];
  return l;
}

void record(ptyb_handle* h, int algorithm, const ptyb_llk& l) {
  ptyb_llk_record r = {};
  r.cycle = h->cycle;
  r.algorithm = algorithm;
  r.llk = l;
  h->history.push_back(r);
}

bool llk_due(int calc_llk, int ic, int ncycle) {
  return calc_llk > 0 && (ic % calc_llk == 0 || ic + 1 == ncycle);
}

// Every epoch's batch order of a call, computed on the host and uploaded once before the
// call's first launch; sizes[e] holds epoch e's batch lengths.
void upload_orders(ptyb_handle* h, int nepoch, int size, uint64_t seed, int64_t epoch0,
                   std::vector<std::vector<int32_t>>* sizes, std::vector<int32_t>* last) {
  std::vector<int32_t> all, order, sz;
  all.reserve((size_t)nepoch * h->P);
  sizes->clear();
  for (int e = 0; e < nepoch; ++e) {
    random_batches(h->P, size, seed, (uint64_t)(epoch0 + e), &order, &sz);
    all.insert(all.end(), order.begin(), order.end());
    sizes->push_back(sz);
  }
  if (last) *last = order;
  if (all.size() > h->order_cap) {
    h->order_all = alloc<int>(h, all.size());
    h->order_cap = all.size();
  }
  if (!all.empty())
    check(h, copy_sync(h, h->order_all, all.data(), all.size() * sizeof(int32_t),
                        cudaMemcpyHostToDevice),
          "order upload");
}

// One rPIE batch (engine/ptycho.rs:904-1085; GPU launch sequence engine/gpu/rpie.rs:239-345).
void rpie_batch(ptyb_handle* h, const ptyb_rpie_params& p, const int* frames, int nslot) {
  FrameArgs a = frame_args(h, frames);
  GatherArgs g = gather_args(h, frames, nslot);
  const int pstride = h->K * h->N * h->N;
  const bool moved = h->have_offsets, refine = h->have_offsets && h->refine_offsets;
  if (moved) {
    // every frame's probe moved by its offset from the batch-start probe (engine/ptycho.rs:
    // 920-935); the views' waves in the frame pass and the object gathers
    ensure_spec(h);
    spectrum_of(h, h->probe, h->spec);
    move_frames(h, frames, nslot, h->spec, h->wave);
    a.probe = h->wave;
    a.probe_stride = pstride;
    g.probe = h->wave;
    g.probe_stride = pstride;
  }
  check(h, launch_frame<kRpie>(h, a, nslot), "rpie frame pass");
  ++h->launches;
  if (p.update_object) {
    check(h, cudaMemsetAsync(h->scal, 0, sizeof(float), h->stream), "memset");
    timed(h, kKObjOverlap, [&] { object_tile_kernel<kGatherOverlap><<<ntiles(h), 1024, 0, h->stream>>>(g); }, nslot);
    launched(h, "overlap max");
  }
  if (refine) {
    // pty-chi's position sums from mode 0 of the batch-start state (engine/ptycho.rs:1037-1064)
    check(h, launch_move<kDerivWindow>(h, move_args(h, frames, h->field), nslot), "window derivative");
    ++h->launches;
    timed(h, kKPositionSums, [&] {
      position_sums_kernel<<<nslot, 256, 0, h->stream>>>(h->field, h->wave, pstride, h->quad,
                                                          h->upd, h->K, h->N, h->pos_sums);
    }, nslot);
    launched(h, "position sums");
  }
  const int count = h->K * h->N * h->N;
  int nchunk = 0;
  if (p.update_probe && moved) {
    // each frame's rPIE probe direction moved back by −d (engine/ptycho.rs:1007-1035)
    timed(h, kKProbePartial, [&] {
      probe_terms_kernel<<<dim3((h->N * h->N + 255) / 256, nslot), 256, 0, h->stream>>>(
          h->object, h->quad, h->upd, frames, h->corners, h->nxo, h->K, h->N, h->field, h->omax,
          (float)p.probe_alpha);
    }, nslot);
    launched(h, "probe terms");
    check(h, launch_move<kMoveBack>(h, move_args(h, frames, h->field), nslot), "probe move back");
    ++h->launches;
  } else if (p.update_probe) {
    // Reads the batch-start object, so it runs before the object update.
    const int chunk = probe_chunk(h, nslot, &nchunk);
    ProbeArgs pa = {};
    pa.object = h->object;
    pa.quad = h->quad;
    pa.upd = h->upd;
    pa.frames = frames;
    pa.corners = h->corners;
    pa.omax = h->omax;
    pa.partial = h->partial;
    pa.alpha = (float)p.probe_alpha;
    pa.nslot = nslot;
    pa.chunk = chunk;
    pa.nxo = h->nxo;
    pa.K = h->K;
    pa.N = h->N;
    pa.mode = 0;
    dim3 grid((h->N * h->N + 255) / 256, nchunk);
    timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(pa); }, pa.nslot);
    launched(h, "probe partial");
  }
  if (p.update_object) {
    g.alpha = (float)p.obj_alpha;
    g.step = (float)p.obj_step;
    timed(h, kKObjRpie, [&] { object_tile_kernel<kGatherRpie><<<ntiles(h), 1024, 0, h->stream>>>(g); }, g.nslot);
    launched(h, "object update");
  }
  if (p.update_probe) {
    // P += step/nbatch · Σ (frames in order); the gathers above read the batch-start probe
    timed(h, kKProbeFinal, [&] {
      probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
          moved ? h->field : h->partial, moved ? nslot : nchunk, count, h->probe, nullptr,
          nullptr, (float)(p.probe_step / nslot), 0);
    });
    launched(h, "probe update");
  }
  if (refine) {
    const double eps = 1e-6 * ((double)h->N * h->N);
    timed(h, kKSolve, [&] {
      position_step_kernel<<<1, 32, 0, h->stream>>>(h->pos_sums, nslot, h->P, eps, frames,
                                                    h->offsets);
    });
    launched(h, "position step");
  }
}

// The preconditioner over every view on pty-chi's schedule (engine/lsqml.rs:676-700).
void lsqml_preconditioner(ptyb_handle* h, bool init) {
  GatherArgs g = gather_args(h, h->iota, h->P);
  g.pre_scale = init ? (float)(h->max_power / (4.0 * h->N * h->N * ((double)h->N * h->N))) : -1.f;
  timed(h, kKIllum, [&] { object_tile_kernel<kGatherIllum><<<ntiles(h), 1024, 0, h->stream>>>(g); });
  launched(h, "illumination");
  check(h, cudaMemsetAsync(h->scal + 1, 0, sizeof(float), h->stream), "memset");
  const size_t n = (size_t)h->nyo * h->nxo;
  timed(h, kKMax, [&] { max_kernel<<<296, 256, 0, h->stream>>>(h->pre, n, h->scal + 1); });
  launched(h, "pre max");
}

// One LSQML step through pty-chi's multislice object (engine/lsqml.rs:581-643 with
// SliceWaves, engine/multislice.rs): forward through the slices, backward χ per slice, every
// slice's object direction from its incident wave, the probe direction from χ of slice 0,
// slice 0's step sizes jointly with the probe and Eq. 23b on the others.
void lsqml_batch_slices(ptyb_handle* h, const ptyb_lsqml_params& p, const int* frames, int nslot,
                        double* log, int log_stride) {
  const int S = h->nslice;
  const size_t plane = (size_t)h->N * h->N, fplanes = (size_t)h->K * plane;
  const size_t slice_stride = (size_t)nslot * fplanes, no = (size_t)h->nyo * h->nxo;
  SliceArgs sa = {};
  sa.f = frame_args(h, frames);
  sa.f.cost = p.cost;
  sa.f.nslot = nslot;
  sa.f.a_prev = h->afar_all;
  sa.f.a_prev_by_frame = 1;
  sa.f.a_out = h->afar1;
  sa.tf = h->tf;
  sa.incident = h->incident;
  sa.chi = h->chi_slices;
  sa.nslice = S;
  sa.obj_plane = no;
  check(h, launch_slice<kSliceForward>(h, sa, nslot), "multislice forward");
  ++h->launches;
  sa.f.a_mid = h->afar1;
  sa.f.a_out = h->afar2;
  check(h, launch_slice<kSliceBackward>(h, sa, nslot), "multislice backward");
  ++h->launches;
  for (int s = 0; s < S; ++s) {
    GatherArgs g = gather_args(h, frames, nslot);
    g.upd = h->chi_slices + s * slice_stride;
    g.out = h->d_obj + s * no;
    g.quad = s + 1 == S ? h->quad : h->ones;
    if (s > 0) {
      g.probe = h->incident + (s - 1) * slice_stride;
      g.probe_stride = (int)fplanes;
    }
    timed(h, kKObjLsqml, [&] { object_tile_kernel<kGatherLsqml><<<ntiles(h), 1024, 0, h->stream>>>(g); }, nslot);
    launched(h, "slice object direction");
  }
  // probe direction from χ of slice 0 through slice 0's windows (no phase when S > 1)
  probe_pass(h, frames, nslot, 1, 0.f, 1.0f / nslot, h->ones, h->chi_slices);
  const double lambda0 = 1.2e-7 * ((double)h->N * h->N) / ((double)h->N * h->N);
  timed(h, kKDots, [&] {
    lsqml_dots_kernel<<<nslot * kDotParts, 512, 0, h->stream>>>(
        h->object, h->d_obj, h->probe, h->d_probe, h->ones, h->chi_slices, frames, h->corners,
        h->nxo, h->K, h->N, lambda0, h->sums, 0);
  }, nslot);
  launched(h, "step sums");
  const double scale = (double)(S * h->K);
  for (int s = 1; s < S; ++s) {
    timed(h, kKDots, [&] {
      slice_dots_kernel<<<nslot, 512, 0, h->stream>>>(
          h->d_obj + s * no, h->incident + (s - 1) * slice_stride,
          s + 1 == S ? h->quad : nullptr, h->chi_slices + s * slice_stride, frames, h->corners,
          h->nxo, h->K, h->N, h->slice_sums);
    }, nslot);
    launched(h, "slice sums");
    timed(h, kKSolve, [&] {
      slice_solve_kernel<<<1, 1024, 0, h->stream>>>(h->slice_sums, nslot, scale, log + 2 + s,
                                                    log_stride, h->scal + 3 + s);
    });
    launched(h, "slice solve");
  }
  timed(h, kKSolve, [&] {
    lsqml_solve_kernel<<<1, 1024, 0, h->stream>>>(h->sums, nslot, scale, h->afar2, frames,
                                                   h->afar_all, log, h->scal + 2, log_stride);
  });
  launched(h, "step solve");
  for (int s = 0; s < S; ++s) {
    const int which = s == 0 ? 0 : 1 + s;  // relative to scal + 2: so_0, sp, so_1, so_2, …
    timed(h, kKAxpy, [&] {
      axpy_scal_kernel<<<(unsigned)((no + 255) / 256), 256, 0, h->stream>>>(
          h->object + s * no, h->d_obj + s * no, h->scal + 2, which, no);
    });
    launched(h, "slice step");
  }
  timed(h, kKAxpy, [&] {
    axpy_scal_kernel<<<(unsigned)((fplanes + 255) / 256), 256, 0, h->stream>>>(
        h->probe, h->d_probe, h->scal + 2, 1, fplanes);
  });
  launched(h, "probe step");
}

// One LSQML step on a batch (engine/lsqml.rs:581-643), with the position model when offsets
// are set: each frame's probe moved by its offset, the probe directions moved back before
// their frame mean, and with refinement pty-chi's position step after the update.
// The probe variation's batch scratch for h->slots frames and the planes of every frame.
void ensure_opr(ptyb_handle* h) {
  const size_t plane = (size_t)h->N * h->N;
  if (h->opr_slots < h->slots) {
    h->opr_vv = alloc<float>(h, (size_t)h->slots * plane);
    h->opr_r = alloc<float2>(h, (size_t)h->slots * plane);
    h->opr_sums = alloc<double>(h, (size_t)h->slots * 3);
    h->opr_p = alloc<double>(h, h->slots);
    h->wave = alloc<float2>(h, (size_t)h->slots * h->K * plane);
    h->opr_slots = h->slots;
  }
  if (!h->opr_e) {
    h->opr_e = alloc<float2>(h, plane);
    h->opr_scal = alloc<double>(h, 4);
  }
  if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * h->K * plane);
}

// Every slot's own probe planes under the probe variation into `out` ([slot][K][N][N]).
void opr_planes(ptyb_handle* h, const int* frames, int nslot, float2* out) {
  const int plane = h->N * h->N;
  timed(h, kKOprStep, [&] {
    opr_planes_kernel<<<dim3((plane + 255) / 256, nslot), 256, 0, h->stream>>>(
        h->probe, h->opr_u, h->opr_w, h->opr_has_c ? h->opr_c : nullptr, frames, h->K, h->opr_k,
        plane, out);
  });
  launched(h, "opr planes");
}

// The OPR step of the batch (engine/opr.rs:122-224) from its frame probe directions, mode-0
// plane of each slot of h->field, and the probe's mode 0 on entry.
void opr_step(ptyb_handle* h, const int* frames, int count) {
  const int plane = h->N * h->N, k = h->opr_k;
  const size_t dstride = (size_t)h->K * plane;
  const unsigned pb = (unsigned)((plane + 255) / 256), pb32 = (unsigned)((plane + 31) / 32);
  timed(h, kKOprStep, [&] {
    window_power_kernel<<<dim3(pb, count), 256, 0, h->stream>>>(h->object, frames, h->corners,
                                                               h->nxo, h->N, h->opr_vv);
  }, count);
  launched(h, "opr window power");
  if (h->opr_has_c && h->opr_refine_c) {
    timed(h, kKOprStep, [&] {
      opr_frame_sums_kernel<<<count, 256, 0, h->stream>>>(h->probe, h->field, dstride, h->opr_vv,
                                                          plane, h->opr_sums);
    });
    launched(h, "opr intensity sums");
    timed(h, kKOprStep, [&] {
      opr_intensity_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(h->opr_sums, frames, count,
                                                                        h->opr_c);
    });
    launched(h, "opr intensity");
  }
  if (k == 0 || count < 2) return;
  timed(h, kKOprStep, [&] {
    opr_residue_kernel<<<pb32, 256, 0, h->stream>>>(h->field, dstride, count, plane, h->opr_r);
  });
  launched(h, "opr residues");
  const double a_u = std::min(0.1, (double)count / h->P);
  for (int i = 0; i < k; ++i) {
    float2* u = h->opr_u + (size_t)i * plane;
    timed(h, kKOprStep, [&] {
      opr_frame_sums_kernel<<<count, 256, 0, h->stream>>>(u, h->opr_r, plane, nullptr, plane,
                                                          h->opr_sums);
    });
    launched(h, "opr dots");
    timed(h, kKOprStep, [&] {
      opr_coef_kernel<<<1, 256, 0, h->stream>>>(h->opr_sums, h->opr_w, frames, k, i, count,
                                                (double)plane, h->opr_p);
    });
    launched(h, "opr coefficients");
    timed(h, kKOprStep, [&] {
      opr_e_kernel<<<pb32, 256, 0, h->stream>>>(h->opr_r, h->opr_p, count, plane, h->opr_e);
    });
    launched(h, "opr e");
    timed(h, kKOprStep, [&] { opr_norm2_kernel<<<1, 1024, 0, h->stream>>>(h->opr_e, plane, h->opr_scal); });
    launched(h, "opr norm");
    timed(h, kKOprStep, [&] {
      opr_u_step_kernel<<<pb, 256, 0, h->stream>>>(u, h->opr_e, h->opr_scal, a_u, plane);
    });
    launched(h, "opr eigenmode step");
    timed(h, kKOprStep, [&] { opr_norm2_kernel<<<1, 1024, 0, h->stream>>>(u, plane, h->opr_scal + 1); });
    launched(h, "opr norm");
    timed(h, kKOprStep, [&] { opr_u_scale_kernel<<<pb, 256, 0, h->stream>>>(u, h->opr_scal + 1, plane); });
    launched(h, "opr eigenmode scale");
    if (h->opr_refine_w) {
      timed(h, kKOprStep, [&] {
        opr_frame_sums_kernel<<<count, 256, 0, h->stream>>>(u, h->field, dstride, h->opr_vv,
                                                            plane, h->opr_sums);
      });
      launched(h, "opr weight sums");
      timed(h, kKOprStep, [&] {
        opr_weights_kernel<<<1, 256, 0, h->stream>>>(h->opr_sums, frames, count, k, i, h->opr_w);
      });
      launched(h, "opr weights");
    }
    if (i + 1 < k) {
      timed(h, kKOprStep, [&] { opr_norm2_kernel<<<1, 1024, 0, h->stream>>>(u, plane, h->opr_scal + 2); });
      launched(h, "opr norm");
      timed(h, kKOprStep, [&] {
        opr_frame_sums_kernel<<<count, 256, 0, h->stream>>>(u, h->opr_r, plane, nullptr, plane,
                                                            h->opr_sums);
      });
      launched(h, "opr projections");
      timed(h, kKOprStep, [&] {
        opr_gs_kernel<<<dim3(pb, count), 256, 0, h->stream>>>(h->opr_r, u, h->opr_sums, h->opr_scal + 2, count,
                                                 plane);
      });
      launched(h, "opr orthogonalisation");
    }
  }
}

void lsqml_batch(ptyb_handle* h, const ptyb_lsqml_params& p, const int* frames, int nslot,
                 double* log) {
  const int pstride = h->K * h->N * h->N;
  FrameArgs a = frame_args(h, frames);
  a.cost = p.cost;
  const bool opr = h->opr_on;
  if (opr) {
    // every frame's own probe (engine/opr.rs:88-120) in place of the shared one
    opr_planes(h, frames, nslot, h->wave);
    a.probe = h->wave;
    a.probe_stride = pstride;
  }
  if (h->have_offsets) {
    ensure_spec(h);
    spectrum_of(h, h->probe, h->spec);
    move_frames(h, frames, nslot, h->spec, h->wave);
    a.probe = h->wave;
    a.probe_stride = pstride;
  }
  if (p.cost == PTYB_COST_POISSON) {
    // Forward pass with the xi solver's first pass, backward pass with its second.
    a.nslot = nslot;
    a.icalc = nullptr;
    a.a_prev = h->afar_all;
    a.a_prev_by_frame = 1;
    a.a_out = h->afar1;
    check(h, launch_frame<kStore>(h, a, nslot), "lsqml forward");
    ++h->launches;
    a.a_mid = h->afar1;
    a.a_out = h->afar2;
    check(h, launch_frame<kFromStore>(h, a, nslot), "lsqml backward");
    ++h->launches;
  } else {
    timed(h, kKMisc, [&] {
      fill_kernel<<<(nslot + 255) / 256, 256, 0, h->stream>>>(h->afar2, 0.5f, nslot);
    });
    launched(h, "a_far");
    check(h, launch_frame<kLsqmlFused>(h, a, nslot), "lsqml pass");
    ++h->launches;
  }
  GatherArgs g = gather_args(h, frames, nslot);
  if (h->have_offsets || opr) {
    g.probe = h->wave;
    g.probe_stride = pstride;
  }
  timed(h, kKObjLsqml, [&] { object_tile_kernel<kGatherLsqml><<<ntiles(h), 1024, 0, h->stream>>>(g); }, nslot);
  launched(h, "object direction");
  if (opr) {
    // each frame's probe direction conj(q·O)·χ (the OPR step reads mode 0), their mean dP
    timed(h, kKProbePartial, [&] {
      probe_terms_kernel<<<dim3((h->N * h->N + 255) / 256, nslot), 256, 0, h->stream>>>(
          h->object, h->quad, h->upd, frames, h->corners, h->nxo, h->K, h->N, h->field);
    });
    launched(h, "probe terms");
    timed(h, kKProbeFinal, [&] {
      probe_finalize_kernel<<<(pstride + 255) / 256, 256, 0, h->stream>>>(
          h->field, nslot, pstride, h->probe, h->d_probe, nullptr, 1.0f / nslot, 1);
    });
    launched(h, "probe direction");
  } else if (h->have_offsets) {
    timed(h, kKProbePartial, [&] {
      probe_terms_kernel<<<dim3((h->N * h->N + 255) / 256, nslot), 256, 0, h->stream>>>(
          h->object, h->quad, h->upd, frames, h->corners, h->nxo, h->K, h->N, h->field);
    });
    launched(h, "probe terms");
    check(h, launch_move<kMoveBack>(h, move_args(h, frames, h->field), nslot), "probe move back");
    ++h->launches;
    timed(h, kKProbeFinal, [&] {
      probe_finalize_kernel<<<(pstride + 255) / 256, 256, 0, h->stream>>>(
          h->field, nslot, pstride, h->probe, h->d_probe, nullptr, 1.0f / nslot, 1);
    });
    launched(h, "probe direction");
  } else {
    probe_pass(h, frames, nslot, 1, 0.f, 1.0f / nslot);
  }
  const double lambda0 = 1.2e-7 * ((double)h->N * h->N) / ((double)h->N * h->N);
  const float2* fprobe = h->have_offsets || opr ? h->wave : h->probe;
  const int fstride = h->have_offsets || opr ? pstride : 0;
  timed(h, kKDots, [&] {
    lsqml_dots_kernel<<<nslot * kDotParts, 512, 0, h->stream>>>(h->object, h->d_obj, fprobe, h->d_probe,
                                                     h->quad, h->upd, frames, h->corners,
                                                     h->nxo, h->K, h->N, lambda0, h->sums,
                                                     fstride);
  }, nslot);
  launched(h, "step sums");
  const bool refine = h->have_offsets && h->refine_offsets;
  if (refine) {
    // position directions from the state on entry (engine/lsqml.rs:237-270)
    check(h, launch_move<kDerivWindow>(h, move_args(h, frames, h->field), nslot), "window derivative");
    ++h->launches;
    timed(h, kKPositionSums, [&] {
      position_sums_kernel<<<nslot, 256, 0, h->stream>>>(h->field, h->wave, pstride, h->quad,
                                                          h->upd, h->K, h->N, h->pos_sums);
    }, nslot);
    launched(h, "position sums");
  }
  timed(h, kKSolve, [&] {
    lsqml_solve_kernel<<<1, 1024, 0, h->stream>>>(h->sums, nslot, (double)(1 * h->K), h->afar2,
                                                   frames, h->afar_all, log, h->scal + 2, 3);
  });
  launched(h, "step solve");
  // the eigenmodes and the refined weights from the state on entry (engine/lsqml.rs:620-621)
  if (opr) opr_step(h, frames, nslot);
  const size_t no = (size_t)h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  timed(h, kKAxpy, [&] {
    axpy_scal_kernel<<<(unsigned)((no + 255) / 256), 256, 0, h->stream>>>(h->object, h->d_obj,
                                                                         h->scal + 2, 0, no);
  });
  launched(h, "object step");
  timed(h, kKAxpy, [&] {
    axpy_scal_kernel<<<(unsigned)((np + 255) / 256), 256, 0, h->stream>>>(h->probe, h->d_probe,
                                                                         h->scal + 2, 1, np);
  });
  launched(h, "probe step");
  if (refine) {
    const double eps = 1e-6 * ((double)h->N * h->N);
    timed(h, kKSolve, [&] {
      position_step_kernel<<<1, 32, 0, h->stream>>>(h->pos_sums, nslot, h->P, eps, frames,
                                                    h->offsets);
    });
    launched(h, "position step");
  }
}

// Every slice's 2·∂L/∂O_s* and the probe's 2·∂L/∂P* of the Poisson LLK sum through a
// multislice object (the adjoint of engine/multislice.rs:87-173, 266-286, 399-438): per stack,
// the exit wave's Poisson gradient back-propagated through the slices on chip, then per slice
// Σ conj(q_s·in_s)·g_s gathered in frame order, the probe's Σ conj(O_0)·g_0.
void ensure_ml(ptyb_handle* h);

void slice_gradients(ptyb_handle* h, bool uo, bool up) {
  const int S = h->nslice, stack = std::min(h->P, h->stack);
  ensure_slots(h, stack);
  ensure_ml(h);
  const size_t plane = (size_t)h->N * h->N, fplanes = (size_t)h->K * plane;
  const size_t no = (size_t)h->nyo * h->nxo;
  if (!h->g_slices) {
    h->g_slices = alloc<float2>(h, (size_t)S * no);
    h->g_slices_c = alloc<float2>(h, (size_t)S * no);
  }
  check(h, cudaMemsetAsync(h->g_slices, 0, (size_t)S * no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_slices_c, 0, (size_t)S * no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe, 0, fplanes * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe_c, 0, fplanes * sizeof(float2), h->stream), "memset");
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    const int* frames = h->iota + s0;
    const size_t slice_stride = (size_t)n * fplanes;
    SliceArgs sa = {};
    sa.f = frame_args(h, frames);
    sa.f.nslot = n;
    sa.tf = h->tf;
    sa.incident = h->incident;
    sa.chi = h->chi_slices;
    sa.nslice = S;
    sa.obj_plane = no;
    check(h, launch_slice<kSliceGrad>(h, sa, n), "multislice gradient");
    ++h->launches;
    for (int s = 0; uo && s < S; ++s) {
      GatherArgs g = gather_args(h, frames, n);
      g.upd = h->chi_slices + s * slice_stride;
      g.out = h->g_slices + s * no;
      g.comp = h->g_slices_c + s * no;
      g.quad = s + 1 == S ? h->quad : h->ones;
      if (s > 0) {
        g.probe = h->incident + (s - 1) * slice_stride;
        g.probe_stride = (int)fplanes;
      }
      timed(h, kKObjMl, [&] { object_tile_kernel<kGatherMl><<<ntiles(h), 1024, 0, h->stream>>>(g); }, n);
      launched(h, "slice gradient");
    }
    if (up) {
      int nchunk = 0;
      const int chunk = probe_chunk(h, n, &nchunk);
      ProbeArgs pa = {};
      pa.object = h->object;
      pa.quad = h->ones;
      pa.upd = h->chi_slices;
      pa.frames = frames;
      pa.corners = h->corners;
      pa.omax = h->omax;
      pa.partial = h->partial;
      pa.nslot = n;
      pa.chunk = chunk;
      pa.nxo = h->nxo;
      pa.K = h->K;
      pa.N = h->N;
      pa.mode = 1;
      dim3 grid((h->N * h->N + 255) / 256, nchunk);
      timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(pa); }, n);
      launched(h, "probe gradient");
      const int count = (int)fplanes;
      timed(h, kKProbeFinal, [&] {
        probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
            h->partial, nchunk, count, nullptr, h->g_probe, h->g_probe_c, 1.f, 2);
      });
      launched(h, "probe gradient sum");
    }
  }
}

// Runs fn(begin, end) over [0, n) on up to eight host threads (one below a million).
template <class F>
void parallel_range(size_t n, F&& fn) {
  const size_t nt = n < (size_t(1) << 20) ? 1 : std::min<size_t>(8, std::thread::hardware_concurrency());
  if (nt <= 1) {
    fn(size_t(0), n);
    return;
  }
  std::vector<std::thread> ts;
  const size_t chunk = (n + nt - 1) / nt;
  for (size_t t = 0; t < nt; ++t) {
    const size_t b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) ts.emplace_back([&fn, b, e] { fn(b, e); });
  }
  for (auto& t : ts) t.join();
}

// The process's page-locked host staging buffer of at least n float2, grown on demand and kept
// (as the device pool keeps device memory), so that a new handle does not pin pages again.
// Callers hold g_stage_mutex while they use it.
std::mutex g_stage_mutex;
float2* g_stage = nullptr;
size_t g_stage_n = 0;

float2* staging(ptyb_handle* h, size_t n) {
  if (n > g_stage_n) {
    if (g_stage) cudaFreeHost(g_stage);
    g_stage = nullptr;
    g_stage_n = 0;
    check(h, cudaMallocHost(&g_stage, n * sizeof(float2)), "cudaMallocHost");
    g_stage_n = n;
  }
  return g_stage;
}

// Device float2 [n] to host complex128 [n] through the staging buffer.
void download_c64(ptyb_handle* h, const float2* src, double* dst, size_t n, const char* what) {
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  float2* st = staging(h, n);
  check(h, copy_sync(h, st, src, n * sizeof(float2), cudaMemcpyDeviceToHost), what);
  parallel_range(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      dst[2 * i] = st[i].x;
      dst[2 * i + 1] = st[i].y;
    }
  });
}

// Host complex128 [n] to device float2 [n] through the staging buffer.
void upload_c64(ptyb_handle* h, const double* src, float2* dst, size_t n, const char* what) {
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  float2* st = staging(h, n);
  parallel_range(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) st[i] = make_float2((float)src[2 * i], (float)src[2 * i + 1]);
  });
  check(h, copy_sync(h, dst, st, n * sizeof(float2), cudaMemcpyHostToDevice), what);
}

template <int N, int C>
cudaError_t launch_gamma_nc(const GammaArgs& a, int nslot, cudaStream_t s) {
  auto kern = gamma_kernel<N, C>;
  const size_t smem = gamma_smem_bytes<N, C>();
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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
  if (C > 1) {
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg);
    if (e != cudaSuccess) return e;
    if (clusters < 1) return cudaErrorLaunchOutOfResources;
  }
  return cudaLaunchKernelEx(&cfg, kern, a);
}

cudaError_t launch_gamma(ptyb_handle* h, const GammaArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  cudaError_t e = cudaErrorInvalidValue;
  timed(h, kKGamma, [&] {
    switch (h->N) {
      case 64: e = launch_gamma_nc<64, 1>(a, nslot, h->stream); break;
      case 96: e = launch_gamma_nc<96, 2>(a, nslot, h->stream); break;
      case 128: e = launch_gamma_nc<128, 4>(a, nslot, h->stream); break;
      case 192: e = launch_gamma_nc<192, 8>(a, nslot, h->stream); break;
      case 256: e = launch_gamma_nc<256, 16>(a, nslot, h->stream); break;
    }
  }, nslot);
  return e;
}

void ensure_ml(ptyb_handle* h) {
  if (h->g_obj) return;
  const size_t no = (size_t)h->nobj * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  h->g_obj = alloc<float2>(h, no);
  h->g_obj_c = alloc<float2>(h, no);
  h->last_obj = alloc<float2>(h, no);
  h->dir_obj = alloc<float2>(h, no);
  h->g_probe = alloc<float2>(h, np);
  h->g_probe_c = alloc<float2>(h, np);
  h->last_probe = alloc<float2>(h, np);
  h->dir_probe = alloc<float2>(h, np);
  h->gamma_sums = alloc<double>(h, (size_t)h->P * 2);
  h->psi_all = alloc<float2>(h, (size_t)h->P * np);
  h->g_all = alloc<float2>(h, (size_t)h->P * np);
  h->g_probe_spec = alloc<float2>(h, np);
  if (!h->partials) h->partials = alloc<double>(h, kPartialBlocks * 2);
}

// Two double sums of an array (mode 0: Polak–Ribière numerator and |h|²; 1: Σ|g|), the block
// partials added in block order on the host.
void array_sums(ptyb_handle* h, const float2* g, const float2* hh, size_t n, int mode, double out[2]) {
  // the block partials, made on first use (ML's set-up, or DM's and RAAR's balance)
  if (!h->partials) h->partials = alloc<double>(h, kPartialBlocks * 2);
  timed(h, kKArraySums, [&] {
    array_sums_kernel<<<kPartialBlocks, 256, 0, h->stream>>>(g, hh, n, mode, h->partials);
  });
  launched(h, "array sums");
  std::vector<double> v(kPartialBlocks * 2);
  check(h, cudaMemcpyAsync(v.data(), h->partials, v.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream),
        "sums");
  check(h, cudaStreamSynchronize(h->stream), "sums");
  out[0] = out[1] = 0.0;
  for (int b = 0; b < kPartialBlocks; ++b) {
    out[0] += v[b * 2];
    out[1] += v[b * 2 + 1];
  }
}

unsigned blocks_for(size_t n) { return (unsigned)((n + 255) / 256); }

// The Poisson gradient numerators of object and probe over every frame, by stacks in frame
// order (engine/ptycho.rs:497-561).
// The Poisson gradients of the object and the probe (engine/ptycho.rs:497-569) from one
// detector field per frame, which is kept for the line search; with `refine`, the position
// sums of AP, DM and ML from the magnitude projection of the same field (engine/ptycho.rs:
// 470-480, engine/features.rs:992-1025). Under the position model the probe gradient goes
// back through the move's adjoint in the spectrum, frame by frame (features.rs:897-957).
void ml_gradients(ptyb_handle* h, bool uo, bool up, bool refine, bool pos_grad = false) {
  const size_t no = (size_t)h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  check(h, cudaMemsetAsync(h->g_obj, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_obj_c, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe, 0, np * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe_c, 0, np * sizeof(float2), h->stream), "memset");
  if (h->have_offsets)
    check(h, cudaMemsetAsync(h->g_probe_spec, 0, np * sizeof(float2), h->stream), "memset");
  const int stack = std::min(h->P, h->stack);
  const int pstride = h->K * h->N * h->N;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    const int* frames = h->iota + s0;
    FrameArgs a = frame_args(h, frames);
    // the gradient field g of these frames, kept for the line search
    float2* gfield = h->g_all + (size_t)s0 * pstride;
    a.out = gfield;
    const float2* waves = h->have_offsets ? h->wave_all + (size_t)s0 * pstride : nullptr;
    if (waves) {
      // each frame's moved probe conj(q)·T_d(q·P) in place of P (engine/ptycho.rs:373-450)
      a.probe = waves;
      a.probe_stride = pstride;
    }
    a.psi_out = h->psi_all + (size_t)s0 * pstride;
    check(h, launch_frame<kMlGrad>(h, a, n), "ml gradient pass");
    ++h->launches;
    if (refine) {
      // the magnitude projection's change of the exit wave from the kept Ψ
      FrameArgs ap = a;
      ap.out = h->field;
      check(h, launch_frame<kProjectKept>(h, ap, n), "magnitude projection");
      ++h->launches;
    }
    if (uo) {
      GatherArgs g = gather_args(h, frames, n);
      g.upd = gfield;
      g.out = h->g_obj;
      g.comp = h->g_obj_c;
      if (waves) {
        g.probe = waves;
        g.probe_stride = pstride;
      }
      timed(h, kKObjMl, [&] { object_tile_kernel<kGatherMl><<<ntiles(h), 1024, 0, h->stream>>>(g); }, n);
      launched(h, "object gradient");
    }
    if (up && h->have_offsets) {
      // DFT(conj(O_win)·g)·exp(+2πi f·d) per frame, summed in frame order
      MoveArgs mb = move_args(h, frames, h->wave2);
      mb.c = gfield;
      check(h, launch_move<kBackSpectrum>(h, mb, n), "probe gradient spectra");
      ++h->launches;
      timed(h, kKProbeFinal, [&] {
        probe_finalize_kernel<<<(pstride + 255) / 256, 256, 0, h->stream>>>(
            h->wave2, n, pstride, nullptr, h->g_probe_spec, h->g_probe_c, 1.f, 2);
      }, n);
      launched(h, "probe gradient sum");
    } else if (up) {
      int nchunk = 0;
      const int chunk = probe_chunk(h, n, &nchunk);
      ProbeArgs pa = {};
      pa.object = h->object;
      pa.quad = h->quad;
      pa.upd = gfield;
      pa.frames = frames;
      pa.corners = h->corners;
      pa.omax = h->omax;
      pa.partial = h->partial;
      pa.nslot = n;
      pa.chunk = chunk;
      pa.nxo = h->nxo;
      pa.K = h->K;
      pa.N = h->N;
      pa.mode = 1;
      dim3 grid((h->N * h->N + 255) / 256, nchunk);
      timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(pa); }, pa.nslot);
      launched(h, "probe gradient");
      const int count = h->K * h->N * h->N;
      timed(h, kKProbeFinal, [&] {
        probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
            h->partial, nchunk, count, nullptr, h->g_probe, h->g_probe_c, 1.f, 2);
      });
      launched(h, "probe gradient sum");
    }
    if (refine || pos_grad) {
      // the moved wave's derivatives from the probe spectra, dotted on chip with the
      // projection's change of the exit wave (refine) or with the gradient field g, whose
      // sums are ∂L/∂d (engine/features.rs:1055-1100)
      MoveArgs md = move_args(h, frames, nullptr);
      md.spec = h->spec;
      md.c = refine ? h->field : gfield;
      md.sums = h->ml_pos_sums;
      check(h, launch_move<kDerivSums>(h, md, n), "position sums");
      ++h->launches;
    }
  }
  if (up && h->have_offsets) {
    // num = conj(q)·IDFT(Σ_f spectra)
    MoveArgs mi = move_args(h, h->iota, h->g_probe);
    mi.spec = h->g_probe_spec;
    check(h, launch_move<kPlainInverse>(h, mi, 1), "probe gradient");
    ++h->launches;
  }
}

// num and den of the Poisson line search along (dir_obj, dir_probe), frames summed in order.
void ml_gamma(ptyb_handle* h, double* num, double* den) {
  const int stack = std::min(h->P, h->stack);
  if (h->have_offsets) spectrum_of(h, h->dir_probe, h->spec_d);
  GammaArgs a = {};
  a.object = h->object;
  a.d_obj = h->dir_obj;
  a.probe = h->probe;
  a.d_probe = h->dir_probe;
  a.quad = h->quad;
  a.tw = h->tw;
  a.iobs = h->iobs;
  a.corners = h->corners;
  a.nyo = h->nyo;
  a.nxo = h->nxo;
  a.nprobe = h->nprobe;
  a.nobj = h->nobj;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    a.frames = h->iota + s0;
    a.out = h->gamma_sums + (size_t)s0 * 2;
    a.psi = h->psi_all + (size_t)s0 * h->K * h->N * h->N;
    a.g = h->g_all + (size_t)s0 * h->K * h->N * h->N;
    if (h->have_offsets) {
      // the probe and its direction, each moved by the frame's offset (engine/ptycho.rs:527-534)
      move_frames(h, a.frames, n, h->spec_d, h->wave2);
      a.probe = h->wave_all + (size_t)s0 * h->K * h->N * h->N;
      a.d_probe = h->wave2;
      a.probe_stride = h->K * h->N * h->N;
    }
    check(h, launch_gamma(h, a, n), "ml line search");
    ++h->launches;
  }
  std::vector<double> v((size_t)h->P * 2);
  check(h, cudaMemcpyAsync(v.data(), h->gamma_sums, v.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream),
        "gamma");
  check(h, cudaStreamSynchronize(h->stream), "gamma");
  *num = *den = 0.0;
  for (int f = 0; f < h->P; ++f) {
    *num += v[(size_t)f * 2];
    *den += v[(size_t)f * 2 + 1];
  }
}

// In-place FFT of n complex doubles, forward, unscaled: radix 2 for a power of 2, else the
// direct sum (sides 96 and 192, host-only work of the phase-ramp removal).
void host_fft(std::vector<double>& re, std::vector<double>& im, size_t off, size_t stride, int n) {
  if (n & (n - 1)) {
    std::vector<double> r(n), i(n);
    for (int k = 0; k < n; ++k) {
      double sr = 0.0, si = 0.0;
      for (int j = 0; j < n; ++j) {
        const double a = -2.0 * M_PI * (double)((long long)j * k % n) / n;
        const double c = std::cos(a), s = std::sin(a);
        const double xr = re[off + j * stride], xi = im[off + j * stride];
        sr += xr * c - xi * s;
        si += xr * s + xi * c;
      }
      r[k] = sr;
      i[k] = si;
    }
    for (int k = 0; k < n; ++k) {
      re[off + k * stride] = r[k];
      im[off + k * stride] = i[k];
    }
    return;
  }
  std::vector<double> r(n), i(n);
  for (int k = 0; k < n; ++k) {
    r[k] = re[off + k * stride];
    i[k] = im[off + k * stride];
  }
  for (int a = 1, j = 0; a < n; ++a) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (a < j) {
      std::swap(r[a], r[j]);
      std::swap(i[a], i[j]);
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    const double ang = -2.0 * M_PI / len;
    for (int s0 = 0; s0 < n; s0 += len)
      for (int k = 0; k < len / 2; ++k) {
        const double wr = std::cos(ang * k), wi = std::sin(ang * k);
        const int u = s0 + k, v = s0 + k + len / 2;
        const double tr = r[v] * wr - i[v] * wi, ti = r[v] * wi + i[v] * wr;
        r[v] = r[u] - tr;
        i[v] = i[u] - ti;
        r[u] += tr;
        i[u] += ti;
      }
  }
  for (int k = 0; k < n; ++k) {
    re[off + k * stride] = r[k];
    im[off + k * stride] = i[k];
  }
}

// PyNX ZeroPhaseRamp (engine/ptycho.rs:1134-1170): the centroid of the probe modes' summed
// far-field intensity on the host, then the probe's and the object's phase ramps on the device.
void zero_phase_ramp(ptyb_handle* h) {
  const int N = h->N;
  const size_t plane = (size_t)N * N;
  std::vector<float2> pr((size_t)h->K * plane);
  check(h, cudaMemcpyAsync(pr.data(), h->probe, pr.size() * sizeof(float2), cudaMemcpyDeviceToHost,
                           h->stream),
        "probe");
  check(h, cudaStreamSynchronize(h->stream), "probe");
  std::vector<double> v(plane, 0.0), re(plane), im(plane);
  for (int m = 0; m < h->K; ++m) {
    // far = FFT of the probe in the shifted layout
    for (int jy = 0; jy < N; ++jy)
      for (int jx = 0; jx < N; ++jx) {
        const float2 p = pr[m * plane + (size_t)((jy + N / 2) % N) * N + (jx + N / 2) % N];
        re[(size_t)jy * N + jx] = p.x;
        im[(size_t)jy * N + jx] = p.y;
      }
    for (int y = 0; y < N; ++y) host_fft(re, im, (size_t)y * N, 1, N);
    for (int x = 0; x < N; ++x) host_fft(re, im, x, N, N);
    // v at natural i = |far[shift(i)]|²
    for (int iy = 0; iy < N; ++iy)
      for (int ix = 0; ix < N; ++ix) {
        const size_t j = (size_t)((iy + N / 2) % N) * N + (ix + N / 2) % N;
        v[(size_t)iy * N + ix] += re[j] * re[j] + im[j] * im[j];
      }
  }
  double w = 0.0, wy = 0.0, wx = 0.0;
  for (size_t i = 0; i < plane; ++i) {
    w += v[i];
    wy += v[i] * (double)(i / N);
    wx += v[i] * (double)(i % N);
  }
  const double dy = wy / w - (double)(N / 2), dx = wx / w - (double)(N / 2);
  const size_t np = (size_t)h->K * plane, no = (size_t)h->nobj * h->nyo * h->nxo;
  timed(h, kKMisc, [&] {
    ramp_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, h->K, N, N, dy, dx, N, N, -1.0);
  });
  launched(h, "probe ramp");
  timed(h, kKMisc, [&] {
    ramp_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->object, h->nobj, h->nyo, h->nxo, dy, dx,
                                                      N, N, 1.0);
  });
  launched(h, "object ramp");
}

// PyNX ScaleObjProbe(absolute=True) without background (engine/ptycho.rs:577-591).
// `waves` (optional): every frame's moved probe of the current probe, scaled along with it.
void split_scale(ptyb_handle* h, double s, float2* waves);

void scale_obj_probe(ptyb_handle* h, float2* waves = nullptr) {
  const ptyb_llk l = llk_pass(h, waves);
  split_scale(h, std::sqrt(h->obs_total / l.nb_photons_calc), waves);
}

// Scales O·P by s and balances Σ|O| and Σ|P| (engine/ptycho.rs:593-603): P *= √(Σ|O|/Σ|P|·s),
// O *= √(Σ|P|/Σ|O|·s); `waves`, every frame's moved probe, scale with the probe.
void split_scale(ptyb_handle* h, double s, float2* waves) {
  const size_t no = (size_t)h->nobj * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  double so[2], sp[2];
  array_sums(h, h->object, nullptr, no, 1, so);
  array_sums(h, h->probe, nullptr, np, 1, sp);
  const double fp = std::sqrt(so[0] / sp[0] * s), fo = std::sqrt(sp[0] / so[0] * s);
  timed(h, kKAxpy, [&] { scale_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, (float)fp, np); });
  launched(h, "scale");
  timed(h, kKAxpy, [&] { scale_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->object, (float)fo, no); });
  launched(h, "scale");
  if (waves) {
    // the moves are linear in the probe: the moved probes scale by the same factor
    const size_t nw = (size_t)h->P * np;
    timed(h, kKAxpy, [&] { scale_kernel<<<blocks_for(nw), 256, 0, h->stream>>>(waves, (float)fp, nw); });
    launched(h, "scale");
  }
}

// AP / DM / RAAR (engine/ptycho.rs:609-754) ---------------------------------------------

// Every frame's carried exit waves (and RAAR's iterate), allocated on first use.
void ensure_carry(ptyb_handle* h, bool iterate) {
  const size_t n = (size_t)h->P * h->K * h->N * h->N;
  if (!h->carry) h->carry = alloc<float2>(h, n);
  if (iterate && !h->carry_it) h->carry_it = alloc<float2>(h, n);
  if (!h->probe_norm) h->probe_norm = alloc<float>(h, (size_t)h->N * h->N);
  if (!h->blend_norm) h->blend_norm = alloc<float>(h, (size_t)h->nyo * h->nxo);
}

// The frame kernel's carry mode over every frame, stack by stack: the carried waves become
// Π(S) + c_refl·(PO − S) with S = c_po·PO + c_psi·carried + c_it·iterate; with `llk`, each
// frame's LLK sums of the field it projects go to h->llk.
void carry_pass(ptyb_handle* h, float c_po, float c_psi, float c_it, float c_refl, bool llk,
                bool iterate, const float2* waves = nullptr) {
  const int stack = std::min(h->P, h->stack);
  const size_t pstride = (size_t)h->K * h->N * h->N;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    FrameArgs a = frame_args(h, h->iota + s0);
    a.carry = h->carry + s0 * pstride;
    a.iter = iterate ? h->carry_it + s0 * pstride : nullptr;
    a.c_po = c_po;
    a.c_psi = c_psi;
    a.c_it = c_it;
    a.c_refl = c_refl;
    a.llk = llk ? h->llk + (size_t)s0 * 4 : nullptr;
    if (waves) {
      // each frame's moved probe in place of P (the position model)
      a.probe = waves + s0 * pstride;
      a.probe_stride = (int)pstride;
    }
    check(h, launch_frame<kCarry>(h, a, n), "carry pass");
    ++h->launches;
  }
}

// psi_to_obj_probe's object blend from the carried waves and the current probe
// (engine/ops.rs:352-381): one tile-owned pass writes the numerator and the norm and takes the
// norm's maximum, then the blend runs per pixel.
void object_blend(ptyb_handle* h, double inertia, const float2* waves = nullptr) {
  GatherArgs g = gather_args(h, h->iota, h->P);
  g.upd = h->carry;
  if (waves) {
    // under the move: num += carried·conj(W), norm += |W|² (engine/features.rs:855-890)
    g.probe = waves;
    g.probe_stride = h->K * h->N * h->N;
  }
  g.pmax = h->scal + kScalObjNorm;
  g.out = h->d_obj;
  g.pre = h->blend_norm;
  check(h, cudaMemsetAsync(g.pmax, 0, sizeof(float), h->stream), "memset");
  timed(h, kKObjBlend, [&] { object_tile_kernel<kGatherBlend><<<ntiles(h), 1024, 0, h->stream>>>(g); }, h->P);
  launched(h, "object blend sums");
  const size_t no = (size_t)h->nyo * h->nxo;
  timed(h, kKAxpy, [&] {
    blend_apply_kernel<<<(unsigned)((no + 255) / 256), 256, 0, h->stream>>>(
        h->object, h->d_obj, h->blend_norm, g.pmax, (float)inertia, no);
  });
  launched(h, "object blend");
}

// The probe blend's chunk sums Σ conj(q·O)·carried and Σ|O|² from the current object; the
// blend itself is probe_blend_finish, so AP's probe sums can read the object before its update.
int probe_blend_sums(ptyb_handle* h, int mode = 2) {
  int nchunk = 0;
  const int chunk = probe_chunk(h, h->P, &nchunk);
  const int plane = h->N * h->N;
  if (nchunk > h->max_den_chunks) {
    h->partial_den = alloc<float>(h, (size_t)nchunk * plane);
    h->max_den_chunks = nchunk;
  }
  ProbeArgs p = {};
  p.object = h->object;
  p.quad = h->quad;
  p.upd = h->carry;
  p.frames = h->iota;
  p.corners = h->corners;
  p.partial = h->partial;
  p.partial_den = h->partial_den;
  p.nslot = h->P;
  p.chunk = chunk;
  p.nxo = h->nxo;
  p.K = h->K;
  p.N = h->N;
  p.mode = mode;
  dim3 grid((plane + 255) / 256, nchunk);
  timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(p); }, h->P);
  launched(h, "probe partial");
  return nchunk;
}

void probe_blend_finish(ptyb_handle* h, int nchunk, double inertia) {
  const int plane = h->N * h->N, count = h->K * plane;
  float* nmax = h->scal + kScalProbeNorm;
  check(h, cudaMemsetAsync(nmax, 0, sizeof(float), h->stream), "memset");
  timed(h, kKProbeFinal, [&] {
    probe_norm_kernel<<<(plane + 255) / 256, 256, 0, h->stream>>>(h->partial_den, nchunk, plane,
                                                                  h->probe_norm, nmax);
  });
  launched(h, "probe norm");
  timed(h, kKProbeFinal, [&] {
    probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
        h->partial, nchunk, count, h->probe, nullptr, nullptr, (float)inertia, 3, h->probe_norm,
        nmax, plane);
  });
  launched(h, "probe blend");
}

// Every frame's moved probe of the current probe and offsets into h->wave_all, and the
// probe's spectrum DFT(q·P) into h->spec.
void move_all_frames(ptyb_handle* h) {
  spectrum_of(h, h->probe, h->spec);
  const int stack = std::min(h->P, h->stack);
  for (int s0 = 0; s0 < h->P; s0 += stack)
    move_frames(h, h->iota + s0, std::min(stack, h->P - s0), h->spec,
                h->wave_all + (size_t)s0 * h->K * h->N * h->N);
}

// Under the position model, the buffers of AP / DM / RAAR: the moved probes, the spectra, a
// stack of planes, the position sums and the probe step's.
void ensure_carry_moves(ptyb_handle* h) {
  const size_t np = (size_t)h->K * h->N * h->N;
  ensure_spec(h);
  if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * np);
  if (h->wave2_slots < h->slots) {
    h->wave2 = alloc<float2>(h, (size_t)h->slots * np);
    h->wave2_slots = h->slots;
  }
  if (!h->ml_pos_sums) h->ml_pos_sums = alloc<double>(h, (size_t)h->P * 4);
  if (!h->pcg_g) {
    h->pcg_g = alloc<float2>(h, np);
    h->pcg_step = alloc<float2>(h, np);
    h->pcg_spec = alloc<float2>(h, np);
    h->pcg_comp = alloc<float2>(h, np);
    h->pcg_norms = alloc<double>(h, (size_t)h->P * h->K);
    h->pcg_modes = alloc<double>(h, (size_t)h->K * 2);
  }
}

// The position sums of the carried waves against the model of the current object and moved
// probes (engine/features.rs:992-1025) into h->ml_pos_sums; h->spec must be the probe's.
void carried_position_sums(ptyb_handle* h) {
  const int stack = std::min(h->P, h->stack);
  const size_t pstride = (size_t)h->K * h->N * h->N;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    MoveArgs md = move_args(h, h->iota + s0, nullptr);
    md.spec = h->spec;
    md.c = h->carry + s0 * pstride;
    md.minus = h->wave_all + s0 * pstride;
    md.sums = h->ml_pos_sums;
    check(h, launch_move<kDerivSums>(h, md, n), "position sums");
    ++h->launches;
  }
}

// The probe's update under the move (engine/features.rs:673-712), from the current object and
// the moved probes in h->wave_all: g = A^H(carried − A·P) through the move's adjoint, frame by
// frame; per mode the step s = g / (Σ|O|² + reg) and α = <g, s> / (‖A·s‖² + reg·‖s‖²) where
// <g, s> > 0; P += α·s.
void probe_pcg_step(ptyb_handle* h, double inertia) {
  const int stack = std::min(h->P, h->stack);
  const int plane = h->N * h->N, K = h->K;
  const size_t pstride = (size_t)K * plane;
  check(h, cudaMemsetAsync(h->pcg_spec, 0, pstride * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->pcg_comp, 0, pstride * sizeof(float2), h->stream), "memset");
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    MoveArgs mb = move_args(h, h->iota + s0, h->wave2);
    mb.c = h->carry + s0 * pstride;
    mb.minus = h->wave_all + s0 * pstride;
    check(h, launch_move<kBackSpectrum>(h, mb, n), "probe residual spectra");
    ++h->launches;
    timed(h, kKProbeFinal, [&] {
      probe_finalize_kernel<<<((int)pstride + 255) / 256, 256, 0, h->stream>>>(
          h->wave2, n, (int)pstride, nullptr, h->pcg_spec, h->pcg_comp, 1.f, 2);
    }, n);
    launched(h, "probe residual sum");
  }
  MoveArgs mi = move_args(h, h->iota, h->pcg_g);
  mi.spec = h->pcg_spec;
  check(h, launch_move<kPlainInverse>(h, mi, 1), "probe residual");
  ++h->launches;
  // Σ|O|² per probe pixel and its maximum
  const int nchunk = probe_blend_sums(h, 3);
  float* nmax = h->scal + kScalProbeNorm;
  check(h, cudaMemsetAsync(nmax, 0, sizeof(float), h->stream), "memset");
  timed(h, kKProbeFinal, [&] {
    probe_norm_kernel<<<(plane + 255) / 256, 256, 0, h->stream>>>(h->partial_den, nchunk, plane,
                                                                  h->probe_norm, nmax);
  });
  launched(h, "probe norm");
  timed(h, kKProbeFinal, [&] {
    probe_pcg_step_kernel<<<K, 1024, 0, h->stream>>>(h->pcg_g, h->probe_norm, nmax,
                                                     (float)inertia, plane, h->pcg_step,
                                                     h->pcg_modes);
  });
  launched(h, "probe step");
  // ‖A·s‖²: the step moved for every frame, weighted by |O|²
  spectrum_of(h, h->pcg_step, h->spec_d);
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    move_frames(h, h->iota + s0, n, h->spec_d, h->wave2);
    timed(h, kKMisc, [&] {
      weighted_norm_kernel<<<dim3(n, K), 256, 0, h->stream>>>(h->wave2, h->object, h->iota + s0,
                                                              h->corners, h->nxo, h->N, K,
                                                              h->pcg_norms + (size_t)s0 * K);
    }, n);
    launched(h, "step norms");
  }
  std::vector<double> modes((size_t)K * 2), norms((size_t)h->P * K);
  check(h, cudaMemcpyAsync(modes.data(), h->pcg_modes, modes.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream),
        "step sums");
  check(h, cudaMemcpyAsync(norms.data(), h->pcg_norms, norms.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream),
        "step sums");
  check(h, cudaStreamSynchronize(h->stream), "step sums");
  ModeCoefs alpha = {};
  for (int m = 0; m < K; ++m) {
    double curv = modes[2 * m + 1];
    for (int f = 0; f < h->P; ++f) curv += norms[(size_t)f * K + m];
    const double slope = modes[2 * m];
    alpha.c[m] = slope > 0.0 ? (float)(slope / curv) : 0.f;
  }
  timed(h, kKAxpy, [&] {
    probe_modes_axpy_kernel<<<((int)pstride + 255) / 256, 256, 0, h->stream>>>(
        h->probe, h->pcg_step, alpha, plane, (int)pstride);
  });
  launched(h, "probe step");
}

// DM's and RAAR's update (engine/ptycho.rs:732-754): `loops` times an object-only then a
// probe-only update, the probe's from the new object; under the position model each from the
// current probe's moves (recomputed after a probe step), the probe's by the step of
// probe_pcg_step, and the position sums come first, from the waves the cycle starts with.
void update_obj_probe(ptyb_handle* h, bool uo, double oi, bool up, double pi, int loops) {
  if (h->have_offsets) {
    bool fresh = true;  // h->wave_all holds the current probe's moves
    for (int l = 0; l < loops; ++l) {
      if (uo) {
        if (!fresh) move_all_frames(h);
        fresh = true;
        object_blend(h, oi, h->wave_all);
      }
      if (up) {
        if (!fresh) move_all_frames(h);
        probe_pcg_step(h, pi);
        fresh = false;
      }
    }
    return;
  }
  for (int l = 0; l < loops; ++l) {
    if (uo) object_blend(h, oi);
    if (up) probe_blend_finish(h, probe_blend_sums(h), pi);
  }
}

// AP, DM and RAAR run on a single-slice object.
int carried_refusal(ptyb_handle* h, int32_t ncycle, const char* what) {
  if (ncycle < 0) {
    h->err = "ncycle must be >= 0";
    return PTYB_INVALID;
  }
  if (h->nslice > 1) {
    h->err = std::string(what) + " runs on a single-slice object";
    return PTYB_INVALID;
  }
  return PTYB_OK;
}

template <typename F>
int guarded(ptyb_handle* h, bool enqueues, F&& body) {
  if (!h) return PTYB_INVALID;
  if (enqueues && h->aborted) {
    h->err = "an earlier call failed part-way; the state is poisoned";
    return PTYB_ABORTED;
  }
  try {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) {
      h->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
      if (enqueues) h->aborted = true;
      return PTYB_GPU;
    }
    return body();
  } catch (const Fail& f) {
    return f.code;
  } catch (const std::exception& ex) {
    // a host failure (out of host memory and the like) must not cross the C ABI
    h->err = std::string("host: ") + ex.what();
    if (enqueues) h->aborted = true;
    return PTYB_GPU;
  }
}

// DM (RAAR when `raar`) cycles (engine/ptycho.rs:653-730): the LLK of the estimate the cycle
// starts from when due, the mix and projection of the carried waves, the updates, and after a
// recorded cycle the balance of Σ|O| and Σ|P|.
int carried_cycles(ptyb_handle* h, bool raar, double mix, bool uo, double oi, bool up, double pi,
                   int loops, int calc_llk, bool ramp, int32_t ncycle) {
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_carry(h, raar);
    const bool moves = h->have_offsets, refine = moves && h->refine_offsets;
    if (moves) ensure_carry_moves(h);
    const float2* waves = moves ? h->wave_all : nullptr;
    begin_call(h);
    for (int ic = 0; ic < ncycle; ++ic) {
      const bool due = llk_due(calc_llk, ic, ncycle);
      if (moves) move_all_frames(h);
      ptyb_llk l = {};
      if (due) l = llk_pass(h, waves);
      if (ic == 0) {
        carry_pass(h, 1.f, 0.f, 0.f, 0.f, false, raar, waves);
      } else if (raar) {
        // psi ← (1 − b/2)·psi + (b/2)·(2·PO − it), the next iterate, then Π
        const double hb = 0.5 * mix;
        carry_pass(h, (float)(2.0 * hb), (float)(1.0 - hb), (float)(-hb), 0.f, false, true,
                   waves);
      } else {
        // refl = (2 − a)·PO − (1 − a)·psi; psi ← Π(refl) + (1 − a)·(PO − refl)
        carry_pass(h, (float)(2.0 - mix), (float)(-(1.0 - mix)), 0.f, (float)(1.0 - mix), false,
                   false, waves);
      }
      if (refine) carried_position_sums(h);
      update_obj_probe(h, uo, oi, up, pi, loops);
      if (refine) {
        timed(h, kKSolve, [&] {
          ml_position_step_kernel<<<1, 1024, 0, h->stream>>>(h->ml_pos_sums, h->P, h->offsets);
        });
        launched(h, "position step");
      }
      if (due) {
        record(h, raar ? kAlgRaar : kAlgDm, l);
        split_scale(h, 1.0, nullptr);
      }
      ++h->cycle;
    }
    if (ramp) zero_phase_ramp(h);
    end_call(h, raar ? "raar" : "dm");
    return PTYB_OK;
  });
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// A handle over `nslice` object slices (each one object mode) with the angular-spectrum gaps
// `gaps` (metres) between them; one slice is the plain object of ptyb_create.
int create_handle(const ptyb_scan* scan, const double* object, int32_t nobj, int32_t nslice,
                  const double* gaps, int32_t nyo, int32_t nxo, const double* probe,
                  int32_t nprobe, const ptyb_options* options, ptyb_handle** out) {
  if (!out) return PTYB_INVALID;
  *out = nullptr;
  if (!scan || !object || !probe || !scan->counts || !scan->pos_y || !scan->pos_x)
    return PTYB_INVALID;
  const int N = scan->ny;
  g_create_error.clear();
  if (nslice < 1 || nslice > kMaxSlices || (nslice > 1 && !gaps)) {
    g_create_error = "need 1 to " + std::to_string(kMaxSlices) + " slices and their gaps";
    return PTYB_INVALID;
  }
  for (int s = 0; s + 1 < nslice; ++s)
    if (!std::isfinite(gaps[s])) {
      g_create_error = "slice gaps must be finite";
      return PTYB_INVALID;
    }
  if (scan->nx != N || !(N == 64 || N == 96 || N == 128 || N == 192 || N == 256)) {
    g_create_error = "frames must be square with a side of 64, 96, 128, 192 or 256";
    return PTYB_INVALID;
  }
  if (scan->nframe <= 0 || nprobe <= 0 || nprobe > kMaxModes || nobj != 1 || nyo < N || nxo < N) {
    g_create_error = "need frames, 1-4 probe modes, one object mode and an object >= the frame";
    return PTYB_INVALID;
  }
  if (!(scan->wavelength > 0 && scan->distance > 0 && scan->detector_pixel > 0)) {
    g_create_error = "wavelength, distance and detector pixel must be > 0";
    return PTYB_INVALID;
  }
  const int K = nprobe * nobj;
  const int C = cluster_for(N, K, options ? options->cluster : 0);
  if (C == 0) {
    g_create_error = "the frame's modes do not fit one cluster's shared memory";
    return PTYB_INVALID;
  }
  auto* h = new ptyb_handle();
  h->device = options ? options->device : 0;
  h->P = scan->nframe;
  h->N = N;
  h->nprobe = nprobe;
  h->nobj = nobj;
  h->K = K;
  h->nyo = nyo;
  h->nxo = nxo;
  h->C = C;
  // The position sums reduce over the whole cluster twice per frame: at side 256 they run on
  // clusters of 8 (measured faster than 16), whatever cluster the frame kernels take.
  h->C_sums = C;
  if (N == 256 && frame_smem_bytes<256, 8>(K) <= 227 * 1024) h->C_sums = 8;
  h->stack = options && options->stack_size > 0 ? options->stack_size : 512;
  h->nslice = nslice;
  h->log_stride = 2 + nslice;
  // Positions: PyNX preprocessing and window corners (base/positions.rs, base/addr.rs).
  const double lz = scan->wavelength * scan->distance;
  h->pixel[0] = lz / (N * scan->detector_pixel);
  h->pixel[1] = lz / (N * scan->detector_pixel);
  std::vector<double> y(scan->pos_y, scan->pos_y + h->P), x(scan->pos_x, scan->pos_x + h->P);
  for (int f = 0; f < h->P; ++f)
    if (!std::isfinite(y[f]) || !std::isfinite(x[f]) || std::fabs(y[f]) > 1e10 ||
        std::fabs(x[f]) > 1e10) {
      g_create_error = "positions must be finite with |pos| <= 1e10";
      delete h;
      return PTYB_INVALID;
    }
  const std::vector<double> py = pynx_axis(y, h->pixel[0]), px = pynx_axis(x, h->pixel[1]);
  if (!corners_of(py, px, h->pixel, N, N, nyo, nxo, &h->corners_h, &g_create_error)) {
    delete h;
    return PTYB_INVALID;
  }
  int rc = guarded(h, true, [&]() -> int {
    check(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    // Observed intensities in the FFT-shifted layout (engine/obs.rs:61-76), converted on the
    // device from the raw counts.
    const size_t plane = (size_t)N * N, nval = (size_t)h->P * plane;
    const size_t esize = scan->counts_kind == PTYB_COUNTS_U16   ? 2
                         : scan->counts_kind == PTYB_COUNTS_F32 ? 4
                                                                : 8;
    h->iobs = alloc<float>(h, nval);
    void* raw = nullptr;
    check(h, pool_alloc(h, &raw, nval * esize), "cudaMallocAsync");
    double* power = alloc<double>(h, h->P);
    int* nobs = alloc<int>(h, h->P + 1);
    check(h, fill_sync(h, nobs, 0, (h->P + 1) * sizeof(int)), "memset");
    cudaError_t e = copy_sync(h, raw, scan->counts, nval * esize, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      if (scan->counts_kind == PTYB_COUNTS_U16)
        counts_kernel<<<h->P, 256, 0, h->stream>>>(static_cast<const uint16_t*>(raw), 1, h->iobs,
                                                   power, nobs, nobs + h->P, N);
      else if (scan->counts_kind == PTYB_COUNTS_F32)
        counts_kernel<<<h->P, 256, 0, h->stream>>>(static_cast<const float*>(raw), 0, h->iobs,
                                                   power, nobs, nobs + h->P, N);
      else
        counts_kernel<<<h->P, 256, 0, h->stream>>>(static_cast<const double*>(raw), 0, h->iobs,
                                                   power, nobs, nobs + h->P, N);
      e = cudaGetLastError();
      ++h->launches;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFreeAsync(raw, h->stream);
    check(h, e, "counts upload");
    std::vector<double> pw(h->P);
    std::vector<int> nb(h->P + 1);
    check(h, copy_sync(h, pw.data(), power, h->P * sizeof(double), cudaMemcpyDeviceToHost), "counts");
    check(h, copy_sync(h, nb.data(), nobs, (h->P + 1) * sizeof(int), cudaMemcpyDeviceToHost), "counts");
    if (nb[h->P]) {
      h->err = "counts must be finite";
      return PTYB_INVALID;
    }
    for (int f = 0; f < h->P; ++f) {
      h->obs_total += pw[f];
      h->max_power = std::max(h->max_power, pw[f]);
      h->nb_obs += nb[f];
    }
    h->corners = alloc<int2>(h, h->P);
    check(h, copy_sync(h, h->corners, h->corners_h.data(), h->P * sizeof(int2), cudaMemcpyHostToDevice),
          "corners upload");
    h->object = alloc<float2>(h, (size_t)nslice * nobj * nyo * nxo);
    upload_c64(h, object, h->object, (size_t)nslice * nobj * nyo * nxo, "object upload");
    h->probe = alloc<float2>(h, (size_t)nprobe * plane);
    upload_c64(h, probe, h->probe, (size_t)nprobe * plane, "probe upload");
    // Far-field plane phase (engine/ops.rs:17-33) and the FFT twiddles, in double.
    std::vector<float2> q(plane), tw(N);
    const double fq = M_PI / (scan->wavelength * scan->distance);
    for (int yy = 0; yy < N; ++yy)
      for (int xx = 0; xx < N; ++xx) {
        const double dy = (double)yy - (double)(N / 2), dx = (double)xx - (double)(N / 2);
        const double ph =
            fq * (dx * dx * h->pixel[1] * h->pixel[1] + dy * dy * h->pixel[0] * h->pixel[0]);
        q[(size_t)yy * N + xx] = make_float2((float)std::cos(ph), (float)std::sin(ph));
      }
    for (int t = 0; t < N; ++t)
      tw[t] = make_float2((float)std::cos(2.0 * M_PI * t / N), (float)-std::sin(2.0 * M_PI * t / N));
    h->quad = alloc<float2>(h, plane);
    check(h, copy_sync(h, h->quad, q.data(), plane * sizeof(float2), cudaMemcpyHostToDevice), "quad");
    h->tw = alloc<float2>(h, N);
    check(h, copy_sync(h, h->tw, tw.data(), N * sizeof(float2), cudaMemcpyHostToDevice), "tw");
    std::vector<int> iota(h->P);
    for (int f = 0; f < h->P; ++f) iota[f] = f;
    h->iota = alloc<int>(h, h->P);
    check(h, copy_sync(h, h->iota, iota.data(), h->P * sizeof(int), cudaMemcpyHostToDevice), "iota");
    h->order = alloc<int>(h, h->P);
    h->afar_all = alloc<float>(h, h->P);
    h->llk = alloc<double>(h, (size_t)h->P * 4);
    h->scal = alloc<float>(h, kScalars);
    h->pre = alloc<float>(h, (size_t)nyo * nxo);
    h->d_obj = alloc<float2>(h, (size_t)nslice * nyo * nxo);
    h->d_probe = alloc<float2>(h, (size_t)K * plane);
    h->steplog = alloc<double>(h, (size_t)h->P * h->log_stride);
    check(h, fill_sync(h, h->scal, 0, kScalars * sizeof(float)), "memset");
    if (nslice > 1) {
      // Angular-spectrum transfer functions exp(2πi z √(1 − r)) of the gaps in DFT order, 0 on
      // the evanescent band (engine/propagate.rs:505-531), in double; the plane of ones is the
      // phase of every slice but the last.
      const double width = h->pixel[1] / scan->wavelength, ar = h->pixel[1] / h->pixel[0];
      std::vector<float2> t((size_t)(nslice - 1) * plane), ones(plane, make_float2(1.f, 0.f));
      for (int g = 0; g + 1 < nslice; ++g) {
        const double i2piz = 2.0 * M_PI * (gaps[g] / scan->wavelength);
        for (int yy = 0; yy < N; ++yy)
          for (int xx = 0; xx < N; ++xx) {
            const double fy = (double)(yy < N / 2 ? yy : yy - N) / N;
            const double fx = (double)(xx < N / 2 ? xx : xx - N) / N;
            const double ratio = (fx * fx + (ar * fy) * (ar * fy)) / (width * width);
            float2 v = make_float2(0.f, 0.f);
            if (ratio < 1.0) {
              const double ph = i2piz * std::sqrt(1.0 - ratio);
              v = make_float2((float)std::cos(ph), (float)std::sin(ph));
            }
            t[(size_t)g * plane + (size_t)yy * N + xx] = v;
          }
      }
      h->tf = alloc<float2>(h, t.size());
      check(h, copy_sync(h, h->tf, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice), "tf");
      h->ones = alloc<float2>(h, plane);
      check(h, copy_sync(h, h->ones, ones.data(), plane * sizeof(float2), cudaMemcpyHostToDevice),
            "ones");
    }
    return PTYB_OK;
  });
  if (rc != PTYB_OK) {
    g_create_error = h->err;
    ptyb_destroy(h);
    return rc;
  }
  *out = h;
  return PTYB_OK;
}

}  // namespace

extern "C" {

int ptyb_create(const ptyb_scan* scan, const double* object, int32_t nobj, int32_t nyo,
                int32_t nxo, const double* probe, int32_t nprobe, const ptyb_options* options,
                ptyb_handle** out) {
  try {
    return create_handle(scan, object, nobj, 1, nullptr, nyo, nxo, probe, nprobe, options, out);
  } catch (const std::exception& ex) {
    // host failures (out of host memory and the like) stop here, as a status and message
    g_create_error = std::string("host: ") + ex.what();
    if (out) *out = nullptr;
    return PTYB_GPU;
  }
}

int ptyb_create_slices(const ptyb_scan* scan, const double* objects, int32_t nslice,
                       const double* gaps, int32_t nyo, int32_t nxo, const double* probe,
                       int32_t nprobe, const ptyb_options* options, ptyb_handle** out) {
  try {
    return create_handle(scan, objects, 1, nslice, gaps, nyo, nxo, probe, nprobe, options, out);
  } catch (const std::exception& ex) {
    g_create_error = std::string("host: ") + ex.what();
    if (out) *out = nullptr;
    return PTYB_GPU;
  }
}

int ptyb_nslice(const ptyb_handle* h) { return h ? h->nslice : 0; }

int ptyb_lsqml_slice_steps(ptyb_handle* h, double* dst) {
  if (!h || !dst) return PTYB_INVALID;
  std::copy(h->slice_steps.begin(), h->slice_steps.end(), dst);
  return PTYB_OK;
}

int ptyb_rpie(ptyb_handle* h, const ptyb_rpie_params* p, int32_t nepoch) {
  if (!h || !p) return PTYB_INVALID;
  if (p->batch_size <= 0 || nepoch < 0) {
    h->err = "rPIE batch_size must be >= 1";
    return PTYB_INVALID;
  }
  if (h->nobj != 1) {
    h->err = "rPIE needs exactly one object mode";
    return PTYB_INVALID;
  }
  if (h->nslice > 1) {
    h->err = "rPIE runs on a single-slice object";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const int bs = std::min(p->batch_size, h->P);
    ensure_slots(h, std::max(bs, std::min(h->P, h->stack)));
    std::vector<std::vector<int32_t>> sizes;
    upload_orders(h, nepoch, p->batch_size, p->seed, h->cycle, &sizes, nullptr);
    begin_call(h);
    for (int ic = 0; ic < nepoch; ++ic) {
      const int* order = h->order_all + (size_t)ic * h->P;
      int off = 0;
      for (int n : sizes[ic]) {
        rpie_batch(h, *p, order + off, n);
        off += n;
      }
      if (llk_due(p->calc_llk, ic, nepoch)) record(h, kAlgRpie, llk_pass(h));
      ++h->cycle;
    }
    end_call(h, "rpie");
    return PTYB_OK;
  });
}

int ptyb_lsqml(ptyb_handle* h, const ptyb_lsqml_params* p, int32_t nepoch, int32_t calc_llk) {
  if (!h || !p) return PTYB_INVALID;
  if (p->batch_size <= 0 || nepoch < 0 ||
      !(p->cost == PTYB_COST_POISSON || p->cost == PTYB_COST_AMPLITUDE)) {
    h->err = "LSQML batch_size must be >= 1 and cost poisson or amplitude";
    return PTYB_INVALID;
  }
  if (std::min(p->batch_size, h->P) > 1024) {
    h->err = "LSQML batches of more than 1024 frames are not supported";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const int size = std::min(p->batch_size, h->P);
    ensure_slots(h, std::max(size, std::min(h->P, h->stack)));
    if (h->opr_on) ensure_opr(h);
    std::vector<std::vector<int32_t>> sizes;
    std::vector<int32_t> last;
    // A fresh run: epochs from 0 (engine/gpu/lsqml.rs:97-105).
    upload_orders(h, nepoch, size, p->seed, 0, &sizes, &last);
    begin_call(h);
    timed(h, kKMisc, [&] {
      fill_kernel<<<(h->P + 255) / 256, 256, 0, h->stream>>>(h->afar_all, 0.5f, h->P);
    });
    launched(h, "a_far");
    for (int ic = 0; ic < nepoch; ++ic) {
      if (ic < 10 || ic % 10 == 0) lsqml_preconditioner(h, ic == 0);
      const int* order = h->order_all + (size_t)ic * h->P;
      int off = 0;
      const int stride = h->log_stride;
      for (int n : sizes[ic]) {
        if (h->nslice > 1)
          lsqml_batch_slices(h, *p, order + off, n, h->steplog + (size_t)off * stride, stride);
        else
          lsqml_batch(h, *p, order + off, n, h->steplog + (size_t)off * stride);
        off += n;
      }
      if (llk_due(calc_llk, ic, nepoch)) {
        if (h->opr_on) {
          // the LLK of every frame's own probe (engine/lsqml.rs:537-551)
          const int stack = std::min(h->P, h->stack);
          for (int s0 = 0; s0 < h->P; s0 += stack)
            opr_planes(h, h->iota + s0, std::min(stack, h->P - s0),
                       h->wave_all + (size_t)s0 * h->K * h->N * h->N);
          record(h, kAlgLsqml, llk_pass(h, h->wave_all));
        } else {
          record(h, kAlgLsqml, llk_pass(h));
        }
      }
      ++h->cycle;
    }
    end_call(h, "lsqml");
    // The last epoch's steps, for `ptyb_lsqml_steps`.
    h->steps.clear();
    h->slice_steps.clear();
    if (nepoch > 0) {
      const int stride = h->log_stride;
      std::vector<double> log((size_t)h->P * stride);
      check(h, copy_sync(h, log.data(), h->steplog, log.size() * sizeof(double),
                          cudaMemcpyDeviceToHost),
            "steps");
      int b = 0, o = 0;
      for (int n : sizes.back()) {
        for (int i = 0; i < n; ++i) {
          const double* row = log.data() + (size_t)(o + i) * stride;
          ptyb_lsqml_step st;
          st.batch = b;
          st.frame = last[o + i];
          st.a_far = row[0];
          st.a_obj = row[1];
          st.a_probe = row[2];
          h->steps.push_back(st);
          for (int sl = 1; sl < h->nslice; ++sl) h->slice_steps.push_back(row[2 + sl]);
        }
        o += n;
        ++b;
      }
    }
    return PTYB_OK;
  });
}

int ptyb_ml(ptyb_handle* h, const ptyb_ml_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (ncycle < 0) {
    h->err = "ncycle must be >= 0";
    return PTYB_INVALID;
  }
  if (h->nslice > 1) {
    h->err = "ML runs on a single-slice object";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_ml(h);
    const bool refine = h->have_offsets && h->refine_offsets;
    if (h->have_offsets && h->wave2_slots < h->slots) {
      h->wave2 = alloc<float2>(h, (size_t)h->slots * h->K * h->N * h->N);
      h->wave2_slots = h->slots;
    }
    if (refine && !h->ml_pos_sums) h->ml_pos_sums = alloc<double>(h, (size_t)h->P * 4);
    if (h->have_offsets) {
      ensure_spec(h);
      if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * h->K * h->N * h->N);
    }
    const bool uo = p->update_object != 0, up = p->update_probe != 0;
    const size_t no = (size_t)h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
    begin_call(h);
    auto move_all = [&] {
      // every frame's moved probe of the current probe, from its spectra
      spectrum_of(h, h->probe, h->spec);
      const int stack = std::min(h->P, h->stack);
      for (int s0 = 0; s0 < h->P; s0 += stack)
        move_frames(h, h->iota + s0, std::min(stack, h->P - s0), h->spec,
                    h->wave_all + (size_t)s0 * h->K * h->N * h->N);
    };
    if (h->have_offsets) move_all();
    // the opening rescale's LLK reads the moved probes, which it scales with the probe
    scale_obj_probe(h, h->have_offsets ? h->wave_all : nullptr);
    check(h, cudaMemsetAsync(h->dir_obj, 0, no * sizeof(float2), h->stream), "memset");
    check(h, cudaMemsetAsync(h->dir_probe, 0, np * sizeof(float2), h->stream), "memset");
    bool have_last = false;
    for (int ic = 0; ic < ncycle; ++ic) {
      const bool due = llk_due(p->calc_llk, ic, ncycle);
      if (h->have_offsets) {
        if (ic == 0)
          spectrum_of(h, h->probe, h->spec);  // the moved probes were scaled above
        else
          move_all();
      }
      ptyb_llk l = {};
      if (due) l = llk_pass(h, h->have_offsets ? h->wave_all : nullptr);
      ml_gradients(h, uo, up, refine);
      double beta = 0.0;
      if (have_last) {
        double a[2], b[2];
        array_sums(h, h->g_obj, h->last_obj, no, 0, a);
        array_sums(h, h->g_probe, h->last_probe, np, 0, b);
        beta = (a[0] + b[0]) / (a[1] + b[1]);
        if (!(std::isfinite(beta) && beta >= 0.0)) beta = 0.0;
      }
      timed(h, kKAxpy, [&] {
        cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_obj, h->g_obj, (float)beta, no);
      });
      launched(h, "direction");
      timed(h, kKAxpy, [&] {
        cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->g_probe, (float)beta, np);
      });
      launched(h, "direction");
      double num = 0.0, den = 0.0;
      ml_gamma(h, &num, &den);
      const double gamma = num / den;
      if (std::isfinite(gamma)) {
        timed(h, kKAxpy, [&] {
          axpy_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->object, h->dir_obj, (float)gamma, no);
        });
        launched(h, "step");
        timed(h, kKAxpy, [&] {
          axpy_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, h->dir_probe, (float)gamma, np);
        });
        launched(h, "step");
      } else {
        // No update; the direction restarts from the gradient.
        timed(h, kKAxpy, [&] {
          cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_obj, h->g_obj, 0.f, no);
        });
        launched(h, "direction");
        timed(h, kKAxpy, [&] {
          cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->g_probe, 0.f, np);
        });
        launched(h, "direction");
      }
      std::swap(h->g_obj, h->last_obj);
      std::swap(h->g_probe, h->last_probe);
      have_last = true;
      if (refine) {
        timed(h, kKSolve, [&] {
          ml_position_step_kernel<<<1, 1024, 0, h->stream>>>(h->ml_pos_sums, h->P, h->offsets);
        });
        launched(h, "position step");
      }
      if (due) record(h, kAlgMl, l);
      ++h->cycle;
    }
    if (p->zero_phase_ramp) zero_phase_ramp(h);
    end_call(h, "ml");
    return PTYB_OK;
  });
}

int ptyb_ap(ptyb_handle* h, const ptyb_ap_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (const int e = carried_refusal(h, ncycle, "AP")) return e;
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_carry(h, false);
    const bool uo = p->update_object != 0, up = p->update_probe != 0;
    const bool moves = h->have_offsets, refine = moves && h->refine_offsets;
    if (moves) ensure_carry_moves(h);
    begin_call(h);
    for (int ic = 0; ic < ncycle; ++ic) {
      // the LLK of the estimate comes from the field the projection reads
      const bool due = llk_due(p->calc_llk, ic, ncycle);
      if (moves) move_all_frames(h);
      carry_pass(h, 1.f, 0.f, 0.f, 0.f, due, false, moves ? h->wave_all : nullptr);
      ptyb_llk l = {};
      if (due) l = llk_of_frames(h);
      if (moves) {
        // under the move (engine/ptycho.rs:627-636): the position sums against the arrays the
        // projection read, the probe's step from the old object, the object's blend under the
        // old probe's moves, then the position step
        if (refine) carried_position_sums(h);
        if (up) probe_pcg_step(h, p->probe_inertia);
        if (uo) object_blend(h, p->obj_inertia, h->wave_all);
        if (refine) {
          timed(h, kKSolve, [&] {
            ml_position_step_kernel<<<1, 1024, 0, h->stream>>>(h->ml_pos_sums, h->P, h->offsets);
          });
          launched(h, "position step");
        }
      } else {
        // both updates from the old arrays: the probe's sums read the object before its blend
        const int nchunk = up ? probe_blend_sums(h) : 0;
        if (uo) object_blend(h, p->obj_inertia);
        if (up) probe_blend_finish(h, nchunk, p->probe_inertia);
      }
      if (due) record(h, kAlgAp, l);
      ++h->cycle;
    }
    if (p->zero_phase_ramp) zero_phase_ramp(h);
    end_call(h, "ap");
    return PTYB_OK;
  });
}

int ptyb_dm(ptyb_handle* h, const ptyb_dm_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (const int e = carried_refusal(h, ncycle, "DM")) return e;
  if (p->loop_obj_probe < 0) {
    h->err = "loop_obj_probe must be >= 0";
    return PTYB_INVALID;
  }
  return carried_cycles(h, false, p->alpha, p->update_object != 0, p->obj_inertia,
                        p->update_probe != 0, p->probe_inertia, p->loop_obj_probe, p->calc_llk,
                        p->zero_phase_ramp != 0, ncycle);
}

int ptyb_raar(ptyb_handle* h, const ptyb_raar_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (const int e = carried_refusal(h, ncycle, "RAAR")) return e;
  if (p->loop_obj_probe < 0) {
    h->err = "loop_obj_probe must be >= 0";
    return PTYB_INVALID;
  }
  return carried_cycles(h, true, p->beta, p->update_object != 0, p->obj_inertia,
                        p->update_probe != 0, p->probe_inertia, p->loop_obj_probe, p->calc_llk,
                        p->zero_phase_ramp != 0, ncycle);
}

namespace {

int batch_run_impl(ptyb_handle* const* handles, int32_t n, const ptyb_rpie_params* rpie,
                   int32_t rpie_epochs, const ptyb_lsqml_params* lsqml, int32_t lsqml_epochs,
                   int32_t calc_llk, int32_t* status, float* device_ms) {
  if (device_ms) *device_ms = -1.f;
  if (!handles || n <= 0 || rpie_epochs < 0 || lsqml_epochs < 0 || (rpie_epochs > 0 && !rpie) ||
      (lsqml_epochs > 0 && !lsqml))
    return PTYB_INVALID;
  std::set<ptyb_handle*> seen;
  for (int i = 0; i < n; ++i)
    if (!handles[i] || !seen.insert(handles[i]).second) return PTYB_INVALID;
  // The batch's device time: every handle's stream waits on a start event recorded on a stream
  // of the batch's own, and that stream waits on every handle's last work before the end event
  // (handles on the first handle's device; the others are not timed).
  const int dev = handles[0]->device;
  cudaStream_t ts = nullptr;
  cudaEvent_t start = nullptr, end = nullptr;
  bool timing = cudaSetDevice(dev) == cudaSuccess &&
                cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreate(&start) == cudaSuccess && cudaEventCreate(&end) == cudaSuccess &&
                cudaEventRecord(start, ts) == cudaSuccess;
  for (int i = 0; i < n && timing; ++i)
    if (handles[i]->device == dev && handles[i]->stream)
      timing = cudaStreamWaitEvent(handles[i]->stream, start, 0) == cudaSuccess;
  std::vector<int32_t> rc(n, PTYB_OK);
  {
    std::vector<std::thread> workers;
    workers.reserve(n);
    try {
      for (int i = 0; i < n; ++i)
        workers.emplace_back([&, i] {
          int r = rpie_epochs > 0 ? ptyb_rpie(handles[i], rpie, rpie_epochs) : PTYB_OK;
          if (r == PTYB_OK && lsqml_epochs > 0)
            r = ptyb_lsqml(handles[i], lsqml, lsqml_epochs, calc_llk);
          rc[i] = r;
        });
    } catch (...) {
      // no thread for the rest: the started ones finish before the failure goes up
      for (auto& w : workers) w.join();
      throw;
    }
    for (auto& w : workers) w.join();
  }
  if (timing) {
    cudaSetDevice(dev);
    for (int i = 0; i < n && timing; ++i) {
      if (handles[i]->device != dev || !handles[i]->stream) continue;
      cudaEvent_t e = nullptr;
      timing = cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventRecord(e, handles[i]->stream) == cudaSuccess &&
               cudaStreamWaitEvent(ts, e, 0) == cudaSuccess;
      if (e) cudaEventDestroy(e);
    }
    float ms = -1.f;
    if (timing && cudaEventRecord(end, ts) == cudaSuccess &&
        cudaEventSynchronize(end) == cudaSuccess &&
        cudaEventElapsedTime(&ms, start, end) == cudaSuccess && device_ms)
      *device_ms = ms;
  }
  if (start) cudaEventDestroy(start);
  if (end) cudaEventDestroy(end);
  if (ts) cudaStreamDestroy(ts);
  int first = PTYB_OK;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = rc[i];
    if (first == PTYB_OK && rc[i] != PTYB_OK) first = rc[i];
  }
  return first;
}

}  // namespace

int ptyb_batch_run(ptyb_handle* const* handles, int32_t n, const ptyb_rpie_params* rpie,
                   int32_t rpie_epochs, const ptyb_lsqml_params* lsqml, int32_t lsqml_epochs,
                   int32_t calc_llk, int32_t* status, float* device_ms) {
  try {
    return batch_run_impl(handles, n, rpie, rpie_epochs, lsqml, lsqml_epochs, calc_llk, status,
                          device_ms);
  } catch (const std::exception&) {
    // a host failure (no thread or host memory for the batch): nothing is reported per handle
    return PTYB_GPU;
  }
}

int ptyb_set_probe_variation(ptyb_handle* h, const double* eigenmodes, int32_t k,
                             const double* weights, int32_t refine_weights,
                             const double* intensity, int32_t refine_intensity) {
  if (!h) return PTYB_INVALID;
  if (k < 0 || (k > 0 && (!eigenmodes || !weights))) {
    h->err = "probe variation: k >= 0 with eigenmodes and weights";
    return PTYB_INVALID;
  }
  if (intensity && k == 0) {
    h->err = "main-mode weights need an eigenmode";
    return PTYB_INVALID;
  }
  if (h->nslice > 1 || h->have_offsets) {
    h->err = "the probe variation runs on a single slice without the position model";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const size_t plane = (size_t)h->N * h->N;
    h->opr_on = k > 0;
    h->opr_k = k;
    h->opr_has_c = intensity != nullptr;
    h->opr_refine_w = refine_weights != 0;
    h->opr_refine_c = refine_intensity != 0;
    if (!h->opr_on) return PTYB_OK;
    h->opr_u = alloc<float2>(h, (size_t)k * plane);
    upload_c64(h, eigenmodes, h->opr_u, (size_t)k * plane, "eigenmodes");
    h->opr_w = alloc<double>(h, (size_t)h->P * k);
    check(h, copy_sync(h, h->opr_w, weights, (size_t)h->P * k * sizeof(double),
                       cudaMemcpyHostToDevice), "weights");
    if (intensity) {
      h->opr_c = alloc<double>(h, h->P);
      check(h, copy_sync(h, h->opr_c, intensity, (size_t)h->P * sizeof(double),
                         cudaMemcpyHostToDevice), "intensity");
    }
    return PTYB_OK;
  });
}

int ptyb_get_probe_variation(ptyb_handle* h, double* eigenmodes, double* weights,
                             double* intensity) {
  if (!h) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    const size_t plane = (size_t)h->N * h->N;
    if (!h->opr_on) return PTYB_OK;
    if (eigenmodes) download_c64(h, h->opr_u, eigenmodes, (size_t)h->opr_k * plane, "eigenmodes");
    if (weights)
      check(h, copy_sync(h, weights, h->opr_w, (size_t)h->P * h->opr_k * sizeof(double),
                         cudaMemcpyDeviceToHost), "weights");
    if (intensity && h->opr_has_c)
      check(h, copy_sync(h, intensity, h->opr_c, (size_t)h->P * sizeof(double),
                         cudaMemcpyDeviceToHost), "intensity");
    return PTYB_OK;
  });
}

int ptyb_get_llk(ptyb_handle* h, ptyb_llk* out) {
  if (!h || !out) return PTYB_INVALID;
  return guarded(h, true, [&]() -> int {
    *out = llk_pass(h);
    return PTYB_OK;
  });
}

int ptyb_gradients(ptyb_handle* h, double* loss, double* d_obj, double* d_probe, double* d_pos) {
  if (!h) return PTYB_INVALID;
  if (h->nslice > 1 && d_pos) {
    h->err = "position gradients run on a single-slice object";
    return PTYB_INVALID;
  }
  if (h->nslice > 1)
    return guarded(h, true, [&]() -> int {
      slice_gradients(h, d_obj != nullptr, d_probe != nullptr);
      const ptyb_llk l = llk_pass(h);
      if (loss) *loss = l.poisson * h->nb_obs;
      const size_t np = (size_t)h->K * h->N * h->N;
      const size_t no = (size_t)h->nslice * h->nyo * h->nxo;
      if (d_obj) {
        download_c64(h, h->g_slices, d_obj, no, "gradient");
      }
      if (d_probe) {
        download_c64(h, h->g_probe, d_probe, np, "gradient");
      }
      return PTYB_OK;
    });
  if (d_pos && !h->have_offsets) {
    h->err = "position gradients need position offsets (ptyb_set_positions)";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_ml(h);
    const size_t np = (size_t)h->K * h->N * h->N, no = (size_t)h->nyo * h->nxo;
    if (h->have_offsets) {
      ensure_spec(h);
      if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * np);
      if (h->wave2_slots < h->slots) {
        h->wave2 = alloc<float2>(h, (size_t)h->slots * np);
        h->wave2_slots = h->slots;
      }
      if (!h->ml_pos_sums) h->ml_pos_sums = alloc<double>(h, (size_t)h->P * 4);
      spectrum_of(h, h->probe, h->spec);
      const int stack = std::min(h->P, h->stack);
      for (int s0 = 0; s0 < h->P; s0 += stack)
        move_frames(h, h->iota + s0, std::min(stack, h->P - s0), h->spec,
                    h->wave_all + (size_t)s0 * np);
    }
    ml_gradients(h, d_obj != nullptr, d_probe != nullptr, false, d_pos != nullptr);
    const ptyb_llk l = llk_pass(h, h->have_offsets ? h->wave_all : nullptr);
    if (loss) *loss = l.poisson * h->nb_obs;
    if (d_obj) {
      download_c64(h, h->g_obj, d_obj, no, "gradient");
    }
    if (d_probe) {
      download_c64(h, h->g_probe, d_probe, np, "gradient");
    }
    if (d_pos) {
      std::vector<double> v((size_t)h->P * 4);
      check(h, copy_sync(h, v.data(), h->ml_pos_sums, v.size() * sizeof(double),
                          cudaMemcpyDeviceToHost),
            "gradient");
      for (int f = 0; f < h->P; ++f) {
        d_pos[2 * f] = v[(size_t)f * 4];
        d_pos[2 * f + 1] = v[(size_t)f * 4 + 1];
      }
    }
    return PTYB_OK;
  });
}

int ptyb_forward_intensity(ptyb_handle* h, const int32_t* frames, int32_t n, float* out) {
  if (!h || !frames || !out || n < 0) return PTYB_INVALID;
  if (h->nslice > 1) {
    h->err = "forward intensity runs on a single-slice object";
    return PTYB_INVALID;
  }
  for (int i = 0; i < n; ++i)
    if (frames[i] < 0 || frames[i] >= h->P) {
      h->err = "frame index out of range";
      return PTYB_INVALID;
    }
  return guarded(h, true, [&]() -> int {
    const int stack = std::min(h->P, h->stack);
    ensure_slots(h, stack);
    const size_t plane = (size_t)h->N * h->N;
    for (int s0 = 0; s0 < n; s0 += stack) {
      const int m = std::min(stack, n - s0);
      check(h, cudaMemcpyAsync(h->order, frames + s0, m * sizeof(int32_t), cudaMemcpyHostToDevice,
                               h->stream),
            "frames");
      FrameArgs a = frame_args(h, h->order);
      check(h, launch_frame<kStore>(h, a, m), "forward");
      ++h->launches;
      check(h, cudaMemcpyAsync(out + (size_t)s0 * plane, h->icalc, m * plane * sizeof(float),
                               cudaMemcpyDeviceToHost, h->stream),
            "intensity");
      check(h, cudaStreamSynchronize(h->stream), "forward");
    }
    return PTYB_OK;
  });
}

int ptyb_forward_intensity_noalloc(ptyb_handle* h, const int32_t* frames, int32_t n,
                                   float* out) {
  if (!h || !frames || !out || n < 0) return PTYB_INVALID;
  if (h->nslice > 1) {
    h->err = "forward intensity runs on a single-slice object";
    return PTYB_INVALID;
  }
  for (int i = 0; i < n; ++i)
    if (frames[i] < 0 || frames[i] >= h->P) {
      h->err = "frame index out of range";
      return PTYB_INVALID;
    }
  // Scratch per frame: its index, its detector field (K planes) and its intensity plane.
  const size_t plane = (size_t)h->N * h->N;
  const size_t per_frame = 256 + (size_t)h->K * plane * sizeof(float2) + plane * sizeof(float);
  const int chunk = (int)std::min<size_t>((size_t)std::max(n, 1), kNoallocScratchBytes / per_frame);
  if (chunk < 1) {
    h->err = "one frame's field and intensity (" + std::to_string(per_frame) +
             " bytes) exceed the 32 MiB no-alloc scratch";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    unsigned char* base = nullptr;
    check(h, noalloc_scratch(h->device, &base), "cudaGetSymbolAddress");
    int* d_frames = reinterpret_cast<int*>(base);
    float2* field = reinterpret_cast<float2*>(base + 256 * (size_t)chunk);
    float* icalc = reinterpret_cast<float*>(field + (size_t)chunk * h->K * plane);
    for (int s0 = 0; s0 < n; s0 += chunk) {
      const int m = std::min(chunk, n - s0);
      check(h, cudaMemcpyAsync(d_frames, frames + s0, m * sizeof(int32_t), cudaMemcpyHostToDevice,
                               h->stream),
            "frames");
      FrameArgs a = frame_args(h, d_frames);
      a.field = field;
      a.icalc = icalc;
      check(h, launch_frame_raw<kStore>(h, a, m), "forward");
      ++h->launches;
      check(h, cudaMemcpyAsync(out + (size_t)s0 * plane, icalc, m * plane * sizeof(float),
                               cudaMemcpyDeviceToHost, h->stream),
            "intensity");
      check(h, cudaStreamSynchronize(h->stream), "forward");
    }
    return PTYB_OK;
  });
}

int ptyb_set_positions(ptyb_handle* h, const double* offsets, int32_t refine) {
  if (!h) return PTYB_INVALID;
  if (h->opr_on && offsets) {
    h->err = "the position model with a probe variation is not built";
    return PTYB_INVALID;
  }
  if (h->nslice > 1 && offsets) {
    h->err = "the position model runs on a single-slice object in this version";
    return PTYB_INVALID;
  }
  if (offsets)
    for (int i = 0; i < 2 * h->P; ++i)
      if (!std::isfinite(offsets[i])) {
        h->err = "position offsets must be finite";
        return PTYB_INVALID;
      }
  return guarded(h, true, [&]() -> int {
    check(h, cudaStreamSynchronize(h->stream), "sync");
    if (!offsets) {
      h->have_offsets = h->refine_offsets = false;
      return PTYB_OK;
    }
    if (!h->offsets) h->offsets = alloc<double>(h, (size_t)h->P * 2);
    check(h, copy_sync(h, h->offsets, offsets, (size_t)h->P * 2 * sizeof(double),
                        cudaMemcpyHostToDevice),
          "offsets");
    if (!h->have_offsets && h->slots > 0) {
      const size_t plane = (size_t)h->N * h->N;
      h->wave = alloc<float2>(h, (size_t)h->slots * h->K * plane);
      h->pos_sums = alloc<double>(h, (size_t)h->slots * 4);
    }
    h->have_offsets = true;
    h->refine_offsets = refine != 0;
    return PTYB_OK;
  });
}

int ptyb_get_positions(ptyb_handle* h, double* dst) {
  if (!h || !dst) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    check(h, cudaStreamSynchronize(h->stream), "sync");
    if (!h->have_offsets) {
      std::fill(dst, dst + 2 * h->P, 0.0);
      return PTYB_OK;
    }
    check(h, copy_sync(h, dst, h->offsets, (size_t)h->P * 2 * sizeof(double), cudaMemcpyDeviceToHost),
          "offsets");
    return PTYB_OK;
  });
}

int ptyb_get_object(ptyb_handle* h, double* dst) {
  if (!h || !dst) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    const size_t n = (size_t)h->nobj * h->nyo * h->nxo;
    download_c64(h, h->object, dst, n, "object");
    return PTYB_OK;
  });
}

int ptyb_get_objects(ptyb_handle* h, double* dst) {
  if (!h || !dst) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    const size_t n = (size_t)h->nslice * h->nobj * h->nyo * h->nxo;
    download_c64(h, h->object, dst, n, "objects");
    return PTYB_OK;
  });
}

int ptyb_set_objects(ptyb_handle* h, const double* src) {
  if (!h || !src) return PTYB_INVALID;
  return guarded(h, true, [&]() -> int {
    const size_t n = (size_t)h->nslice * h->nobj * h->nyo * h->nxo;
    upload_c64(h, src, h->object, n, "objects");
    return PTYB_OK;
  });
}

int ptyb_get_probe(ptyb_handle* h, double* dst) {
  if (!h || !dst) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    const size_t n = (size_t)h->nprobe * h->N * h->N;
    download_c64(h, h->probe, dst, n, "probe");
    return PTYB_OK;
  });
}

int ptyb_set_object(ptyb_handle* h, const double* src) {
  if (!h || !src) return PTYB_INVALID;
  return guarded(h, true, [&]() -> int {
    const size_t n = (size_t)h->nobj * h->nyo * h->nxo;
    upload_c64(h, src, h->object, n, "object");
    return PTYB_OK;
  });
}

int ptyb_set_probe(ptyb_handle* h, const double* src) {
  if (!h || !src) return PTYB_INVALID;
  return guarded(h, true, [&]() -> int {
    const size_t n = (size_t)h->nprobe * h->N * h->N;
    upload_c64(h, src, h->probe, n, "probe");
    return PTYB_OK;
  });
}

int ptyb_corners(ptyb_handle* h, int32_t* dst) {
  if (!h || !dst) return PTYB_INVALID;
  std::memcpy(dst, h->corners_h.data(), h->corners_h.size() * sizeof(int32_t));
  return PTYB_OK;
}

int ptyb_history_len(ptyb_handle* h) { return h ? (int)h->history.size() : 0; }

int ptyb_history(ptyb_handle* h, ptyb_llk_record* dst, int32_t cap) {
  if (!h || (!dst && cap > 0)) return PTYB_INVALID;
  const int n = std::min<int>(cap, (int)h->history.size());
  for (int i = 0; i < n; ++i) dst[i] = h->history[i];
  return PTYB_OK;
}

int64_t ptyb_cycle(ptyb_handle* h) { return h ? h->cycle : 0; }

int ptyb_lsqml_steps_len(ptyb_handle* h) { return h ? (int)h->steps.size() : 0; }

int ptyb_lsqml_steps(ptyb_handle* h, ptyb_lsqml_step* dst, int32_t cap) {
  if (!h || (!dst && cap > 0)) return PTYB_INVALID;
  const int n = std::min<int>(cap, (int)h->steps.size());
  for (int i = 0; i < n; ++i) dst[i] = h->steps[i];
  return PTYB_OK;
}

int ptyb_synchronize(ptyb_handle* h) {
  if (!h) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    check(h, cudaStreamSynchronize(h->stream), "synchronize");
    return PTYB_OK;
  });
}

int64_t ptyb_launches(ptyb_handle* h) { return h ? h->launches : 0; }

int ptyb_set_timing(ptyb_handle* h, int32_t on) {
  if (!h) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    check(h, cudaStreamSynchronize(h->stream), "sync");
    harvest(h);
    h->timing = on != 0;
    for (int k = 0; k < kNumKinds; ++k) {
      h->kind_ms[k] = 0.0;
      h->kind_n[k] = 0;
      h->kind_frames[k] = 0;
    }
    return PTYB_OK;
  });
}

int32_t ptyb_kernel_kinds(void) { return kNumKinds; }

const char* ptyb_kernel_name(int32_t kind) {
  return kind >= 0 && kind < kNumKinds ? kKindNames[kind] : "";
}

int ptyb_kernel_times(ptyb_handle* h, double* ms, int64_t* launches, int32_t cap) {
  if (!h || !ms || !launches) return PTYB_INVALID;
  for (int k = 0; k < std::min<int>(cap, kNumKinds); ++k) {
    ms[k] = h->kind_ms[k];
    launches[k] = h->kind_n[k];
  }
  return PTYB_OK;
}

int ptyb_kernel_frames(ptyb_handle* h, int64_t* frames, int32_t cap) {
  if (!h || !frames) return PTYB_INVALID;
  for (int k = 0; k < std::min<int>(cap, kNumKinds); ++k) frames[k] = h->kind_frames[k];
  return PTYB_OK;
}

double ptyb_last_call_ms(ptyb_handle* h) { return h ? h->last_call_ms : 0.0; }

int ptyb_random_batches(int32_t nframe, int32_t size, uint64_t seed, uint64_t epoch,
                        int32_t* order) {
  if (nframe < 0 || size <= 0 || (!order && nframe > 0)) return PTYB_INVALID;
  std::vector<int32_t> o, sizes;
  random_batches(nframe, size, seed, epoch, &o, &sizes);
  std::memcpy(order, o.data(), o.size() * sizeof(int32_t));
  return PTYB_OK;
}

int ptyb_view_corners(const double* y, const double* x, int32_t nframe, double pixel_y,
                      double pixel_x, int32_t ny, int32_t nx, int32_t nyo, int32_t nxo,
                      int32_t* corners) {
  if (nframe < 0 || !y || !x || !corners) return PTYB_INVALID;
  const double pixel[2] = {pixel_y, pixel_x};
  std::vector<double> yy(y, y + nframe), xx(x, x + nframe);
  std::vector<int32_t> c;
  std::string err;
  if (!corners_of(pynx_axis(yy, pixel_y), pynx_axis(xx, pixel_x), pixel, ny, nx, nyo, nxo, &c,
                  &err)) {
    g_create_error = err;
    return PTYB_INVALID;
  }
  std::memcpy(corners, c.data(), c.size() * sizeof(int32_t));
  return PTYB_OK;
}

const char* ptyb_last_error(ptyb_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

void ptyb_destroy(ptyb_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto& b : h->bufs) cudaFreeAsync(b.p, h->stream);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto e : h->event_pool) cudaEventDestroy(e);
  for (auto& p : h->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : h->call_ev)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

}  // extern "C"
