// Internal interface of the reconstruction engine behind the C ABI (include/ptyb200.h): the
// device state of one scan (`ptyb_handle`) and the host helpers every algorithm's launch
// sequence shares. The algorithms' host loops live in their own files: rpie.cu, lsqml.cu,
// ml.cu, carried.cu (AP / DM / RAAR), batch.cu; the per-frame cluster kernels are instantiated
// once per frame side in kernels_<side>.cu behind the launch functions of launch.cuh.
//
// Reference engine (physwkim/ptyrs): `GpuPtycho` (ptyrs/src/engine/gpu/mod.rs:533-881).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ptyb200.h"
#include "gather.cuh"
#include "launch.cuh"
#include "lsqml.cuh"
#include "ml.cuh"
#include "multislice.cuh"
#include "opr.cuh"
#include "position.cuh"
#include "scan.h"

// Object slices of a multislice handle, and the float scalars on the device (maxima, the
// batch's object and probe steps, one step per further slice).
constexpr int kMaxSlices = 16;
// Room for the kernel kinds of the per-kernel timing (the Kind enum below fits it).
constexpr int kMaxKinds = 48;
constexpr int kScalars = 8 + kMaxSlices + 2;
// The maxima of the AP / DM / RAAR blends' object and probe norms.
constexpr int kScalObjNorm = 8 + kMaxSlices, kScalProbeNorm = kScalObjNorm + 1;

namespace ptyb::eng {

// Devices a process may use (per-device tables of the pool and the no-alloc scratch).
constexpr int kMaxDevices = 64;

constexpr int kAlgAp = 0, kAlgDm = 1, kAlgRaar = 2, kAlgRpie = 3, kAlgMl = 4, kAlgLsqml = 6,
              kAlgBh = 5;

// One device allocation, freed with the handle.
struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace ptyb::eng

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
  // ML through the slices: the previous gradients and the directions of every slice.
  float2* last_slices = nullptr;  // [S][nyo][nxo]
  float2* dir_slices = nullptr;   // [S][nyo][nxo]
  float2* bh_tmp = nullptr;       // [S][nyo][nxo] then [K][N][N]: BH's u ± v through slices
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
  float2* opr_r = nullptr;       // [slots][N][N]
  float2* opr_moved = nullptr;   // [slots][K][N][N] frame probe directions moved back
  float2* opr_e = nullptr;       // [N][N]
  double* opr_sums = nullptr;    // [slots][parts][≤ 4] per-frame partials, then [slots][2]
                                 // the Gram–Schmidt sums
  double* opr_p = nullptr;       // [slots]
  double* opr_scal = nullptr;    // [4]
  unsigned* opr_count = nullptr; // the per-frame passes' count of finished blocks
  // Their probe step under the position model: the residual's back-projection g, the step,
  // g's spectrum summed over frames with its compensation, each frame's ‖A·step‖² per mode
  // and the modes' slope and regulariser sums.
  float2 *pcg_g = nullptr, *pcg_step = nullptr, *pcg_spec = nullptr, *pcg_comp = nullptr;
  double* pcg_norms = nullptr;    // [P][K]
  double* pcg_modes = nullptr;    // [K][2]
  double* partials = nullptr;    // [kPartialBlocks][2]
  std::vector<ptyb::eng::Buf> bufs;
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
  std::vector<ptyb_bh_step> bh_steps;  // the last BH epoch's steps
  // BH under the position model: per stack slot the planes its Hessian reads, [bh_slots][K][N][N]
  // each (M(P), M(u_P), M(v_P), then with refined offsets ∂y, ∂x of each and ∂y∂y, ∂y∂x, ∂x∂x of
  // M(P)), the spectra of u_P and v_P, and the displacements' offsets parts [bh_slots][2]
  float2* bh_planes[12] = {};
  int bh_slots = 0;
  float2 *bh_spec_u = nullptr, *bh_spec_v = nullptr;
  double *bh_ud = nullptr, *bh_vd = nullptr;
  int log_stride = 3;
  bool aborted = false;
  std::string err;
};

namespace ptyb::eng {

// A CUDA failure part-way through a call: the handle is poisoned and the call returns `code`.
struct Fail {
  int code;
};

// Host error messages of ptyb_create / ptyb_view_corners (no handle to hold them).
extern thread_local std::string g_create_error;

void check(ptyb_handle* h, cudaError_t e, const char* what);
cudaError_t pool_alloc(ptyb_handle* h, void** p, size_t bytes);
cudaError_t copy_sync(ptyb_handle* h, void* dst, const void* src, size_t bytes,
                      cudaMemcpyKind kind);
cudaError_t fill_sync(ptyb_handle* h, void* dst, int value, size_t bytes);
void launched(ptyb_handle* h, const char* what);
// Whether `p` is device (or managed) memory of the handle's device.
bool on_device(ptyb_handle* h, const void* p);

// `count` elements of T from the device pool, freed with the handle.
template <typename T>
T* alloc(ptyb_handle* h, size_t count) {
  void* p = nullptr;
  check(h, pool_alloc(h, &p, count * sizeof(T) + 16), "cudaMallocAsync");
  h->bufs.push_back({p, count * sizeof(T)});
  return static_cast<T*>(p);
}

constexpr int kPartialBlocks = 296;

// Kernel kinds for the per-kernel timing (ptyb_kernel_name).
enum Kind : int {
  kKFrameRpie = 0, kKFrameLsqml, kKFrameMl, kKFrameLlk, kKFrameStore, kKFrameFromStore,
  kKObjRpie, kKObjOverlap, kKObjLsqml, kKObjMl, kKIllum, kKProbePartial, kKProbeFinal,
  kKAfar, kKDots, kKSolve, kKAxpy, kKMax, kKCounts, kKMisc, kKGamma, kKArraySums, kKMove,
  kKPositionSums, kKSliceForward, kKSliceBackward, kKSliceLlk, kKFrameProject, kKSpectrum,
  kKDerivSums, kKBackSpectrum, kKSliceGrad, kKFrameCarry, kKObjBlend, kKOprStep, kKBhHessian,
  kNumKinds
};
static_assert(kNumKinds <= kMaxKinds, "the timing arrays hold kMaxKinds kinds");
extern const char* const kKindNames[kNumKinds];

cudaEvent_t take_event(ptyb_handle* h);

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

void harvest(ptyb_handle* h);
void begin_call(ptyb_handle* h);
void end_call(ptyb_handle* h, const char* what);
int cluster_for(int N, int K, int want);

// The per-frame cluster kernels on the handle's stream, in its cluster shape.
template <int MODE>
cudaError_t launch_frame_raw(ptyb_handle* h, const FrameArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  return launch_frame_side(h->N, h->C, MODE, a, nslot, h->K, h->stream);
}

template <int MODE>
cudaError_t launch_frame(ptyb_handle* h, const FrameArgs& a, int nslot) {
  constexpr int kind = MODE == kRpie ? kKFrameRpie
                       : MODE == kLsqmlFused ? kKFrameLsqml
                       : MODE == kMlGrad || MODE == kBhGrad ? kKFrameMl
                       : MODE == kLlk ? kKFrameLlk
                       : MODE == kStore ? kKFrameStore
                       : MODE == kProject || MODE == kProjectKept ? kKFrameProject
                       : MODE == kCarry ? kKFrameCarry
                                        : kKFrameFromStore;
  cudaError_t e = cudaSuccess;
  timed(h, kind, [&] { e = launch_frame_raw<MODE>(h, a, nslot); }, nslot);
  return e;
}

// Plane transforms of the position model over `nslot` frames (the frame kernel's cluster
// shape; window derivatives carry two planes, the position sums at least two).
template <int MODE>
cudaError_t launch_move(ptyb_handle* h, const MoveArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  const int K = MODE == kDerivWindow ? 2 : MODE == kDerivSums ? std::max(h->K, 2) : h->K;
  constexpr int kind = MODE == kDerivSums      ? kKDerivSums
                       : MODE == kSpectrum     ? kKSpectrum
                       : MODE == kBackSpectrum ? kKBackSpectrum
                                               : kKMove;
  const int C = MODE == kDerivSums ? h->C_sums : h->C;
  cudaError_t e = cudaErrorInvalidValue;
  timed(h, kind, [&] { e = launch_move_side(h->N, C, MODE, a, nslot, K, h->stream); }, nslot);
  return e;
}

template <int MODE>
cudaError_t launch_slice(ptyb_handle* h, const SliceArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  constexpr int kind = MODE == kSliceForward ? kKSliceForward
                       : MODE == kSliceBackward ? kKSliceBackward
                       : MODE == kSliceGrad     ? kKSliceGrad
                                                : kKSliceLlk;
  cudaError_t e = cudaErrorInvalidValue;
  timed(h, kind, [&] { e = launch_slice_side(h->N, h->C, MODE, a, nslot, h->K, h->stream); },
        nslot);
  return e;
}

cudaError_t launch_gamma(ptyb_handle* h, const GammaArgs& a, int nslot);

MoveArgs move_args(ptyb_handle* h, const int* frames, float2* planes);
void spectrum_of(ptyb_handle* h, const float2* probe, float2* spec);
void move_frames(ptyb_handle* h, const int* frames, int n, const float2* spec, float2* out);
void ensure_spec(ptyb_handle* h);
FrameArgs frame_args(ptyb_handle* h, const int* frames);
GatherArgs gather_args(ptyb_handle* h, const int* frames, int nslot);
int ntiles(ptyb_handle* h);
void ensure_slots(ptyb_handle* h, int n);
int probe_chunk(ptyb_handle* h, int nslot, int* nchunk);
void probe_pass(ptyb_handle* h, const int* frames, int nslot, int mode, float alpha, float coef,
                const float2* quad = nullptr, const float2* upd = nullptr);
ptyb_llk llk_pass(ptyb_handle* h, const float2* waves = nullptr);
ptyb_llk llk_of_frames(ptyb_handle* h);
void record(ptyb_handle* h, int algorithm, const ptyb_llk& l);
bool llk_due(int calc_llk, int ic, int ncycle);
void upload_orders(ptyb_handle* h, int nepoch, int size, uint64_t seed, int64_t epoch0,
                   std::vector<std::vector<int32_t>>* sizes, std::vector<int32_t>* last);

// Runs fn(begin, end) over [0, n) on up to eight host threads (one below a million).
template <class F>
void parallel_range(size_t n, F&& fn) {
  const size_t nt =
      n < (size_t(1) << 20) ? 1 : std::min<size_t>(8, std::thread::hardware_concurrency());
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

void download_c64(ptyb_handle* h, const float2* src, double* dst, size_t n, const char* what);
void upload_c64(ptyb_handle* h, const double* src, float2* dst, size_t n, const char* what);
void ensure_ml(ptyb_handle* h);
// 2·∂F/∂x* over every slice (h->g_slices) and the probe (h->g_probe) through a multislice
// object, over `n` frames (every frame when null), Poisson or with kCostBh BH's amplitude cost.
void slice_gradients(ptyb_handle* h, bool uo, bool up, const int* frames = nullptr, int n = 0,
                     int cost = kCostPoisson);
// Shared memory of the multislice line search (and BH's quadratic form) at side N, K modes.
size_t slice_gamma_bytes(int N, int K);
void array_sums(ptyb_handle* h, const float2* g, const float2* hh, size_t n, int mode,
                double out[2]);
unsigned blocks_for(size_t n);
void finish_state(ptyb_handle* h, const double* object, const double* probe, double wavelength,
                  double distance, const double* gaps);
// Raw counts of `nframe` frames (PTYB_COUNTS_*, detector order) to the FFT-shifted float layout
// with masked pixels −1, each frame's photon sum and unmasked count; `*bad` set by a non-finite
// unmasked value (engine/obs.rs:61-76).
cudaError_t convert_counts(const void* raw, int kind, float* iobs, double* power, int* nobs,
                           int* bad, int nframe, int N, cudaStream_t s);
void zero_phase_ramp(ptyb_handle* h);
void scale_obj_probe(ptyb_handle* h, float2* waves = nullptr);
void split_scale(ptyb_handle* h, double s, float2* waves);

// Runs `body` for an ABI call: the abort gate (engine/gpu/gate.rs:8-71), the handle's device,
// and failures turned into a status and message.
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

}  // namespace ptyb::eng
