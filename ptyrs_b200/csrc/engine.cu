// The engine's core behind the C ABI (include/ptyb200.h): the handle's creation and device
// memory, the launch helpers every algorithm shares (frame arguments, probe passes, the LLK
// pass, batch orders, timing), host staging of complex arrays, the phase-ramp removal and the
// object/probe rescale, and the state accessors.
//
// Reference engine (physwkim/ptyrs): `GpuPtycho` (ptyrs/src/engine/gpu/mod.rs:533-881), the LLK
// pass (engine/gpu/device.rs:3379-3395).
#include "engine.cuh"

using namespace ptyb;

namespace ptyb {

cudaError_t launch_frame_side(int N, int C, int mode, const FrameArgs& a, int nslot, int K,
                              cudaStream_t s) {
  switch (N) {
    case 64: return SideKernels<64>::frame(C, mode, a, nslot, K, s);
    case 96: return SideKernels<96>::frame(C, mode, a, nslot, K, s);
    case 128: return SideKernels<128>::frame(C, mode, a, nslot, K, s);
    case 192: return SideKernels<192>::frame(C, mode, a, nslot, K, s);
    case 256: return SideKernels<256>::frame(C, mode, a, nslot, K, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_move_side(int N, int C, int mode, const MoveArgs& a, int nslot, int K,
                             cudaStream_t s) {
  switch (N) {
    case 64: return SideKernels<64>::move(C, mode, a, nslot, K, s);
    case 96: return SideKernels<96>::move(C, mode, a, nslot, K, s);
    case 128: return SideKernels<128>::move(C, mode, a, nslot, K, s);
    case 192: return SideKernels<192>::move(C, mode, a, nslot, K, s);
    case 256: return SideKernels<256>::move(C, mode, a, nslot, K, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_slice_side(int N, int C, int mode, const SliceArgs& a, int nslot, int K,
                              cudaStream_t s) {
  switch (N) {
    case 64: return SideKernels<64>::slice(C, mode, a, nslot, K, s);
    case 96: return SideKernels<96>::slice(C, mode, a, nslot, K, s);
    case 128: return SideKernels<128>::slice(C, mode, a, nslot, K, s);
    case 192: return SideKernels<192>::slice(C, mode, a, nslot, K, s);
    case 256: return SideKernels<256>::slice(C, mode, a, nslot, K, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_gamma_side(int N, const GammaArgs& a, int nslot, cudaStream_t s) {
  switch (N) {
    case 64: return SideKernels<64>::gamma(a, nslot, s);
    case 96: return SideKernels<96>::gamma(a, nslot, s);
    case 128: return SideKernels<128>::gamma(a, nslot, s);
    case 192: return SideKernels<192>::gamma(a, nslot, s);
    case 256: return SideKernels<256>::gamma(a, nslot, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_bh_side(int N, const BhArgs& a, int nslot, cudaStream_t s) {
  switch (N) {
    case 64: return SideKernels<64>::bh(a, nslot, s);
    case 96: return SideKernels<96>::bh(a, nslot, s);
    case 128: return SideKernels<128>::bh(a, nslot, s);
    case 192: return SideKernels<192>::bh(a, nslot, s);
    case 256: return SideKernels<256>::bh(a, nslot, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_slice_gamma_side(int N, const SliceGammaArgs& a, int nslot, int K,
                                    cudaStream_t s) {
  switch (N) {
    case 64: return SideKernels<64>::slice_gamma(a, nslot, K, s);
    case 96: return SideKernels<96>::slice_gamma(a, nslot, K, s);
    case 128: return SideKernels<128>::slice_gamma(a, nslot, K, s);
    case 192: return SideKernels<192>::slice_gamma(a, nslot, K, s);
    case 256: return SideKernels<256>::slice_gamma(a, nslot, K, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ptyb

namespace ptyb::eng {

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
bool on_device(ptyb_handle* h, const void* p) {
  cudaPointerAttributes a = {};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // not a pointer the runtime knows: clear the error it left
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) &&
         a.device == h->device;
}

void launched(ptyb_handle* h, const char* what) {
  ++h->launches;
  check(h, cudaGetLastError(), what);
}

const char* const kKindNames[kNumKinds] = {
    "frame_rpie", "frame_lsqml", "frame_ml_grad", "frame_llk", "frame_store",
    "frame_from_store", "object_rpie", "object_overlap", "object_lsqml", "object_ml",
    "illumination", "probe_partial", "probe_finalize", "lsqml_afar", "lsqml_dots",
    "lsqml_solve", "axpy", "max", "counts", "misc", "ml_gamma", "array_sums", "move",
    "position_sums", "slice_forward", "slice_backward", "slice_llk", "frame_project", "spectrum",
    "deriv_sums", "back_spectrum", "slice_grad", "frame_carry", "object_blend", "opr_step",
    "bh_hessian"};


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

MoveArgs move_args(ptyb_handle* h, const int* frames, float2* planes) {
  MoveArgs m = {};
  m.probe = h->probe;
  // the phase the probe moves with: the exit's on one slice, none on slice 0 of a multislice
  // object (engine/lsqml.rs:500-523, `optics.slice_quad(0)`)
  m.quad = h->nslice > 1 ? h->ones : h->quad;
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
  // the detector field (K planes per slot), also the window derivatives of the position model
  // (two planes per slot)
  h->field = alloc<float2>(h, (size_t)n * std::max(h->K, 2) * plane);
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
                const float2* quad, const float2* upd) {
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
ptyb_llk llk_pass(ptyb_handle* h, const float2* waves) {
  const int stack = std::min(h->P, h->stack);
  const size_t pstride = (size_t)h->K * h->N * h->N;
  ensure_slots(h, stack);
  if (h->have_offsets && !waves) {
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
      if (waves) {
        // each frame's own (moved or varied) probe enters slice 0
        sa.f.probe = waves + s0 * pstride;
        sa.f.probe_stride = (int)pstride;
      } else if (h->have_offsets) {
        // each frame's moved probe enters slice 0
        move_frames(h, h->iota + s0, n, h->spec, h->wave);
        sa.f.probe = h->wave;
        sa.f.probe_stride = (int)pstride;
      }
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
// Per frame, Σ_pixels Σ_modes |P_m·O_window|² in double (one block per frame, the modes'
// probes shared or, with `waves`, the frame's own moved planes): by Parseval the photons of the
// model's detector fields, Σ|Ψ|² under the unitary transform (|q| = 1).
__global__ void __launch_bounds__(256) exit_power_kernel(const float2* object,
                                                         const float2* probe, size_t stride,
                                                         const int2* corners, int nxo, int K,
                                                         int N, double* out) {
  __shared__ double part[8];
  const int f = blockIdx.x;
  const int2 c = corners[f];
  const float2* p = probe + (size_t)f * stride;
  const float2* ow = object + (size_t)c.x * nxo + c.y;
  double s = 0.0;
  // Two neighbouring pixels of a row per thread and step (N is even), the probe planes read as
  // 16-byte pairs; rows and columns carried along the 512-pixel strides.
  int y = 2 * threadIdx.x / N, x = 2 * threadIdx.x % N;
#pragma unroll 4
  for (int pp = threadIdx.x; pp < N * N / 2; pp += 256) {
    const float2* orow = ow + (size_t)y * nxo + x;
    const float2 o0 = orow[0], o1 = orow[1];
    float p0 = 0.f, p1 = 0.f;
    for (int m = 0; m < K; ++m) {
      const float4 v = reinterpret_cast<const float4*>(p + (size_t)m * N * N)[pp];
      p0 += v.x * v.x + v.y * v.y;
      p1 += v.z * v.z + v.w * v.w;
    }
    s += (double)p0 * (o0.x * o0.x + o0.y * o0.y) + (double)p1 * (o1.x * o1.x + o1.y * o1.y);
    y += 512 / N;
    x += 512 % N;
    if (x >= N) {
      x -= N;
      ++y;
    }
  }
  s = warp_sum(s);
  if (threadIdx.x % 32 == 0) part[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += part[w];
    out[f] = t;
  }
}

// The opening rescale of ML (engine/ptycho.rs:577-591): object and probe scaled so that the
// model holds the data's photons, from the LLK pass's Σ over the unmasked pixels of |Ψ|². With
// no pixel masked anywhere that sum is every pixel's, which Parseval gives in the exit plane
// without a transform (exit_power_kernel); otherwise the LLK pass takes it.
void scale_obj_probe(ptyb_handle* h, float2* waves) {
  double calc = 0.0;
  if (h->nslice == 1 && h->nobj == 1 && h->nb_obs == (double)h->P * h->N * h->N) {
    const size_t np = (size_t)h->K * h->N * h->N;
    timed(h, kKMisc, [&] {
      exit_power_kernel<<<h->P, 256, 0, h->stream>>>(h->object, waves ? waves : h->probe,
                                                     waves ? np : 0, h->corners, h->nxo, h->K,
                                                     h->N, h->llk);
    }, h->P);
    launched(h, "exit power");
    std::vector<double> v(h->P);
    check(h, copy_sync(h, v.data(), h->llk, h->P * sizeof(double), cudaMemcpyDeviceToHost),
          "exit power");
    for (double x : v) calc += x;
  } else {
    calc = llk_pass(h, waves).nb_photons_calc;
  }
  split_scale(h, std::sqrt(h->obs_total / calc), waves);
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

// The state every handle holds past its counts (h->iobs, h->obs_total, h->max_power,
// h->nb_obs) and its corners (h->corners_h): the corners, object and probe on the device, the
// far-field phase, the twiddles, the angular-spectrum gaps of a multislice object and the
// per-frame scratch. The handle's stream exists; the caller runs this inside `guarded`.
void finish_state(ptyb_handle* h, const double* object, const double* probe, double wavelength,
                  double distance, const double* gaps) {
  const int N = h->N, nslice = h->nslice, nobj = h->nobj, nprobe = h->nprobe, K = h->K;
  const int nyo = h->nyo, nxo = h->nxo;
  const size_t plane = (size_t)N * N;
  h->corners = alloc<int2>(h, h->P);
  check(h, copy_sync(h, h->corners, h->corners_h.data(), h->P * sizeof(int2), cudaMemcpyHostToDevice),
        "corners upload");
  h->object = alloc<float2>(h, (size_t)nslice * nobj * nyo * nxo);
  upload_c64(h, object, h->object, (size_t)nslice * nobj * nyo * nxo, "object upload");
  h->probe = alloc<float2>(h, (size_t)nprobe * plane);
  upload_c64(h, probe, h->probe, (size_t)nprobe * plane, "probe upload");
  // Far-field plane phase (engine/ops.rs:17-33) and the FFT twiddles, in double.
  std::vector<float2> q(plane), tw(N);
  const double fq = M_PI / (wavelength * distance);
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
    const double width = h->pixel[1] / wavelength, ar = h->pixel[1] / h->pixel[0];
    std::vector<float2> t((size_t)(nslice - 1) * plane), ones(plane, make_float2(1.f, 0.f));
    for (int g = 0; g + 1 < nslice; ++g) {
      const double i2piz = 2.0 * M_PI * (gaps[g] / wavelength);
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
}

cudaError_t convert_counts(const void* raw, int kind, float* iobs, double* power, int* nobs,
                           int* bad, int nframe, int N, cudaStream_t s) {
  if (nframe <= 0) return cudaSuccess;
  if (kind == PTYB_COUNTS_U16)
    counts_kernel<<<nframe, 256, 0, s>>>(static_cast<const uint16_t*>(raw), 1, iobs, power, nobs,
                                         bad, N);
  else if (kind == PTYB_COUNTS_F32)
    counts_kernel<<<nframe, 256, 0, s>>>(static_cast<const float*>(raw), 0, iobs, power, nobs,
                                         bad, N);
  else
    counts_kernel<<<nframe, 256, 0, s>>>(static_cast<const double*>(raw), 0, iobs, power, nobs,
                                         bad, N);
  return cudaGetLastError();
}

thread_local std::string g_create_error;

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
  // The position sums reduce over the whole cluster once per frame: at side 256 they run on
  // clusters of 8 (measured faster than 16), whatever cluster the frame kernels take.
  h->C_sums = C;
  if (N == 256 && frame_smem_bytes<256, 8>(std::max(K, 2)) <= 227 * 1024) h->C_sums = 8;
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
      e = convert_counts(raw, scan->counts_kind, h->iobs, power, nobs, nobs + h->P, h->P, N,
                         h->stream);
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
    finish_state(h, object, probe, scan->wavelength, scan->distance, gaps);
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


cudaError_t launch_gamma(ptyb_handle* h, const GammaArgs& a, int nslot) {
  if (nslot <= 0) return cudaSuccess;
  cudaError_t e = cudaErrorInvalidValue;
  timed(h, kKGamma, [&] { e = launch_gamma_side(h->N, a, nslot, h->stream); }, nslot);
  return e;
}
}  // namespace ptyb::eng

using namespace ptyb::eng;

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


int ptyb_get_llk(ptyb_handle* h, ptyb_llk* out) {
  if (!h || !out) return PTYB_INVALID;
  return guarded(h, true, [&]() -> int {
    *out = llk_pass(h);
    return PTYB_OK;
  });
}

int ptyb_set_positions(ptyb_handle* h, const double* offsets, int32_t refine) {
  if (!h) return PTYB_INVALID;
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

int ptyb_set_object_device(ptyb_handle* h, int32_t nobj, int32_t nyo, int32_t nxo,
                           const void* src) {
  if (!h || !src) return PTYB_INVALID;
  if (nobj != h->nobj || nyo != h->nyo || nxo != h->nxo) {
    h->err = "object dims differ from the handle's";
    return PTYB_INVALID;
  }
  if (!on_device(h, src)) {
    h->err = "the object must be device memory of the handle's device";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const size_t n = (size_t)h->nobj * h->nyo * h->nxo;
    check(h, copy_sync(h, h->object, src, n * sizeof(float2), cudaMemcpyDeviceToDevice),
          "object");
    return PTYB_OK;
  });
}

int ptyb_set_objects_device(ptyb_handle* h, int32_t nslice, int32_t nyo, int32_t nxo,
                            const void* src) {
  if (!h || !src) return PTYB_INVALID;
  if (nslice != h->nslice || nyo != h->nyo || nxo != h->nxo) {
    h->err = "slice dims differ from the handle's";
    return PTYB_INVALID;
  }
  if (!on_device(h, src)) {
    h->err = "the slices must be device memory of the handle's device";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const size_t n = (size_t)h->nslice * h->nobj * h->nyo * h->nxo;
    check(h, copy_sync(h, h->object, src, n * sizeof(float2), cudaMemcpyDeviceToDevice),
          "objects");
    return PTYB_OK;
  });
}

int ptyb_set_probe_device(ptyb_handle* h, int32_t nprobe, int32_t ny, int32_t nx,
                          const void* src) {
  if (!h || !src) return PTYB_INVALID;
  if (nprobe != h->nprobe || ny != h->N || nx != h->N) {
    h->err = "probe dims differ from the handle's";
    return PTYB_INVALID;
  }
  if (!on_device(h, src)) {
    h->err = "the probe must be device memory of the handle's device";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const size_t n = (size_t)h->nprobe * h->N * h->N;
    check(h, copy_sync(h, h->probe, src, n * sizeof(float2), cudaMemcpyDeviceToDevice),
          "probe");
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
