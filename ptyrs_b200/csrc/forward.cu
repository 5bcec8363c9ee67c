// The forward model's intensities for chosen frames: `ptyb_forward_intensity` on the handle's
// scratch and `ptyb_forward_intensity_noalloc` on a fixed device array.
#include "engine.cuh"

using namespace ptyb;

// Scratch of `ptyb_forward_intensity_noalloc`: a fixed 32 MiB per device that loads this
// library, held until the process exits. Host code must not pass `g_noalloc_scratch` itself
// to a kernel (on the host it names a stand-in, not the device array): it takes the device
// address from `noalloc_scratch()`.
constexpr size_t kNoallocScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];


namespace ptyb::eng {
namespace {

// Device address of the no-alloc scratch on the current device, looked up once per device
// (with that device current) by cudaGetSymbolAddress.
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

}  // namespace
}  // namespace ptyb::eng

using namespace ptyb::eng;

extern "C" {

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
  // Scratch: the chunk's frame indices at the front (rounded up to 256 bytes), then per frame
  // its detector field (K planes) and its intensity plane. A chunk is at most the handle's
  // stack, as the allocating entry point batches, and at most what fits the array.
  const size_t plane = (size_t)h->N * h->N;
  const size_t per_frame = (size_t)h->K * plane * sizeof(float2) + plane * sizeof(float);
  auto head = [](size_t m) { return (m * sizeof(int32_t) + 255) / 256 * 256; };
  size_t fit = kNoallocScratchBytes / per_frame;
  while (fit > 0 && head(fit) + fit * per_frame > kNoallocScratchBytes) --fit;
  const int chunk = (int)std::min<size_t>(
      {(size_t)std::max(n, 1), (size_t)std::max(1, std::min(h->P, h->stack)), fit});
  if (fit < 1) {
    h->err = "one frame's field and intensity (" + std::to_string(per_frame) +
             " bytes) exceed the 32 MiB no-alloc scratch";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    unsigned char* base = nullptr;
    check(h, noalloc_scratch(h->device, &base), "cudaGetSymbolAddress");
    int* d_frames = reinterpret_cast<int*>(base);
    float2* field = reinterpret_cast<float2*>(base + head(chunk));
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

}  // extern "C"
