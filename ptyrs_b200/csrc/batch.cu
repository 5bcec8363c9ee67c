// Many independent scans at once: `ptyb_batch_run` over their handles, one host thread and
// stream each, with the batch's device time.
#include "engine.cuh"

using namespace ptyb;

namespace ptyb::eng {
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
}  // namespace ptyb::eng

using namespace ptyb::eng;

extern "C" {

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

}  // extern "C"
