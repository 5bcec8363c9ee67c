// Live ingestion (reference live/ring.rs:1-31, live/pos.rs): a pinned host ring of frames,
// written by workers under reservations and committed with each frame's uid, a table of
// positions by uid, and an uploader thread that lands committed frames in sequence order into
// a device store once their position is in, converting each on the device, and releases a
// slot only after the copy out of it has completed.
//
// Sequencing: `next` counts reservations; frame `seq` lives in slot seq % slots and may be
// reserved only when seq < released + slots. `done[slot] == seq + 1` publishes a commit. The
// uploader joins frames below `joined` (landed, or dropped) and keeps each landed frame's
// completion event in `inflight`; it advances `released` past a frame once every copy queued
// up to it has completed (a dropped frame releases with the frames before it).
#include <chrono>
#include <condition_variable>
#include <deque>
#include <unordered_map>

#include "engine.cuh"

using namespace ptyb;

struct ptyb_live {
  // Set at create.
  int device = 0, N = 0, kind = 0, slots = 0, capacity = 0, batch = 0;
  size_t frame_bytes = 0;
  double wavelength = 0, distance = 0, detector_pixel = 0;
  int64_t pos_wait_ns = 0;
  unsigned char* ring = nullptr;  // [slots][frame_bytes] pinned host
  // Device store: landed frames in landing order.
  unsigned char* raw = nullptr;   // [capacity][frame_bytes]
  float* iobs = nullptr;          // [capacity][N][N] FFT-shifted, masked −1
  double* power = nullptr;        // [capacity]
  int* nobs = nullptr;            // [capacity]: unmasked counts
  int* bad = nullptr;             // [capacity]: at a copy batch's first place, set by a
                                  // non-finite unmasked value in the batch
  cudaStream_t stream = nullptr;
  std::vector<cudaEvent_t> events;  // [slots]: a copy batch's completion, by its first slot
  // Shared state, under `mu`.
  std::mutex mu;
  std::condition_variable cv;
  int64_t next = 0, released = 0, joined = 0;
  std::vector<int64_t> done, uid;  // [slots]
  std::vector<std::chrono::steady_clock::time_point> t_commit;
  std::unordered_map<int64_t, std::pair<double, double>> positions;  // uid → (y, x)
  std::unordered_map<int64_t, bool> invalid;                         // uid → invalid arrival
  struct Flight {
    int64_t end;        // the frames below this sequence number are joined with it
    int64_t landed;     // frames of a copy batch (0: a dropped frame)
    cudaEvent_t event;  // the batch's copy and conversion; null for a dropped frame
  };
  std::deque<Flight> inflight;
  bool issuing = false;             // the uploader is queueing joined batches
  std::vector<int64_t> landed_uid;  // [landed]
  std::vector<double> landed_y, landed_x;
  int64_t ready = 0;                // landed frames whose copy and conversion completed
  int64_t committed = 0, dropped_no_position = 0, dropped_crowded = 0, dropped_invalid = 0,
          dropped_full = 0, stalls = 0, pos_waits = 0, batches = 0;
  int64_t waited_seq = -1;          // the last head frame counted in pos_waits
  bool stop = false, failed = false;
  std::string err;
  std::thread uploader;
};

namespace ptyb::eng {
namespace {

constexpr double kPosLimit = 1e10;

// Releases the batches and dropped frames at the front of the flight list whose copies have
// completed, in order. Called with `mu` held.
bool retire(ptyb_live* l) {
  bool any = false;
  while (!l->inflight.empty()) {
    auto& f = l->inflight.front();
    if (f.event) {
      const cudaError_t e = cudaEventQuery(f.event);
      if (e == cudaErrorNotReady) break;
      if (e != cudaSuccess) {
        l->failed = true;
        l->err = std::string("live copy: ") + cudaGetErrorString(e);
        break;
      }
      l->ready += f.landed;
    }
    l->released = f.end;
    l->inflight.pop_front();
    any = true;
  }
  return any;
}

// One pass's joined frames: a copy batch of n frames from ring slots slot0 .. slot0 + n − 1 to
// store places place0 .., or (n = 0) a dropped frame.
struct Plan {
  int64_t end, n;
  int slot0;
  int64_t place0;
};

void upload_loop(ptyb_live* l) {
  cudaSetDevice(l->device);
  const size_t np = (size_t)l->N * l->N;
  std::vector<Plan> plans;
  std::vector<cudaEvent_t> evs;
  std::unique_lock<std::mutex> lock(l->mu);
  while (!l->stop) {
    if (retire(l)) l->cv.notify_all();  // slots released: reservations may go on
    if (l->failed) {
      l->cv.notify_all();
      break;
    }
    // Join committed frames in sequence order (reference live/ring.rs:830-880).
    plans.clear();
    int64_t hold_ns = -1;  // the head frame waits this long at most for its position
    for (;;) {
      const int64_t seq = l->joined;
      const int slot = (int)(seq % l->slots);
      if (l->done[slot] != seq + 1) break;
      const int64_t uid = l->uid[slot];
      const auto pos = l->positions.find(uid);
      if (pos != l->positions.end()) {
        const int64_t place = (int64_t)l->landed_uid.size();
        if (place >= l->capacity) {
          ++l->dropped_full;
          plans.push_back({seq + 1, 0, slot, 0});
        } else {
          Plan* run = plans.empty() ? nullptr : &plans.back();
          if (run && run->n > 0 && run->n < l->batch && run->slot0 + run->n == slot) {
            ++run->n;
            run->end = seq + 1;
          } else {
            plans.push_back({seq + 1, 1, slot, place});
          }
          l->landed_uid.push_back(uid);
          l->landed_y.push_back(pos->second.first);
          l->landed_x.push_back(pos->second.second);
        }
        l->positions.erase(pos);
      } else if (l->invalid.erase(uid)) {
        ++l->dropped_invalid;
        plans.push_back({seq + 1, 0, slot, 0});
      } else {
        // a worker waits for this frame's slot (reference live/ring.rs:850-857)
        const bool crowded = l->next > seq + l->slots;
        const int64_t waited = std::chrono::duration_cast<std::chrono::nanoseconds>(
                                   std::chrono::steady_clock::now() - l->t_commit[slot])
                                   .count();
        if (!crowded && waited <= l->pos_wait_ns) {
          if (l->waited_seq != seq) {
            ++l->pos_waits;
            l->waited_seq = seq;
          }
          hold_ns = l->pos_wait_ns - waited + 1;
          break;
        }
        ++l->dropped_no_position;
        l->dropped_crowded += crowded;
        plans.push_back({seq + 1, 0, slot, 0});
      }
      ++l->joined;
    }
    if (!plans.empty()) {
      // Queue the batches outside the lock: their slots stay committed and unreleased, and no
      // pass of this thread starts two batches at one slot.
      l->issuing = true;
      lock.unlock();
      evs.assign(plans.size(), nullptr);
      cudaError_t e = cudaSuccess;
      for (size_t i = 0; i < plans.size() && e == cudaSuccess; ++i) {
        const Plan& p = plans[i];
        if (p.n == 0) continue;
        e = cudaMemcpyAsync(l->raw + p.place0 * l->frame_bytes,
                            l->ring + (size_t)p.slot0 * l->frame_bytes, p.n * l->frame_bytes,
                            cudaMemcpyHostToDevice, l->stream);
        if (e == cudaSuccess)
          e = convert_counts(l->raw + p.place0 * l->frame_bytes, l->kind, l->iobs + p.place0 * np,
                             l->power + p.place0, l->nobs + p.place0, l->bad + p.place0,
                             (int)p.n, l->N, l->stream);
        if (e == cudaSuccess) e = cudaEventRecord(l->events[p.slot0], l->stream);
        evs[i] = l->events[p.slot0];
      }
      lock.lock();
      l->issuing = false;
      if (e != cudaSuccess) {
        l->failed = true;
        l->err = std::string("live upload: ") + cudaGetErrorString(e);
        l->cv.notify_all();
        break;
      }
      for (size_t i = 0; i < plans.size(); ++i) {
        l->inflight.push_back({plans[i].end, plans[i].n, plans[i].n ? evs[i] : nullptr});
        l->batches += plans[i].n > 0;
      }
      l->cv.notify_all();
      continue;
    }
    // Nothing joined: sleep until a commit, a position or a waiting worker, polling the copies
    // in flight and the head frame's wait.
    int64_t ns = l->inflight.empty() ? 2000000 : 50000;
    if (hold_ns >= 0) ns = std::min<int64_t>(ns, std::max<int64_t>(hold_ns, 1000));
    l->cv.wait_for(lock, std::chrono::nanoseconds(ns));
  }
}

// Records `what` as the ring's last error; `mu` held.
int live_fail(ptyb_live* l, const std::string& what) {
  l->err = what;
  return PTYB_INVALID;
}

int live_fail_locked(ptyb_live* l, const std::string& what) {
  std::lock_guard<std::mutex> lock(l->mu);
  return live_fail(l, what);
}

}  // namespace
}  // namespace ptyb::eng

using namespace ptyb::eng;

extern "C" {

int ptyb_live_create(const ptyb_live_params* p, ptyb_live** out) {
  if (!out) return PTYB_INVALID;
  *out = nullptr;
  g_create_error.clear();
  if (!p || !(p->n == 64 || p->n == 96 || p->n == 128 || p->n == 192 || p->n == 256) ||
      !(p->counts_kind == PTYB_COUNTS_U16 || p->counts_kind == PTYB_COUNTS_F32) ||
      p->slots < 1 || p->capacity < 1 || p->batch < 0 || p->pos_wait_ns < 0 ||
      !(p->wavelength > 0 && p->distance > 0 && p->detector_pixel > 0)) {
    g_create_error = "live: a side of 64, 96, 128, 192 or 256, u16 or f32 counts, slots and "
                     "capacity >= 1, batch >= 0, pos_wait_ns >= 0 and a positive geometry";
    return PTYB_INVALID;
  }
  auto* l = new ptyb_live();
  l->device = p->device;
  l->N = p->n;
  l->kind = p->counts_kind;
  l->slots = p->slots;
  l->capacity = p->capacity;
  l->batch = p->batch > 0 ? p->batch : 32;
  l->frame_bytes = (size_t)p->n * p->n * (p->counts_kind == PTYB_COUNTS_U16 ? 2 : 4);
  l->wavelength = p->wavelength;
  l->distance = p->distance;
  l->detector_pixel = p->detector_pixel;
  l->pos_wait_ns = p->pos_wait_ns;
  l->done.assign(l->slots, 0);
  l->uid.assign(l->slots, 0);
  l->t_commit.resize(l->slots);
  auto bail = [&](const char* what, cudaError_t e) {
    g_create_error = std::string(what) + ": " + cudaGetErrorString(e);
    ptyb_live_destroy(l);
    return PTYB_GPU;
  };
  cudaError_t e = cudaSetDevice(l->device);
  if (e != cudaSuccess) return bail("cudaSetDevice", e);
  const size_t np = (size_t)l->N * l->N;
  if ((e = cudaMallocHost(&l->ring, l->slots * l->frame_bytes)) != cudaSuccess)
    return bail("cudaMallocHost", e);
  if ((e = cudaMalloc(&l->raw, l->capacity * l->frame_bytes)) != cudaSuccess ||
      (e = cudaMalloc(&l->iobs, l->capacity * np * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc(&l->power, l->capacity * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc(&l->nobs, l->capacity * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&l->bad, l->capacity * sizeof(int))) != cudaSuccess)
    return bail("cudaMalloc", e);
  if ((e = cudaMemset(l->bad, 0, l->capacity * sizeof(int))) != cudaSuccess)
    return bail("cudaMemset", e);
  if ((e = cudaStreamCreateWithFlags(&l->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail("cudaStreamCreate", e);
  l->events.assign(l->slots, nullptr);
  for (auto& ev : l->events)
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
      return bail("cudaEventCreate", e);
  try {
    l->uploader = std::thread(upload_loop, l);
  } catch (const std::exception& ex) {
    g_create_error = std::string("host: ") + ex.what();
    ptyb_live_destroy(l);
    return PTYB_GPU;
  }
  *out = l;
  return PTYB_OK;
}

int ptyb_live_reserve(ptyb_live* l, int64_t* seq, void** frame) {
  if (!l || !seq || !frame) return PTYB_INVALID;
  std::unique_lock<std::mutex> lock(l->mu);
  const int64_t s = l->next++;
  if (s >= l->released + l->slots) {
    ++l->stalls;
    l->cv.notify_all();  // the uploader may be holding this slot for a position
    l->cv.wait(lock, [&] { return l->stop || l->failed || s < l->released + l->slots; });
  }
  if (l->stop || l->failed) {
    l->err = l->failed ? l->err : "live: stopped";
    return l->failed ? PTYB_GPU : PTYB_INVALID;
  }
  *seq = s;
  *frame = l->ring + (size_t)(s % l->slots) * l->frame_bytes;
  return PTYB_OK;
}

int ptyb_live_commit(ptyb_live* l, int64_t seq, int64_t uid) {
  if (!l) return PTYB_INVALID;
  std::lock_guard<std::mutex> lock(l->mu);
  if (seq < l->released || seq >= l->next) return live_fail(l, "live: not a reserved sequence");
  const int slot = (int)(seq % l->slots);
  if (l->done[slot] == seq + 1) return live_fail(l, "live: committed twice");
  l->uid[slot] = uid;
  l->t_commit[slot] = std::chrono::steady_clock::now();
  l->done[slot] = seq + 1;
  ++l->committed;
  l->cv.notify_all();
  return PTYB_OK;
}

int ptyb_live_position(ptyb_live* l, int64_t uid, double y, double x) {
  if (!l) return PTYB_INVALID;
  std::lock_guard<std::mutex> lock(l->mu);
  // a position that is not a scan position (reference live/pos.rs: Entry::Invalid)
  if (!(std::isfinite(y) && std::isfinite(x) && std::fabs(y) <= kPosLimit &&
        std::fabs(x) <= kPosLimit))
    l->invalid[uid] = true;
  else
    l->positions[uid] = {y, x};
  l->cv.notify_all();
  return PTYB_OK;
}

int ptyb_live_flush(ptyb_live* l, int32_t timeout_ms) {
  if (!l) return PTYB_INVALID;
  std::unique_lock<std::mutex> lock(l->mu);
  const bool ok = l->cv.wait_for(lock, std::chrono::milliseconds(std::max(timeout_ms, 0)), [&] {
    if (l->failed) return true;
    const int slot = (int)(l->joined % l->slots);
    const bool all_joined = l->joined == l->next || l->done[slot] != l->joined + 1;
    return all_joined && !l->issuing && l->inflight.empty();
  });
  if (l->failed) return PTYB_GPU;
  if (!ok) return live_fail(l, "live: flush timed out");
  return PTYB_OK;
}

int ptyb_live_get_stats(ptyb_live* l, ptyb_live_stats* out) {
  if (!l || !out) return PTYB_INVALID;
  std::lock_guard<std::mutex> lock(l->mu);
  out->committed = l->committed;
  out->landed = (int64_t)l->landed_uid.size();
  out->ready = l->ready;
  out->dropped_no_position = l->dropped_no_position;
  out->dropped_crowded = l->dropped_crowded;
  out->dropped_invalid = l->dropped_invalid;
  out->dropped_full = l->dropped_full;
  out->stalls = l->stalls;
  out->pos_waits = l->pos_waits;
  out->batches = l->batches;
  return PTYB_OK;
}

int ptyb_live_landed(ptyb_live* l, int64_t* uids, double* y, double* x, int32_t cap) {
  if (!l || cap < 0) return PTYB_INVALID;
  std::lock_guard<std::mutex> lock(l->mu);
  const int n = std::min<int>(cap, (int)l->landed_uid.size());
  if (uids) std::copy(l->landed_uid.begin(), l->landed_uid.begin() + n, uids);
  if (y) std::copy(l->landed_y.begin(), l->landed_y.begin() + n, y);
  if (x) std::copy(l->landed_x.begin(), l->landed_x.begin() + n, x);
  return n;
}

int ptyb_live_handle(ptyb_live* l, const double* object, int32_t nyo, int32_t nxo,
                     const double* probe, int32_t nprobe, const ptyb_options* options,
                     ptyb_handle** out, int32_t* nframe) {
  if (!out) return PTYB_INVALID;
  *out = nullptr;
  if (nframe) *nframe = 0;
  if (!l || !object || !probe) return PTYB_INVALID;
  std::vector<double> y, x;
  int64_t n = 0;
  {
    std::lock_guard<std::mutex> lock(l->mu);
    if (l->failed) return PTYB_GPU;
    n = l->ready;
    y.assign(l->landed_y.begin(), l->landed_y.begin() + n);
    x.assign(l->landed_x.begin(), l->landed_x.begin() + n);
  }
  const int N = l->N;
  if (n < 1) return live_fail_locked(l, "live: no frame has landed");
  if (nprobe <= 0 || nprobe > kMaxModes || nyo < N || nxo < N)
    return live_fail_locked(l, "live: 1-4 probe modes and an object >= the frame");
  const int C = cluster_for(N, nprobe, options ? options->cluster : 0);
  if (C == 0) return live_fail_locked(l, "live: the frame's modes do not fit one cluster");
  auto* h = new ptyb_handle();
  h->device = l->device;
  h->P = (int)n;
  h->N = N;
  h->nprobe = nprobe;
  h->nobj = 1;
  h->K = nprobe;
  h->nyo = nyo;
  h->nxo = nxo;
  h->C = C;
  h->C_sums = C;
  if (N == 256 && frame_smem_bytes<256, 8>(std::max(nprobe, 2)) <= 227 * 1024) h->C_sums = 8;
  h->stack = options && options->stack_size > 0 ? options->stack_size : 512;
  h->nslice = 1;
  h->log_stride = 3;
  const double lz = l->wavelength * l->distance;
  h->pixel[0] = h->pixel[1] = lz / (N * l->detector_pixel);
  const std::vector<double> py = pynx_axis(y, h->pixel[0]), px = pynx_axis(x, h->pixel[1]);
  std::string err;
  if (!corners_of(py, px, h->pixel, N, N, nyo, nxo, &h->corners_h, &err)) {
    delete h;
    return live_fail_locked(l, "live: " + err);
  }
  const int rc = guarded(h, true, [&]() -> int {
    check(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    const size_t plane = (size_t)N * N;
    h->iobs = alloc<float>(h, (size_t)n * plane);
    // the landed frames are converted (ready): the store's places 0 .. n − 1 as they are
    check(h, copy_sync(h, h->iobs, l->iobs, (size_t)n * plane * sizeof(float),
                       cudaMemcpyDeviceToDevice),
          "live counts");
    std::vector<double> pw(n);
    std::vector<int> nb(n), bad(n);
    check(h, copy_sync(h, pw.data(), l->power, n * sizeof(double), cudaMemcpyDeviceToHost),
          "live counts");
    check(h, copy_sync(h, nb.data(), l->nobs, n * sizeof(int), cudaMemcpyDeviceToHost),
          "live counts");
    check(h, copy_sync(h, bad.data(), l->bad, n * sizeof(int), cudaMemcpyDeviceToHost),
          "live counts");
    if (std::any_of(bad.begin(), bad.end(), [](int b) { return b != 0; })) {
      h->err = "counts must be finite";
      return PTYB_INVALID;
    }
    for (int64_t f = 0; f < n; ++f) {
      h->obs_total += pw[f];
      h->max_power = std::max(h->max_power, pw[f]);
      h->nb_obs += nb[f];
    }
    finish_state(h, object, probe, l->wavelength, l->distance, nullptr);
    return PTYB_OK;
  });
  if (rc != PTYB_OK) {
    live_fail_locked(l, h->err);
    ptyb_destroy(h);
    return rc;
  }
  *out = h;
  if (nframe) *nframe = h->P;
  return PTYB_OK;
}

const char* ptyb_live_last_error(ptyb_live* l) {
  return l ? l->err.c_str() : g_create_error.c_str();
}

void ptyb_live_destroy(ptyb_live* l) {
  if (!l) return;
  {
    std::lock_guard<std::mutex> lock(l->mu);
    l->stop = true;
    l->cv.notify_all();
  }
  if (l->uploader.joinable()) l->uploader.join();
  cudaSetDevice(l->device);
  if (l->stream) cudaStreamSynchronize(l->stream);
  for (auto ev : l->events)
    if (ev) cudaEventDestroy(ev);
  if (l->stream) cudaStreamDestroy(l->stream);
  if (l->ring) cudaFreeHost(l->ring);
  if (l->raw) cudaFree(l->raw);
  if (l->iobs) cudaFree(l->iobs);
  if (l->power) cudaFree(l->power);
  if (l->nobs) cudaFree(l->nobs);
  if (l->bad) cudaFree(l->bad);
  delete l;
}

}  // extern "C"
