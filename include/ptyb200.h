/* ptyb200 — B200-native ptychography reconstruction hot path behind a C ABI.
 *
 * One handle is one reconstruction state of one scan on one CUDA device, as the reference
 * engine's `GpuPtycho` (physwkim/ptyrs, ptyrs/src/engine/gpu/mod.rs:533-881) is; the handle
 * owns every device buffer. Inputs are copied (and rounded to single precision) at create;
 * outputs are copied out on request as complex128 (interleaved re, im doubles).
 *
 * Errors follow the reference's `EngineError` (ptyrs/src/engine/mod.rs:106-123): every call
 * returns a status; PTYB_INVALID leaves the state unchanged; a device failure part-way
 * through an algorithm poisons the handle (PTYB_ABORTED for every later call that would
 * enqueue work, while downloads still work, the reference's abort gate,
 * ptyrs/src/engine/gpu/gate.rs:8-71). `ptyb_last_error` gives the message. A handle is not
 * thread-safe; several handles may coexist.
 */
#ifndef PTYB200_H
#define PTYB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum ptyb_status {
  PTYB_OK = 0,
  PTYB_INVALID = 1, /* bad shape or parameter; nothing changed */
  PTYB_GPU = 2,     /* CUDA failure; the handle is poisoned */
  PTYB_ABORTED = 3, /* an earlier call failed part-way; enqueueing calls are refused */
};

/* Counts encodings of `ptyb_scan.counts`. */
enum ptyb_counts_kind {
  PTYB_COUNTS_U16 = 0, /* uint16, 65535 masked (reference `Counts`, base/counts.rs:377-379) */
  PTYB_COUNTS_F32 = 1, /* float32, negative masked (counts past 65534 photons) */
  PTYB_COUNTS_F64 = 2, /* float64, negative masked */
};

/* A far-field scan (reference `Scan` + `Geometry`, ptyrs-py/src/lib.rs:435-463): counts
 * [nframe][ny][nx] in detector order (zero frequency at the centre), positions in metres;
 * square frames of side 64, 96, 128, 192 or 256. */
typedef struct ptyb_scan {
  int32_t nframe, ny, nx;
  int32_t counts_kind;
  const void* counts;
  const double* pos_y;
  const double* pos_x;
  double wavelength, distance, detector_pixel;
} ptyb_scan;

/* Reference `GpuOptions` (engine/gpu/mod.rs:63-112): frames per launch of the passes over the
 * whole scan (LLK, ML), 0 for the default; `cluster` the CTAs per frame of the frame kernel
 * (1 at frame side 64; 2 or 4 at 128; 8 or 16 at 256), 0 to let the engine choose. */
typedef struct ptyb_options {
  int32_t device;
  int32_t stack_size;
  int32_t cluster;
} ptyb_options;

/* Reference `RpieParams` (engine/ptycho.rs:148-186). A step flag of 0 holds that array. */
typedef struct ptyb_rpie_params {
  int32_t update_object, update_probe;
  double obj_step, probe_step, obj_alpha, probe_alpha;
  int32_t batch_size, calc_llk;
  uint64_t seed;
} ptyb_rpie_params;

enum ptyb_cost { PTYB_COST_POISSON = 0, PTYB_COST_AMPLITUDE = 1 };

/* Reference `LsqmlParams` (engine/lsqml.rs:34-53). */
typedef struct ptyb_lsqml_params {
  int32_t batch_size, cost;
  uint64_t seed;
} ptyb_lsqml_params;

/* Reference `MlParams` (engine/ptycho.rs:123-143). */
typedef struct ptyb_ml_params {
  int32_t update_object, update_probe, calc_llk, zero_phase_ramp;
} ptyb_ml_params;

/* Reference `ApParams` (engine/ptycho.rs:48-68): an update flag of 0 is the reference's `None`
 * inertia (that array stays fixed). Defaults: object on at 0.01, probe off (0.001). */
typedef struct ptyb_ap_params {
  int32_t update_object, update_probe;
  double obj_inertia, probe_inertia;
  int32_t calc_llk, zero_phase_ramp;
} ptyb_ap_params;

/* Reference `DmParams` (engine/ptycho.rs:71-96): alpha the AP/DM mix (0 plain DM, default
 * 0.02), loop_obj_probe object-then-probe updates per cycle (default 1). */
typedef struct ptyb_dm_params {
  int32_t update_object, update_probe;
  double obj_inertia, probe_inertia, alpha;
  int32_t loop_obj_probe, calc_llk, zero_phase_ramp;
} ptyb_dm_params;

/* Reference `RaarParams` (engine/ptycho.rs:98-123): beta the relaxation (default 0.9). */
typedef struct ptyb_raar_params {
  int32_t update_object, update_probe;
  double obj_inertia, probe_inertia, beta;
  int32_t loop_obj_probe, calc_llk, zero_phase_ramp;
} ptyb_raar_params;

/* Reference `Llk` (engine/ops.rs:257-277), normalised by the unmasked pixel count. */
typedef struct ptyb_llk {
  double poisson, gaussian, euclidian, nb_photons_calc;
} ptyb_llk;

/* Reference `LlkRecord` (engine/ptycho.rs:36-41); algorithm 0 = AP, 1 = DM, 2 = RAAR,
 * 3 = rPIE, 4 = ML, 5 = BH, 6 = LSQML (the reference's `Algorithm` order Ap, Dm, Raar, Rpie,
 * Ml, Bh, Lsqml). */
typedef struct ptyb_llk_record {
  int64_t cycle;
  int32_t algorithm;
  int32_t pad_;
  ptyb_llk llk;
} ptyb_llk_record;

/* One frame's LSQML step sizes (reference `LsqmlStep`, engine/lsqml.rs:56-66). */
typedef struct ptyb_lsqml_step {
  int32_t batch, frame;
  double a_far, a_obj, a_probe;
} ptyb_lsqml_step;

/* Reference `BhParams` (engine/bh.rs:29-49): frames per batch (one batch of every frame runs
 * conjugate directions across epochs, smaller batches steepest descent), pty-chi's probe
 * `rho` (the probe variable is the probe over rho·√k), the offsets' rho (under refined
 * offsets the offsets' gradient is scaled by position_rho²) and the batches' seed. */
typedef struct ptyb_bh_params {
  int32_t batch_size, pad_;
  double probe_rho, position_rho;
  uint64_t seed;
} ptyb_bh_params;

/* One batch's BH step (reference `BhStep`, engine/bh.rs:58-70): its place in the epoch, its
 * frame count, the conjugate weight beta, the step alpha, −⟨g, D⟩ and H(D, D). */
typedef struct ptyb_bh_step {
  int32_t batch, count;
  double beta, alpha, top, bottom;
} ptyb_bh_step;

typedef struct ptyb_handle ptyb_handle;

/* Reference `GpuPtycho::new` (engine/gpu/mod.rs:601-617): object complex128 [nobj][nyo][nxo],
 * probe complex128 [nprobe][ny][nx]. Positions go through PyNX's preprocessing and every
 * window must lie inside the object (PTYB_INVALID otherwise). */
int ptyb_create(const ptyb_scan* scan, const double* object, int32_t nobj, int32_t nyo,
                int32_t nxo, const double* probe, int32_t nprobe, const ptyb_options* options,
                ptyb_handle** out);

/* Reference `GpuPtycho::with_slices` (engine/gpu/mod.rs:629-660) on `Optics::with_slices`
 * (engine/propagate.rs:81-99): pty-chi's multislice object, `objects` complex128
 * [nslice][nyo][nxo] in the order the wave crosses them, `gaps` the nslice - 1 slice spacings in
 * metres, each gap an angular-spectrum propagation at the object pixel; the exit is the scan's
 * far field with its phase on the last slice. 1 <= nslice <= 16. A handle of more than one
 * slice runs LSQML alone (ptyb_rpie, ptyb_ml, ptyb_set_positions and the forward-intensity
 * calls return PTYB_INVALID on it); ptyb_get_object / ptyb_set_object read and replace slice 0
 * as the reference's `object` / `set_object` do. */
int ptyb_create_slices(const ptyb_scan* scan, const double* objects, int32_t nslice,
                       const double* gaps, int32_t nyo, int32_t nxo, const double* probe,
                       int32_t nprobe, const ptyb_options* options, ptyb_handle** out);

/* The handle's object slices (1 for ptyb_create). */
int ptyb_nslice(const ptyb_handle* h);

/* Reference `GpuPtycho::objects` (engine/gpu/mod.rs:772-779): every slice, [nslice][nyo][nxo]. */
int ptyb_get_objects(ptyb_handle* h, double* dst);
/* No counterpart in the reference (its `set_object` replaces slice 0 alone): replaces every
 * slice, [nslice][nyo][nxo], as the torch function of the adjoint needs. */
int ptyb_set_objects(ptyb_handle* h, const double* src);

/* Reference `GpuPtycho::rpie` (engine/gpu/rpie.rs:31-63). */
int ptyb_rpie(ptyb_handle* h, const ptyb_rpie_params* params, int32_t nepoch);

/* Reference `GpuPtycho::lsqml` with `ProbeVariation::none` (engine/gpu/lsqml.rs:75-121). */
int ptyb_lsqml(ptyb_handle* h, const ptyb_lsqml_params* params, int32_t nepoch,
               int32_t calc_llk);

/* Reference `GpuPtycho::ml` (engine/gpu/ml.rs:38-83). */
int ptyb_ml(ptyb_handle* h, const ptyb_ml_params* params, int32_t ncycle);

/* Reference `GpuPtycho::ap` (engine/gpu/ap.rs:28-44; CPU twin `Ptycho::ap`,
 * engine/ptycho.rs:609-641): per cycle every frame's exit waves, the magnitude projection (the
 * LLK record is of the estimate it projects), then both updates from the old arrays. Under
 * the position model (ptyb_set_positions) every frame's probe is moved by its offset, the
 * probe takes the reference's line-searched step through the move's adjoint
 * (engine/features.rs:653-725) and refined offsets take the position step from the projected
 * waves. Single slice (PTYB_INVALID otherwise). */
int ptyb_ap(ptyb_handle* h, const ptyb_ap_params* params, int32_t ncycle);

/* Reference `GpuPtycho::dm` (engine/gpu/dm.rs:32-38; CPU twin `Ptycho::dm`,
 * engine/ptycho.rs:653-691): cycle 0 of a call starts from the estimate's exit waves, later
 * cycles reflect the carried waves; the LLK record is of the estimate the cycle starts from,
 * and a recorded cycle ends by balancing Σ|O| and Σ|P|. Under the position model as ptyb_ap,
 * each update from the current probe's moves and the position sums from the carried waves.
 * Single slice. */
int ptyb_dm(ptyb_handle* h, const ptyb_dm_params* params, int32_t ncycle);

/* Reference `GpuPtycho::raar` (engine/gpu/raar.rs:17-23; CPU twin `Ptycho::raar`,
 * engine/ptycho.rs:698-730): DM's cycle with RAAR's mix of the carried projection and iterate. */
int ptyb_raar(ptyb_handle* h, const ptyb_raar_params* params, int32_t ncycle);

/* No counterpart in the reference (its engine runs one scan per call; this is the batch of
 * independent uneven-size scans): `rpie_epochs` rPIE epochs then `lsqml_epochs` LSQML epochs on
 * every handle at once, one host thread per handle and each handle on its own stream, so the
 * scans' kernels share the GPU. status[i] (may be NULL) gets handle i's return code; the call
 * returns PTYB_OK when every handle succeeded, else the first failing handle's code (the
 * others keep their results). *device_ms (may be NULL) gets the batch's device time from the
 * first launch to the last of the handles on the first handle's device, -1 if it could not be
 * taken. The handles must be distinct. */
int ptyb_batch_run(ptyb_handle* const* handles, int32_t n, const ptyb_rpie_params* rpie,
                   int32_t rpie_epochs, const ptyb_lsqml_params* lsqml, int32_t lsqml_epochs,
                   int32_t calc_llk, int32_t* status, float* device_ms);

/* Reference `ProbeVariation` (engine/opr.rs:17-88) for the LSQML calls that follow (the
 * reference passes it to `GpuPtycho::lsqml`, engine/gpu/lsqml.rs:75-121): pty-chi's OPR of
 * probe mode 0 with k eigenmodes, complex128 [k][ny][nx], weights [nframe][k] and, when not
 * NULL, the main mode's weights [nframe]; each moves with the LSQML steps when its refine flag
 * is set. k = 0 returns to the shared probe. Single slice, without the position model
 * (PTYB_INVALID otherwise). */
int ptyb_set_probe_variation(ptyb_handle* h, const double* eigenmodes, int32_t k,
                             const double* weights, int32_t refine_weights,
                             const double* intensity, int32_t refine_intensity);
/* The variation's eigenmodes, weights and main-mode weights (when modelled); NULL skips one. */
int ptyb_get_probe_variation(ptyb_handle* h, double* eigenmodes, double* weights,
                             double* intensity);

/* Reference `GpuPtycho::llk` (engine/gpu/mod.rs:871-881): normalised LLK of the estimate. */
int ptyb_get_llk(ptyb_handle* h, ptyb_llk* out);

/* The hand-written adjoint of the far-field model: the Poisson LLK sum L over the unmasked
 * pixels of the current estimate (not normalised, reference `llk` engine/ops.rs:119-154) into
 * *loss, its gradients over the object's and the probe's real and imaginary parts packed as
 * 2·∂L/∂X* = ∂L/∂Re X + i·∂L/∂Im X (reference `Ptycho::obj_grad` / `probe_grad`,
 * engine/ptycho.rs:492-515; complex128 [nyo][nxo] and [nprobe][ny][nx]) and over each frame's
 * sub-pixel offset ∂L/∂d [nframe][2] (reference `position_grad`, engine/features.rs:1055-1100),
 * all under the position model when offsets are set. Any output may be NULL; d_pos needs
 * offsets (ptyb_set_positions). On a multislice handle the model is the walk through every
 * slice and d_obj is every slice's gradient, [nslice][nyo][nxo] (d_pos must be NULL). The
 * handle's arrays are not changed. */
int ptyb_gradients(ptyb_handle* h, double* loss, double* d_obj, double* d_probe, double* d_pos);
/* ptyb_gradients with the object and probe gradients written as complex64 (interleaved float
 * re, im) to device memory of the handle's device, d_obj [nslice][nyo][nxo] and d_probe
 * [nprobe][ny][nx] (either NULL to skip), the torch function's path; loss and d_pos on the
 * host as there. No counterpart in the reference. */
int ptyb_gradients_device(ptyb_handle* h, double* loss, void* d_obj, void* d_probe,
                          double* d_pos);

/* The model intensity Σ_modes |Ψ|² of the current estimate for frames[0..n) into out[n][ny][nx]
 * in the FFT-shifted detector layout (zero frequency at [0, 0]), the far-field forward model of
 * the reference binding's `forward` (ptyrs-py/src/cpu.rs) summed over modes. */
int ptyb_forward_intensity(ptyb_handle* h, const int32_t* frames, int32_t n, float* out);

/* No counterpart in the reference. `ptyb_forward_intensity` without any device allocation,
 * for callers that cannot call cudaMalloc at that point (a host runtime whose device memory
 * is fixed once the handle exists, or a memory-capped service that must not grow its
 * footprint per request): the same model intensity, computed with the same kernel, its
 * scratch (frame list, detector field, intensities) in one fixed 32 MiB device array that
 * every GPU loading this library holds until exit. Frames are processed in chunks that fit it;
 * PTYB_INVALID when a single frame (K field planes and one intensity plane) does not. The
 * first call on a device looks the array's address up (cudaGetSymbolAddress) and keeps it for
 * the life of the process, which assumes the device's primary context lives as long (a host
 * program that calls cudaDeviceReset must not call this entry point afterwards); make that
 * first call before any stream capture. Every call shares the array and leaves its last contents there:
 * every byte a call reads it writes first, and calls that overlap on the GPU (other handles or
 * threads at the same time) race on it. */
int ptyb_forward_intensity_noalloc(ptyb_handle* h, const int32_t* frames, int32_t n, float* out);

/* Reference `GpuPtycho::set_features` with `Features::position` (engine/gpu/mod.rs:848-859,
 * engine/features.rs:20-130): per-frame sub-pixel offsets [nframe][2] (dy, dx) in object pixels
 * on top of the views' corners, modelled under Patch sampling (each frame's probe moved by its
 * offset) by rPIE, LSQML and ML, and refined when `refine` is set: rPIE and LSQML take
 * pty-chi's step (engine/ptycho.rs:1037-1085, engine/lsqml.rs:237-270), ML the step of AP and
 * DM from the magnitude projection (engine/ptycho.rs:775-842, engine/features.rs:1028-1047).
 * NULL clears them. Read back with ptyb_get_positions. */
int ptyb_set_positions(ptyb_handle* h, const double* offsets, int32_t refine);
int ptyb_get_positions(ptyb_handle* h, double* dst);

/* Reference `GpuPtycho::bh` (engine/gpu/bh.rs:29-66; CPU twin `Bh::epoch`, engine/bh.rs:
 * 645-760): pty-chi's bilinear-Hessian method on the amplitude cost, `nepoch` epochs from a
 * fresh run (epoch e's batches `random_batches(nframe, batch_size, seed, e)`), every batch
 * moving object and probe by α·D; an LLK record after every due epoch (calc_llk as
 * ptyb_lsqml's). On a multislice handle every slice and the probe are the variables (no position
 * model there: PTYB_INVALID). With ptyb_set_positions every
 * frame's probe is moved by its offset (Patch sampling, engine/bh.rs:92-275); refined offsets
 * are BH variables (their part of the gradient and the directions, 0.3·α·D_d added to them,
 * engine/bh.rs:725-745), held ones only move the probe. */
int ptyb_bh(ptyb_handle* h, const ptyb_bh_params* p, int32_t nepoch, int32_t calc_llk);
/* Reference `GpuPtycho::bh_steps` (engine/gpu/bh.rs:68-72): the last epoch's steps. */
int ptyb_bh_steps_len(ptyb_handle* h);
int ptyb_bh_steps(ptyb_handle* h, ptyb_bh_step* dst, int32_t cap);

/* Live ingestion: the reference's pinned host ring of frames and the thread that streams it
 * into the device store (live/ring.rs:1-31), with the position table the uploader joins each
 * frame with (live/pos.rs). Workers reserve a slot (ptyb_live_reserve, which blocks while the
 * ring is full), write the frame's counts into its pinned host memory and commit it with the
 * frame's uid; positions arrive by uid on their own (ptyb_live_position). The uploader takes
 * committed frames in sequence order: a frame lands once its position is in (the next place of
 * the device store, in landing order, converted on the device as ptyb_create converts counts);
 * one whose position is not valid (a coordinate not finite or |pos| > 1e10) is dropped at once;
 * one still without its position is dropped pos_wait_ns after its commit, or sooner as soon as
 * a worker waits for its slot. A slot is released only after its copy to the device has
 * completed. The uploader copies runs of landed frames that sit in consecutive ring slots (at most
 * `batch` frames, 0 for 32) in one copy and one conversion launch, as soon as they are joined.
 * ptyb_live_handle makes a reconstruction handle over the frames landed so far. */
typedef struct ptyb_live ptyb_live;

typedef struct ptyb_live_params {
  int32_t device, n, counts_kind; /* frame side; PTYB_COUNTS_U16 or PTYB_COUNTS_F32 */
  int32_t slots, capacity;        /* ring slots; device store places (frames that can land) */
  int32_t batch;                  /* most frames in one copy to the device (0: 32) */
  double wavelength, distance, detector_pixel;
  int64_t pos_wait_ns;
} ptyb_live_params;

/* Frames committed, landed (given a store place) and ready (copied and converted); dropped
 * without a position (pos_wait_ns passed, or, dropped_crowded of them, a worker needed the
 * slot first), with an invalid position, or with the device store full; reservations that
 * waited for a slot; frames that reached the head of the ring before their position; copy
 * batches queued (reference live/ring.rs:570-600, UploadReport). */
typedef struct ptyb_live_stats {
  int64_t committed, landed, ready, dropped_no_position, dropped_crowded, dropped_invalid,
      dropped_full, stalls, pos_waits, batches;
} ptyb_live_stats;

int ptyb_live_create(const ptyb_live_params* p, ptyb_live** out);
/* A slot for the next frame (sequence number *seq) and its pinned host frame to fill. */
int ptyb_live_reserve(ptyb_live* l, int64_t* seq, void** frame);
int ptyb_live_commit(ptyb_live* l, int64_t seq, int64_t uid);
/* The position (metres) of frame `uid`. */
int ptyb_live_position(ptyb_live* l, int64_t uid, double y, double x);
/* Waits (at most timeout_ms) until every committed frame has landed or dropped and every
 * landed frame's copy and conversion has completed; PTYB_GPU on a device failure, PTYB_INVALID
 * on the timeout. */
int ptyb_live_flush(ptyb_live* l, int32_t timeout_ms);
int ptyb_live_get_stats(ptyb_live* l, ptyb_live_stats* out);
/* The uids and positions of the landed frames in landing order (at most cap; any of the three
 * arrays may be NULL); returns how many were written. */
int ptyb_live_landed(ptyb_live* l, int64_t* uids, double* y, double* x, int32_t cap);
/* A handle (as ptyb_create, on the ring's device: options->device is not read) over the frames
 * landed and converted so far, in landing order, with their positions; the counts are copied on
 * the device. *nframe (if not NULL) receives the handle's frame count. */
int ptyb_live_handle(ptyb_live* l, const double* object, int32_t nyo, int32_t nxo,
                     const double* probe, int32_t nprobe, const ptyb_options* options,
                     ptyb_handle** out, int32_t* nframe);
const char* ptyb_live_last_error(ptyb_live* l);
void ptyb_live_destroy(ptyb_live* l);

/* Scan files (reference ptyrs/src/io/cxi.rs:130-200 `read_cxi`): the CXI layout PyNX's
 * `save_ptycho_data_cxi` writes, read by the library's own HDF5 reader (libhdf5's default
 * layouts: superblocks 0-3, symbol-table and compact groups, soft links, contiguous, compact and
 * chunked datasets with deflate and shuffle). Counts are `u16 [nframe][ny][nx]` in detector
 * order with 65535 masked: raw u16 data with the detector mask applied, or float data under the
 * reference's `Counts::from_f64` rule (masked or negative → 65535, a non-integer or a value past
 * 65534 refused). Positions come from the f32 translation rows (x, y), the wavelength from the
 * energy by PyNX's 12.3984 keV·Å and 1.60218e-16 J/keV. The arrays are the library's; free the
 * scan with ptyb_free_cxi. A handle takes counts, y and x as they are (counts_kind
 * PTYB_COUNTS_U16). */
typedef struct ptyb_cxi_scan {
  int32_t nframe, ny, nx, pad_;
  uint16_t* counts;
  double* y; /* [nframe] metres */
  double* x;
  double wavelength, distance, detector_pixel;
} ptyb_cxi_scan;
int ptyb_read_cxi(const char* path, ptyb_cxi_scan* out);
void ptyb_free_cxi(ptyb_cxi_scan* s);

/* Reference `read_ptyr` (ptyrs/src/io/ptyr.rs): the object and probe of a PtyPy `.ptyr`
 * reconstruction (the one storage under content/obj and content/probe, complex64 or
 * complex128), as complex128 interleaved `[obj_shape]` and `[probe_shape]`, with the object
 * storage's pixel size and origin ([y, x]). Free with ptyb_free_ptyr. */
typedef struct ptyb_ptyr {
  int32_t obj_shape[3], probe_shape[3];
  double* object;
  double* probe;
  double psize[2], origin[2];
} ptyb_ptyr;
int ptyb_read_ptyr(const char* path, ptyb_ptyr* out);
void ptyb_free_ptyr(ptyb_ptyr* r);
/* The reason the last ptyb_read_* call of this thread failed. */
const char* ptyb_io_last_error(void);

/* Reference `GpuPtycho::{object, probe, set_object}` (engine/gpu/mod.rs:763-817). */
int ptyb_get_object(ptyb_handle* h, double* dst);
int ptyb_get_probe(ptyb_handle* h, double* dst);
int ptyb_set_object(ptyb_handle* h, const double* src);
int ptyb_set_probe(ptyb_handle* h, const double* src);

/* Reference `GpuPtycho::set_object_device` (engine/gpu/mod.rs:795-805): the object (of a
 * multislice object its first slice) from `src`, complex64 [nobj][nyo][nxo] (interleaved
 * float re, im) in device memory of the handle's device whose writes have finished; the copy
 * is waited for, so `src` may be released or rewritten on return. PTYB_INVALID, changing
 * nothing, when the dims differ from the handle's or `src` is not memory of that device. */
int ptyb_set_object_device(ptyb_handle* h, int32_t nobj, int32_t nyo, int32_t nxo,
                           const void* src);
/* No counterpart in the reference: as ptyb_set_object_device for every slice
 * ([nslice][nyo][nxo]) and for the probe ([nprobe][ny][nx]). */
int ptyb_set_objects_device(ptyb_handle* h, int32_t nslice, int32_t nyo, int32_t nxo,
                            const void* src);
int ptyb_set_probe_device(ptyb_handle* h, int32_t nprobe, int32_t ny, int32_t nx,
                          const void* src);

/* Window corners [nframe][2] (oy, ox) of the address table (reference `AddrTable`,
 * base/addr.rs:35-81). */
int ptyb_corners(ptyb_handle* h, int32_t* dst);

/* Reference `GpuPtycho::history` / `cycle` (engine/gpu/mod.rs:818-864). */
int ptyb_history_len(ptyb_handle* h);
int ptyb_history(ptyb_handle* h, ptyb_llk_record* dst, int32_t cap);
int64_t ptyb_cycle(ptyb_handle* h);

/* Reference `GpuPtycho::lsqml_steps`: the steps of the last LSQML epoch, one per frame in
 * batch order. */
int ptyb_lsqml_steps_len(ptyb_handle* h);
int ptyb_lsqml_steps(ptyb_handle* h, ptyb_lsqml_step* dst, int32_t cap);
/* Of a multislice handle, the object steps of slices 1.. for the same frames,
 * [ptyb_lsqml_steps_len][nslice - 1] (the reference `LsqmlStep::a_obj` of those slices). */
int ptyb_lsqml_slice_steps(ptyb_handle* h, double* dst);

/* Reference `GpuPtycho::synchronize` (engine/gpu/mod.rs:865-870). */
int ptyb_synchronize(ptyb_handle* h);

/* Host-only (no device needed): reference `random_batches` (engine/batch.rs:18-38), the
 * frames of `epoch` in seeded sorted batches of `size`, concatenated into order[nframe]. */
int ptyb_random_batches(int32_t nframe, int32_t size, uint64_t seed, uint64_t epoch,
                        int32_t* order);

/* Host-only: PyNX position preprocessing and the window corners [nframe][2] (oy, ox) of
 * positions in metres on an object pixel (pixel_y, pixel_x) (reference
 * `Positions::pynx_preprocess` + `AddrTable::new`, base/positions.rs:274-315,
 * base/addr.rs:35-127); PTYB_INVALID when a window leaves the object. */
int ptyb_view_corners(const double* y, const double* x, int32_t nframe, double pixel_y,
                      double pixel_x, int32_t ny, int32_t nx, int32_t nyo, int32_t nxo,
                      int32_t* corners);

/* Per-kernel device timing: `on` resets the totals and brackets every later launch of this
 * handle with CUDA events on its stream (kernel names by ptyb_kernel_name). */
int ptyb_set_timing(ptyb_handle* h, int32_t on);
int32_t ptyb_kernel_kinds(void);
const char* ptyb_kernel_name(int32_t kind);
int ptyb_kernel_times(ptyb_handle* h, double* ms, int64_t* launches, int32_t cap);
/* The frames the timed launches of each kind processed (0 for kinds not per frame). */
int ptyb_kernel_frames(ptyb_handle* h, int64_t* frames, int32_t cap);

/* Device time (ms, CUDA events on the handle's stream) of the last rPIE / LSQML / ML call. */
double ptyb_last_call_ms(ptyb_handle* h);

/* Device-side launch count of this handle's own kernels since create (observability). */
int64_t ptyb_launches(ptyb_handle* h);

const char* ptyb_last_error(ptyb_handle* h);
void ptyb_destroy(ptyb_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* PTYB200_H */
