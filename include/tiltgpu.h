/*
 * tiltgpu.h -- C ABI of libtiltgpu.so, the B200 (sm_100a) implementation of the
 * imod-rs `tilt` reconstruction path: R-weighted radial filtering of every
 * projection row, cosine stretch, weighted back-projection with linear
 * interpolation, and the SIRT reproject -> difference -> backproject loop, with
 * projections and volume resident in device memory.
 *
 * Plain C types only (no CUDA or torch types cross this boundary).  Every
 * function returns a tg_status (0 = TG_OK, negative = error); the library never
 * falls back to a CPU implementation.  A session is single-thread-affine; the
 * server object (tg_server_*) is thread-safe.
 *
 * Reference interfaces that each entry point replaces are cited as
 * file:line inside the imod-rs project.
 */
#ifndef TILTGPU_H
#define TILTGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TG_ABI_VERSION 1

typedef enum {
  TG_OK = 0,
  TG_ERR_INVALID_ARG = -1,  /* bad sizes/pointers/options */
  TG_ERR_OOM = -2,          /* device allocation failed */
  TG_ERR_CUDA = -3,         /* a CUDA call failed (message via tg_last_error) */
  TG_ERR_TIMEOUT = -4,      /* a bounded device wait gave up */
  TG_ERR_BUDGET = -5,       /* job larger than the server's memory budget */
  TG_ERR_UNSUPPORTED = -6,  /* option combination not implemented */
  TG_ERR_NO_DEVICE = -7,    /* no CUDA device / not sm_100 */
  TG_ERR_PANIC = -8,        /* input on which the reference panics (e.g. fewer
                               tilt angles than views with cosine stretch on) */
  TG_ERR_NOT_READY = -9,    /* tg_server_wait: job still running */
  TG_ERR_NOT_FOUND = -10,   /* unknown job id */
  TG_ERR_CANCELLED = -11,   /* job dropped by tg_server_destroy before admission */
  TG_ERR_RANGE = -12        /* FP16 staging: a filtered projection or SIRT residual exceeds the
                               FP16 range (|v| >= 65520), e.g. a diverging SIRT run; the
                               volume is not valid.  FP32/BF16 staging never report it. */
} tg_status;

/* Fill modes of apps/tilt/src/main.rs:122-128 */
typedef enum { TG_FILL_MEAN = 0, TG_FILL_ZERO = 1, TG_FILL_EDGE = 2 } tg_fill_mode;

/* Storage precision of the filtered projections staged for back-projection
 * (accumulation is always FP32). */
typedef enum { TG_STORE_FP32 = 0, TG_STORE_FP16 = 1, TG_STORE_BF16 = 2 } tg_storage;

/* Geometry of one tilt series.  Replaces the dimension handling of
 * apps/tilt/src/main.rs:560-571 and the per-view inputs of 550, 656-700. */
typedef struct {
  int32_t nx, ny, nz;        /* input stack: width, rows (tilt-axis direction), views */
  int32_t out_nx;            /* output width  (--width);     <=0: nx  */
  int32_t out_nz;            /* output thickness (-z);       <=0: nx  */
  int32_t n_angles;          /* angles as read from the .tlt file (degrees, f32) */
  const float *angles;
  int32_t n_xtilt;           /* --xtilt-file values (degrees) or 0/NULL */
  const float *xtilt;
  int32_t n_zfactor;         /* --zfactor-file values or 0/NULL */
  const float *zfactor;
  int32_t n_local;           /* --local-file rows (view, x, y, dx, dy) or 0/NULL */
  const float *local;
  int32_t has_local;         /* --local-file given (even if it held no rows) */
} tg_geometry;

/* Options of apps/tilt/src/main.rs:18-120 (defaults via tg_options_default). */
typedef struct {
  float radial_cutoff;       /* --radial cutoff   (0.35) */
  float radial_falloff;      /* --radial falloff  (0.05) */
  int32_t hamming;           /* --hamming */
  int32_t exact_filter_size; /* --exact-filter-size, <=0: none */
  int32_t no_weight;         /* --no-weight */
  int32_t fill_mode;         /* tg_fill_mode (--fill-mode) */
  int32_t no_cosine_stretch; /* --no-cosine-stretch */
  int32_t cosine_cubic;      /* --cosine-interp cubic */
  float max_cosine_tilt;     /* --max-cosine-tilt (80) */
  int32_t log_transform;     /* --log */
  int32_t sirt_iters;        /* --sirt (0 = WBP) */
  float sirt_relax;          /* --sirt-relax (1.0) */
  int32_t fake_sirt;         /* --fake-sirt */
  float densweight, outscale, outadd;  /* output transform (1, 1, 0) */
  int32_t gpu_compat;        /* --gpu: semantics of apps/tilt/src/backproject.wgsl */
  int32_t storage;           /* tg_storage of the staged filtered projections */
  int32_t device;            /* CUDA device ordinal */
  int32_t use_graphs;        /* capture each SIRT iteration in a CUDA graph (1) */
  int32_t exact_xtilt;       /* x-tilt shared by all views: 0 (default) sums each projection row
                                over the views, then blends the two rows of every voxel (the
                                reference's per-view blend up to f32 rounding order); 1 blends
                                per view, bit-identical to main.rs:802-817 (addition) */
} tg_options;

/* Output header statistics (amin, amax, amean) of apps/tilt/src/main.rs:1077-1093 */
typedef struct { float amin, amax, amean; } tg_stats;

/* Per-call timing/accounting filled by tg_session_last_run. */
typedef struct {
  double updates;            /* voxel-view updates performed (onx*onz*ny*views per pass) */
  double ms_total;           /* device time of the last tg_reconstruct (CUDA events) */
  double ms_filter;          /* filter stage (R-weighting, stretch, staging format) */
  double ms_backproject;     /* back-projection passes */
  double ms_reproject;       /* SIRT reprojection passes */
  int32_t passes;            /* back-projection passes (1 + sirt_iters) */
  int32_t kernel_launches;   /* kernels launched by the last tg_reconstruct */
} tg_run_info;

typedef struct tg_session tg_session;

void tg_options_default(tg_options *opt);
const char *tg_status_string(int status);
/* Message of the last error on this thread ("" if none). */
const char *tg_last_error(void);
int tg_abi_version(void);

/* Replaces GpuSession::new (apps/tilt/src/gpu.rs:43-221) plus the CPU
 * preprocessing of apps/tilt/src/main.rs:602-700: plans one tilt series and
 * allocates its device buffers (projections, staged filtered rows, volume). */
int tg_session_create(const tg_geometry *geom, const tg_options *opt, tg_session **out);
/* Copies nx*ny*nz floats ([view][row][x], as read by MrcReader::read_slice_f32,
 * crates/imod-mrc/src/read.rs:127-231) from host memory into the session. */
int tg_upload_projections(tg_session *s, const float *host, size_t n);
/* Same from device memory (cudaMemcpyDeviceToDevice on the session stream). */
int tg_set_projections_device(tg_session *s, const float *dev, size_t n);
/* Runs the whole path (log, means, R-weighting, stretch, WBP or SIRT, fake-SIRT,
 * output transform, statistics) asynchronously on the session stream.
 * Replaces the body of main() in apps/tilt/src/main.rs:607-1093. */
int tg_reconstruct(tg_session *s);
int tg_synchronize(tg_session *s);
/* Copies output slices [y0, y1) ([y][out_nz][out_nx] f32) to host memory and
 * returns the whole-volume header statistics. Synchronises the session. */
int tg_download_slices(tg_session *s, int32_t y0, int32_t y1, float *host_out, tg_stats *stats);
/* Queues the same copy on the session's stream and returns at once (no
 * counterpart in the reference, which writes each slice as it is made): the
 * caller keeps host_out alive and calls tg_synchronize before reading it.
 * Lets one series' download overlap the next series' upload and compute. */
int tg_download_slices_async(tg_session *s, int32_t y0, int32_t y1, float *host_out);
/* Queues the copy of sections (views) [z0, z1) ([view][row][x] floats) from host
 * memory into the session on its stream and returns at once: the caller keeps
 * `host` unchanged until tg_synchronize, then may reuse it.  Lets a reader
 * stream a stack in as MrcReader::read_slice_f32 produces it
 * (crates/imod-mrc/src/read.rs:127-231, apps/tilt/src/main.rs:602-605); every
 * section must be uploaded before tg_reconstruct. */
int tg_upload_sections(tg_session *s, int32_t z0, int32_t z1, const float *host);
/* Queues output slices [y0, y1) converted on the device to IEEE half (round to
 * nearest even) into host_out (2 bytes per voxel, little-endian), for MRC mode
 * 12 output at half the bytes.  The reference reads mode 12
 * (crates/imod-mrc/src/read.rs:468-499) but its write_slice_f32
 * (write.rs:58-104) has no half case; this is an addition.  Values beyond the
 * half range become infinities.  Synchronise before reading host_out. */
int tg_download_slices_f16_async(tg_session *s, int32_t y0, int32_t y1, uint16_t *host_out);
/* Page-locked host memory (cudaHostAlloc), for copies that overlap with other
 * work; free with tg_host_free.  No counterpart in the reference. */
int tg_host_alloc(size_t bytes, void **out);
int tg_host_free(void *p);
int tg_get_stats(tg_session *s, tg_stats *stats);
/* Device pointer of the resident volume [ny][out_nz][out_nx]. */
const float *tg_volume_device(tg_session *s);
int tg_session_last_run(tg_session *s, tg_run_info *info);
/* Resolved output dims (out_nx, out_nz, out_ny = ny). */
int tg_session_dims(tg_session *s, int32_t *out_nx, int32_t *out_nz, int32_t *out_ny);
/* Device bytes held by the session. */
size_t tg_session_device_bytes(tg_session *s);
/* Runs the session's work on the caller's CUDA stream (a cudaStream_t passed as
 * void*; NULL restores the session's own stream).  No counterpart in the
 * reference (its wgpu queue is private); lets a host runtime order the work
 * with its own copies and timers. */
int tg_session_set_stream(tg_session *s, void *cuda_stream);
/* Test hook of the bounded device waits (no counterpart in the reference).  The
 * pipelined back-projector's waits give up after wait_limit_us (0: the default
 * 2 s) and report TG_ERR_TIMEOUT through tg_synchronize.  skip_stage >= 0 makes
 * its producer issue no copy for that pipeline stage of every tile, so the
 * consumers' bounded wait on it runs out: the timeout path runs without any
 * device fault, and the session stays usable (skip_stage -1 and wait_limit_us 0
 * restore normal operation).  TG_ERR_UNSUPPORTED for sessions that do not use
 * that back-projector (local alignment, per-view x-tilts). */
int tg_session_inject_wait_fault(tg_session *s, int32_t skip_stage, uint32_t wait_limit_us);
/* ---- SIRT in steps, with checkpoints (no counterpart in the reference, whose
 * SIRT loop apps/tilt/src/main.rs:919-975 runs to the end in one process) ----
 * tg_sirt_begin runs what tg_reconstruct runs before the first SIRT iteration
 * (log, means, R-weighting and the WBP start: iteration count 0);
 * tg_sirt_iterate runs n more iterations (at most the session's sirt_iters in
 * all); tg_sirt_end runs the output stage (fake SIRT, output transform,
 * statistics), after which the volume and statistics are those of
 * tg_reconstruct with the iterations run so far.  Between them, tg_sirt_save
 * copies the raw SIRT volume ([y][out_nz][out_nx] f32, before the output
 * transform) and the iteration count to the host (synchronising), and
 * tg_sirt_restore puts them back into a session with the same geometry and
 * options whose projections are uploaded (it recomputes the log and means),
 * so that iterating on continues the saved run: begin, k iterations, save,
 * then restore, n - k iterations, end gives tg_reconstruct's n-iteration result
 * bit for bit.  TG_ERR_INVALID_ARG without SIRT (sirt_iters 0, --gpu), out of
 * order, or with more iterations than sirt_iters. */
int tg_sirt_begin(tg_session *s);
int tg_sirt_iterate(tg_session *s, int32_t n);
int tg_sirt_end(tg_session *s);
int tg_sirt_save(tg_session *s, float *host_volume, int32_t *iterations_done);
int tg_sirt_restore(tg_session *s, const float *host_volume, int32_t iterations_done);
int tg_session_destroy(tg_session *s);

/* ---- Batched reconstruction of many series (no counterpart in the reference,
 * which reconstructs one series per process) ----
 * Sessions (already holding their projections, all on the batch's device) are
 * added to a batch; tg_batch_reconstruct runs every series' whole path.  The
 * back-projection passes of all series that take the fast kernel and share a
 * staging precision run as one persistent launch per round (round 0: WBP,
 * round r: r-th SIRT update), with a longest-first tile queue.  Each series'
 * result is identical to tg_reconstruct on that session alone.  Call
 * tg_batch_synchronize before reading a session's results. */
typedef struct tg_batch tg_batch;
int tg_batch_create(int32_t device, tg_batch **out);
int tg_batch_add(tg_batch *b, tg_session *s);
int tg_batch_clear(tg_batch *b);
int tg_batch_reconstruct(tg_batch *b);
int tg_batch_synchronize(tg_batch *b);
int tg_batch_last_run(tg_batch *b, tg_run_info *info);
int tg_batch_destroy(tg_batch *b);

/* ---- Serving: a request loop with continuous batching (no counterpart in the
 * reference, which reconstructs one series per process) ----
 * Jobs (WBP or SIRT, any size) are submitted from any thread.  One device
 * thread per server admits them first-in first-out while the device bytes of the
 * admitted jobs stay within the budget and fewer than max_active run (a job that
 * does not fit yet may be passed by later ones for at most 2 s), copies
 * their projections in on a copy stream, and runs rounds: every round takes each
 * running job one step further (its filter + WBP pass, or one SIRT
 * reproject/residual/update) with the back-projections of all those jobs in one
 * persistent launch; jobs join and leave at round boundaries.  A finished job's
 * volume is copied out on a third stream and its memory returns to the server's
 * stream-ordered pool.  Each job's result is identical to tg_reconstruct of the
 * same series alone.  A device error word set by a job's kernels fails that job
 * only. */
typedef struct tg_server tg_server;
typedef enum { TG_JOB_QUEUED = 0, TG_JOB_RUNNING = 1, TG_JOB_DONE = 2, TG_JOB_FAILED = 3 } tg_job_state;
typedef struct {
  tg_geometry geometry;     /* copied at submit (the arrays may be freed afterwards) */
  tg_options options;       /* options.device is ignored (the server's device) */
  const float *projections; /* host, nx*ny*nz floats; must stay valid until the job ends */
  size_t n_projections;
  float *volume_out;        /* host, ny*out_nz*out_nx floats (slice-major), or NULL; written
                               before the job reports TG_JOB_DONE.  Pinned memory copies fastest. */
  uint64_t tag;             /* returned in tg_job_result */
} tg_job;
typedef struct {
  int32_t state;            /* tg_job_state */
  int32_t status;           /* TG_OK, or the failure of a TG_JOB_FAILED job */
  tg_stats stats;           /* header statistics (main.rs:1080-1093) of a done job */
  int32_t rounds;           /* 1 + SIRT iterations */
  double submit_ms, admit_ms, done_ms;  /* server clock (ms since tg_server_create); -1 if not yet */
  double updates;           /* voxel-view updates of the job */
  uint64_t device_bytes;    /* device memory the job held while running */
  uint64_t tag;
  char message[128];        /* why a failed job failed (empty otherwise) */
} tg_job_result;
typedef struct {
  uint64_t submitted, completed, failed, queued, running;
  uint64_t budget_bytes, bytes_in_use, bytes_peak;
  uint64_t rounds, bp_launches;
  double updates_done;
  uint64_t oom_requeues;    /* admissions put back after a device allocation failure */
  double gpu_round_ms;      /* device time of the completed rounds */
  double host_round_ms;     /* server time spent issuing rounds */
  double host_admit_ms;     /* server time spent creating the sessions of admitted jobs */
} tg_server_info;
typedef enum {
  TG_FAULT_ALLOC = 1,  /* the next `count` admissions fail their device allocation (TG_ERR_OOM) */
  TG_FAULT_ADMIT = 2   /* the next `count` admissions are refused (TG_ERR_BUDGET) */
} tg_fault;
/* budget_bytes 0: 80% of the device's free memory; max_active <= 0: 64. */
int tg_server_create(int32_t device, uint64_t budget_bytes, int32_t max_active, tg_server **out);
/* TG_ERR_BUDGET if the job alone exceeds the budget; other validation errors as tg_session_create. */
int tg_server_submit(tg_server *sv, const tg_job *job, uint64_t *id);
/* Current state of a job (TG_OK), or TG_ERR_NOT_FOUND. */
int tg_server_poll(tg_server *sv, uint64_t id, tg_job_result *out);
/* Waits up to timeout_ms (<0: no limit) for the job to end; TG_ERR_NOT_READY on timeout. */
int tg_server_wait(tg_server *sv, uint64_t id, int32_t timeout_ms, tg_job_result *out);
/* Forgets an ended job's record; TG_ERR_NOT_READY while it runs. */
int tg_server_release(tg_server *sv, uint64_t id);
int tg_server_get_info(tg_server *sv, tg_server_info *out);
/* Host-side fault injection (tg_fault); no device fault is ever injected. */
int tg_server_inject(tg_server *sv, int32_t fault, int32_t count);
/* Drops queued jobs (TG_ERR_CANCELLED), lets running jobs finish, stops the device thread. */
int tg_server_destroy(tg_server *sv);
/* Short names of tg_server_submit / tg_server_poll. */
int tg_submit(tg_server *sv, const tg_job *job, uint64_t *id);
int tg_poll(tg_server *sv, uint64_t id, tg_job_result *out);

/* ---- The reference's GPU seam, same arguments and meaning ----
 * GpuSession::new(projections, tilt_cos_sin, in_nx, in_ny, n_projs, out_nx, out_nz)
 * (apps/tilt/src/gpu.rs:43-51): projections are already filtered/stretched,
 * tilt_cos_sin holds n_projs (cos, sin) pairs.  Returns TG_OK or an error
 * where the reference returns None. */
typedef struct tg_gpu_session tg_gpu_session;
int tg_gpu_session_new(const float *projections, const float *tilt_cos_sin, size_t in_nx,
                       size_t in_ny, size_t n_projs, size_t out_nx, size_t out_nz,
                       int32_t device, tg_gpu_session **out);
/* reconstruct_row(iy) (apps/tilt/src/gpu.rs:224-269): writes out_nx*out_nz floats. */
int tg_gpu_session_reconstruct_row(tg_gpu_session *s, size_t iy, float *out);
void tg_gpu_session_free(tg_gpu_session *s);

/* ---- Stage function ----
 * apply_rweighting(proj_data, in_nx, in_ny, nz, cutoff, falloff,
 * exact_filter_size, use_hamming) (apps/tilt/src/main.rs:333): in place on a
 * host array of in_nx*in_ny*nz floats, computed on the device. */
int tg_apply_rweighting(float *proj_data, size_t in_nx, size_t in_ny, size_t nz, float cutoff,
                        float falloff, int32_t exact_filter_size, int32_t use_hamming,
                        int32_t device);

/* ---- Allocation-free R-weighting ----
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * hosts that hand out all device memory from their own pool or arena, and
 * services that must avoid cudaMalloc's implicit device-wide synchronisation.
 * Filters nz*in_ny rows of in_nx floats in place in caller-owned DEVICE memory
 * (same arithmetic as tg_apply_rweighting), asynchronously on cuda_stream
 * (a cudaStream_t as void*, NULL = legacy default stream).  Allocates nothing:
 * its weight/twiddle tables live in a static 128 KB device array, which limits
 * rows to in_nx <= 8192 (larger rows are rejected with TG_ERR_INVALID_ARG).
 * Each call writes its tables into the array with small kernels that carry
 * them in their launch parameters, then filters with the generic mixed-radix
 * kernel (for 2^k and 3*2^k rows the allocating paths use a faster
 * register-resident FFT kernel; the results agree to rounding).  The first call
 * in a device's context looks the array up (cudaGetSymbolAddress); make that
 * first call before any stream capture.  All calls on a device share the array
 * and it keeps the last call's tables: calls whose GPU work overlaps race, so
 * order them on one stream. */
int tg_apply_rweighting_device_noalloc(float *dev_proj, size_t in_nx, size_t in_ny, size_t nz,
                                       float cutoff, float falloff, int32_t exact_filter_size,
                                       int32_t use_hamming, int32_t device, void *cuda_stream);

/* ---- imod-studio's reconstruction step ----
 * Replaces step_reconstruction (apps/imod-studio/src/main.rs:725-776): reads the
 * aligned stack (MRC) and tilt file, back-projects every row on the GPU without
 * R-weighting or cosine stretch (zero fill, thickness = width, sum / sections;
 * the tilt path with --no-weight --no-cosine-stretch --fill-mode zero -z nx)
 * and writes the volume with MrcHeader::new(nx, nx, ny, Float), the label
 * "imod-studio: reconstruction" and statistics (0, 0, 0), as the step does.
 * TG_ERR_INVALID_ARG with "<path> not found" where the step returns that Err. */
int tg_studio_reconstruct(const char *ali_path, const char *tlt_path, const char *rec_path,
                          int32_t device);

/* ---- ctfphaseflip: CTF phase flip of a tilt series (the step before tilt) ----
 * Options of apps/ctfphaseflip/src/main.rs:19-88 (defaults via
 * tg_ctf_options_default).  pixel_size is the caller's resolved value (the
 * reference takes -p or the header's xlen/mx). */
typedef struct {
  float defocus;             /* -d, nm, used when no per-view values are given (-3000) */
  float voltage;             /* -v, kV (300) */
  float cs;                  /* -c, mm (2.7) */
  float pixel_size;          /* -p or header, Angstrom */
  int32_t strip_width;       /* -w (256) */
  float tilt_axis_angle;     /* --tilt-axis-angle, degrees (0) */
  int32_t max_strip_width;   /* --max-strip-width, <= 0: automatic (main.rs:297-320) */
  float amplitude_contrast;  /* --amplitude-contrast (0.07) */
  float cuton_freq;          /* --cuton-freq, 1/Angstrom (0) */
  float plate_phase;         /* --plate-phase, degrees (0) */
  int32_t device;            /* CUDA device ordinal */
} tg_ctf_options;
void tg_ctf_options_default(tg_ctf_options *o);
/* The strip width the correction uses: strip_width clamped to the given or
 * automatic maximum (main.rs:284-324).  view_defocus as in tg_ctf_phaseflip. */
int tg_ctf_strip_width(const tg_ctf_options *o, int32_t nx, const float *view_defocus,
                       int32_t n_view_defocus, int32_t *out);
/* Replaces the per-view loop of main() (apps/ctfphaseflip/src/main.rs:385-700):
 * host_in and host_out are [nz][ny][nx] floats (MrcReader::read_slice_f32
 * order); angles are the .tlt values (missing views: 0); view_defocus holds 3
 * floats per view (defocus1 nm, defocus2 nm, astigmatism angle degrees) after
 * the reference's interpolation of the defocus file, or NULL to use
 * o->defocus.  Every strip's 2D FFT, CTF sign flip (the CPU path's f64 CTF),
 * inverse and weighted blend run on the GPU; stats receives the header
 * statistics of main.rs:681-693. */
int tg_ctf_phaseflip(const tg_ctf_options *o, const float *host_in, int32_t nx, int32_t ny, int32_t nz,
                     const float *angles, int32_t n_angles, const float *view_defocus,
                     int32_t n_view_defocus, float *host_out, tg_stats *stats);
/* The shader's parameters (CtfParams of apps/ctfphaseflip/src/gpu.rs:8-26). */
typedef struct {
  uint32_t sw, sh;
  float pixel_a, wavelength, cs_a, amp_contrast, cuton_freq, defocus1, defocus2, astig_angle_rad;
  uint32_t has_astigmatism;
  float plate_phase_rad, tilt_axis_rad;
} tg_ctf_strip_params;
/* Replaces GpuCtfSession::correct_strip (apps/ctfphaseflip/src/gpu.rs:107-262,
 * ctf_correct.wgsl): flips, in place, the real and imaginary parts (sw*sh
 * floats each, host memory) of one strip's 2D FFT where the CTF is negative,
 * in the shader's f32 arithmetic. */
int tg_ctf_correct_strip(float *strip_re, float *strip_im, const tg_ctf_strip_params *p, int32_t device);

/* ---- Synthetic seeded inputs (no counterpart in the reference; the
 * workload generator for tests and benchmarks) ----
 * Projects a seeded random ellipsoid phantom (n_ell ellipsoids with semi-axes
 * in [rmin, rmax] px and densities U(dmin, dmax), plus n_beads spheres of
 * radius bead_r and density bead_d) of size px_nx x ny x pz_nz along the given
 * angles (degrees) with the reference geometry (x = dx*cos + dz*sin + nx/2,
 * row = y), then adds noise:
 *   noise_kind 0: none; 1: Gaussian with sigma = noise * std(signal);
 *   2: counts = Poisson(noise * exp(-mu * line integral)) (noise = base
 *      counts, mu = 1/pz_nz) written as counts, ready for --log.
 * out: device or host pointer (is_device) of nz*ny*nx floats. */
typedef struct {
  uint64_t seed;
  int32_t nx, ny, nz;         /* projection width, rows, views */
  int32_t vol_nx, vol_nz;     /* phantom width and thickness (rows = ny) */
  int32_t n_ell;
  float rmin, rmax, dmin, dmax;
  int32_t n_beads;
  float bead_r, bead_d;
  int32_t noise_kind;
  float noise;
  float xtilt_deg;            /* x-axis tilt of the projection geometry */
} tg_phantom_spec;
int tg_synth_projections(const tg_phantom_spec *spec, const float *angles, float *out,
                         int32_t is_device, int32_t device);

/* ---- MRC / tilt-file boundary (host only; usable without a GPU) ----
 * Byte-compatible with crates/imod-mrc (header.rs:10-258, read.rs:28-231,
 * write.rs:20-153) and crates/imod-transforms/src/tilt.rs:6-33. */
typedef struct {
  int32_t nx, ny, nz, mode, next;
  int32_t swapped;           /* file was big-endian (MrcReader::is_swapped) */
  float xlen, ylen, zlen;
  float amin, amax, amean;
  int32_t nlabl;
  int32_t imod;              /* IMOD stamp present */
  uint8_t header[1024];      /* the parsed header re-serialised little-endian */
} tg_mrc_info;
/* MrcHeader::new(nx, ny, nz, mode) serialised (header.rs:181-241), plus
 * add_label(label) when label != NULL (header.rs:244-258). */
int tg_mrc_header_new(int32_t nx, int32_t ny, int32_t nz, int32_t mode, const char *label,
                      uint8_t out[1024]);
/* MrcReader::open + read_slice_f32 for sections [z0, z1) (out may be NULL to
 * read the header only).  out receives (z1-z0) * values-per-section floats. */
int tg_mrc_read(const char *path, tg_mrc_info *info, int32_t z0, int32_t z1, float *out);
/* MrcWriter::create(path, header) + write_slice_f32 for nsec sections +
 * finish(amin, amax, amean).  header: 1024 little-endian bytes. */
int tg_mrc_write_f32(const char *path, const uint8_t header[1024], const float *data,
                     int32_t nsec, float amin, float amax, float amean);
/* Output header of a reconstruction (apps/tilt/src/main.rs:710-717): from the
 * input stack's header bytes, the output width/thickness and the number of
 * sections; statistics are filled in by tg_mrc_write_f32's finish. */
int tg_tilt_output_header(const uint8_t in_header[1024], int32_t out_nx, int32_t out_nz,
                          uint8_t out[1024]);
/* read_tilt_file: up to cap angles into out, count in *n. */
int tg_read_tilt_file(const char *path, float *out, int32_t cap, int32_t *n);
/* write_tilt_file ("{:10.2}" per line). */
int tg_write_tilt_file(const char *path, const float *angles, int32_t n);

#ifdef __cplusplus
}
#endif
#endif /* TILTGPU_H */
