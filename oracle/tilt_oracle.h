/*
 * tilt_oracle.h -- CPU restatement of the imod-rs `tilt` reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA product path is
 * compared against (and the timed CPU baseline); nothing in the product links it.
 *
 * Two precisions of the same semantics:
 *   ref32  -- f32 arithmetic in the reference's operation order
 *             (apps/tilt/src/main.rs), compiled with -ffp-contract=off so no
 *             multiply-add is fused, exactly as Rust/LLVM evaluates it.
 *   ref64  -- the same semantics evaluated in FP64 (FP64 FFT, FP64 geometry):
 *             the accuracy oracle.
 *
 * Parity status: the reference is Rust (no cargo/rustc in this image) and its
 * FFT is the third-party crate rustfft 6.x (apps/tilt/Cargo.toml, no lockfile,
 * not vendored).  The reference's own tests pin only the MRC/.tlt boundary, not
 * the arithmetic, so the arithmetic of this oracle is PARITY UNPINNED against
 * the reference binary; it is pinned by analytic known-answer tests instead
 * (tests/test_oracle_kat.py).  rustfft's published algorithm is a
 * mixed-radix Cooley-Tukey FFT with twiddles computed in f64 and rounded to the
 * working type; this file restates that method (not rustfft's code).
 */
#ifndef TILT_ORACLE_H
#define TILT_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { OR_FILL_MEAN = 0, OR_FILL_ZERO = 1, OR_FILL_EDGE = 2 };

/* Mirrors the reference `Args` (apps/tilt/src/main.rs:18-120) after parsing. */
typedef struct {
  int32_t nx, ny, nz;          /* input stack: width, rows, sections (views) */
  int32_t out_nx, out_nz;      /* output width and thickness (already resolved) */
  int32_t n_angles;            /* number of angles read from the .tlt file */
  const float *angles;         /* degrees */
  int32_t n_xtilt;  const float *xtilt;    /* NULL/0 if no --xtilt-file */
  int32_t n_zfac;   const float *zfac;     /* NULL/0 if no --zfactor-file */
  int32_t n_local;  const float *local;    /* rows of (view, x, y, dx, dy); NULL/0 if none */
  int32_t has_local;                       /* --local-file given */
  float cutoff, falloff;
  int32_t no_weight;
  int32_t exact_filter_size;   /* <= 0: None */
  int32_t hamming;
  int32_t sirt_iters;
  float sirt_relax;
  int32_t no_cosine_stretch;
  int32_t cosine_cubic;
  float max_cosine_tilt;
  int32_t log_transform;
  float densweight, outscale, outadd;
  int32_t fill_mode;
  int32_t fake_sirt;
  int32_t gpu_compat;          /* --gpu: restate backproject.wgsl semantics */
} or_params;

typedef struct { float amin, amax, amean; } or_stats;

/* ---- stage functions (in place on a [nz][ny][nx] f32 stack) ---- */
void or_log_transform32(float *data, size_t n);
void or_view_means32(const float *data, int nx, int ny, int nz, float *means);
/* weight table of length n exactly as apply_rweighting builds it (main.rs:349-369) */
void or_weight_table32(int n, float cutoff, float falloff, int exact_filter_size,
                       int hamming, float *w);
void or_weight_table64(int n, double cutoff, double falloff, int exact_filter_size,
                       int hamming, double *w);
void or_rweight32(float *data, int nx, int nrows, float cutoff, float falloff,
                  int exact_filter_size, int hamming, int nthreads);
void or_rweight64(double *data, int nx, int nrows, double cutoff, double falloff,
                  int exact_filter_size, int hamming, int nthreads);
void or_cosine_stretch32(float *data, int nx, int ny, int nz, const float *angles,
                         int n_angles, int cubic, float max_tilt);
/* f32 FFT / FP64 FFT of one complex row (interleaved re,im), sign -1 forward */
void or_fft32(float *reim, int n, int inverse);
void or_fft64(double *reim, int n, int inverse);

/* WBP core (main.rs:756-828 / 1002-1090): vol is [out_ny=ny][out_nz][out_nx],
 * already multiplied by 1/nz.  Slices [y0, y1) only (y0=0,y1=ny for all). */
int or_backproject32(const or_params *p, const float *proj, const float *means,
                     float *vol, int y0, int y1, int nthreads);
int or_backproject64(const or_params *p, const double *proj, const double *means,
                     double *vol, int y0, int y1, int nthreads);
/* reprojection (main.rs:831-896): sino [nz][ny][nx] is overwritten */
int or_forward_project32(const or_params *p, const float *vol, float *sino);
int or_forward_project64(const or_params *p, const double *vol, double *sino);
/* fake-SIRT smoothing pass (main.rs:493-538), vol [ny][out_nz][out_nx] */
void or_lowpass32(float *vol, int out_nx, int out_nz, int out_ny);
void or_lowpass64(double *vol, int out_nx, int out_nz, int out_ny);

/* ---- whole path: everything main() does between reading and writing ----
 * proj: raw input stack as read (f32).  vol32/vol64: [ny][out_nz][out_nx].
 * Returns 0, or a negative code for the reference's panics/exits. */
int or_run32(const or_params *p, const float *proj, float *vol, or_stats *st, int nthreads);
int or_run64(const or_params *p, const float *proj, double *vol, or_stats *st, int nthreads);
/* ref64g: FP64 data path (FFT, interpolation, sums) with the reference's f32
 * sampling geometry, so both make the same floor/bounds decisions.  This is
 * the accuracy oracle for storage-precision error (FP16/BF16 vs FP32). */
int or_run64g(const or_params *p, const float *proj, double *vol, or_stats *st, int nthreads);
int or_backproject64g(const or_params *p, const double *proj, const double *means,
                      double *vol, int y0, int y1, int nthreads);
int or_forward_project64g(const or_params *p, const double *vol, double *sino);

/* Output transform + header statistics of main.rs:1077-1093 applied to a volume
 * in place (f32, reference order). */
void or_output_stats32(float *vol, int out_nx, int out_nz, int out_ny, float densweight,
                       float outscale, float outadd, or_stats *st);

/* WBP of the first y-rows only, for the timed CPU baseline: filter+stretch on
 * rows [y0,y1) of every view then backprojection of those slices. */
int or_wbp_rows32(const or_params *p, const float *proj, float *vol_rows, int y0, int y1,
                  int nthreads);
int or_wbp_rows64g(const or_params *p, const float *proj, double *vol_rows, int y0, int y1,
                   int nthreads);

/* ---- ctfphaseflip (apps/ctfphaseflip/src/main.rs, ctf_correct.wgsl) ---- */
typedef struct {
  float defocus;             /* -d, nm (used without per-view values) */
  float voltage;             /* kV */
  float cs;                  /* mm */
  float pixel_a;             /* pixel size, Angstrom */
  int32_t strip_width;       /* -w */
  float tilt_axis_angle;     /* degrees */
  int32_t max_strip_width;   /* <= 0: automatic */
  float amplitude_contrast;
  float cuton_freq;          /* 1/Angstrom */
  float plate_phase;         /* degrees */
} or_ctf_params;
typedef struct {             /* the shader's Params (ctf_correct.wgsl) */
  uint32_t sw, sh;
  float pixel_a, wavelength, cs_a, amp_contrast, cuton_freq, defocus1, defocus2, astig_angle_rad;
  uint32_t has_astigmatism;
  float plate_phase_rad, tilt_axis_rad;
} or_ctf_strip;
double or_ctf_wavelength(float kv);
int or_ctf_strip_width(const or_ctf_params *p, int nx, const float *view_def, int nviews);
int or_ctfphaseflip32(const or_ctf_params *p, const float *in, int nx, int ny, int nz, const float *angles,
                      int n_angles, const float *view_def, int n_view_def, float *out, or_stats *st);
void or_ctf_correct_strip32(float *re, float *im, const or_ctf_strip *p);

/* imod-studio's reconstruction step (apps/imod-studio/src/main.rs:725-776) restated
 * directly: out[ny][nx][nx]. */
void or_studio_reconstruct32(const float *proj, int nx, int ny, int nz, const float *angles,
                             int n_angles, float *out);

#ifdef __cplusplus
}
#endif
#endif
