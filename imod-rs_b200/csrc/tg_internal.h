// tg_internal.h -- shared declarations of libtiltgpu (kernels + host plumbing).
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/tiltgpu.h"

#include <nvtx3/nvToolsExt.h>  // header-only NVTX v3: no-ops unless a profiler is attached

namespace tg {

// Staged-projection formats written by the filter stage and read by the
// back-projectors.  Element k of a row holds the samples needed to interpolate
// anywhere in [k, k+1):
//   FP32 : (row[k], row[k+1]); out-of-range k holds (fill, fill) and the
//          kernel forces the fraction to 0 there, which reproduces the
//          reference's `sample_row_with_fill` bit for bit.
//   FP16/BF16 : (row[k], row[k+1]-row[k]); out-of-range k holds (fill, 0).
// ROWPAIR interleaves rows 2j and 2j+1 of a view in one element
// ([view][row-pair][PW]): FP32 float4 (a0, a1, b0, b1), FP16/BF16 uint2
// (h2(a0,a1), h2(d0,d1)).  SINGLE keeps one row per element ([view][row][PW]):
// FP32 float2 (a, b), FP16/BF16 uint32 h2(a, d).
enum Fmt { FMT_ROWPAIR = 0, FMT_SINGLE = 1, FMT_ROWS = 2 /* plain filtered rows, in place */ };

inline int elem_bytes(int fmt, int store) {
  if (fmt == FMT_ROWPAIR) return store == TG_STORE_FP32 ? 16 : 8;
  return store == TG_STORE_FP32 ? 8 : 4;
}

struct StatPartial {
  float mn, mx;
  double sum;
};

// ---- log transform + per-view means (main.rs:608-623) ----
// logd == nullptr: means of raw; else logd = log10(max(raw, 0.001)) and its means
// (means == nullptr: partial sums only)
void launch_log_means(const float *raw, float *logd, int npix, int nviews, double *partials,
                      float *means, cudaStream_t st);
// per-view f64 sums from the partials of launch_log_means
void launch_view_sums(const double *partials, int nviews, double *sums, cudaStream_t st);

// ---- filter stage: R-weighting (main.rs:333-381), cosine stretch
// (main.rs:446-488) and staging-format packing ----
struct FftPlanDev {
  int n;
  int nfac;
  int fac[24];
};
bool fft_plan(int n, FftPlanDev *p);  // false if n has a prime factor > 7

struct FilterArgs {
  const float *in;          // [nviews_all][ny][nx]
  const float *sub;         // optional: value = in - sub (SIRT residual)
  void *out;                // staged format
  const float *weights;     // n weights, nullptr = no R-weighting
  const float2 *tw;         // n twiddles exp(-2 pi i k/n)
  const float2 *tw2;        // register-resident kernel's per-pass twiddles (p2_twiddle_table), or nullptr
  const float *conv_h;      // circulant kernel for n without a radix plan (else nullptr)
  const float *stretch;     // per view 1/cos (f32) or 0: no stretch; nullptr = none
  const float *fill;        // per view fill value for mean mode
  int nx, ny, nviews;
  int rows_alloc;           // rows (SINGLE) or row-pairs (ROWPAIR) per view in `out`
  int PW, padL;
  int fill_mode, cubic, fmt, store;
  float inv_n;
  FftPlanDev plan;
  int *err;                 // session error word: bit 2 set when a value exceeds the FP16 range
};
void launch_filter(const FilterArgs &a, cudaStream_t st);
// Twiddles of the register-resident filter kernel for rows of n samples, per
// forward pass p with span NS > 1 and radix R: exp(-2 pi i r k / (NS R)) at
// offset_p + (r-1)*NS + k (k-major, so a warp's lanes read neighbouring entries);
// fewer than n entries in all.  False (table empty) when n has no such kernel.
bool p2_twiddle_table(int n, std::vector<float2> &out);
// ---- the register-resident filter over many series of one width in one launch ----
struct FilterBatchDev {
  const FilterArgs *jobs;   // device array
  const int *blk0;          // njobs + 1 prefix sums of ((ny + 1) / 2) * nviews blocks
  int njobs;
};
// the row width a series' filter shares launches by, or 0 when it runs on its own
int filter_batch_width(const FilterArgs &a);
void launch_filter_batch(int n, int fmt, int store, const FilterBatchDev &fb, int nblocks, cudaStream_t st);
// radial weight table of apps/tilt/src/main.rs:348-369 in f32 (host)
void weight_table(int n, float cutoff, float falloff, int efs, int hamming, float *wt);

// ---- back-projection ----
struct LocalDev {
  // per view: offset into xs/ys (nxs, nys) and into grids; empty view: nxs=0
  const int4 *vinfo;        // (x_off, nxs, y_off, nys)
  const int *goff;          // grid offset per view
  const float *xs, *ys, *gdx, *gdy;
  // per (view, slice, column): the interpolated (dx, dy) of local_interp, or null.
  // Views without patches hold (0, 0); adding 0 changes no position.
  const float2 *table;
  int table_nx;             // columns per table row (the output width)
};
struct BpArgs {
  const void *pairs;
  const float4 *vg;         // per view (cos_t, sin_t, zf, cos_xt)
  const float4 *vg2;        // per view (sin_xt, 0, 0, 0)
  float *vol;               // [ny][onz][onx]
  StatPartial *partial;     // [ny][ntiles]
  int *err;
  int nx, ny, nviews, onx, onz;
  int PW, padL, rows_alloc;
  float cx, cz, ocx, inv_n, dw, os, oa, relax;
  int mode;                 // 0: final (transform + stats), 1: store acc/N, 2: vol += relax*acc/N
  int has_local;
  LocalDev loc;
  int nbx, ntiles_xz;       // tile grid of the fast kernel (set by its launcher)
  int tile0;                // batched launch: index of this series' first tile
  // bounded pipeline waits of the fast kernel: give up after wait_limit_ns (error bit 0)
  unsigned long long wait_limit_ns;
  // test hook (tg_session_inject_wait_fault): the producer issues no copy for this
  // stage of each tile, so the consumers' wait on it runs out; -1: none
  int fault_skip_stage;
  int pad_;
};
// A persistent back-projection launch over the tiles of several series.  Tile t
// belongs to the series j with jobs[j].tile0 <= t < jobs[j+1].tile0 (series in
// queue order, longest first); inside a series tiles run x fastest, then z,
// then the row group.
struct BatchLaunch {
  const BpArgs *jobs;       // device array of per-series arguments (nbx, ntiles_xz, tile0 filled)
  int njobs;
  int ntiles;
  int *counter;             // device int, reset by the launcher
  int max_views;
};
int launch_bp_batch(const BatchLaunch &bl, int store, bool zf, int variant, cudaStream_t st);
void bp_fast_tile_shape(int variant, int *S, int *TX, int *TZ);
struct BpTile { int S, K, TX, NT, VPS, wmax; };
// Fast kernel: no x-tilt, no local alignment, ROWPAIR format.
// zf: 0 none, 1 z-factors, 2 z-factors and one x-tilt in the positions (row sums)
int launch_bp_fast(const BpArgs &a, int store, int zf, int variant, cudaStream_t st,
                   int *ntiles_out);
int bp_fast_variants();
const char *bp_fast_variant_name(int v);
// General kernel: x-tilt, z-factor, local alignment, SINGLE format.
int launch_bp_general(const BpArgs &a, int store, cudaStream_t st, int *ntiles_out);
// x-tilt back-projection with staged rows (no local alignment); same tile grid
// and partial-stat layout as the general kernel
int launch_bp_xtilt(const BpArgs &a, int store, cudaStream_t st, int *ntiles_out);
// max_abs_sin_xt: over the views; max_x_extent_per_tile: max over views of
// 31*|cos*cos_xt| + 15*|sin*zf| (a 32-column, 16-depth tile)
bool bp_xtilt_supported(int onx, float max_abs_sin_xt, float max_x_extent_per_tile);
int bp_fast_ntiles(const BpArgs &a, int variant);
int bp_fast_row_align();  // slices per tile of the widest fast variant
// Second half of the x-tilt back-projection of a series whose views share one
// x-tilt: rows holds, per projection row r, the fast kernel's mode-1 output
// (sum over views of the row-r sample) * 1/N; every voxel (ox, iy) takes rows
// floor(iy + dx*sin_xt) and the next, blended as the reference blends each
// view's pair.  a.vol, a.mode (0, 1, 2), a.partial and the output constants as
// in BpArgs; mode 0 writes XB_TILES partial-stat tiles per slice.
constexpr int XB_TILES = 16;  // depth tiles per slice (each block walks onz/16 depths)
int launch_xt_blend(const BpArgs &a, const float *rows, float sin_xt, cudaStream_t st, int *ntiles_out);

// ---- reprojection (main.rs:831-896) ----
struct FpArgs {
  const float *vol;         // [ny][onz][onx]
  float *sino;              // [nviews_all][ny][nx] (views >= nviews are zeroed)
  const float4 *vg, *vg2;
  int nx, ny, nviews, nviews_all, onx, onz;
  float cx, cz, ocx;
  int has_local;
  LocalDev loc;
  int fast;                 // fp_fast_kernel: 1 no x-tilt (bit-exact), 2 with x-tilt; 0 general
  float *volg;              // fast == 1: row-group interleaved copy of vol, or null;
                            // fast == 2: the blended copy (one x-tilt for all views), or null
  float sin_xt_common;      // fast == 2 with volg: the x-tilt sine shared by every view
  void *volh;               // fast == 1, half staging: scaled FP16 interleaved copy, or null
  unsigned *maxbits;        // with volh: max |vol| as float bits (sets the copy's scale)
  int variant;              // bit 0: 16 rows per thread (else 8); bit 1: interleaved copy;
                            // bit 2: 32 rows per thread in the half path (else 16);
                            // bit 3: FP32 reprojection also for half staging
  // local alignment: per (view, tile t of LB_TILE slices, column) the min and max of the
  // table's dx over slices [LB_TILE*(t-1), LB_TILE*(t+2)) (clipped to the series), or null
  const float2 *lbnd;
};
constexpr int LB_TILE = 16;
int launch_reproject(const FpArgs &a, cudaStream_t st);  // returns the kernels launched
// fills L.table for every (view < nviews, slice < ny, column < onx)
void launch_local_table(const LocalDev &L, int nviews, int ny, int onx, float2 *table, cudaStream_t st);
// fills FpArgs::lbnd from the table: nviews * ceil(ny / LB_TILE) * onx entries
void launch_local_bounds(const float2 *table, int nviews, int ny, int onx, float2 *bnd, cudaStream_t st);
int fp_group_rows(int variant);
int fp_half_rows(int variant);
// ---- batched reprojection (one launch per phase over the series of a group) ----
struct FpBatchDev {
  const FpArgs *jobs;       // device array of per-series arguments
  const int *blk0;          // njobs + 1 prefix sums of the phase's blocks per series
  int njobs;
};
// blocks of the max|vol| pass of a volume of n values (one series)
inline __host__ __device__ int fp_absmax_blocks(size_t n) {
  const size_t b = (n + 4095) / 4096;
  return (int)(b < 1 ? 1 : b > 1184 ? 1184 : b);
}
// the batched form a series' reprojection takes (series with equal keys share
// launches), or -1 when it is launched on its own (local alignment, general kernel)
int fp_batch_key(const FpArgs &a);
// blocks of each phase of one series in its group: max|vol|, copy, projection
void fp_batch_blocks(const FpArgs &a, int key, int *absmax, int *copy, int *fp);
// the phases of one group; jobs and the three prefix arrays in device memory,
// totals = the last prefix entries.  Returns the kernels launched.
int launch_reproject_batch(int key, const FpArgs *jobs, int njobs, const int *blk_abs, int nabs,
                           const int *blk_copy, int ncopy, const int *blk_fp, int nfp, cudaStream_t st);

// ---- volume operations ----
void launch_lowpass(float *vol, float *tmp, int onx, int onz, int ny, cudaStream_t st);
// in-place output transform + per-(slice, tile) partial stats
void launch_transform_stats(float *vol, int onx, int onz, int ny, float dw, float os, float oa,
                            StatPartial *partial, int *ntiles_out, cudaStream_t st);
// per slice (min,max,mean) -> whole-volume stats in the reference's order
void launch_stats_reduce(const StatPartial *partial, int ny, int ntiles, int slice_count,
                         float *slice_stats, float *out3, cudaStream_t st);

// f32 -> IEEE half (round to nearest even) of n values (mode-12 output)
void launch_to_half(const float *in, void *out, size_t n, cudaStream_t st);

// ---- synthetic data ----
int synth_projections(const tg_phantom_spec *spec, const float *angles, float *d_out,
                      cudaStream_t st);

// ---- errors ----
void set_error(const std::string &msg);
// NVTX range over a host scope (the kernels launched inside it, for ncu --nvtx filters)
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};
int cuda_fail(cudaError_t e, const char *what);
// tg_status of a nonzero device error word (bit 0: a bounded wait gave up; bit 1:
// staging window outside the padded row; bit 2: a value beyond the FP16 range),
// with its message set
int device_error_status(int word);
#define TG_STR2(x) #x
#define TG_STR(x) TG_STR2(x)
#define TG_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t _e = (call);                                                                \
    if (_e != cudaSuccess) return ::tg::cuda_fail(_e, #call " at " __FILE__ ":" TG_STR(__LINE__)); \
  } while (0)

}  // namespace tg
