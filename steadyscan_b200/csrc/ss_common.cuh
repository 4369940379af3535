// Shared types and device helpers of the B200 align_group_to_template engine.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>

namespace ss {

// Values the reference leaves in buffers it allocates (task_allocate.cu:226, :244).
constexpr double kPnewFill = 1e6;
constexpr double kErrvalFill = 1e6;
// Bound on line-search trials per frame; the reference has none (task_linesearch.cu:95-149).
constexpr int kTrialCap = 2048;

// Evaluation modes of k_eval.
enum EvalMode : int { kAssemble = 0, kTrial = 1, kCorr = 2, kFinal = 3 };

// Group phases of the device-side control state machine.
// kPhWait: the group's frames are still on their way to the device (streamed uploads).
enum Phase : int { kPhHalf = 0, kPhIterEnd = 1, kPhFinal = 2, kPhDone = 3, kPhWait = 4 };

// StopCriterion (interface/stopcriterion.h:4-10).
enum Stop : int { kStopCorrInc = 0, kStopHaltCorr = 1, kStopMovement = 2, kStopIterLimit = 3, kStopError = 4 };

// Flag bits parsed from the gpu_flags string (mex/configuration.cpp:83-152).
enum FlagBits : int {
  kFlagMaskInactive = 1 << 0,   // M
  kFlagIterCorr = 1 << 1,       // C
  kFlagFrameCorr = 1 << 2,      // c
  kFlagIterErrvals = 1 << 3,    // e
  kFlagMedianBefore = 1 << 4,   // R
  kFlagRawParams = 1 << 5,      // P
  kFlagFrameOrdered = 1 << 6,   // p
  kFlagTimeExec = 1 << 7,       // T: execution timing (outputs 9 and 10)
  kFlagTimeSub = 1 << 8,        // t: sub-function timing, TimedMainIteration (outputs 9, 10, 14)
};

// The device's global clock in nanoseconds (the iteration times of flags T and t).
__device__ __forceinline__ unsigned long long device_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Per-column sums written by k_eval. Assembly uses all slots; other modes a prefix.
enum ColSum : int {
  kCsSsd = 0,
  kCsAxx, kCsAyy, kCsAxy,   // sum g g' (1-f)^2            (diagonal, own knot)
  kCsBxx, kCsByy, kCsBxy,   // sum g g' f'^2, f' of column (c+1) mod W (diagonal, next knot)
  kCsOxx, kCsOyy, kCsOxy,   // sum g g' (f - f^2)          (coupling c, c+1)
  kCsJ1x, kCsJ1y,           // sum d (1-f) g               (gradient, own knot)
  kCsJ2x, kCsJ2y,           // sum d f g                   (gradient, next knot)
  kCsAssemble = 14,
  // correlation / final pass
  kCsSumD = 0,              // sum over all pixels of the swapped difference image D'
  kCsSetN, kCsSetD, kCsSetDD, kCsSetI, kCsSetII, kCsSetDI,  // leading-valid-run set
  kCsFrD, kCsFrI, kCsFrDD, kCsFrII, kCsFrDI,                 // valid pixels (per-frame corr)
  kCsFinalSsd,              // final pass: SSD at the mask knots
  kCsCorr = 13,
  kCsStride = 16,
};

// Batch counters of shared-memory staging and column reuse (ss_batch_stats.staging and
// .assembly_columns_kept): assembly/final CTAs, of them with a template row window, line-search
// CTAs, of them with a window, of them on the packed pixel-pair path, assembly block columns
// evaluated as pixel pairs, assembly block columns that kept their sums.
constexpr int kStagingCounters = 7;

struct GroupCtl {
  int phase, iteration, shift, improved, exec_result;
  int filter_active, filter_kind, filter_id, n_filter_iter;
  int stop_reason, cap_hit, eig_size, n_used;
  int ls_state;    // 1 from the half-step solve until the line search is post-processed
  int ls_pending;  // frames of the half-step whose line search still runs (trial rounds)
  int solve_now;          // 1 while the group's half-step solve of this cycle runs (set by k_solve_compact)
  int par_sel;            // flag M: the parity bitmap (0 or 1) of the last global correlation
  int retry;              // the iteration is being retried without the filter
  int rg_slot;            // flag t: rgParams slot of the half-step that just ended, -1 if none
  double correlation, corr;
  long long n_eval;      // frame evaluations the reference would count: errval passes and trials
  long long passes[4];   // frames read per evaluation kind (EvalMode)
  unsigned long long t_mark;  // flags T and t: device clock (ns) at the start of the iteration
};

struct GroupDesc {
  // geometry (mexgateway.cpp:176-198)
  int Hb, W, nF, fW, N, Ht, Wt;
  int group_size, n_rg;
  int chunk_base;   // first frame chunk of this group in the batch's chunk table
  int frame_base;   // first global frame index of this group
  // settings
  int max_iter, solver_id, max_filter_iter, filter_id, flags, frac_uniform;
  int frames_per_cta;       // frames of an evaluation tile (a tuning choice): W * ceil(nF / it) tiles
  double move_thresh, halt_corr, corr_inc_thr, filter_strength, filter_corr_thr, lambda, ls_mult;
  // inputs on the device
  const double* frac;       // Hb x W column-major
  const double* basex;
  const double* basey;
  const float* frac_f;      // FP32 copies for precision 'S'
  const float* basex_f;
  const float* basey_f;
  // Affine geometry (precision 'S'; geo_k == 0: use the tables). Row r of block column cc holds
  // line cc*k + l, pixel j of that line (l = r mod k, j = r div k), with
  // basex = geo_ax*j + geo_bx, basey = geo_ay*(cc*k + l) + geo_by, tfrac = (l*L + j + 1/2) * geo_fs.
  int geo_k, geo_L;
  float geo_ax, geo_bx, geo_ay, geo_by, geo_fs;
  // Precision 'S': the template as FP32 rows of tpitch floats (16-byte aligned rows) for staging
  // row windows in shared memory, and per block column the [min, max] of basey over valid rows.
  const float* tplain;
  int tpitch;
  const float* col_yrange;  // W x 2
  int* err;                 // device error word of the batch (bit 0: a staging copy timed out)
  int pair_ok;              // precision 'S' pixel pairs: affine geometry, Hb % 64 == 0, aligned frames
  int quad_ok;              // pair_ok with 16-bit frames, knots every 1 or 2 lines, Hb % 256 == 0 and
                            // 16-byte aligned frames: trial columns by 16-byte loads
  unsigned long long* staging;  // batch counters of shared-memory staging (ss_batch_stats.staging)
  int ls_rounds;            // 1: the line search runs in trial rounds (precision 'S')
  int* ls_max_trials;       // batch: most trials of a frame whose search ended in the current cycle
  int* ls_done;             // nF: columns of the frame evaluated in the current trial round
  const uint8_t* base_mask;
  const int* min_points;    // W
  const void* image;        // Hb x fW column-major, engine frame type
  const void* tquad;        // (Ht-1)(Wt-1) template quads, engine template type
  const void* gquad;        // gradient quads or nullptr when derived from the template
  const double* sum_image; // sum of the frame data over all Hb x fW entries
  // state
  double *p, *p_last, *p_snap, *delta_p, *ndp;
  double* colsum;           // fW x kCsStride
  int* colcnt;              // fW
  // Assembly sums kept apart from the other passes' column sums, with the 8 knots each column was
  // assembled at (mask knots, then difference-image knots): a column whose knots are unchanged at
  // the next assembly keeps its sums instead of reading its frame again.
  double* asmsum;           // fW x kCsStride
  int* asmcnt;              // fW
  double* asmk;             // fW x 8
  uint8_t *params_used, *blocks_present, *grp_active;
  double* errval;           // 2 nF
  double *kmask, *kdiff;    // nF x 2 x (W+1)
  uint32_t* dparity;        // flag M: 2 x fW x ceil(Hb/32) words, bit r of a column's word r/32 set
                            // where the difference-image buffer holds image - difference: the
                            // bitmap of the last global correlation (GroupCtl::par_sel) and the one
                            // the next correlation pass writes; else nullptr
  uint8_t* fstate;          // nF: 2 while the frame's line search runs
  int* ls_trials;           // nF
  double* eig_c;            // N x 4
  uint8_t* eig_valid;       // N
  int* list;                // 2N: knot of each list position, then list position of each knot
  double* cr;               // N x 13
  double* ilu;              // 11 N: ILU(0) factors and forward solve (solver id 0 only)
  // outputs on the device
  double *o_frame_corr, *o_residrms, *o_iter_corr, *o_frame_corr_hist, *o_iter_errvals, *o_all_params;
  double *o_dx, *o_dy, *o_frame_params, *o_raw;
  double* o_rg_params;      // flag t: 2N x 2 max_iter, the chain after every half-step
  double* o_iter_times;     // flags T and t: max_iter seconds
  uint8_t* o_mask;          // Hb x fW column-major, may be null
  uint8_t* o_blocks_used;   // fW: block column has a valid pixel in the final mask, may be null
  const double* p0;         // 2N: the initial parameter vector, copied into p when a run starts
};

// ---------------------------------------------------------------------------------------------
// element loads

__device__ __forceinline__ double to_double(double v) { return v; }
__device__ __forceinline__ double to_double(float v) { return (double)v; }
__device__ __forceinline__ double to_double(uint16_t v) { return (double)v; }
__device__ __forceinline__ double to_double(__half v) { return (double)__half2float(v); }
__device__ __forceinline__ float to_float(double v) { return (float)v; }
__device__ __forceinline__ float to_float(float v) { return v; }
__device__ __forceinline__ float to_float(uint16_t v) { return (float)v; }
__device__ __forceinline__ float to_float(__half v) { return __half2float(v); }

template <class T>
struct Quad {
  T v[4];
};

// Template quad (T[iy][ix], T[iy][ix+1], T[iy+1][ix], T[iy+1][ix+1]) as Acc values.
template <class Acc, class TplT>
__device__ __forceinline__ void load_quad(const void* base, size_t i, Acc& t00, Acc& t01, Acc& t10, Acc& t11);

template <>
__device__ __forceinline__ void load_quad<double, double>(const void* base, size_t i, double& a, double& b,
                                                          double& c, double& d) {
  const double2* q = reinterpret_cast<const double2*>(base) + 2 * i;
  double2 lo = __ldg(q), hi = __ldg(q + 1);
  a = lo.x; b = lo.y; c = hi.x; d = hi.y;
}
template <>
__device__ __forceinline__ void load_quad<float, float>(const void* base, size_t i, float& a, float& b, float& c,
                                                        float& d) {
  float4 q = __ldg(reinterpret_cast<const float4*>(base) + i);
  a = q.x; b = q.y; c = q.z; d = q.w;
}
template <>
__device__ __forceinline__ void load_quad<float, __half>(const void* base, size_t i, float& a, float& b, float& c,
                                                         float& d) {
  uint2 raw = __ldg(reinterpret_cast<const uint2*>(base) + i);
  __half2 lo = *reinterpret_cast<__half2*>(&raw.x), hi = *reinterpret_cast<__half2*>(&raw.y);
  float2 l = __half22float2(lo), h = __half22float2(hi);
  a = l.x; b = l.y; c = h.x; d = h.y;
}

// ---------------------------------------------------------------------------------------------
// warp reductions

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------------------------
// 2x2 blocks: symmetric S = (s0 s2; s2 s1); general M = (m0 m1; m2 m3)

struct M2 {
  double a, b, c, d;  // (a b; c d)
};
__device__ __forceinline__ M2 m2_mul(const M2& x, const M2& y) {
  return {x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
}
__device__ __forceinline__ M2 m2_inv(const M2& x) {
  double det = x.a * x.d - x.b * x.c;
  double r = 1.0 / det;
  return {x.d * r, -x.b * r, -x.c * r, x.a * r};
}
__device__ __forceinline__ M2 m2_neg(const M2& x) { return {-x.a, -x.b, -x.c, -x.d}; }
__device__ __forceinline__ M2 m2_sub(const M2& x, const M2& y) { return {x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d}; }

}  // namespace ss
