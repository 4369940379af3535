// Evaluation of the warp model over block columns, and the per-frame line search.
//
// A warp evaluates one block column c (the pixels of the k scan lines between knots c and c+1 of
// one frame, Hb rows in the reference's block-matrix order, steady_scan.m:601-613); its lanes stride
// the rows, so frame and geometry loads are coalesced. Per pixel it evaluates the reference's
// d_applyParameters (task_applyparameters.cuh:33-82), d_createDifferenceImage
// (task_differenceimage.cuh:13-33) and d_updateGradients (task_updategradients.cu:3-29) in registers
// and reduces, per column, the sums that d_fillDiagonals (task_filldiagonals.cu:47-159), d_fillJTr
// (task_filljtr.cu:3-58), d_calcBaseErrval (task_calcerrval.cu:6-18) and the correlation kernels
// (task_correlation.cu:16-183) form from them. Nothing per pixel is written back.
//
// The reference keeps x, y, mask and the difference image as device buffers that later kernels
// read; here each frame carries two knot vectors instead: kmask (the knots of the last warp of the
// frame: x, y, mask) and kdiff (the knots of its last difference image). A pass that must see the
// reference's buffers evaluates both knot sets when they differ.
//
// Precision: Acc = double reproduces the reference's 'D' build (FP64 coordinates and sums, fma where
// nvcc contracts the reference source). Acc = float is the mixed 'S' path: FP32 geometry,
// coordinates, template samples and per-lane partial sums; the warp reductions, knots, solve and
// line-search comparison stay FP64.
#pragma once

#include <cooperative_groups.h>

#include "ss_common.cuh"
#include "ss_sched.cuh"

namespace ss {

namespace cg = cooperative_groups;

constexpr int kEvalWarps = 8;       // warps per assembly/final CTA
constexpr int kLsCluster = 8;       // CTAs per frame in the line-search cluster
constexpr int kLsMaxKnots = 256;    // knots per cluster CTA: frame_w <= kLsCluster * kLsMaxKnots
constexpr int kMaxFrameW = kLsCluster * kLsMaxKnots;
// frames of a tile worth staging a template window for (2: trial rounds 61.96 -> 61.57 ms against
// 4; 8 cost 1%)
constexpr int kMinWinFrames = 2;

// Resident 256-thread CTAs per SM requested from the register allocator: the FP32 correlation and
// final passes are latency-bound on frame loads and template gathers and need the warps (three
// CTAs, 80 registers); the FP32 assembly, whose 14 packed sums spill at 80 registers, runs two CTAs
// of up to 128 registers (assembly -5%, the correlation pass +41% when it ran two); the FP64 path
// keeps its registers.
template <class Acc, int MODE>
struct MinBlocks {
  static constexpr int value = 2;
};
#ifndef SS_EVAL_MIN_BLOCKS
#define SS_EVAL_MIN_BLOCKS 3
#endif
#ifndef SS_ASM_MIN_BLOCKS
#define SS_ASM_MIN_BLOCKS 2
#endif
template <int MODE>
struct MinBlocks<float, MODE> {
  static constexpr int value = MODE == 0 ? SS_ASM_MIN_BLOCKS : SS_EVAL_MIN_BLOCKS;
};

// Trial-round CTAs per SM (register bound) and the bytes of their template window; both must fit
// one SM's shared memory together (build-time tuning).
#ifndef SS_TRIAL_MIN_BLOCKS
#define SS_TRIAL_MIN_BLOCKS 4
#endif
#ifndef SS_TRIAL_WIN_KB
#define SS_TRIAL_WIN_KB 52
#endif
constexpr int kTrialMinBlocks = SS_TRIAL_MIN_BLOCKS;
constexpr int kTrialWinBytes = SS_TRIAL_WIN_KB * 1024;

// Line-search CTA: 256 threads; two (FP64) or four (FP32) CTAs per SM. A launch given window bytes
// keeps the template rows of the CTA's knot range in shared memory for the whole search.
template <class Acc>
struct LsShape {
  static constexpr int threads = 256, min_blocks = 2;
};
template <>
struct LsShape<float> {
  static constexpr int threads = 256, min_blocks = 4;
};

__device__ __forceinline__ bool frame_active(const GroupDesc& G, int f, int shift) {
  // groupActive[groupId + shift * nGroups] with zero-filled reads past the array
  // (task_calcerrval.cu:164-166, task_linesearch.cu:86-88).
  int gid = (f * G.W) / G.group_size + shift * G.n_rg;
  return gid < 2 * G.n_rg && G.grp_active[gid];
}

// The reference's difference-image buffer between its rewrites. hd_globalCorrelation swaps every
// valid pixel to image - difference and swaps back only the first 256 ceil(fW / 256) pixels in
// row-major order, the grid of its per-column kernel (task_correlation.cu:86-98); frames rewrite
// the buffer in d_calcAllGroupErrval and the line search, so with every group active the swapped
// pixels are rewritten before anything reads them, except hd_frameCorrelation of the same
// iteration (flag c), which then correlates the difference image itself past that index. With
// flag M a frame that is inactive in both half-steps keeps its buffer, and each later global
// correlation swaps its valid pixels past the index once more: the parity bitmap records which
// buffer pixels hold image - difference.
//
// DiffState of one block column: row_s, the first row whose pixel lies past the swap-back (kCorr);
// par_in, the column's parity words where its frame was not rewritten since the last global
// correlation (else nullptr: nothing swapped); par_out, the words the correlation pass writes. The
// correlation pass writes the other bitmap of the pair, which becomes current when the group moves
// to its iteration end (k_after_ls): a pass after which MainIteration retries the iteration without
// its filter (mainiteration.cpp:62-119) is followed by no global correlation and changes nothing.
struct DiffState {
  int row_s;
  const uint32_t* par_in;
  uint32_t* par_out;
};

__device__ __forceinline__ DiffState no_diff_state() { return DiffState{INT_MAX, nullptr, nullptr}; }

template <int MODE>
__device__ __forceinline__ DiffState diff_state(const GroupDesc& G, int par_sel, int shift, int f, int col) {
  DiffState d = no_diff_state();
  if (MODE == kCorr) {
    const int s = 256 * ((G.fW + 255) / 256);
    d.row_s = (s - col + G.fW - 1) / G.fW;  // first r with r * fW + col >= s
  }
  if (G.dparity) {
    const size_t nw = (size_t)((G.Hb + 31) >> 5), plane = (size_t)G.fW * nw;
    uint32_t* w = G.dparity + (size_t)par_sel * plane + (size_t)col * nw;
    bool stale;  // not rewritten since the last global correlation
    if (MODE == kAssemble) stale = !frame_active(G, f, shift) && !(shift == 1 && frame_active(G, f, 0));
    else if (MODE == kCorr) stale = !frame_active(G, f, 0) && !frame_active(G, f, 1);
    else stale = !frame_active(G, f, 0);  // kFinal, after the final hd_calculateGroupErrvals(mem, 0)
    if (stale) d.par_in = w;
    if (MODE == kCorr) d.par_out = G.dparity + (size_t)(par_sel ^ 1) * plane + (size_t)col * nw;
  }
  return d;
}

template <class Acc>
struct Limits;
template <>
struct Limits<double> {  // templateW - eps<double>() (task_applyparameters.cuh:44-45, eps.h:14-22)
  __device__ static double lim(int n) { return (double)(n - 1) - 2.220446049250313e-16; }
};
template <>
struct Limits<float> {   // templateW - eps<float>()
  __device__ static float lim(int n) { return (float)(n - 1) - 1.1920928955078125e-7f; }
};

// Warped position and validity of one pixel (task_applyparameters.cuh:57-62); a*b+c is contracted
// into fma the way nvcc contracts the reference source.
template <class Acc>
__device__ __forceinline__ bool warp_pixel(Acc kx0, Acc kx1, Acc ky0, Acc ky1, Acc f, Acc bx, Acc by, bool bm, Acc tw,
                                           Acc th, Acc& x, Acc& y) {
  const Acc one = (Acc)1;
  x = fma(kx1, f, fma(kx0, one - f, bx));
  y = fma(ky1, f, fma(ky0, one - f, by));
  return bm && x >= (Acc)0 && x < tw && y >= (Acc)0 && y < th;
}

// Integer part and fraction of a non-negative coordinate, as static_cast<int> in the reference.
__device__ __forceinline__ int split(double x, double& frac) {
  int i = (int)x;
  frac = x - (double)i;
  return i;
}
__device__ __forceinline__ int split(float x, float& frac) {
  // x + 2^23 rounded down holds floor(x) in its mantissa (0 <= x < 2^23)
  float v = __fadd_rd(x, 8388608.0f);
  frac = x - (v - 8388608.0f);
  return __float_as_int(v) - 0x4B000000;
}

template <class Acc>
struct Sample {
  Acc wI, wx, wy;
};

// Bilinear template value and warped gradients at a valid pixel (task_differenceimage.cuh:118-126,
// task_updategradients.cu:12-20). With gquad == nullptr the gradients are the template's forward
// differences (steady_scan.m:178-179), taken from the same four template values.
template <class Acc, class TplT, bool kGrad>
__device__ __forceinline__ Sample<Acc> sample(const GroupDesc& G, Acc x, Acc y) {
  Acc xf, yf;
  const int ix = split(x, xf), iy = split(y, yf);
  const size_t qi = (size_t)iy * (size_t)(G.Wt - 1) + (size_t)ix;
  Acc t00, t01, t10, t11;
  load_quad<Acc, TplT>(G.tquad, qi, t00, t01, t10, t11);
  const Acc one = (Acc)1;
  Acc a = fma(yf, t10, (one - yf) * t00);
  Acc b = fma(yf, t11, (one - yf) * t01);
  Sample<Acc> s;
  s.wI = fma(xf, b, (one - xf) * a);
  if (kGrad) {
    Acc gx0, gx1, gy0, gy1;
    if (G.gquad) {
      load_quad<Acc, TplT>(G.gquad, qi, gx0, gx1, gy0, gy1);
    } else {
      gx0 = t01 - t00; gx1 = t11 - t10; gy0 = t10 - t00; gy1 = t11 - t01;
    }
    s.wx = fma(yf, gx1, (one - yf) * gx0);
    s.wy = fma(xf, gy1, (one - xf) * gy0);
  } else {
    s.wx = s.wy = (Acc)0;
  }
  return s;
}

}  // namespace ss

#include "ss_pairs.cuh"

namespace ss {

// Template sample from the staged window (kWin, precision 'S'), else from the global template quads.
template <class Acc, class TplT, bool kGrad, bool kWin>
__device__ __forceinline__ Sample<Acc> samp(const GroupDesc& G, const TWin& w, Acc x, Acc y) {
  if constexpr (kWin && sizeof(Acc) == 4) return sample_win<kGrad>(w, x, y);
  else return sample<Acc, TplT, kGrad>(G, x, y);
}

template <class FrameT>
__device__ __forceinline__ FrameT ld_frame(const void* base, size_t i) {
  return __ldg(reinterpret_cast<const FrameT*>(base) + i);
}
template <>
__device__ __forceinline__ __half ld_frame<__half>(const void* base, size_t i) {
  unsigned short raw = __ldg(reinterpret_cast<const unsigned short*>(base) + i);
  return __ushort_as_half(raw);
}
template <class Acc, class FrameT>
__device__ __forceinline__ Acc ld_pixel(const void* base, size_t i) {
  return (Acc)to_double(ld_frame<FrameT>(base, i));
}
template <>
__device__ __forceinline__ float ld_pixel<float, uint16_t>(const void* base, size_t i) {
  return (float)ld_frame<uint16_t>(base, i);
}
template <>
__device__ __forceinline__ float ld_pixel<float, __half>(const void* base, size_t i) {
  return __half2float(ld_frame<__half>(base, i));
}
template <>
__device__ __forceinline__ float ld_pixel<float, float>(const void* base, size_t i) {
  return ld_frame<float>(base, i);
}

// Knots of one block column: set A (mask, position, gradients) and set B (difference image).
template <class Acc>
struct ColKnots {
  Acc ax0, ax1, ay0, ay1, bx0, bx1, by0, by1;
  bool dual;
};

template <class Acc>
__device__ __forceinline__ void set_knots(ColKnots<Acc>& k, double ax0, double ax1, double ay0, double ay1, double bx0,
                                          double bx1, double by0, double by1) {
  k.ax0 = (Acc)ax0; k.ax1 = (Acc)ax1; k.ay0 = (Acc)ay0; k.ay1 = (Acc)ay1;
  k.bx0 = (Acc)bx0; k.bx1 = (Acc)bx1; k.by0 = (Acc)by0; k.by1 = (Acc)by1;
  k.dual = bx0 != ax0 || bx1 != ax1 || by0 != ay0 || by1 != ay1;
}

// Geometry of one block column; generic pointers (global or shared memory).
template <class Acc>
struct ColGeo {
  const Acc* frac;
  const Acc* bx;
  const Acc* by;
  const uint8_t* bm;
  const Acc* fnext;  // tfrac of column (c+1) mod W; equals frac when all columns match
};

template <class Acc>
__device__ __forceinline__ ColGeo<Acc> global_geo(const GroupDesc& G, int cc);
template <>
__device__ __forceinline__ ColGeo<double> global_geo<double>(const GroupDesc& G, int cc) {
  const size_t o = (size_t)cc * G.Hb, on = (size_t)((cc + 1) % G.W) * G.Hb;
  return {G.frac + o, G.basex + o, G.basey + o, G.base_mask + o, G.frac_uniform ? G.frac + o : G.frac + on};
}
template <>
__device__ __forceinline__ ColGeo<float> global_geo<float>(const GroupDesc& G, int cc) {
  const size_t o = (size_t)cc * G.Hb, on = (size_t)((cc + 1) % G.W) * G.Hb;
  return {G.frac_f + o, G.basex_f + o, G.basey_f + o, G.base_mask + o, G.frac_uniform ? G.frac_f + o : G.frac_f + on};
}

__host__ __device__ constexpr int nsums(int mode) {
  return mode == kAssemble ? kCsAssemble : (mode == kTrial ? 1 : kCsStride - 2);
}

// Evaluates one block column with one warp and returns the warp-reduced sums (all lanes) and the
// valid-pixel count. coli is the column's offset in the frame data; mask_out (kFinal) receives the
// reference's mask output.
template <class Acc, class FrameT, class TplT, int MODE, bool AFFINE = false, bool WIN = false, bool DS = false>
__device__ __forceinline__ void eval_column(const GroupDesc& G, size_t coli, const ColGeo<Acc>& geo,
                                            const ColKnots<Acc>& k, double (&out)[kCsStride], int& cnt_out,
                                            uint8_t* mask_out, int cc = 0, const TWin& win = TWin{nullptr, 0, 0, 0},
                                            const DiffState& ds = no_diff_state()) {
  const int lane = threadIdx.x & 31;
  const int Hb = G.Hb;
  const Acc tw = Limits<Acc>::lim(G.Wt), th = Limits<Acc>::lim(G.Ht);
  const Acc one = (Acc)1;
  const bool split_fn = AFFINE ? false : geo.fnext != geo.frac;
  constexpr int NS = nsums(MODE);
  Acc s[NS];
#pragma unroll
  for (int i = 0; i < NS; i++) s[i] = (Acc)0;
  int cnt = 0;
  bool run = true;  // leading run of valid pixels (task_correlation.cu:24-34)
  // affine geometry: the lane's line offset l is fixed (k divides 32) and its pixel index j
  // advances by 32/k per row step
  Acc a_j = 0, a_dj = 0, a_f0 = 0, a_by = 0;
  if (AFFINE) {
    const int l = lane % G.geo_k;
    a_j = (Acc)(lane / G.geo_k);
    a_dj = (Acc)(32 / G.geo_k);
    a_f0 = ((Acc)(l * G.geo_L) + (Acc)0.5) * (Acc)G.geo_fs;
    a_by = fma((Acc)G.geo_ay, (Acc)(cc * G.geo_k + l), (Acc)G.geo_by);
  }

#pragma unroll 2
  for (int r0 = 0; r0 < Hb; r0 += 32) {
    const int r = r0 + lane;
    const bool in = r < Hb;
    Acc f = 0, bxv = 0, byv = 0;
    bool bm = false;
    if (AFFINE) {
      f = fma((Acc)G.geo_fs, a_j, a_f0);
      bxv = fma((Acc)G.geo_ax, a_j, (Acc)G.geo_bx);
      byv = a_by;
      bm = in;
      a_j += a_dj;
    } else if (in) {
      f = geo.frac[r];
      bxv = geo.bx[r];
      byv = geo.by[r];
      bm = geo.bm[r] != 0;
    }
    Acc x, y;
    const bool mA = warp_pixel<Acc>(k.ax0, k.ax1, k.ay0, k.ay1, f, bxv, byv, bm, tw, th, x, y) && in;
    cnt += mA ? 1 : 0;
    // the buffer pixel holds image - difference (flag M: swapped by earlier global correlations)
    const bool par = DS && ds.par_in != nullptr && in && ((ds.par_in[r0 >> 5] >> lane) & 1u);

    if (MODE == kAssemble) {
      Acc img = (mA || ((k.dual || par) && in)) ? ld_pixel<Acc, FrameT>(G.image, coli + r) : (Acc)0;
      Acc wx = 0, wy = 0, d = 0;
      if (mA) {
        Sample<Acc> sa = samp<Acc, TplT, true, WIN>(G, win, x, y);
        wx = sa.wx;
        wy = sa.wy;
        d = img - sa.wI;
      }
      if (k.dual) {
        Acc xb, yb;
        bool mB = warp_pixel<Acc>(k.bx0, k.bx1, k.by0, k.by1, f, bxv, byv, bm, tw, th, xb, yb) && in;
        d = mB ? img - samp<Acc, TplT, false, WIN>(G, win, xb, yb).wI : (Acc)0;
      }
      if (par) d = img - d;
      const Acc fn = split_fn ? (in ? geo.fnext[r] : (Acc)0) : f;
      const Acc fsq = f * f, csq = (one - f) * (one - f), fc = f - fsq, fnsq = fn * fn;
      const Acc gxx = wx * wx, gyy = wy * wy, gxy = wx * wy;
      s[kCsSsd] = fma(d, d, s[kCsSsd]);
      s[kCsAxx] = fma(gxx, csq, s[kCsAxx]);
      s[kCsAyy] = fma(gyy, csq, s[kCsAyy]);
      s[kCsAxy] = fma(gxy, csq, s[kCsAxy]);
      s[kCsBxx] = fma(gxx, fnsq, s[kCsBxx]);
      s[kCsByy] = fma(gyy, fnsq, s[kCsByy]);
      s[kCsBxy] = fma(gxy, fnsq, s[kCsBxy]);
      s[kCsOxx] = fma(gxx, fc, s[kCsOxx]);
      s[kCsOyy] = fma(gyy, fc, s[kCsOyy]);
      s[kCsOxy] = fma(gxy, fc, s[kCsOxy]);
      const Acc d1 = d * (one - f), d2 = d * f;
      s[kCsJ1x] = fma(d1, wx, s[kCsJ1x]);
      s[kCsJ1y] = fma(d1, wy, s[kCsJ1y]);
      s[kCsJ2x] = fma(d2, wx, s[kCsJ2x]);
      s[kCsJ2y] = fma(d2, wy, s[kCsJ2y]);
    } else if (MODE == kTrial) {
      if (mA) {
        Acc d = ld_pixel<Acc, FrameT>(G.image, coli + r) - samp<Acc, TplT, false, WIN>(G, win, x, y).wI;
        s[kCsSsd] = fma(d, d, s[kCsSsd]);
      }
    } else {
      // swapped difference image D' of task_correlation.cu:51-60 over the state (kmask, kdiff)
      Acc img = in ? ld_pixel<Acc, FrameT>(G.image, coli + r) : (Acc)0;
      Acc wA = 0;
      if (mA) wA = samp<Acc, TplT, false, WIN>(G, win, x, y).wI;
      bool mB = mA;
      Acc wB = wA;
      if (k.dual) {
        Acc xb, yb;
        mB = warp_pixel<Acc>(k.bx0, k.bx1, k.by0, k.by1, f, bxv, byv, bm, tw, th, xb, yb) && in;
        wB = mB ? samp<Acc, TplT, false, WIN>(G, win, xb, yb).wI : (Acc)0;
      }
      Acc dstate = mB ? img - wB : (Acc)0;  // differenceImage
      if (par) dstate = img - dstate;       // the buffer as the earlier swaps left it
      Acc dp = mA ? img - dstate : dstate;  // after d_swapWIDiff
      if (DS && MODE == kCorr && ds.par_out) {
        const unsigned nb = __ballot_sync(0xffffffffu, par != (mA && r >= ds.row_s));
        if (lane == 0) ds.par_out[r0 >> 5] = nb;
      }
      s[kCsSumD] += dp;
      unsigned bal = __ballot_sync(0xffffffffu, mA);
      unsigned le = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);
      if (run && ((~bal & le) == 0u) && mA) {
        s[kCsSetN] += one;
        s[kCsSetD] += dp;
        s[kCsSetDD] = fma(dp, dp, s[kCsSetDD]);
        s[kCsSetI] += img;
        s[kCsSetII] = fma(img, img, s[kCsSetII]);
        s[kCsSetDI] = fma(dp, img, s[kCsSetDI]);
      }
      run = run && (bal == 0xffffffffu);
      if (mA) {
        // hd_frameCorrelation after the global correlation (flag c) swaps back to the buffer the
        // pixels past the swap-back (kCorr); the final one sees the whole swapped image
        const Acc da = (DS && MODE == kCorr && r >= ds.row_s) ? dstate : dp;
        s[kCsFrD] += da;
        s[kCsFrI] += img;
        s[kCsFrDD] = fma(da, da, s[kCsFrDD]);
        s[kCsFrII] = fma(img, img, s[kCsFrII]);
        s[kCsFrDI] = fma(da, img, s[kCsFrDI]);
        if (MODE == kFinal) {
          Acc dA = img - wA;
          s[kCsFinalSsd] = fma(dA, dA, s[kCsFinalSsd]);
        }
      }
      if (MODE == kFinal && mask_out && in) mask_out[r] = mA ? 1 : 0;
    }
  }
  cnt_out = warp_sum(cnt);
#pragma unroll
  for (int i = 0; i < NS; i++) out[i] = warp_sum((double)s[i]);
}

// Trial SSD and valid count of up to NC block columns of one frame with one warp, their rows
// interleaved so that the frame loads and template gathers of all columns are in flight together.
// Loads are predicated by index clamping (a masked pixel reads row 0 / quad 0 and is discarded), so
// the column loop has no divergent branches. tq: frame-local column indices, nq <= NC of them valid.
template <class Acc, class FrameT, class TplT, bool AFFINE, int NC, bool WIN = false>
__device__ __forceinline__ void trial_columns(const GroupDesc& G, int b0, const TWin& win, const int (&tq)[NC], int nq,
                                              const Acc (&qx0)[NC], const Acc (&qx1)[NC], const Acc (&qy0)[NC],
                                              const Acc (&qy1)[NC], double (&ssd)[NC], int (&cnt)[NC]) {
  const int lane = threadIdx.x & 31;
  const int Hb = G.Hb;
  const Acc tw = Limits<Acc>::lim(G.Wt), th = Limits<Acc>::lim(G.Ht);
  Acc s[NC];
  int c[NC];
  size_t coli[NC];
  ColGeo<Acc> geo[NC];
  Acc aby[NC];
  Acc a_j = 0, a_dj = 0, a_f0 = 0;
  if (AFFINE) {
    const int l = lane % G.geo_k;
    a_j = (Acc)(lane / G.geo_k);
    a_dj = (Acc)(32 / G.geo_k);
    a_f0 = ((Acc)(l * G.geo_L) + (Acc)0.5) * (Acc)G.geo_fs;
#pragma unroll
    for (int q = 0; q < NC; q++) aby[q] = fma((Acc)G.geo_ay, (Acc)(tq[q] * G.geo_k + l), (Acc)G.geo_by);
  }
#pragma unroll
  for (int q = 0; q < NC; q++) {
    s[q] = (Acc)0;
    c[q] = 0;
    coli[q] = (size_t)(b0 + tq[q]) * Hb;
    if (!AFFINE) geo[q] = global_geo<Acc>(G, tq[q]);
  }
  for (int r0 = 0; r0 < Hb; r0 += 32) {
    const int r = r0 + lane;
    const bool in = r < Hb;
    const int rr = in ? r : 0;
    Acc fa = 0, bxa = 0;
    if (AFFINE) {
      fa = fma((Acc)G.geo_fs, a_j, a_f0);
      bxa = fma((Acc)G.geo_ax, a_j, (Acc)G.geo_bx);
      a_j += a_dj;
    }
#pragma unroll
    for (int q = 0; q < NC; q++) {
      if (q < nq) {
        const Acc f = AFFINE ? fa : geo[q].frac[rr];
        const Acc bx = AFFINE ? bxa : geo[q].bx[rr];
        const Acc by = AFFINE ? aby[q] : geo[q].by[rr];
        const bool bm = AFFINE ? in : (in && geo[q].bm[rr] != 0);
        Acc x, y;
        const bool m = warp_pixel<Acc>(qx0[q], qx1[q], qy0[q], qy1[q], f, bx, by, bm, tw, th, x, y);
        const Acc img = ld_pixel<Acc, FrameT>(G.image, coli[q] + rr);
        const Acc wI = samp<Acc, TplT, false, WIN>(G, win, m ? x : (Acc)0, m ? y : (Acc)0).wI;
        const Acc d = img - wI;
        s[q] = m ? fma(d, d, s[q]) : s[q];
        c[q] += m ? 1 : 0;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NC; q++) {
    ssd[q] = warp_sum((double)s[q]);
    cnt[q] = warp_sum(c[q]);
  }
}

// Shared-memory bytes of one staged block column of geometry (tfrac, basex, basey, the next
// column's tfrac, base_mask), rounded up to 16.
template <class Acc>
__host__ __device__ constexpr size_t stage_bytes(int hb) {
  return ((size_t)hb * (4 * sizeof(Acc) + 1) + 15) & ~(size_t)15;
}

// Knots of block column cc of frame f in the assembly pass: the mask knots (p) and the knots of the
// difference image (p, or the stale kdiff of a frame that is not active in this half-step).
__device__ __forceinline__ void assembly_knots(const GroupDesc& G, int f, int cc, int shift, double (&k)[8]) {
  const int W = G.W, N = G.N, c = f * W + cc;
  k[0] = G.p[c];
  k[1] = G.p[c + 1];
  k[2] = G.p[N + c];
  k[3] = G.p[N + c + 1];
  if (frame_active(G, f, shift)) {
    k[4] = k[0]; k[5] = k[1]; k[6] = k[2]; k[7] = k[3];
  } else {
    const double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
    k[4] = kd[cc]; k[5] = kd[cc + 1]; k[6] = kd[W + 1 + cc]; k[7] = kd[W + 1 + cc + 1];
  }
}

// Assembly (at p), correlation and final (at kmask) passes of one tile: block column cc of one group
// and frames fb*fpc .. of its chunk fb, a warp per frame at a time; the column's geometry is staged in
// shared memory once for all of them (at smem), and the frames share the template rows around the
// column (a window staged after the geometry, for precision 'S', or L1).
template <class Acc, class FrameT, class TplT, int MODE>
__device__ __forceinline__ void eval_tile(const GroupDesc& G, const GroupCtl& C, int cc, int fb, unsigned char* smem,
                                          uint64_t* bar, unsigned& bar_phase, bool& win_ok, int stage_rows,
                                          int win_bytes) {
  if (!group_has_work<MODE>(C)) return;
  const int W = G.W, N = G.N, Hb = G.Hb, fpc = G.frames_per_cta;
  const int warp = threadIdx.x >> 5;
  const int f0 = fb * fpc;

  // assembly: the frames of the tile whose column knots differ from those of the column's last
  // assembly (bit f - f0); the others keep their sums (the same knots give the same sums)
  unsigned long long need = ~0ull;
  if (MODE == kAssemble) {
    __shared__ unsigned long long s_need;
    const int lane = threadIdx.x & 31, fe = min(G.nF, f0 + fpc);
    if (warp == 0) {
      unsigned long long m = 0;
      for (int fa = f0; fa < fe; fa += 32) {
        const int f = fa + lane;
        bool changed = false;
        if (f < fe) {
          double k[8];
          assembly_knots(G, f, cc, C.shift, k);
          const double* prev = G.asmk + (size_t)(f * W + cc) * 8;
#pragma unroll
          for (int i = 0; i < 8; i++) changed |= __double_as_longlong(k[i]) != __double_as_longlong(prev[i]);
          // a swapped buffer changes with every global correlation, the knots staying the same
          changed |= diff_state<kAssemble>(G, C.par_sel, C.shift, f, f * W + cc).par_in != nullptr;
        }
        m |= (unsigned long long)__ballot_sync(0xffffffffu, changed) << (fa - f0);
      }
      if (lane == 0) {
        s_need = m;
        const int kept = (fe - f0) - __popcll(m);
        if (kept) atomicAdd(G.staging + 6, (unsigned long long)kept);
      }
    }
    __syncthreads();
    need = s_need;
    if (need == 0) return;  // uniform over the CTA
  }

  ColGeo<Acc> geo = global_geo<Acc>(G, cc);
  const bool affine = sizeof(Acc) == 4 && G.geo_k > 0;
  if (!affine && Hb <= stage_rows) {
    Acc* sf = reinterpret_cast<Acc*>(smem);
    Acc* sx = sf + Hb;
    Acc* sy = sx + Hb;
    Acc* sn = sy + Hb;
    uint8_t* sm = reinterpret_cast<uint8_t*>(sn + Hb);
    const bool split_fn = geo.fnext != geo.frac;
    for (int r = threadIdx.x; r < Hb; r += blockDim.x) {
      sf[r] = __ldg(geo.frac + r);
      sx[r] = __ldg(geo.bx + r);
      sy[r] = __ldg(geo.by + r);
      sm[r] = __ldg(geo.bm + r);
      if (split_fn) sn[r] = __ldg(geo.fnext + r);
    }
    __syncthreads();
    geo = {sf, sx, sy, sm, split_fn ? sn : sf};
  }
  const int f_end = min(G.nF, (fb + 1) * fpc);

  // Precision 'S': stage the template rows every pixel of this CTA can sample (the column's basey
  // range widened by its frames' y knots) into shared memory; windows that would not fit, and
  // tiles of too few frames to repay the copy, use the global template.
  TWin win{nullptr, 0, 0, 0};
  if constexpr (sizeof(Acc) == 4) {
    const int win_cap = G.tplain ? win_bytes / (G.tpitch * (int)sizeof(float)) : 0;
    if (win_ok && win_cap >= 2 && !G.gquad && f_end - fb * fpc >= kMinWinFrames) {
      const size_t geo_bytes = (!affine && Hb <= stage_rows) ? stage_bytes<Acc>(Hb) : 0;
      float* wbuf = reinterpret_cast<float*>(smem + geo_bytes);
      float klo = INFINITY, khi = -INFINITY;
      for (int f = fb * fpc + threadIdx.x; f < f_end; f += blockDim.x) {
        const int c = f * W + cc;
        const double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
        float a0, a1, b0 = NAN, b1 = NAN;
        if (MODE == kAssemble) {
          a0 = (float)G.p[N + c];
          a1 = (float)G.p[N + c + 1];
          if (!frame_active(G, f, C.shift)) {
            b0 = (float)kd[W + 1 + cc];
            b1 = (float)kd[W + 1 + cc + 1];
          }
        } else {
          const double* km = G.kmask + (size_t)f * 2 * (W + 1);
          a0 = (float)km[W + 1 + cc];
          a1 = (float)km[W + 1 + cc + 1];
          b0 = (float)kd[W + 1 + cc];
          b1 = (float)kd[W + 1 + cc + 1];
        }
        klo = fminf(klo, fminf(fminf(a0, a1), fminf(b0, b1)));
        khi = fmaxf(khi, fmaxf(fmaxf(a0, a1), fmaxf(b0, b1)));
      }
      block_minmax(klo, khi);
      int r0, rows;
      window_rows(G, G.col_yrange[2 * cc] + klo, G.col_yrange[2 * cc + 1] + khi, win_cap, r0, rows);
      if (rows > 0) {
        if (stage_window(G, wbuf, r0, rows, bar, bar_phase)) win = {wbuf, r0, rows, G.tpitch};
        else win_ok = false;  // a copy may still be in flight: no further windows in this CTA
      }
    }
  }

  if (threadIdx.x == 0) {
    atomicAdd(G.staging + 0, 1ull);
    if (win.p) atomicAdd(G.staging + 1, 1ull);
  }
  for (int f = fb * fpc + warp; f < f_end; f += kEvalWarps) {
    const int c = f * W + cc;
    ColKnots<Acc> k;
    if (MODE == kAssemble) {
      if (!((need >> (f - f0)) & 1ull)) continue;
      double ka[8];
      assembly_knots(G, f, cc, C.shift, ka);  // (the difference image of an inactive frame is stale)
      set_knots(k, ka[0], ka[1], ka[2], ka[3], ka[4], ka[5], ka[6], ka[7]);
      // the knots the column's sums belong to (no other tile reads this column's entry meanwhile),
      // stored before the evaluation so that they hold no registers across it
      if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int i = 0; i < 8; i++) G.asmk[(size_t)c * 8 + i] = ka[i];
    } else {
      const double* km = G.kmask + (size_t)f * 2 * (W + 1);
      const double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
      set_knots(k, km[cc], km[cc + 1], km[W + 1 + cc], km[W + 1 + cc + 1], kd[cc], kd[cc + 1], kd[W + 1 + cc],
                kd[W + 1 + cc + 1]);
    }
    const size_t coli = (size_t)c * Hb;
    double out[kCsStride];
    int cnt;
    uint8_t* mo = G.o_mask ? G.o_mask + coli : nullptr;
    const DiffState ds = diff_state<MODE>(G, C.par_sel, C.shift, f, c);
    if (ds.par_in || ds.par_out || (MODE == kCorr && (G.flags & kFlagFrameCorr))) {
      // the buffer state of flags M and c (DiffState), on the table-geometry path
      eval_column<Acc, FrameT, TplT, MODE, false, false, true>(G, coli, geo, k, out, cnt, mo, cc,
                                                               TWin{nullptr, 0, 0, 0}, ds);
    } else if constexpr (sizeof(Acc) == 4) {
      const bool pairs = win.p && G.pair_ok && !k.dual;
      if (MODE == kAssemble && pairs) {
        bool quads = false;
        if constexpr (sizeof(FrameT) == 2) quads = G.quad_ok;  // 16-byte loads handed round by shuffles
        if (quads) {
          if constexpr (sizeof(FrameT) == 2)
            assemble_pairs16<FrameT>(G, coli, pair_col(G, cc, k.ax0, k.ax1, k.ay0, k.ay1), pair_win(win), out, cnt);
        } else {
          assemble_pairs<FrameT>(G, coli, pair_col(G, cc, k.ax0, k.ax1, k.ay0, k.ay1), pair_win(win), out, cnt);
        }
        if ((threadIdx.x & 31) == 0) atomicAdd(G.staging + 5, 1ull);
      } else if (MODE != kAssemble && pairs) {
        corr_pairs<FrameT, MODE>(G, coli, pair_col(G, cc, k.ax0, k.ax1, k.ay0, k.ay1), pair_win(win), out, cnt, mo);
      } else if (win.p) {
        if (affine) eval_column<Acc, FrameT, TplT, MODE, true, true>(G, coli, geo, k, out, cnt, mo, cc, win);
        else eval_column<Acc, FrameT, TplT, MODE, false, true>(G, coli, geo, k, out, cnt, mo, cc, win);
      } else {
        if (affine) eval_column<Acc, FrameT, TplT, MODE, true>(G, coli, geo, k, out, cnt, mo, cc);
        else eval_column<Acc, FrameT, TplT, MODE>(G, coli, geo, k, out, cnt, mo);
      }
    } else {
      eval_column<Acc, FrameT, TplT, MODE>(G, coli, geo, k, out, cnt, mo);
    }
    if ((threadIdx.x & 31) == 0) {
      double* dst = (MODE == kAssemble ? G.asmsum : G.colsum) + (size_t)c * kCsStride;
#pragma unroll
      for (int i = 0; i < nsums(MODE); i++) dst[i] = out[i];
      if (MODE == kAssemble) {
        G.asmcnt[c] = cnt;
      } else {
        G.colcnt[c] = cnt;
      }
    }
  }
}

// The evaluation passes over the tiles of the launch's schedule (ss_sched.cuh), one tile at a time
// per CTA. Dynamic shared memory: the window's mbarrier (16 bytes), the column geometry, the window.
template <class Acc, class FrameT, class TplT, int MODE>
__global__ void __launch_bounds__(32 * kEvalWarps, MinBlocks<Acc, MODE>::value)
    k_eval(const GroupDesc* __restrict__ gds, int* __restrict__ sched, int cap, const GroupCtl* __restrict__ ctl,
           int stage_rows, int win_bytes) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_tile[3];
  __shared__ GroupDesc s_gd;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  if (threadIdx.x == 0) mbar_init(bar);
  __syncthreads();
  unsigned bar_phase = 0;
  bool win_ok = true;
  while (fetch_tile(sched, cap, s_tile)) {
    const int g = s_tile[0];
    load_desc(gds + g, &s_gd);
    eval_tile<Acc, FrameT, TplT, MODE>(s_gd, ctl[g], s_tile[1], s_tile[2], smem + 16, bar, bar_phase, win_ok,
                                       stage_rows, win_bytes);
    __syncthreads();  // s_tile, s_gd and the shared buffers are reused by the next tile
  }
  if (!win_ok) drain_window(bar, bar_phase);  // a timed-out copy may still write this CTA's memory
}

// Line search of one frame per thread-block cluster (task_linesearch.cu:76-149), for every frame of
// every group in kPhHalf. The cluster's CTAs split the frame's block columns; each trial's SSD,
// valid count, block presence and largest step are reduced across the cluster through distributed
// shared memory, rank 0 decides, and every CTA applies the decision to its own copy of the knots, so
// the frame's whole search runs without leaving the kernel. The frame's right boundary knot is the
// committed knot at line-search start (p_snap), or the never-written 1e6 for the last frame.
// After shift 1 the cluster also evaluates the frame's correlation sums (the iteration-end state).
template <class Acc, class FrameT, class TplT>
__global__ void __launch_bounds__(LsShape<Acc>::threads, LsShape<Acc>::min_blocks)
    k_linesearch(const GroupDesc* __restrict__ gds, const int* __restrict__ frame_group, GroupCtl* __restrict__ ctl,
                 int win_bytes) {
  constexpr int kLsThreads = LsShape<Acc>::threads;
  extern __shared__ __align__(16) unsigned char ls_smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int gf = blockIdx.x / kLsCluster;
  const int g = frame_group[gf];
  const GroupDesc& G = gds[g];
  GroupCtl& C = ctl[g];
  if (C.phase != kPhHalf || C.ls_state != 1) return;  // uniform over the cluster
  const int f = gf - G.frame_base;
  const int W = G.W, N = G.N, Hb = G.Hb, b0 = f * W;
  const int shift = C.shift;
  const bool searching = G.fstate[f] & 2;
  if (!searching && shift == 0) return;

  const int cpc = (W + kLsCluster - 1) / kLsCluster;
  const int lo = min(W, rank * cpc), hi = min(W, lo + cpc);  // own knots [lo, hi); copies [lo, hi]
  const int nk = hi - lo + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = kLsThreads / 32;
  const bool last_frame = f + 1 == G.nF;

  // knot copies: p, deltaP, kmask, kdiff over [lo, hi] for x (first) and y (second)
  __shared__ double s_p[2][kLsMaxKnots + 1], s_dp[2][kLsMaxKnots + 1], s_km[2][kLsMaxKnots + 1],
      s_kd[2][kLsMaxKnots + 1];
  __shared__ double s_part[5][kLsThreads / 32];
  __shared__ double s_red[5];      // this CTA's partials: ssd, cnt, present, max|dp|, regulariser
  __shared__ double s_dec[2];      // rank 0's decision: action, errval
  const double bxv = last_frame ? kPnewFill : G.p_snap[b0 + W];
  const double byv = last_frame ? kPnewFill : G.p_snap[N + b0 + W];
  for (int i = threadIdx.x; i < nk; i += blockDim.x) {
    const int t = lo + i;
    for (int d = 0; d < 2; d++) {
      const size_t o = (size_t)d * N + b0 + t;
      if (t < W) {
        s_p[d][i] = G.p[o];
        s_dp[d][i] = G.delta_p[o];
      } else {  // the frame's boundary knot: fixed trial value, no step
        s_p[d][i] = d ? byv : bxv;
        s_dp[d][i] = 0.0;
      }
      s_km[d][i] = G.kmask[(size_t)f * 2 * (W + 1) + d * (W + 1) + t];
      s_kd[d][i] = G.kdiff[(size_t)f * 2 * (W + 1) + d * (W + 1) + t];
    }
  }
  __syncthreads();

  // Precision 'S': stage the template rows of this CTA's lines for every knot vector the search
  // and the correlation pass can evaluate (trial knots lie between p and p + deltaP; kmask and
  // kdiff are earlier states); a range that does not fit uses the global template.
  TWin win{nullptr, 0, 0, 0};
  uint64_t* stage_bar = nullptr;  // set when a staging copy timed out (drained before the CTA exits)
  unsigned stage_phase = 0;
  if constexpr (sizeof(Acc) == 4) {
    const int win_cap = G.tplain ? win_bytes / (G.tpitch * (int)sizeof(float)) : 0;
    if (win_cap >= 2 && !G.gquad && hi > lo) {
      float klo = INFINITY, khi = -INFINITY;
      for (int i = threadIdx.x; i < nk; i += blockDim.x) {
        const float a = (float)s_p[1][i], b = (float)(s_p[1][i] + s_dp[1][i]);
        const float c = (float)s_km[1][i], d = (float)s_kd[1][i];
        klo = fminf(klo, fminf(fminf(a, b), fminf(c, d)));
        khi = fmaxf(khi, fmaxf(fmaxf(a, b), fmaxf(c, d)));
      }
      float ylo = INFINITY, yhi = -INFINITY;
      for (int t = lo + threadIdx.x; t < hi; t += blockDim.x) {
        ylo = fminf(ylo, G.col_yrange[2 * t]);
        yhi = fmaxf(yhi, G.col_yrange[2 * t + 1]);
      }
      block_minmax(klo, khi);
      block_minmax(ylo, yhi);
      int r0, rows;
      window_rows(G, ylo + klo, yhi + khi, win_cap, r0, rows);
      if (rows > 0) {
        float* wbuf = reinterpret_cast<float*>(ls_smem);
        uint64_t* bar = reinterpret_cast<uint64_t*>(ls_smem + (size_t)win_bytes);
        if (threadIdx.x == 0) mbar_init(bar);
        __syncthreads();
        if (stage_window(G, wbuf, r0, rows, bar, stage_phase)) win = {wbuf, r0, rows, G.tpitch};
        else stage_bar = bar;
      }
    }
  }
  bool pairs = false;
  if constexpr (sizeof(Acc) == 4) pairs = win.p && G.pair_ok;
  if (threadIdx.x == 0) {
    atomicAdd(G.staging + 2, 1ull);
    if (win.p) atomicAdd(G.staging + 3, 1ull);
    if (pairs) atomicAdd(G.staging + 4, 1ull);
  }

  const double thr = G.move_thresh, rho = G.ls_mult;
  int trials = 0;
  while (searching) {
    // trial knots: pnew = p + deltaP for own knots (task_linesearch.cu:50-54), boundary as is
    double ssd = 0, maxabs = 0, reg = 0;
    long long cnt = 0;
    bool present = false;
    constexpr int NC = 4;
    if (pairs) {
      for (int t = lo + warp; t < hi; t += nw) {
        const int i = t - lo;
        const float x0 = (float)(s_p[0][i] + s_dp[0][i]), y0 = (float)(s_p[1][i] + s_dp[1][i]);
        const float x1 = (float)((t + 1 < W) ? s_p[0][i + 1] + s_dp[0][i + 1] : s_p[0][i + 1]);
        const float y1 = (float)((t + 1 < W) ? s_p[1][i + 1] + s_dp[1][i + 1] : s_p[1][i + 1]);
        double qs;
        int qc;
        trial_pairs<FrameT>(G, (size_t)(b0 + t) * Hb, pair_col(G, t, x0, x1, y0, y1), pair_win(win), qs, qc);
        ssd += qs;
        cnt += qc;
        present |= qc >= G.min_points[t];
      }
    }
    for (int t0 = lo + warp; !pairs && t0 < hi; t0 += nw * NC) {
      int tq[NC], nq = 0;
      Acc qx0[NC], qx1[NC], qy0[NC], qy1[NC];
#pragma unroll
      for (int q = 0; q < NC; q++) {
        int t = t0 + q * nw;
        if (t >= hi) t = t0;  // padding column, not evaluated (nq excludes it)
        else nq = q + 1;
        const int i = t - lo;
        tq[q] = t;
        qx0[q] = (Acc)(s_p[0][i] + s_dp[0][i]);
        qy0[q] = (Acc)(s_p[1][i] + s_dp[1][i]);
        qx1[q] = (Acc)((t + 1 < W) ? s_p[0][i + 1] + s_dp[0][i + 1] : s_p[0][i + 1]);
        qy1[q] = (Acc)((t + 1 < W) ? s_p[1][i + 1] + s_dp[1][i + 1] : s_p[1][i + 1]);
      }
      double qs[NC];
      int qc[NC];
      bool aff = false;
      if constexpr (sizeof(Acc) == 4) aff = G.geo_k > 0;
      if (win.p) {
        if (aff) trial_columns<Acc, FrameT, TplT, true, NC, true>(G, b0, win, tq, nq, qx0, qx1, qy0, qy1, qs, qc);
        else trial_columns<Acc, FrameT, TplT, false, NC, true>(G, b0, win, tq, nq, qx0, qx1, qy0, qy1, qs, qc);
      } else {
        if (aff) trial_columns<Acc, FrameT, TplT, true, NC>(G, b0, win, tq, nq, qx0, qx1, qy0, qy1, qs, qc);
        else trial_columns<Acc, FrameT, TplT, false, NC>(G, b0, win, tq, nq, qx0, qx1, qy0, qy1, qs, qc);
      }
#pragma unroll
      for (int q = 0; q < NC; q++) {
        if (q < nq) {
          ssd += qs[q];
          cnt += qc[q];
          present |= qc[q] >= G.min_points[tq[q]];
        }
      }
    }
    for (int i = threadIdx.x; i < hi - lo; i += blockDim.x) {
      const int t = lo + i;
      maxabs = fmax(maxabs, fmax(fabs(s_dp[0][i]), fabs(s_dp[1][i])));
      if (G.lambda != 0.0) {  // knot-difference regulariser of the trial (extension)
        double x0 = s_p[0][i] + s_dp[0][i], y0 = s_p[1][i] + s_dp[1][i];
        double x1 = t + 1 < W ? s_p[0][i + 1] + s_dp[0][i + 1] : G.p_snap[b0 + W];
        double y1 = t + 1 < W ? s_p[1][i + 1] + s_dp[1][i + 1] : G.p_snap[N + b0 + W];
        reg += (x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxabs = fmax(maxabs, __shfl_xor_sync(0xffffffffu, maxabs, o));
    reg = warp_sum(reg);
    if (lane == 0) {
      s_part[0][warp] = ssd;
      s_part[1][warp] = (double)cnt;
      s_part[2][warp] = present ? 1.0 : 0.0;
      s_part[3][warp] = maxabs;
      s_part[4][warp] = reg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0, b = 0, pr = 0, m = 0, rg = 0;
      for (int w = 0; w < nw; w++) {
        a += s_part[0][w];
        b += s_part[1][w];
        pr = fmax(pr, s_part[2][w]);
        m = fmax(m, s_part[3][w]);
        rg += s_part[4][w];
      }
      s_red[0] = a; s_red[1] = b; s_red[2] = pr; s_red[3] = m; s_red[4] = rg;
    }
    cluster.sync();
    if (rank == 0 && threadIdx.x == 0) {
      double a = 0, b = 0, pr = 0, m = 0, rg = 0;
      for (int q = 0; q < kLsCluster; q++) {
        const double* r = cluster.map_shared_rank(s_red, q);
        a += r[0]; b += r[1]; pr = fmax(pr, r[2]); m = fmax(m, r[3]); rg += r[4];
      }
      // actions: 0 accept, 1 reduce and retry, 2 stop; bit 4: a block was present (the
      // difference image was written)
      int action;
      double ev = 0;
      if (pr > 0) {
        ev = (G.lambda != 0.0) ? (a + G.lambda * rg) / b : a / b;
        if (ev < G.errval[shift * G.nF + f]) action = 0;
        else action = (m > thr) ? 1 : 2;  // d_checkMovement before d_reduceDeltaP
        action |= 16;
      } else {
        action = (m * rho > thr) ? 1 : 2;  // d_reduceDeltaP before d_checkMovement
      }
      ++trials;
      atomicAdd((unsigned long long*)&C.n_eval, 1ull);
      atomicAdd((unsigned long long*)&C.passes[kTrial], 1ull);
      if ((action & 15) == 1 && trials >= kTrialCap) {
        action = (action & 16) | 2;
        C.cap_hit = 1;
      }
      if ((action & 15) == 0 && b0 == 0) G.errval[shift * G.nF] = ev;  // only idx == 0 writes (:135)
      s_dec[0] = (double)action;
      s_dec[1] = ev;
    }
    cluster.sync();
    const int action = (int)*cluster.map_shared_rank(&s_dec[0], 0);
    // the reference's buffers now hold this trial's x, y, mask; the difference image only if a
    // block was present; then p or deltaP change
    for (int i = threadIdx.x; i < nk; i += blockDim.x) {
      const int t = lo + i;
      for (int d = 0; d < 2; d++) {
        const double v = (t < W) ? s_p[d][i] + s_dp[d][i] : s_p[d][i];
        s_km[d][i] = v;
        if (action & 16) s_kd[d][i] = v;
        if (t < W) {
          if ((action & 15) == 0) s_p[d][i] = v;
          else if ((action & 15) == 1) s_dp[d][i] *= rho;
          else if (!(action & 16)) s_dp[d][i] *= rho;  // absent block: reduced before the stop test
        }
      }
    }
    __syncthreads();
    if ((action & 15) != 1) break;
  }

  if (searching) {  // write back own knots (and the boundary copies) of the search
    for (int i = threadIdx.x; i < nk; i += blockDim.x) {
      const int t = lo + i;
      for (int d = 0; d < 2; d++) {
        if (t < hi) {
          G.p[(size_t)d * N + b0 + t] = s_p[d][i];
          G.delta_p[(size_t)d * N + b0 + t] = s_dp[d][i];
        }
        if (t < hi || t == W) {
          G.kmask[(size_t)f * 2 * (W + 1) + d * (W + 1) + t] = s_km[d][i];
          G.kdiff[(size_t)f * 2 * (W + 1) + d * (W + 1) + t] = s_kd[d][i];
        }
      }
    }
    if (rank == 0 && threadIdx.x == 0) G.fstate[f] = 0;
  }

  if (shift == 1) {  // iteration-end correlation sums of this frame's state (task.cpp:284)
    for (int t = lo + warp; t < hi; t += nw) {
      const int i = t - lo;
      ColKnots<Acc> k;
      set_knots(k, s_km[0][i], s_km[0][i + 1], s_km[1][i], s_km[1][i + 1], s_kd[0][i], s_kd[0][i + 1], s_kd[1][i],
                s_kd[1][i + 1]);
      double out[kCsStride];
      int c;
      const DiffState ds = diff_state<kCorr>(G, C.par_sel, shift, f, b0 + t);
      if (ds.par_out || (G.flags & kFlagFrameCorr)) {  // the buffer state of flags M and c (DiffState)
        eval_column<Acc, FrameT, TplT, kCorr, false, false, true>(G, (size_t)(b0 + t) * Hb, global_geo<Acc>(G, t), k,
                                                                  out, c, nullptr, t, TWin{nullptr, 0, 0, 0}, ds);
      } else if constexpr (sizeof(Acc) == 4) {
        const size_t coli = (size_t)(b0 + t) * Hb;
        if (win.p) {
          if (G.geo_k > 0)
            eval_column<Acc, FrameT, TplT, kCorr, true, true>(G, coli, global_geo<Acc>(G, t), k, out, c, nullptr, t, win);
          else
            eval_column<Acc, FrameT, TplT, kCorr, false, true>(G, coli, global_geo<Acc>(G, t), k, out, c, nullptr, t,
                                                               win);
        } else if (G.geo_k > 0) {
          eval_column<Acc, FrameT, TplT, kCorr, true>(G, coli, global_geo<Acc>(G, t), k, out, c, nullptr, t);
        } else {
          eval_column<Acc, FrameT, TplT, kCorr>(G, coli, global_geo<Acc>(G, t), k, out, c, nullptr);
        }
      } else {
        eval_column<Acc, FrameT, TplT, kCorr>(G, (size_t)(b0 + t) * Hb, global_geo<Acc>(G, t), k, out, c, nullptr);
      }
      if (lane == 0) {
        double* dst = G.colsum + (size_t)(b0 + t) * kCsStride;
        for (int q = 0; q < nsums(kCorr); q++) dst[q] = out[q];
        G.colcnt[b0 + t] = c;
      }
    }
  }
  if (stage_bar) drain_window(stage_bar, stage_phase);  // uniform over the CTA
  cluster.sync();  // no CTA leaves while others may still read its shared memory
}


// ---------------------------------------------------------------------------------------------
// Line search in trial rounds (precision 'S')
//
// A round evaluates one trial (pnew = p + deltaP on the frame's own knots, the right boundary knot
// fixed: task_linesearch.cu:50-54) of every frame still searching, over the assembly tiles (block
// column cc x a chunk of frames) with the template rows of the tile in shared memory. Each column
// writes its SSD and valid count; the warp that completes a frame's last column (a device-wide
// arrival count per frame) makes the frame's decision of task_linesearch.cu:95-149: accept, halve
// deltaP and search on, or stop. Rounds repeat until no frame searches.

constexpr int kMaxChunk = 64;       // frames_per_cta bound

// Device-scope fetch-and-add with acquire-release order: the writes before it are visible to a
// thread that observes the new count, and the caller sees every write released before the count
// it read.
__device__ __forceinline__ int atomic_add_acq_rel(int* p, int v) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Device-scope load with acquire order.
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Decision for frame f after all its columns of the round were evaluated (one warp).
__device__ __forceinline__ void ls_decide(const GroupDesc& G, GroupCtl& C, int f) {
  const int lane = threadIdx.x & 31;
  const int W = G.W, N = G.N, b0 = f * W, shift = C.shift;
  const bool last_frame = f + 1 == G.nF;
  const double bx = G.p_snap[b0 + W], by = G.p_snap[N + b0 + W];
  double a = 0, m = 0, rg = 0, b = 0;
  bool pr = false;
  for (int t = lane; t < W; t += 32) {
    const int c = b0 + t;
    a += __ldcg(G.colsum + (size_t)c * kCsStride + kCsSsd);
    const int n = __ldcg(G.colcnt + c);
    b += (double)n;
    pr |= n >= G.min_points[t];
    const double dx = G.delta_p[c], dy = G.delta_p[N + c];
    m = fmax(m, fmax(fabs(dx), fabs(dy)));
    if (G.lambda != 0.0) {  // knot-difference regulariser of the trial (extension)
      const double x0 = G.p[c] + dx, y0 = G.p[N + c] + dy;
      const double x1 = t + 1 < W ? G.p[c + 1] + G.delta_p[c + 1] : bx;
      const double y1 = t + 1 < W ? G.p[N + c + 1] + G.delta_p[N + c + 1] : by;
      rg += (x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0);
    }
  }
  a = warp_sum(a);
  b = warp_sum(b);
  rg = warp_sum(rg);
  pr = __any_sync(0xffffffffu, pr);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  // actions: 0 accept, 1 reduce and retry, 2 stop; bit 4: a block was present (the difference
  // image was written)
  int action = 0;
  if (lane == 0) {
    const double thr = G.move_thresh, rho = G.ls_mult;
    double ev = 0;
    if (pr) {
      ev = (G.lambda != 0.0) ? (a + G.lambda * rg) / b : a / b;
      if (ev < G.errval[shift * G.nF + f]) action = 0;
      else action = (m > thr) ? 1 : 2;  // d_checkMovement before d_reduceDeltaP
      action |= 16;
    } else {
      action = (m * rho > thr) ? 1 : 2;  // d_reduceDeltaP before d_checkMovement
    }
    const int trials = ++G.ls_trials[f];
    atomicAdd((unsigned long long*)&C.n_eval, 1ull);
    atomicAdd((unsigned long long*)&C.passes[kTrial], 1ull);
    if ((action & 15) == 1 && trials >= kTrialCap) {
      action = (action & 16) | 2;
      C.cap_hit = 1;
    }
    if ((action & 15) == 0 && b0 == 0) G.errval[shift * G.nF] = ev;  // only idx == 0 writes (:135)
  }
  action = __shfl_sync(0xffffffffu, action, 0);
  const double rho = G.ls_mult;
  double* km = G.kmask + (size_t)f * 2 * (W + 1);
  double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
  for (int t = lane; t <= W; t += 32) {
    for (int d = 0; d < 2; d++) {
      const size_t o = (size_t)d * N + b0 + t;
      const double v = t < W ? G.p[o] + G.delta_p[o] : (last_frame ? kPnewFill : (d ? by : bx));
      km[d * (W + 1) + t] = v;
      if (action & 16) kd[d * (W + 1) + t] = v;
      if (t < W) {
        if ((action & 15) == 0) G.p[o] = v;
        else if ((action & 15) == 1) G.delta_p[o] *= rho;
        else if (!(action & 16)) G.delta_p[o] *= rho;  // absent block: reduced before the stop test
      }
    }
  }
  if (lane == 0) {
    G.ls_done[f] = 0;
    if ((action & 15) != 1) {
      G.fstate[f] = 0;
      atomicSub(&C.ls_pending, 1);
      atomicMax(G.ls_max_trials, G.ls_trials[f]);
    }
  }
}

// One trial of the line search for the frames of one trial tile: block column cc of the
// ns <= kTrialTileFrames searching frames listed at list[pos..pos+ns) (batch frame indices,
// ss_sched.cuh); the last column of a frame to arrive decides for the frame (ls_decide).
template <class FrameT, class TplT>
__device__ __forceinline__ void trial_tile(const GroupDesc& G, GroupCtl& C, int cc, int pos, int ns,
                                           const int* __restrict__ list, unsigned char* smem, uint64_t* bar,
                                           unsigned& bar_phase, bool& win_ok, int win_bytes, int* s_list,
                                           float4* s_kn) {
  const int W = G.W, N = G.N, Hb = G.Hb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the tile's frames (searching when the round's schedule was built; a frame's fstate changes only
  // in its decision, which follows the evaluation of all its columns of the round)
  if (threadIdx.x < ns) s_list[threadIdx.x] = list[pos + threadIdx.x] - G.frame_base;
  __syncthreads();

  // trial knots of this column: own knots p + deltaP, the frame's right boundary fixed
  auto knots = [&](int f, float& x0, float& x1, float& y0, float& y1) {
    const int b0 = f * W, c = b0 + cc;
    x0 = (float)(G.p[c] + G.delta_p[c]);
    y0 = (float)(G.p[N + c] + G.delta_p[N + c]);
    if (cc + 1 < W) {
      x1 = (float)(G.p[c + 1] + G.delta_p[c + 1]);
      y1 = (float)(G.p[N + c + 1] + G.delta_p[N + c + 1]);
    } else if (f + 1 == G.nF) {
      x1 = y1 = (float)kPnewFill;
    } else {
      x1 = (float)G.p_snap[b0 + W];
      y1 = (float)G.p_snap[N + b0 + W];
    }
  };

  // every searching frame's trial knots at once (one round trip to memory for the tile)
  for (int i = threadIdx.x; i < ns; i += blockDim.x) {
    float x0, x1, y0, y1;
    knots(s_list[i], x0, x1, y0, y1);
    s_kn[i] = make_float4(x0, x1, y0, y1);
  }
  __syncthreads();

  TWin win{nullptr, 0, 0, 0};
  const int win_cap = G.tplain ? win_bytes / (G.tpitch * (int)sizeof(float)) : 0;
  if (win_ok && win_cap >= 2 && !G.gquad && ns >= kMinWinFrames) {
    float klo = INFINITY, khi = -INFINITY;
    for (int i = threadIdx.x; i < ns; i += blockDim.x) {
      const float4 k = s_kn[i];
      klo = fminf(klo, fminf(k.z, k.w));
      khi = fmaxf(khi, fmaxf(k.z, k.w));
    }
    block_minmax(klo, khi);
    int r0, rows;
    window_rows(G, G.col_yrange[2 * cc] + klo, G.col_yrange[2 * cc + 1] + khi, win_cap, r0, rows);
    if (rows > 0) {
      float* wbuf = reinterpret_cast<float*>(smem);
      if (stage_window(G, wbuf, r0, rows, bar, bar_phase, G.tplain)) win = {wbuf, r0, rows, G.tpitch};
      else win_ok = false;  // a copy may still be in flight: no further windows in this CTA
    }
  }
  if (threadIdx.x == 0) {
    atomicAdd(G.staging + 2, 1ull);
    if (win.p) atomicAdd(G.staging + 3, 1ull);
    if (win.p && G.pair_ok) atomicAdd(G.staging + 4, 1ull);
  }

  const bool affine = G.geo_k > 0;
  // without a staged window the pixel-pair paths read the template rows in global memory (L1)
  const bool grows = !win.p && G.tplain != nullptr && !G.gquad;
  for (int i = warp; i < ns; i += kEvalWarps) {
    const int f = s_list[i];
    const int c = f * W + cc;
    const size_t coli = (size_t)c * Hb;
    const float4 kn = s_kn[i];
    const float x0 = kn.x, x1 = kn.y, y0 = kn.z, y1 = kn.w;
    double ssd;
    int cnt;
    bool quads = false;
    if constexpr (sizeof(FrameT) == 2) quads = G.quad_ok;
    // separate call sites for the staged window and the global rows keep the window's loads in
    // shared memory
    if (quads && win.p) {
      if constexpr (sizeof(FrameT) == 2)
        trial_pairs16<FrameT>(G, coli, pair_col(G, cc, x0, x1, y0, y1), pair_win(win), ssd, cnt);
    } else if (quads && grows) {  // the whole template's rows in global memory as the window
      if constexpr (sizeof(FrameT) == 2)
        trial_pairs16<FrameT>(G, coli, pair_col(G, cc, x0, x1, y0, y1), pair_win(TWin{G.tplain, 0, G.Ht, G.tpitch}),
                              ssd, cnt);
    } else if (win.p && G.pair_ok) {
      trial_pairs<FrameT>(G, coli, pair_col(G, cc, x0, x1, y0, y1), pair_win(win), ssd, cnt);
    } else if (grows && G.pair_ok) {
      trial_pairs<FrameT>(G, coli, pair_col(G, cc, x0, x1, y0, y1), pair_win(TWin{G.tplain, 0, G.Ht, G.tpitch}), ssd,
                          cnt);
    } else {
      ColKnots<float> k;
      set_knots(k, x0, x1, y0, y1, x0, x1, y0, y1);
      double out[kCsStride];
      const ColGeo<float> geo = global_geo<float>(G, cc);
      if (win.p) {
        if (affine) eval_column<float, FrameT, TplT, kTrial, true, true>(G, coli, geo, k, out, cnt, nullptr, cc, win);
        else eval_column<float, FrameT, TplT, kTrial, false, true>(G, coli, geo, k, out, cnt, nullptr, cc, win);
      } else {
        if (affine) eval_column<float, FrameT, TplT, kTrial, true>(G, coli, geo, k, out, cnt, nullptr, cc);
        else eval_column<float, FrameT, TplT, kTrial>(G, coli, geo, k, out, cnt, nullptr);
      }
      ssd = out[kCsSsd];
    }
    int prev = 0;
    if (lane == 0) {
      G.colsum[(size_t)c * kCsStride + kCsSsd] = ssd;
      G.colcnt[c] = cnt;
      prev = atomic_add_acq_rel(G.ls_done + f, 1);  // releases this column's results
    }
    prev = __shfl_sync(0xffffffffu, prev, 0);
    if (prev == W - 1) {
      // lane 0's acquire covers lane 0 only and a shuffle orders no memory: every lane reads the
      // arrival count with acquire order (it reads the value of lane 0's add, the last in the
      // count's release sequence) before it reads the other CTAs' column results
      (void)ld_acquire(G.ls_done + f);
      ls_decide(G, C, f);  // acquired every column of the frame
    }
  }
}

// One line-search trial round of precision 'S' over the tiles of the round's trial schedule (the
// searching frames, ss_sched.cuh), one tile at a time per CTA. Dynamic shared memory: the window's
// mbarrier (16 bytes), then the template window.
template <class FrameT, class TplT>
__global__ void __launch_bounds__(32 * kEvalWarps, kTrialMinBlocks)
    k_trial_round(const GroupDesc* __restrict__ gds, int* __restrict__ ts, int n_frames, int n_groups,
                  GroupCtl* __restrict__ ctl, int win_bytes) {
  static_assert(kTrialTileFrames <= kEvalWarps * 32, "one thread per tile frame");
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_list[kTrialTileFrames];
  __shared__ float4 s_kn[kTrialTileFrames];
  __shared__ int s_tile[4];
  __shared__ GroupDesc s_gd;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  if (threadIdx.x == 0) mbar_init(bar);
  __syncthreads();
  unsigned bar_phase = 0;
  bool win_ok = true;
  const int* list = ts + kTsHdr;
  while (fetch_trial_tile(ts, n_frames, n_groups, s_tile)) {
    const int g = s_tile[0];
    load_desc(gds + g, &s_gd);
    trial_tile<FrameT, TplT>(s_gd, ctl[g], s_tile[1], s_tile[2], s_tile[3], list, smem + 16, bar, bar_phase, win_ok,
                             win_bytes, s_list, s_kn);
    __syncthreads();  // s_tile, s_gd, s_list, s_kn and the window are reused by the next tile
  }
  if (!win_ok) drain_window(bar, bar_phase);  // a timed-out copy may still write this CTA's memory
}

}  // namespace ss
