// k_eval: one pass of the warp model over block columns of every group in a batch.
//
// A warp owns one block column c (the pixels of the k scan lines between knots c and c+1 of one
// frame, Hb rows in the reference's block-matrix order, steady_scan.m:601-613); its lanes stride the
// rows, so frame and geometry loads are coalesced. Per pixel it evaluates the reference's
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
#pragma once

#include "ss_common.cuh"

namespace ss {

__device__ __forceinline__ bool frame_active(const GroupDesc& G, int f, int shift) {
  // groupActive[groupId + shift * nGroups] with zero-filled reads past the array
  // (task_calcerrval.cu:164-166, task_linesearch.cu:86-88).
  int gid = (f * G.W) / G.group_size + shift * G.n_rg;
  return gid < 2 * G.n_rg && G.grp_active[gid];
}

// Warped position and validity of one pixel (task_applyparameters.cuh:57-62), FP64 as in the
// reference's 'D' build; a*b+c is contracted into fma the way nvcc contracts the reference source.
__device__ __forceinline__ bool warp_pixel(double kx0, double kx1, double ky0, double ky1, double f, double bx,
                                           double by, bool bm, double tw, double th, double& x, double& y) {
  x = fma(kx1, f, fma(kx0, 1.0 - f, bx));
  y = fma(ky1, f, fma(ky0, 1.0 - f, by));
  return bm && x >= 0.0 && x < tw && y >= 0.0 && y < th;
}

template <class Acc, class TplT>
struct Sample {
  Acc wI, wx, wy;
};

// Bilinear template value and warped gradients at a valid pixel (task_differenceimage.cuh:118-126,
// task_updategradients.cu:12-20). With gquad == nullptr the gradients are the template's forward
// differences (steady_scan.m:178-179), taken from the same four template values.
template <class Acc, class TplT, bool kGrad>
__device__ __forceinline__ Sample<Acc, TplT> sample(const GroupDesc& G, double x, double y) {
  int ix = (int)x, iy = (int)y;
  Acc xf = (Acc)(x - (double)ix), yf = (Acc)(y - (double)iy);
  size_t qi = (size_t)iy * (size_t)(G.Wt - 1) + (size_t)ix;
  Acc t00, t01, t10, t11;
  load_quad<Acc, TplT>(G.tquad, qi, t00, t01, t10, t11);
  Acc one = (Acc)1;
  Acc a = fma(yf, t10, (one - yf) * t00);
  Acc b = fma(yf, t11, (one - yf) * t01);
  Sample<Acc, TplT> s;
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

template <class FrameT>
__device__ __forceinline__ FrameT ld_frame(const void* base, size_t i) {
  return __ldg(reinterpret_cast<const FrameT*>(base) + i);
}
template <>
__device__ __forceinline__ __half ld_frame<__half>(const void* base, size_t i) {
  unsigned short raw = __ldg(reinterpret_cast<const unsigned short*>(base) + i);
  return __ushort_as_half(raw);
}

template <class Acc, class FrameT, class TplT, int MODE>
__global__ void __launch_bounds__(256) k_eval(const GroupDesc* __restrict__ gds, const int* __restrict__ tile_group,
                                              const GroupCtl* __restrict__ ctl) {
  const int g = tile_group[blockIdx.x];
  const GroupDesc& G = gds[g];
  const GroupCtl& C = ctl[g];
  const int want = (MODE == kCorr) ? kPhIterEnd : (MODE == kFinal ? kPhFinal : kPhHalf);
  if (C.phase != want) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = (blockIdx.x - G.tile_base) * 8 + warp;
  if (c >= G.fW) return;
  const int f = c / G.W, cc = c - f * G.W;
  const int W = G.W, N = G.N, Hb = G.Hb;
  const int shift = C.shift;

  // knots of set A (mask, position, gradients) and set B (difference image)
  double ax0, ax1, ay0, ay1, bx0, bx1, by0, by1;
  bool dual = false;
  bool active = true;
  if (MODE == kAssemble) {
    ax0 = G.p[c]; ax1 = G.p[c + 1]; ay0 = G.p[N + c]; ay1 = G.p[N + c + 1];
    active = frame_active(G, f, shift);
    if (!active) {
      const double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
      bx0 = kd[cc]; bx1 = kd[cc + 1]; by0 = kd[W + 1 + cc]; by1 = kd[W + 1 + cc + 1];
      dual = bx0 != ax0 || bx1 != ax1 || by0 != ay0 || by1 != ay1;
    }
  } else if (MODE == kTrial) {
    if (!(G.fstate[f] & 2)) return;
    // pnew = p + deltaP (task_linesearch.cu:50-54); the frame's right boundary knot is the
    // committed knot at line-search start, or the never-written 1e6 for the last frame.
    ax0 = G.p[c] + G.delta_p[c];
    ay0 = G.p[N + c] + G.delta_p[N + c];
    if (cc + 1 < W) {
      ax1 = G.p[c + 1] + G.delta_p[c + 1];
      ay1 = G.p[N + c + 1] + G.delta_p[N + c + 1];
    } else if (f + 1 < G.nF) {
      ax1 = G.p_snap[c + 1];
      ay1 = G.p_snap[N + c + 1];
    } else {
      ax1 = kPnewFill;
      ay1 = kPnewFill;
    }
  } else {
    const double* km = G.kmask + (size_t)f * 2 * (W + 1);
    ax0 = km[cc]; ax1 = km[cc + 1]; ay0 = km[W + 1 + cc]; ay1 = km[W + 1 + cc + 1];
    const double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
    bx0 = kd[cc]; bx1 = kd[cc + 1]; by0 = kd[W + 1 + cc]; by1 = kd[W + 1 + cc + 1];
    dual = bx0 != ax0 || bx1 != ax1 || by0 != ay0 || by1 != ay1;
  }

  const double tw = (double)(G.Wt - 1) - 2.220446049250313e-16;  // templateW - eps<double>() (eps.h:14-22)
  const double th = (double)(G.Ht - 1) - 2.220446049250313e-16;
  const size_t colm = (size_t)cc * Hb;
  const size_t coli = (size_t)c * Hb;
  const size_t coln = (size_t)((cc + 1) % W) * Hb;
  const Acc one = (Acc)1;

  Acc s[kCsStride];
#pragma unroll
  for (int k = 0; k < kCsStride; k++) s[k] = (Acc)0;
  int cnt = 0;
  bool run = true;  // leading run of valid pixels (task_correlation.cu:24-34)

  for (int r0 = 0; r0 < Hb; r0 += 32) {
    const int r = r0 + lane;
    const bool in = r < Hb;
    double f = 0, bxv = 0, byv = 0;
    bool bm = false;
    if (in) {
      f = __ldg(G.frac + colm + r);
      bxv = __ldg(G.basex + colm + r);
      byv = __ldg(G.basey + colm + r);
      bm = __ldg(G.base_mask + colm + r) != 0;
    }
    double x, y;
    bool mA = warp_pixel(ax0, ax1, ay0, ay1, f, bxv, byv, bm, tw, th, x, y) && in;
    cnt += mA ? 1 : 0;

    if (MODE == kAssemble) {
      Acc img = in ? (Acc)to_double(ld_frame<FrameT>(G.image, coli + r)) : (Acc)0;
      Acc wx = 0, wy = 0, d = 0;
      if (mA) {
        Sample<Acc, TplT> sa = sample<Acc, TplT, true>(G, x, y);
        wx = sa.wx;
        wy = sa.wy;
        d = img - sa.wI;
      }
      if (dual) {
        double xb, yb;
        bool mB = warp_pixel(bx0, bx1, by0, by1, f, bxv, byv, bm, tw, th, xb, yb) && in;
        d = mB ? img - sample<Acc, TplT, false>(G, xb, yb).wI : (Acc)0;
      }
      Acc fa = (Acc)f;
      Acc fn = G.frac_uniform ? fa : (in ? (Acc)__ldg(G.frac + coln + r) : (Acc)0);
      Acc fsq = fa * fa, csq = (one - fa) * (one - fa), fc = fa - fsq, fnsq = fn * fn;
      Acc gxx = wx * wx, gyy = wy * wy, gxy = wx * wy;
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
      Acc d1 = d * (one - fa), d2 = d * fa;
      s[kCsJ1x] = fma(d1, wx, s[kCsJ1x]);
      s[kCsJ1y] = fma(d1, wy, s[kCsJ1y]);
      s[kCsJ2x] = fma(d2, wx, s[kCsJ2x]);
      s[kCsJ2y] = fma(d2, wy, s[kCsJ2y]);
    } else if (MODE == kTrial) {
      if (mA) {
        Acc img = (Acc)to_double(ld_frame<FrameT>(G.image, coli + r));
        Acc d = img - sample<Acc, TplT, false>(G, x, y).wI;
        s[kCsSsd] = fma(d, d, s[kCsSsd]);
      }
    } else {
      // swapped difference image D' of task_correlation.cu:51-60 over the state (kmask, kdiff)
      Acc img = in ? (Acc)to_double(ld_frame<FrameT>(G.image, coli + r)) : (Acc)0;
      Acc wA = 0;
      if (mA) wA = sample<Acc, TplT, false>(G, x, y).wI;
      bool mB = mA;
      Acc wB = wA;
      if (dual) {
        double xb, yb;
        mB = warp_pixel(bx0, bx1, by0, by1, f, bxv, byv, bm, tw, th, xb, yb) && in;
        wB = mB ? sample<Acc, TplT, false>(G, xb, yb).wI : (Acc)0;
      }
      Acc dstate = mB ? img - wB : (Acc)0;         // differenceImage
      Acc dp = mA ? img - dstate : dstate;         // after d_swapWIDiff
      s[kCsSumD] += dp;
      unsigned bal = __ballot_sync(0xffffffffu, mA);
      unsigned le = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);
      bool inset = run && ((~bal & le) == 0u) && mA;
      if (inset) {
        s[kCsSetN] += one;
        s[kCsSetD] += dp;
        s[kCsSetDD] = fma(dp, dp, s[kCsSetDD]);
        s[kCsSetI] += img;
        s[kCsSetII] = fma(img, img, s[kCsSetII]);
        s[kCsSetDI] = fma(dp, img, s[kCsSetDI]);
      }
      run = run && (bal == 0xffffffffu);
      if (mA) {
        s[kCsFrD] += dp;
        s[kCsFrI] += img;
        s[kCsFrDD] = fma(dp, dp, s[kCsFrDD]);
        s[kCsFrII] = fma(img, img, s[kCsFrII]);
        s[kCsFrDI] = fma(dp, img, s[kCsFrDI]);
        if (MODE == kFinal) {
          Acc dA = img - wA;
          s[kCsFinalSsd] = fma(dA, dA, s[kCsFinalSsd]);
        }
      }
      if (MODE == kFinal && G.o_mask && in) G.o_mask[coli + r] = mA ? 1 : 0;
    }
  }

  // Leading-run rows past Hb do not exist; the run simply ends at Hb.
  cnt = warp_sum(cnt);
  const int nsum = (MODE == kAssemble) ? kCsAssemble : (MODE == kTrial ? 1 : kCsStride - 2);
  double out[kCsStride];
#pragma unroll
  for (int k = 0; k < kCsStride; k++) out[k] = (k < nsum) ? warp_sum((double)s[k]) : 0.0;
  if (lane == 0) {
    double* dst = G.colsum + (size_t)c * kCsStride;
#pragma unroll
    for (int k = 0; k < kCsStride; k++)
      if (k < nsum) dst[k] = out[k];
    G.colcnt[c] = cnt;
  }
}

}  // namespace ss
