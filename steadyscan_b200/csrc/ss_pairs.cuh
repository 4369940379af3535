// Pixel-pair evaluation of precision 'S' on the packed FP32 pipe (f32x2 fma/add/mul of sm_100).
//
// Applies to a block column with the default scan geometry (affine in the pixel index, k lines per
// knot, k dividing 32, Hb a multiple of 64) whose template rows are staged in a shared-memory
// window. Lane `lane` of a warp takes rows 64 t + 2 lane and 64 t + 2 lane + 1 of step t as the
// two halves of float2 values, so every arithmetic instruction serves two pixels; the two frame
// samples are one 32-bit (16-bit storage) or 64-bit (FP32 storage) load.
//
// The warp model is the reference's (task_applyparameters.cuh:33-62): with f = fs (l L + j + 1/2)
// and basex = ax j + bx0, basey = ay (cc k + l) + by0 for pixel j of line l of knot span cc,
//   x = basex + kx0 (1 - f) + kx1 f = (ax + (kx1 - kx0) fs) j + (bx0 + kx0 + (kx1 - kx0) f0(l)),
// and y likewise: one fma per coordinate. Bilinear values and gradients follow
// task_differenceimage.cuh:118-126 and task_updategradients.cu:12-20 in lerp form. The FP32 results
// differ from the FP64 path by rounding only.
#pragma once

#include "ss_stage.cuh"

namespace ss {

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  float2 r;
  asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n sub.rn.f32x2 rd, ra, rb;\n"
      " mov.b64 {%0, %1}, rd;\n}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// Two frame samples of rows (2i, 2i + 1) of a column as floats.
template <class FrameT>
struct PairLoad;
template <>
struct PairLoad<uint16_t> {
  using W = uint32_t;
  __device__ static W load(const void* col, int i) { return __ldg(reinterpret_cast<const uint32_t*>(col) + i); }
  __device__ static float2 cvt(W w) {
    // 2^23 + v has v in its mantissa: exact for 16-bit v
    const float lo = __uint_as_float(0x4B000000u | (w & 0xFFFFu)) - 8388608.0f;
    const float hi = __uint_as_float(0x4B000000u | (w >> 16)) - 8388608.0f;
    return make_float2(lo, hi);
  }
};
template <>
struct PairLoad<__half> {
  using W = uint32_t;
  __device__ static W load(const void* col, int i) { return __ldg(reinterpret_cast<const uint32_t*>(col) + i); }
  __device__ static float2 cvt(W w) {
    __half2 h = *reinterpret_cast<__half2*>(&w);
    return __half22float2(h);
  }
};
template <>
struct PairLoad<float> {
  using W = float2;
  __device__ static W load(const void* col, int i) { return __ldg(reinterpret_cast<const float2*>(col) + i); }
  __device__ static float2 cvt(W w) { return w; }
};
template <>
struct PairLoad<double> {
  using W = double2;
  __device__ static W load(const void* col, int i) { return __ldg(reinterpret_cast<const double2*>(col) + i); }
  __device__ static float2 cvt(W w) { return make_float2((float)w.x, (float)w.y); }
};

// Steps (64 rows) of frame samples a warp keeps in flight: trial evaluation (32-bit sample pairs;
// fewer for wider frame types), assembly (whose 14 accumulators leave fewer registers).
constexpr int kPrefetch = 8;
constexpr int kPrefetchAsm = 2;
// Correlation and final passes: 64-row steps of frame samples in flight, by the width of a lane's
// sample word (16-bit pairs: 16 steps, a whole 1024-row column; the pass took 17.2 ms with 2, 16.5
// with 6, 15.7 with 8 and 14.3 with 16 steps over the 2000-frame run).
template <class W>
struct CorrPrefetch {
  static constexpr int value = sizeof(W) <= 4 ? 16 : (sizeof(W) <= 8 ? 8 : 4);
};

// Per-warp constants of one block column for the pair loop.
struct PairCol {
  float2 bxj, cx, byj, cy;  // x = bxj * j + cx, y = byj * j + cy (both halves)
  float2 fsj, f0;           // f = fsj * j + f0
  float2 j0;                // j of step 0 for both halves
  float dj;                 // j advance per step (64 / k)
};

// Column constants for knots (kx0, kx1, ky0, ky1) of block column cc (lane-dependent halves); the
// lane's first pair holds rows row0 and row0 + 1 (default 2 lane).
__device__ __forceinline__ PairCol pair_col(const GroupDesc& G, int cc, float kx0, float kx1, float ky0, float ky1,
                                            int row0 = -1) {
  const int lane = threadIdx.x & 31, k = G.geo_k, L = G.geo_L, ks = __ffs(k) - 1;  // k = 2^ks
  const int rA = row0 >= 0 ? row0 : 2 * lane, rB = rA + 1;
  const int lA = rA & (k - 1), lB = rB & (k - 1);
  const float fs = G.geo_fs;
  const float f0A = ((float)(lA * L) + 0.5f) * fs, f0B = ((float)(lB * L) + 0.5f) * fs;
  const float dkx = kx1 - kx0, dky = ky1 - ky0;
  PairCol p;
  p.bxj = f2(fmaf(dkx, fs, G.geo_ax));
  p.cx = f2(fmaf(dkx, f0A, G.geo_bx + kx0), fmaf(dkx, f0B, G.geo_bx + kx0));
  p.byj = f2(dky * fs);
  p.cy = f2(fmaf(dky, f0A, fmaf(G.geo_ay, (float)(cc * k + lA), G.geo_by) + ky0),
            fmaf(dky, f0B, fmaf(G.geo_ay, (float)(cc * k + lB), G.geo_by) + ky0));
  p.fsj = f2(fs);
  p.f0 = f2(f0A, f0B);
  p.j0 = f2((float)(rA >> ks), (float)(rB >> ks));
  p.dj = (float)(64 >> ks);
  return p;
}

// Window addressing: element (iy, ix) of the template sits at index (iy - r0) pitch + ix of the
// window; from v = 2^23 + floor(c) (the bits of a round-down add) that index is
// vy pitch + vx - kbias in wrapping 32-bit arithmetic, clamped so masked pixels stay in bounds.
struct PairWin {
  const float* p;
  unsigned pitch, kbias, emax;
};
__device__ __forceinline__ PairWin pair_win(const TWin& w) {
  PairWin q;
  q.p = w.p;
  q.pitch = (unsigned)w.pitch;
  q.kbias = 0x4B000000u * ((unsigned)w.pitch + 1u) + (unsigned)w.r0 * (unsigned)w.pitch;
  q.emax = (unsigned)((w.rows - 1) * w.pitch - 2);
  return q;
}

// Floor / fraction of both halves (0 <= c < 2^23 for valid pixels) and the window corner values.
__device__ __forceinline__ void pair_sample(const PairWin& w, float2 x, float2 y, float2& xf, float2& yf, float2& t00,
                                            float2& t01, float2& t10, float2& t11) {
  const float2 big = f2(8388608.0f);
  const float2 vx = __fadd2_rd(x, big), vy = __fadd2_rd(y, big);
  xf = sub2(x, sub2(vx, big));
  yf = sub2(y, sub2(vy, big));
  unsigned eA = __float_as_uint(vy.x) * w.pitch + __float_as_uint(vx.x) - w.kbias;
  unsigned eB = __float_as_uint(vy.y) * w.pitch + __float_as_uint(vx.y) - w.kbias;
  eA = min(eA, w.emax);
  eB = min(eB, w.emax);
  const float* qA = w.p + eA;
  const float* qB = w.p + eB;
  t00 = f2(qA[0], qB[0]);
  t01 = f2(qA[1], qB[1]);
  t10 = f2(qA[w.pitch], qB[w.pitch]);
  t11 = f2(qA[w.pitch + 1], qB[w.pitch + 1]);
}

// Validity of both halves: 0 <= c < lim as an unsigned compare of the bit patterns (negative
// values and NaN have larger patterns).
__device__ __forceinline__ bool in_range(float c, unsigned lim_bits) { return __float_as_uint(c) < lim_bits; }

// The assembly sums of one lane's pixel pairs (kCsSsd .. kCsJ2y, in that order) and its valid count.
struct AsmAcc {
  float2 v[kCsAssemble];
  int cnt;
  __device__ __forceinline__ AsmAcc() : cnt(0) {
#pragma unroll
    for (int i = 0; i < kCsAssemble; i++) v[i] = f2(0.f);
  }
  // the pixel pair at j (both halves) with frame samples img: warp, mask, bilinear sample and
  // gradients, residual, and the sums of JᵀJ blocks ((1-f)², f², f(1-f)), Jᵀr and SSD
  __device__ __forceinline__ void add(const PairCol& pc, const PairWin& w, float2 j, float2 img, unsigned twb,
                                      unsigned thb) {
    const float2 x = fma2(pc.bxj, j, pc.cx), y = fma2(pc.byj, j, pc.cy), f = fma2(pc.fsj, j, pc.f0);
    const bool mA = in_range(x.x, twb) && in_range(y.x, thb);
    const bool mB = in_range(x.y, twb) && in_range(y.y, thb);
    cnt += (mA ? 1 : 0) + (mB ? 1 : 0);
    float2 xf, yf, t00, t01, t10, t11;
    pair_sample(w, x, y, xf, yf, t00, t01, t10, t11);
    const float2 gy0 = sub2(t10, t00), gy1 = sub2(t11, t01);
    const float2 gx0 = sub2(t01, t00), gx1 = sub2(t11, t10);
    const float2 a = fma2(yf, gy0, t00), b = fma2(yf, gy1, t01);
    const float2 wI = fma2(xf, sub2(b, a), a);
    float2 wx = fma2(yf, sub2(gx1, gx0), gx0);
    float2 wy = fma2(xf, sub2(gy1, gy0), gy0);
    float2 d2 = sub2(img, wI);
    d2 = f2(mA ? d2.x : 0.f, mB ? d2.y : 0.f);
    wx = f2(mA ? wx.x : 0.f, mB ? wx.y : 0.f);
    wy = f2(mA ? wy.x : 0.f, mB ? wy.y : 0.f);
    const float2 c = sub2(f2(1.0f), f);
    const float2 csq = mul2(c, c), fsq = mul2(f, f), fc = mul2(f, c);
    const float2 gxx = mul2(wx, wx), gyy = mul2(wy, wy), gxy = mul2(wx, wy);
    v[0] = fma2(d2, d2, v[0]);
    v[1] = fma2(gxx, csq, v[1]);
    v[2] = fma2(gyy, csq, v[2]);
    v[3] = fma2(gxy, csq, v[3]);
    v[4] = fma2(gxx, fsq, v[4]);
    v[5] = fma2(gyy, fsq, v[5]);
    v[6] = fma2(gxy, fsq, v[6]);
    v[7] = fma2(gxx, fc, v[7]);
    v[8] = fma2(gyy, fc, v[8]);
    v[9] = fma2(gxy, fc, v[9]);
    const float2 d1 = mul2(d2, c), dd2 = mul2(d2, f);
    v[10] = fma2(d1, wx, v[10]);
    v[11] = fma2(d1, wy, v[11]);
    v[12] = fma2(dd2, wx, v[12]);
    v[13] = fma2(dd2, wy, v[13]);
  }
  // the block's partials reduced in FP32 over the warp, combined in FP64 by the solve
  __device__ __forceinline__ void reduce(double (&out)[kCsStride], int& cnt_out) const {
    cnt_out = warp_sum(cnt);
#pragma unroll
    for (int i = 0; i < kCsAssemble; i++) out[i] = (double)warp_sumf(v[i].x + v[i].y);
  }
};

// Assembly sums (kCsSsd .. kCsJ2y) and valid count of one block column at knots that are both the
// mask and the difference-image knots. out/cnt are warp-reduced (all lanes).
template <class FrameT>
__device__ __forceinline__ void assemble_pairs(const GroupDesc& G, size_t coli, const PairCol& pc, const PairWin& w,
                                               double (&out)[kCsStride], int& cnt_out) {
  using PL = PairLoad<FrameT>;
  const int lane = threadIdx.x & 31;
  const unsigned twb = __float_as_uint(Limits<float>::lim(G.Wt)), thb = __float_as_uint(Limits<float>::lim(G.Ht));
  const FrameT* col = reinterpret_cast<const FrameT*>(G.image) + coli;
  const int steps = G.Hb >> 6;
  AsmAcc acc;
  float2 j = pc.j0;
  const float2 dj = f2(pc.dj);
  // kPrefetchAsm steps of frame samples in flight (a register ring)
  typename PL::W ring[kPrefetchAsm];
#pragma unroll
  for (int d = 0; d < kPrefetchAsm; d++) ring[d] = d < steps ? PL::load(col, d * 32 + lane) : typename PL::W{};
#pragma unroll 1
  for (int t0 = 0; t0 < steps; t0 += kPrefetchAsm) {
#pragma unroll
    for (int d = 0; d < kPrefetchAsm; d++) {
      const int t = t0 + d;
      if (t >= steps) break;
      const typename PL::W cur = ring[d];
      if (t + kPrefetchAsm < steps) ring[d] = PL::load(col, (t + kPrefetchAsm) * 32 + lane);
      acc.add(pc, w, j, PL::cvt(cur), twb, thb);
      j = add2(j, dj);
    }
  }
  acc.reduce(out, cnt_out);
}

// assemble_pairs for 16-bit frame samples with knots every 1 or 2 lines, Hb a multiple of 256 and a
// 16-byte aligned column: the frame samples of a 256-row step arrive as one 16-byte load per lane
// and are handed round by four shuffles as in trial_pairs16 (lane L = 4 a + b takes pair L + 32 m,
// m = (b - rho) mod 4, in round rho), so the lanes of a round read consecutive template columns.
// One load per lane covers four pairs of work: twice the bytes in flight of assemble_pairs' ring.
template <class FrameT>
__device__ __forceinline__ void assemble_pairs16(const GroupDesc& G, size_t coli, const PairCol& pc, const PairWin& w,
                                                 double (&out)[kCsStride], int& cnt_out) {
  static_assert(sizeof(FrameT) == 2, "16-bit frame samples");
  using PL = PairLoad<FrameT>;
  const int lane = threadIdx.x & 31;
  const unsigned twb = __float_as_uint(Limits<float>::lim(G.Wt)), thb = __float_as_uint(Limits<float>::lim(G.Ht));
  const uint4* col = reinterpret_cast<const uint4*>(reinterpret_cast<const FrameT*>(G.image) + coli);
  const int steps = G.Hb >> 8;
  const int ks = __ffs(G.geo_k) - 1;
  const float d64 = (float)(64 >> ks), dt = (float)(256 >> ks);
  const int b = lane & 3, a = lane >> 2, rot = lane >> 3;
  AsmAcc acc;
  uint4 next = __ldg(col + lane);
#pragma unroll 1
  for (int t = 0; t < steps; t++) {
    uint4 cur = next;
    if (t + 1 < steps) next = __ldg(col + (t + 1) * 32 + lane);
    if (rot & 1) cur = make_uint4(cur.y, cur.z, cur.w, cur.x);
    if (rot & 2) cur = make_uint4(cur.z, cur.w, cur.x, cur.y);
    const float2 jb = add2(pc.j0, f2(dt * (float)t));
    const uint32_t wv[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
    for (int rho = 0; rho < 4; rho++) {
      const int m = (b - rho) & 3;
      const uint32_t v = __shfl_sync(0xffffffffu, wv[rho], (m << 3) | a);
      acc.add(pc, w, add2(jb, f2(d64 * (float)m)), PL::cvt(v), twb, thb);
    }
  }
  acc.reduce(out, cnt_out);
}

// Trial SSD and valid count of one block column (task_linesearch.cu:50-74 with the SSD of
// task_calcerrval.cu:6-18); out values are warp-reduced (all lanes).
template <class FrameT>
__device__ __forceinline__ void trial_pairs(const GroupDesc& G, size_t coli, const PairCol& pc, const PairWin& w,
                                            double& ssd_out, int& cnt_out) {
  using PL = PairLoad<FrameT>;
  const int lane = threadIdx.x & 31;
  const unsigned twb = __float_as_uint(Limits<float>::lim(G.Wt)), thb = __float_as_uint(Limits<float>::lim(G.Ht));
  const FrameT* col = reinterpret_cast<const FrameT*>(G.image) + coli;
  const int steps = G.Hb >> 6;
  float2 ssd = f2(0.f);
  int cnt = 0;
  float2 j = pc.j0;
  const float2 dj = f2(pc.dj);
  constexpr int kPf = sizeof(typename PL::W) <= 4 ? kPrefetch : (sizeof(typename PL::W) <= 8 ? 4 : 2);
  typename PL::W ring[kPf];
#pragma unroll
  for (int d = 0; d < kPf; d++) ring[d] = d < steps ? PL::load(col, d * 32 + lane) : typename PL::W{};
#pragma unroll 1
  for (int t0 = 0; t0 < steps; t0 += kPf) {
#pragma unroll
    for (int d = 0; d < kPf; d++) {
      const int t = t0 + d;
      if (t >= steps) break;
      const typename PL::W cur = ring[d];
      if (t + kPf < steps) ring[d] = PL::load(col, (t + kPf) * 32 + lane);
      const float2 x = fma2(pc.bxj, j, pc.cx), y = fma2(pc.byj, j, pc.cy);
      j = add2(j, dj);
      const bool mA = in_range(x.x, twb) && in_range(y.x, thb);
      const bool mB = in_range(x.y, twb) && in_range(y.y, thb);
      cnt += (mA ? 1 : 0) + (mB ? 1 : 0);
      float2 xf, yf, t00, t01, t10, t11;
      pair_sample(w, x, y, xf, yf, t00, t01, t10, t11);
      const float2 a = fma2(yf, sub2(t10, t00), t00), b = fma2(yf, sub2(t11, t01), t01);
      const float2 wI = fma2(xf, sub2(b, a), a);
      float2 d2 = sub2(PL::cvt(cur), wI);
      d2 = f2(mA ? d2.x : 0.f, mB ? d2.y : 0.f);
      ssd = fma2(d2, d2, ssd);
    }
  }
  cnt_out = warp_sum(cnt);
  ssd_out = (double)warp_sumf(ssd.x + ssd.y);
}

// trial_pairs for 16-bit frame samples with knots every 1 or 2 lines, Hb a multiple of 256 and a
// 16-byte aligned column, on the plain window rows: each lane loads rows 8 lane .. 8 lane + 7 of
// every 256-row step as one 16-byte load (four pixel pairs), and four shuffles hand the pairs round
// so that in round rho lane L = 4 a + b takes pair L + 32 m of the step, m = (b - rho) mod 4, from
// lane 8 m + a, which sends its word b (each lane first rotates its words by lane / 8, so the word
// it sends in round rho is its rotated word rho). The lanes of a round then take pairs 32 apart on
// consecutive template columns: no bank conflicts on the plain rows, whose index needs no plane
// arithmetic. pc is pair_col's with row0 = 2 lane; pair L + 32 m + 128 t sits at
// j0 + (64 m + 256 t) / k. One step in flight keeps the kernel within its registers.
template <class FrameT>
__device__ __forceinline__ void trial_pairs16(const GroupDesc& G, size_t coli, const PairCol& pc, const PairWin& w,
                                               double& ssd_out, int& cnt_out) {
  static_assert(sizeof(FrameT) == 2, "16-bit frame samples");
  using PL = PairLoad<FrameT>;
  const int lane = threadIdx.x & 31;
  const unsigned twb = __float_as_uint(Limits<float>::lim(G.Wt)), thb = __float_as_uint(Limits<float>::lim(G.Ht));
  const uint4* col = reinterpret_cast<const uint4*>(reinterpret_cast<const FrameT*>(G.image) + coli);
  const int steps = G.Hb >> 8;
  const int ks = __ffs(G.geo_k) - 1;
  const float d64 = (float)(64 >> ks), dt = (float)(256 >> ks);
  const int b = lane & 3, a = lane >> 2, rot = lane >> 3;
  float2 ssd = f2(0.f);
  int cnt = 0;
  uint4 next = __ldg(col + lane);
#pragma unroll 1
  for (int t = 0; t < steps; t++) {
    uint4 cur = next;
    if (t + 1 < steps) next = __ldg(col + (t + 1) * 32 + lane);
    if (rot & 1) cur = make_uint4(cur.y, cur.z, cur.w, cur.x);
    if (rot & 2) cur = make_uint4(cur.z, cur.w, cur.x, cur.y);
    const float2 jb = add2(pc.j0, f2(dt * (float)t));
    const uint32_t wv[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
    for (int rho = 0; rho < 4; rho++) {
      const int m = (b - rho) & 3;
      const uint32_t v = __shfl_sync(0xffffffffu, wv[rho], (m << 3) | a);
      const float2 j = add2(jb, f2(d64 * (float)m));
      const float2 x = fma2(pc.bxj, j, pc.cx), y = fma2(pc.byj, j, pc.cy);
      const bool mA = in_range(x.x, twb) && in_range(y.x, thb);
      const bool mB = in_range(x.y, twb) && in_range(y.y, thb);
      cnt += (mA ? 1 : 0) + (mB ? 1 : 0);
      float2 xf, yf, t00, t01, t10, t11;
      pair_sample(w, x, y, xf, yf, t00, t01, t10, t11);
      const float2 a2 = fma2(yf, sub2(t10, t00), t00), b2 = fma2(yf, sub2(t11, t01), t01);
      const float2 wI = fma2(xf, sub2(b2, a2), a2);
      float2 d2 = sub2(PL::cvt(v), wI);
      d2 = f2(mA ? d2.x : 0.f, mB ? d2.y : 0.f);
      ssd = fma2(d2, d2, ssd);
    }
  }
  cnt_out = warp_sum(cnt);
  ssd_out = (double)warp_sumf(ssd.x + ssd.y);
}

// Correlation sums (kCsSumD .. kCsFrDI) of one block column whose mask and difference-image knots
// agree, in the reference's definitions (task_correlation.cu:16-60, swapped difference image D'),
// and for the final pass also the SSD at the mask knots and the mask output. The leading run of
// valid pixels follows the row order: within a 64-row step lane L holds rows 2L and 2L + 1.
template <class FrameT, int MODE>
__device__ __forceinline__ void corr_pairs(const GroupDesc& G, size_t coli, const PairCol& pc, const PairWin& w,
                                           double (&out)[kCsStride], int& cnt_out, uint8_t* mask_out) {
  using PL = PairLoad<FrameT>;
  constexpr int kPrefetchCorr = CorrPrefetch<typename PL::W>::value;
  const int lane = threadIdx.x & 31;
  const unsigned twb = __float_as_uint(Limits<float>::lim(G.Wt)), thb = __float_as_uint(Limits<float>::lim(G.Ht));
  const FrameT* col = reinterpret_cast<const FrameT*>(G.image) + coli;
  const int steps = G.Hb >> 6;
  const unsigned lt = (1u << lane) - 1u;
  float2 sumd = f2(0.f), sn = f2(0.f), sd = f2(0.f), sdd = f2(0.f), si = f2(0.f), sii = f2(0.f), sdi = f2(0.f),
         fd = f2(0.f), fi = f2(0.f), fdd = f2(0.f), fii = f2(0.f), fdi = f2(0.f), fssd = f2(0.f);
  int cnt = 0;
  bool run = true;
  float2 j = pc.j0;
  const float2 dj = f2(pc.dj);
  typename PL::W ring[kPrefetchCorr];
#pragma unroll
  for (int d = 0; d < kPrefetchCorr; d++) ring[d] = d < steps ? PL::load(col, d * 32 + lane) : typename PL::W{};
#pragma unroll 1
  for (int t0 = 0; t0 < steps; t0 += kPrefetchCorr) {
#pragma unroll
    for (int d = 0; d < kPrefetchCorr; d++) {
      const int t = t0 + d;
      if (t >= steps) break;
      const typename PL::W cur = ring[d];
      if (t + kPrefetchCorr < steps) ring[d] = PL::load(col, (t + kPrefetchCorr) * 32 + lane);
      const float2 x = fma2(pc.bxj, j, pc.cx), y = fma2(pc.byj, j, pc.cy);
      j = add2(j, dj);
      const bool mA = in_range(x.x, twb) && in_range(y.x, thb);
      const bool mB = in_range(x.y, twb) && in_range(y.y, thb);
      cnt += (mA ? 1 : 0) + (mB ? 1 : 0);
      float2 xf, yf, t00, t01, t10, t11;
      pair_sample(w, x, y, xf, yf, t00, t01, t10, t11);
      const float2 a = fma2(yf, sub2(t10, t00), t00), b = fma2(yf, sub2(t11, t01), t01);
      const float2 wI = fma2(xf, sub2(b, a), a);
      const float2 img = PL::cvt(cur);
      const float2 diff = sub2(img, wI);          // differenceImage at valid pixels
      float2 dp = sub2(img, diff);                // after d_swapWIDiff
      dp = f2(mA ? dp.x : 0.f, mB ? dp.y : 0.f);
      sumd = add2(sumd, dp);
      const float2 im = f2(mA ? img.x : 0.f, mB ? img.y : 0.f);
      fd = add2(fd, dp);
      fi = add2(fi, im);
      fdd = fma2(dp, dp, fdd);
      fii = fma2(im, im, fii);
      fdi = fma2(dp, im, fdi);
      const unsigned bothv = __ballot_sync(0xffffffffu, mA && mB);
      const bool pre = run && (bothv & lt) == lt;
      const bool inA = pre && mA, inB = inA && mB;
      run = run && bothv == 0xffffffffu;
      const float2 ds = f2(inA ? dp.x : 0.f, inB ? dp.y : 0.f);
      const float2 is = f2(inA ? img.x : 0.f, inB ? img.y : 0.f);
      sn = add2(sn, f2(inA ? 1.f : 0.f, inB ? 1.f : 0.f));
      sd = add2(sd, ds);
      sdd = fma2(ds, ds, sdd);
      si = add2(si, is);
      sii = fma2(is, is, sii);
      sdi = fma2(ds, is, sdi);
      if (MODE == kFinal) {
        const float2 dm = f2(mA ? diff.x : 0.f, mB ? diff.y : 0.f);
        fssd = fma2(dm, dm, fssd);
        if (mask_out)
          reinterpret_cast<uint16_t*>(mask_out)[t * 32 + lane] = (uint16_t)((mA ? 1u : 0u) | (mB ? 0x100u : 0u));
      }
    }
  }
  cnt_out = warp_sum(cnt);
  out[kCsSumD] = (double)warp_sumf(sumd.x + sumd.y);
  out[kCsSetN] = (double)warp_sumf(sn.x + sn.y);
  out[kCsSetD] = (double)warp_sumf(sd.x + sd.y);
  out[kCsSetDD] = (double)warp_sumf(sdd.x + sdd.y);
  out[kCsSetI] = (double)warp_sumf(si.x + si.y);
  out[kCsSetII] = (double)warp_sumf(sii.x + sii.y);
  out[kCsSetDI] = (double)warp_sumf(sdi.x + sdi.y);
  out[kCsFrD] = (double)warp_sumf(fd.x + fd.y);
  out[kCsFrI] = (double)warp_sumf(fi.x + fi.y);
  out[kCsFrDD] = (double)warp_sumf(fdd.x + fdd.y);
  out[kCsFrII] = (double)warp_sumf(fii.x + fii.y);
  out[kCsFrDI] = (double)warp_sumf(fdi.x + fdi.y);
  out[kCsFinalSsd] = MODE == kFinal ? (double)warp_sumf(fssd.x + fssd.y) : 0.0;
}

}  // namespace ss
