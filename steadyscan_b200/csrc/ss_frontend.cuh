// Caller-side preparation of frames on the GPU: the part of the reference's MATLAB driver that
// turns raw frames into the block matrix the alignment reads (steady_scan.m:229-234), with
// prefilter_foralignment (steady_scan.m:625-643) and cropimage (steady_scan.m:830-834).
//
// Blur: the reference multiplies the frame's 2-D FFT on a grid padded by L rows and columns with
// the FFT of a periodic Gaussian, i.e. it convolves the zero-padded frame circularly (period H + L
// down a column, W + L along a row) with exp(-(dy^2 + dx^2) / (2 s^2)), dy and dx the circular
// distances, normalised to sum 1. The Gaussian is separable and its normalising sum is the product
// of the two axes' sums, so here the convolution runs as two 1-D circular passes in FP64 (down the
// columns, then along the rows), each over the taps within R = ceil(9.6 s) of the centre, where the
// weights fall below 1e-20 of the centre tap: the terms left out lie below FP64 rounding of the sum.
// Median normalisation divides each (blurred) frame by the median of its H x W samples, found
// exactly by a radix select over order-preserving 64-bit keys (NaN anywhere gives NaN, as MATLAB's
// median). Block reorder: entry (r, b) of a frame's block matrix is the cropped frame's pixel whose
// column-major index the caller's gather map holds there, or 0 where it holds -1
// (image2blockmatrix, steady_scan.m:601-613).
#pragma once

#include <type_traits>

#include "ss_common.cuh"

namespace ss {

template <class T>
__device__ __forceinline__ double fe_load(const void* base, size_t i) {
  return to_double(reinterpret_cast<const T*>(base)[i]);
}

// One 1-D circular pass of the blur over frames of h x w column-major samples, n frames in a row.
// axis 0: down each column (period h + L), axis 1: along each row (period w + L). taps[d], d in
// [0, R], are the normalised weights at circular distance d; `period` is the padded length.
// Grid: (ceil(h / blockDim.x), w, frames); a thread per output sample, lanes on consecutive rows, so
// every tap's loads are coalesced along the column. An output whose window lies inside the frame
// sums its taps in symmetric pairs; near the ends the window wraps over the period and skips the
// zero padding.
template <class InT, int AXIS>
__global__ void __launch_bounds__(256) k_blur_pass(const void* __restrict__ in, double* __restrict__ out, int h, int w,
                                                   int period, const double* __restrict__ taps, int R) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= h) return;
  const int j = blockIdx.y;
  const size_t base = (size_t)blockIdx.z * h * w;
  const int len = AXIS == 0 ? h : w;
  const int pos = AXIS == 0 ? i : j;
  const size_t stride = AXIS == 0 ? 1 : (size_t)h;
  const size_t at = base + (size_t)j * h + i;  // this output; the tap at offset d reads at + d stride
  double s;
  if (pos >= R && pos + R < len) {
    s = fe_load<InT>(in, at) * taps[0];
    for (int d = 1; d <= R; d++)
      s = fma(fe_load<InT>(in, at - d * stride) + fe_load<InT>(in, at + d * stride), taps[d], s);
  } else {
    s = 0.0;
    for (int d = -R; d <= R; d++) {
      int a = pos + d;
      if (a < 0) a += period;
      else if (a >= period) a -= period;
      if (a >= len) continue;  // the zero padding
      s = fma(fe_load<InT>(in, at + (ptrdiff_t)(a - pos) * (ptrdiff_t)stride), taps[d < 0 ? -d : d], s);
    }
  }
  out[at] = s;
}

// Order-preserving 64-bit key of a double and back.
__device__ __forceinline__ unsigned long long fe_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double fe_unkey(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
  return __longlong_as_double((long long)b);
}

// Adds 1 to hist[bin] for every lane of the warp with `take`: the lanes that share the bin of the
// first taking lane add with one shared atomic, the others one each (a frame's samples share their
// leading key digits, which would otherwise serialise the warp's atomics on one address).
__device__ __forceinline__ void fe_hist_add(unsigned* hist, unsigned bin, bool take) {
  const unsigned act = __activemask();
  const unsigned tk = __ballot_sync(act, take);
  if (!tk) return;
  const unsigned b0 = __shfl_sync(act, bin, __ffs(tk) - 1);
  const bool same = take && bin == b0;
  const unsigned sm = __ballot_sync(act, same);
  if (same) {
    if ((threadIdx.x & 31) == (unsigned)(__ffs(sm) - 1)) atomicAdd(&hist[b0], (unsigned)__popc(sm));
  } else if (take) {
    atomicAdd(&hist[bin], 1u);
  }
}

constexpr int kFeUnroll = 4;

// The k-th smallest (0-based) of the n samples at x (whole CTA; result in every thread): eight
// passes over 8-bit digits of the keys, most significant first, kFeUnroll loads in flight per
// thread. With `nan_flag`, the first pass also sets *nan_flag when a sample is NaN (the caller
// stops on it: NaN keys sort above every number).
template <class T>
__device__ unsigned long long fe_select_key(const void* x, size_t n, size_t k, unsigned* hist, int* nan_flag) {
  unsigned long long prefix = 0, mask = 0;
  __shared__ unsigned long long s_prefix;
  __shared__ size_t s_k;
  const size_t step = (size_t)blockDim.x * kFeUnroll;
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    bool nan = false;
    for (size_t i0 = threadIdx.x; i0 < n; i0 += step) {
      double v[kFeUnroll];
#pragma unroll
      for (int u = 0; u < kFeUnroll; u++) {
        const size_t i = i0 + (size_t)u * blockDim.x;
        v[u] = i < n ? fe_load<T>(x, i) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kFeUnroll; u++) {
        const bool in = i0 + (size_t)u * blockDim.x < n;
        const unsigned long long key = fe_key(v[u]);
        if (nan_flag && shift == 56) nan |= in && isnan(v[u]);
        fe_hist_add(hist, (unsigned)((key >> shift) & 0xFF), in && (key & mask) == prefix);
      }
    }
    if (nan) *nan_flag = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
      size_t below = 0;
      int b = 0;
      for (; b < 255; b++) {
        if (below + hist[b] > k) break;
        below += hist[b];
      }
      s_prefix = prefix | ((unsigned long long)b << shift);
      s_k = k - below;
    }
    __syncthreads();
    prefix = s_prefix;
    k = s_k;
    mask |= 0xFFull << shift;
    if (nan_flag && shift == 56 && *nan_flag) return 0;
    __syncthreads();
  }
  return prefix;
}

// Median of each frame's h * w samples (a CTA per frame): the middle sample, or the mean of the two
// middle samples for an even count; NaN when a sample is NaN. For an even count the upper middle
// sample follows from the lower one by one more pass: the lower one again when more than k samples
// are at most it, else the smallest sample above it.
template <class T>
__global__ void __launch_bounds__(1024) k_frame_median(const void* __restrict__ x, size_t per_frame,
                                                       double* __restrict__ med) {
  __shared__ unsigned hist[256];
  __shared__ int s_nan;
  __shared__ unsigned long long s_min;
  __shared__ unsigned long long s_le;
  const size_t off = (size_t)blockIdx.x * per_frame;
  const void* fx = reinterpret_cast<const T*>(x) + off;
  if (threadIdx.x == 0) {
    s_nan = 0;
    s_min = ~0ull;
    s_le = 0;
  }
  __syncthreads();
  const size_t k = (per_frame - 1) / 2;  // the (lower) middle sample
  const unsigned long long ka = fe_select_key<T>(fx, per_frame, k, hist, &s_nan);
  if (s_nan) {
    if (threadIdx.x == 0) med[blockIdx.x] = NAN;
    return;
  }
  const double a = fe_unkey(ka);
  if (per_frame & 1) {
    if (threadIdx.x == 0) med[blockIdx.x] = a;
    return;
  }
  unsigned long long mn = ~0ull, le = 0;
  for (size_t i = threadIdx.x; i < per_frame; i += blockDim.x) {
    const unsigned long long key = fe_key(fe_load<T>(fx, i));
    if (key <= ka) le++;
    else mn = key < mn ? key : mn;
  }
  for (int o = 16; o > 0; o >>= 1) {
    le += __shfl_xor_sync(0xffffffffu, le, o);
    const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mn, o);
    mn = m2 < mn ? m2 : mn;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&s_le, le);
    atomicMin(&s_min, mn);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double b = s_le > k + 1 ? a : fe_unkey(s_min);
    med[blockIdx.x] = (a + b) / 2.0;
  }
}

// x /= med[frame], in place (FP64 samples).
__global__ void k_frame_divide(double* __restrict__ x, size_t per_frame, size_t total, const double* __restrict__ med) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
    x[e] = x[e] / med[e / per_frame];
}

// Block matrices of frames: out (Hb x nb * n) entry (r, b + f nb) = frame f's cropped pixel
// gather[r + b Hb] (column-major in the cropped hc x wc frame; -1: 0), the cropped frame being rows
// [r0, r0 + hc) and columns [c0, c0 + wc) of the h x w frame.
template <class InT, class OutT>
__global__ void __launch_bounds__(256) k_block_gather(const void* __restrict__ in, OutT* __restrict__ out, int h, int w,
                                                      int n, int r0, int c0, int hc, const int* __restrict__ gather,
                                                      int hb, int nb) {
  const size_t per = (size_t)hb * nb, total = per * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t f = e / per;
    const int g = gather[e - f * per];
    OutT v = OutT(0);
    if (g >= 0) {
      const int ci = g % hc, cj = g / hc;
      const size_t src = f * (size_t)h * w + (size_t)(cj + c0) * h + (ci + r0);
      if constexpr (std::is_same<InT, OutT>::value) v = reinterpret_cast<const InT*>(in)[src];
      else v = (OutT)to_double(reinterpret_cast<const InT*>(in)[src]);
    }
    out[e] = v;
  }
}

}  // namespace ss
