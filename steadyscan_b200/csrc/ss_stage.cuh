// Staging of template row windows in shared memory with the bulk-copy (TMA) engine.
//
// A window holds rows [r0, r0 + rows) of the FP32 template at its row pitch. It is filled by
// cp.async.bulk from global memory completing on an mbarrier; no multicast is used. Waits are
// bounded: if a copy does not complete within the bound the kernel records bit 0 in the batch's
// error word and evaluates from the global template instead.
#pragma once

#include "ss_common.cuh"

namespace ss {

constexpr long long kWaitPolls = 1LL << 20;

struct TWin {
  const float* p;  // nullptr: no window, use the global template quads
  int r0, rows, pitch;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One thread: expects `bytes` on the barrier and copies them (16-byte aligned, multiple of 16).
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  const char* s = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  for (unsigned off = 0; off < bytes; off += 32768u) {
    const unsigned n = bytes - off < 32768u ? bytes - off : 32768u;
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(d + off)),
                 "l"(s + off), "r"(n), "r"(smem_u32(bar))
                 : "memory");
  }
}

// Bounded wait for the barrier phase; true when the copy completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase) {
  const unsigned a = smem_u32(bar);
  for (long long i = 0; i < kWaitPolls; i++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Window rows that contain every bilinear footprint of pixels whose y lies in [ylo, yhi], with a
// one-row margin for FP32 rounding; rows <= 0 when the bound is not finite or exceeds max_rows.
__device__ __forceinline__ void window_rows(const GroupDesc& G, float ylo, float yhi, int max_rows, int& r0,
                                            int& rows) {
  rows = 0;
  r0 = 0;
  if (!(ylo <= yhi) || !isfinite(ylo) || !isfinite(yhi)) return;
  const float lo = fmaxf(ylo, -2.0f), hi = fminf(yhi, (float)G.Ht + 2.0f);
  int a = max(0, (int)floorf(lo) - 1);
  int b = min(G.Ht - 1, (int)floorf(hi) + 2);
  if (b < a + 1) {  // no pixel can be inside the template: a two-row window keeps indexing in range
    b = min(max(a, 1), G.Ht - 1);
    a = b - 1;
  }
  if (b - a + 1 > max_rows) return;
  r0 = a;
  rows = b - a + 1;
}

// Stages rows [r0, r0 + rows) of the FP32 template into win (whole CTA; barrier already
// initialised, phase tracked by the caller). Returns false after recording a timeout in bit 0 of the
// batch's error word: the copy may then still be in flight, so the phase is left as it is, the
// caller stages no further window in this CTA (its later tiles and passes sample the global
// template instead) and calls drain_window before the CTA exits.
// src: the rows to copy from (G.tplain when null).
__device__ __forceinline__ bool stage_window(const GroupDesc& G, float* win, int r0, int rows, uint64_t* bar,
                                           unsigned& phase, const float* src = nullptr) {
  __syncthreads();  // the previous window is no longer read
  if (!src) src = G.tplain;
  if (threadIdx.x == 0)
    bulk_copy(win, src + (size_t)r0 * G.tpitch, (unsigned)((size_t)rows * G.tpitch * sizeof(float)), bar);
  bool ok = mbar_wait(bar, phase);
  if (!ok) ok = mbar_wait(bar, phase);  // second bounded wait for the copy still in flight
  if (!ok && threadIdx.x == 0) atomicOr(G.err, 1);
  ok = __syncthreads_and(ok ? 1 : 0) != 0;
  if (ok) phase ^= 1u;
  return ok;
}

// Before a CTA whose staging timed out exits: one more bounded wait for the copy into its shared
// memory (whole CTA).
__device__ __forceinline__ void drain_window(uint64_t* bar, unsigned phase) {
  (void)mbar_wait(bar, phase);
  __syncthreads();
}

// CTA-wide min of lo and max of hi (all threads call; result in every thread).
__device__ __forceinline__ void block_minmax(float& lo, float& hi) {
  __shared__ float s_lo[32], s_hi[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    s_lo[w] = lo;
    s_hi[w] = hi;
  }
  __syncthreads();
  lo = s_lo[0];
  hi = s_hi[0];
  for (int i = 1; i < nw; i++) {
    lo = fminf(lo, s_lo[i]);
    hi = fmaxf(hi, s_hi[i]);
  }
}

// Bilinear template value and warped gradients from a staged window (see sample() for the
// arithmetic); the row index is clamped into the window.
template <bool kGrad>
__device__ __forceinline__ Sample<float> sample_win(const TWin& w, float x, float y) {
  float xf, yf;
  const int ix = split(x, xf), iy = split(y, yf);
  const int ry = min(max(iy - w.r0, 0), w.rows - 2);
  const float* q = w.p + ry * w.pitch + ix;
  const float t00 = q[0], t01 = q[1], t10 = q[w.pitch], t11 = q[w.pitch + 1];
  const float a = fmaf(yf, t10, (1.0f - yf) * t00);
  const float b = fmaf(yf, t11, (1.0f - yf) * t01);
  Sample<float> s;
  s.wI = fmaf(xf, b, (1.0f - xf) * a);
  if (kGrad) {
    s.wx = fmaf(yf, t11 - t10, (1.0f - yf) * (t01 - t00));
    s.wy = fmaf(xf, t11 - t01, (1.0f - xf) * (t10 - t00));
  } else {
    s.wx = s.wy = 0.0f;
  }
  return s;
}

}  // namespace ss
