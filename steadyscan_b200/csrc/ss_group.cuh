// Per-group kernels: the half-step solve, the line-search decision and the iteration control.
#pragma once

#include "ss_common.cuh"
#include "ss_eval.cuh"

namespace ss {

constexpr int kSolveThreads = 1024;
constexpr int kCrStride = 13;  // D(3: xx yy xy) L(4) R(4) b(2)

__device__ __forceinline__ void cr_load(const double* n, double& d0, double& d1, double& d2, M2& L, M2& R, double& b0,
                                        double& b1) {
  d0 = n[0]; d1 = n[1]; d2 = n[2];
  L = {n[3], n[4], n[5], n[6]};
  R = {n[7], n[8], n[9], n[10]};
  b0 = n[11]; b1 = n[12];
}

// Solves a symmetric positive definite block-tridiagonal system with 2x2 blocks in place by block
// cyclic reduction, with the whole CTA. Node i of cr holds (D_i: xx yy xy, L_i: coupling to its left
// neighbour, R_i: coupling to its right neighbour, b_i) in kCrStride doubles; on return b_i holds
// x_i. At stride s every multiple of 2s absorbs its two odd-multiple neighbours (each elimination is
// a Schur complement on 2x2 blocks), so the reduction takes ceil(log2 h) levels; back substitution
// runs the levels in reverse. In exact arithmetic this is the LDL^T of the system in a nested
// dissection order, so it solves the same equations as the reference's exact sparse solvers
// (eigensolve.cpp:35-38, cusolversolver.cu:53-56).
__device__ void cr_solve(double* cr, int h) {
  const int t = threadIdx.x, nt = blockDim.x;
  int top = 1;
  while (top < h) top <<= 1;
  for (int s = 1; s < h; s <<= 1) {
    for (int j = t * 2 * s; j < h; j += nt * 2 * s) {
      double* n = cr + (size_t)j * kCrStride;
      double d0, d1, d2, b0, b1;
      M2 L, R;
      cr_load(n, d0, d1, d2, L, R, b0, b1);
      M2 D = {d0, d2, d2, d1};
      if (j - s >= 0) {
        double e0, e1, e2, c0, c1;
        M2 Ll, Rl;
        cr_load(cr + (size_t)(j - s) * kCrStride, e0, e1, e2, Ll, Rl, c0, c1);
        M2 Di = m2_inv({e0, e2, e2, e1});
        M2 T = m2_mul(L, Di);
        D = m2_sub(D, m2_mul(T, Rl));
        b0 -= T.a * c0 + T.b * c1;
        b1 -= T.c * c0 + T.d * c1;
        L = m2_neg(m2_mul(T, Ll));
      }
      if (j + s < h) {
        double e0, e1, e2, c0, c1;
        M2 Lr, Rr;
        cr_load(cr + (size_t)(j + s) * kCrStride, e0, e1, e2, Lr, Rr, c0, c1);
        M2 Di = m2_inv({e0, e2, e2, e1});
        M2 T = m2_mul(R, Di);
        D = m2_sub(D, m2_mul(T, Lr));
        b0 -= T.a * c0 + T.b * c1;
        b1 -= T.c * c0 + T.d * c1;
        R = m2_neg(m2_mul(T, Rr));
      }
      n[0] = D.a; n[1] = D.d; n[2] = 0.5 * (D.b + D.c);
      n[3] = L.a; n[4] = L.b; n[5] = L.c; n[6] = L.d;
      n[7] = R.a; n[8] = R.b; n[9] = R.c; n[10] = R.d;
      n[11] = b0; n[12] = b1;
    }
    __syncthreads();
  }
  if (t == 0 && h > 0) {
    double* n = cr;
    M2 Di = m2_inv({n[0], n[2], n[2], n[1]});
    double b0 = n[11], b1 = n[12];
    n[11] = Di.a * b0 + Di.b * b1;
    n[12] = Di.c * b0 + Di.d * b1;
  }
  __syncthreads();
  for (int s = top >> 1; s >= 1; s >>= 1) {
    for (int i = s + t * 2 * s; i < h; i += nt * 2 * s) {
      double* n = cr + (size_t)i * kCrStride;
      double d0, d1, d2, b0, b1;
      M2 L, R;
      cr_load(n, d0, d1, d2, L, R, b0, b1);
      const double* l = cr + (size_t)(i - s) * kCrStride;
      b0 -= L.a * l[11] + L.b * l[12];
      b1 -= L.c * l[11] + L.d * l[12];
      if (i + s < h) {
        const double* r = cr + (size_t)(i + s) * kCrStride;
        b0 -= R.a * r[11] + R.b * r[12];
        b1 -= R.c * r[11] + R.d * r[12];
      }
      M2 Di = m2_inv({d0, d2, d2, d1});
      n[11] = Di.a * b0 + Di.b * b1;
      n[12] = Di.c * b0 + Di.d * b1;
    }
    __syncthreads();
  }
}


__device__ __forceinline__ M2 m2_t(const M2& x) { return {x.a, x.c, x.b, x.d}; }
__device__ __forceinline__ M2 m2_add(const M2& x, const M2& y) { return {x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d}; }
__device__ __forceinline__ void m2_mv(const M2& m, double v0, double v1, double& r0, double& r1) {
  r0 = m.a * v0 + m.b * v1;
  r1 = m.c * v0 + m.d * v1;
}
__device__ __forceinline__ M2 sym_inv(double d0, double d1, double d2) { return m2_inv({d0, d2, d2, d1}); }

// Node layout of the partitioned block-tridiagonal solve: the h nodes are split into P =
// min(blockDim.x, h) contiguous partitions, the first rem = h - q P of q + 1 nodes and the rest of q;
// every field of every node has a plane of h doubles in which node k of partition t sits at
// k P + t, so the threads of a warp, each walking its own partition, touch consecutive doubles.
constexpr int kRelStride = 10;                      // uL (4), uR (4), u0 (2)
constexpr int kPartSmemStride = kCrStride + kRelStride;  // shared doubles per partition

enum PartPlane : int {
  kPD0 = 0, kPD1, kPD2,         // D (xx yy xy); after the forward sweep D~^-1
  kPR0, kPR1, kPR2, kPR3,       // R, the block coupling the node to the next: [[R0 R1] [R2 R3]]
  kPB0, kPB1,                   // b; after the forward sweep b~
  kPS0, kPS1, kPS2, kPS3,       // forward spike S~
  kPlanes
};

struct PartLayout {
  int h, P, q, rem;
  __device__ PartLayout(int h_, int nt) : h(h_), P(min(nt, h_)), q(h_ / min(nt, h_)), rem(h_ - (h_ / min(nt, h_)) * min(nt, h_)) {}
  __device__ int a(int t) const { return t * q + min(t, rem); }
  __device__ int m(int t) const { return q + (t < rem ? 1 : 0); }
  __device__ size_t pos(int t, int k) const { return (size_t)k * P + t; }
  __device__ size_t pos_of(int i) const {  // plane position of node i
    const int lo = rem * (q + 1);
    if (i < lo) {
      const int t = i / (q + 1);
      return pos(t, i - t * (q + 1));
    }
    const int j = i - lo, t = rem + j / q;
    return pos(t, j - (t - rem) * q);
  }
};

// Solves the symmetric positive definite block-tridiagonal system of h nodes given in the planes
// of pl (PartLayout of h and blockDim.x; L_i = R_{i-1}^T) with the whole CTA and writes x_i to
// xo[i * xs] and yo[i * ys]. Partition method: thread t eliminates the interior of its partition
// by block Thomas sweeps (backward for the relation of the first interior node, forward storing
// D~^-1, S~ and b~), leaving its last node as separator; the separators' Schur complement is block
// tridiagonal again and is solved by block cyclic reduction in shared memory (red: blockDim.x x
// kCrStride doubles); the interior follows by back substitution. For SPD systems every block
// elimination is a Schur complement of an SPD matrix, so this solves the same equations as the
// reference's exact solvers (eigensolve.cpp:35-38, cusolversolver.cu:53-56) in another
// elimination order. red holds blockDim.x x kPartSmemStride doubles: the separator system and
// each partition's first-interior relation.
__device__ void part_solve(double* pl, int h, double* red, double* xo, int xs, double* yo, int ys) {
  const int t = threadIdx.x;
  if (h <= 0) return;
  const PartLayout L(h, blockDim.x);
  const int P = L.P;
  const bool own = t < P;
  const int mt = own ? L.m(t) : 0;
  const int a = own ? L.a(t) : 0;
  const int e = a + mt - 1;
  double* const D0 = pl + (size_t)kPD0 * h;
  double* const D1 = pl + (size_t)kPD1 * h;
  double* const D2 = pl + (size_t)kPD2 * h;
  double* const R0 = pl + (size_t)kPR0 * h;
  double* const R1 = pl + (size_t)kPR1 * h;
  double* const R2 = pl + (size_t)kPR2 * h;
  double* const R3 = pl + (size_t)kPR3 * h;
  double* const B0 = pl + (size_t)kPB0 * h;
  double* const B1 = pl + (size_t)kPB1 * h;
  double* const S0 = pl + (size_t)kPS0 * h;
  double* const S1 = pl + (size_t)kPS1 * h;
  double* const S2 = pl + (size_t)kPS2 * h;
  double* const S3 = pl + (size_t)kPS3 * h;
  auto ldR = [&](size_t q) -> M2 { return {R0[q], R1[q], R2[q], R3[q]}; };
  const M2 Z = {0, 0, 0, 0};
  // coupling of node a to the previous separator (the last node of partition t - 1)
  const M2 La = (own && t > 0) ? m2_t(ldR(L.pos(t - 1, L.m(t - 1) - 1))) : Z;

  // backward sweep: relation x_a = u0 + uL x_(previous separator) + uR x_e of the first interior node
  if (own && mt >= 2) {
    size_t q = L.pos(t, mt - 2);
    M2 Dc = {D0[q], D2[q], D2[q], D1[q]};
    double b0 = B0[q], b1 = B1[q];
    M2 S = ldR(q);
    for (int k = mt - 3; k >= 0; k--) {
      q = L.pos(t, k);
      const M2 Ri = ldR(q);
      const M2 Nm = m2_mul(Ri, m2_inv(Dc));
      Dc = m2_sub({D0[q], D2[q], D2[q], D1[q]}, m2_mul(Nm, m2_t(Ri)));
      double c0, c1;
      m2_mv(Nm, b0, b1, c0, c1);
      b0 = B0[q] - c0;
      b1 = B1[q] - c1;
      S = m2_neg(m2_mul(Nm, S));
    }
    const M2 Di = m2_inv(Dc);
    const M2 uL = m2_neg(m2_mul(Di, La)), uR = m2_neg(m2_mul(Di, S));
    double u0, u1;
    m2_mv(Di, b0, b1, u0, u1);
    double* r = red + (size_t)blockDim.x * kCrStride + (size_t)t * kRelStride;
    r[0] = uL.a; r[1] = uL.b; r[2] = uL.c; r[3] = uL.d;
    r[4] = uR.a; r[5] = uR.b; r[6] = uR.c; r[7] = uR.d;
    r[8] = u0; r[9] = u1;
  }
  // forward sweep storing D~^-1, S~ and b~ of each interior node; relation of the last one
  M2 uLe = Z, uRe = Z;
  double u0e = 0, u1e = 0;
  if (own && mt >= 2) {
    size_t q = L.pos(t, 0);
    M2 Di = m2_inv({D0[q], D2[q], D2[q], D1[q]});
    double b0 = B0[q], b1 = B1[q];
    M2 S = La;
    M2 Rp = ldR(q);
    for (int k = 0;; k++) {
      D0[q] = Di.a; D1[q] = Di.d; D2[q] = 0.5 * (Di.b + Di.c);
      S0[q] = S.a; S1[q] = S.b; S2[q] = S.c; S3[q] = S.d;
      B0[q] = b0; B1[q] = b1;
      if (k + 1 >= mt - 1) break;
      q = L.pos(t, k + 1);
      const M2 M = m2_mul(m2_t(Rp), Di);  // L_{i+1} D~_i^-1 with L_{i+1} = R_i^T
      Di = m2_inv(m2_sub({D0[q], D2[q], D2[q], D1[q]}, m2_mul(M, Rp)));
      double c0, c1;
      m2_mv(M, b0, b1, c0, c1);
      b0 = B0[q] - c0;
      b1 = B1[q] - c1;
      S = m2_neg(m2_mul(M, S));
      Rp = ldR(q);
    }
    // Rp = R_{e-1}, Di = D~_{e-1}^-1
    uRe = m2_neg(m2_mul(Di, Rp));
    uLe = m2_neg(m2_mul(Di, S));
    m2_mv(Di, b0, b1, u0e, u1e);
  }
  __syncthreads();
  // separator rows of the reduced system
  if (own) {
    const size_t qe = L.pos(t, mt - 1);
    M2 Dr = {D0[qe], D2[qe], D2[qe], D1[qe]};
    double b0 = B0[qe], b1 = B1[qe];
    // L_e = R_{e-1}^T: node e - 1 is an interior node, or the previous separator
    const M2 Le = mt >= 2 ? m2_t(ldR(L.pos(t, mt - 2))) : La;
    const M2 Re = e + 1 < h ? ldR(qe) : Z;
    M2 Lr = Z, Rr = Z;
    double c0, c1;
    if (mt >= 2) {
      Dr = m2_add(Dr, m2_mul(Le, uRe));
      Lr = m2_mul(Le, uLe);
      m2_mv(Le, u0e, u1e, c0, c1);
      b0 -= c0;
      b1 -= c1;
    } else {
      Lr = Le;  // coupled directly to the previous separator (zero for the first node)
    }
    if (t + 1 < P) {
      if (L.m(t + 1) >= 2) {
        const double* w = red + (size_t)blockDim.x * kCrStride + (size_t)(t + 1) * kRelStride;
        const M2 uL1 = {w[0], w[1], w[2], w[3]}, uR1 = {w[4], w[5], w[6], w[7]};
        Dr = m2_add(Dr, m2_mul(Re, uL1));
        Rr = m2_mul(Re, uR1);
        m2_mv(Re, w[8], w[9], c0, c1);
        b0 -= c0;
        b1 -= c1;
      } else {
        Rr = Re;
      }
    }
    double* r = red + (size_t)t * kCrStride;
    r[0] = Dr.a; r[1] = Dr.d; r[2] = 0.5 * (Dr.b + Dr.c);
    r[3] = Lr.a; r[4] = Lr.b; r[5] = Lr.c; r[6] = Lr.d;
    r[7] = Rr.a; r[8] = Rr.b; r[9] = Rr.c; r[10] = Rr.d;
    r[11] = b0; r[12] = b1;
  }
  __syncthreads();
  cr_solve(red, P);
  // back substitution of the interior
  if (own) {
    const double xl0 = t > 0 ? red[(size_t)(t - 1) * kCrStride + 11] : 0.0;
    const double xl1 = t > 0 ? red[(size_t)(t - 1) * kCrStride + 12] : 0.0;
    double x0 = red[(size_t)t * kCrStride + 11], x1 = red[(size_t)t * kCrStride + 12];
    xo[(size_t)e * xs] = x0;
    yo[(size_t)e * ys] = x1;
    for (int k = mt - 2; k >= 0; k--) {
      const size_t q = L.pos(t, k);
      const M2 Di = {D0[q], D2[q], D2[q], D1[q]};
      double c0, c1, s0, s1;
      m2_mv({S0[q], S1[q], S2[q], S3[q]}, xl0, xl1, s0, s1);
      m2_mv(ldR(q), x0, x1, c0, c1);  // R_i x_{i+1}
      m2_mv(Di, B0[q] - s0 - c0, B1[q] - s1 - c1, x0, x1);
      xo[(size_t)(a + k) * xs] = x0;
      yo[(size_t)(a + k) * ys] = x1;
    }
  }
  __syncthreads();
}

// Standalone solve of a block-tridiagonal system given as diag (n x 3: xx yy xy), coupling
// ((n-1) x 4: [[c0 c2] [c3 c1]] between block i and i+1) and rhs (n x 2) into x (n x 2), with
// the caller's workspace cr (n x kCrStride doubles). One CTA with blockDim.x x kPartSmemStride
// doubles of dynamic shared memory.
__global__ void __launch_bounds__(kSolveThreads) k_block_tridiag(int n, const double* __restrict__ diag,
                                                                 const double* __restrict__ coupling,
                                                                 const double* __restrict__ rhs,
                                                                 double* __restrict__ x, double* __restrict__ cr) {
  const PartLayout L(n, blockDim.x);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const size_t q = L.pos_of(i);
    cr[(size_t)kPD0 * n + q] = diag[3 * i];
    cr[(size_t)kPD1 * n + q] = diag[3 * i + 1];
    cr[(size_t)kPD2 * n + q] = diag[3 * i + 2];
    const double* c = coupling + 4 * (size_t)i;
    const bool has = i + 1 < n;
    cr[(size_t)kPR0 * n + q] = has ? c[0] : 0.0;
    cr[(size_t)kPR1 * n + q] = has ? c[2] : 0.0;
    cr[(size_t)kPR2 * n + q] = has ? c[3] : 0.0;
    cr[(size_t)kPR3 * n + q] = has ? c[1] : 0.0;
    cr[(size_t)kPB0 * n + q] = rhs[2 * i];
    cr[(size_t)kPB1 * n + q] = rhs[2 * i + 1];
  }
  __syncthreads();
  extern __shared__ double sh_red[];  // blockDim.x x kPartSmemStride
  part_solve(cr, n, sh_red, x, 2, x + 1, 2);
}

// Knot-difference regulariser of frame f (extension; lambda = 0 reproduces the reference): sum of
// |k_{t+1}-k_t|^2 over its W edges, own knots from own (+N for y), right boundary (bx, by). All
// lanes of a warp call; the result is in every lane.
__device__ inline double frame_reg_warp(const double* own, int W, int N, double bx, double by) {
  double r = 0;
  for (int t = threadIdx.x & 31; t < W; t += 32) {
    double x0 = own[t], y0 = own[t + N];
    double x1 = t + 1 < W ? own[t + 1] : bx, y1 = t + 1 < W ? own[t + 1 + N] : by;
    r += (x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0);
  }
  return warp_sum(r);
}

// Chunked scan of SmearingFilter::apply (smearingfilter.cpp:24-33), v_i = s v_{i-1} + (1-s) v_i with
// v_{-1} = 0, over n values. Each thread runs the exact recurrence on its chunk from a carry-in that
// composes the preceding chunks' affine maps.
__device__ void smear_scan(double* v, int n, double s, double* sh_a, double* sh_b) {
  const int nt = blockDim.x, t = threadIdx.x;
  const int chunk = (n + nt - 1) / nt;
  const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
  const double om = 1.0 - s;
  double y = 0.0, a = 1.0;
  for (int i = lo; i < hi; i++) {
    y = __dadd_rn(__dmul_rn(y, s), __dmul_rn(v[i], om));
    a = a * s;
  }
  // carry-in of each chunk: exclusive scan of the chunks' affine maps c -> a c + y (composition
  // (a2, b2) after (a1, b1) = (a2 a1, a2 b1 + b2)), warp scans then a scan of the warp totals
  const int lane = t & 31, warp = t >> 5, nw = (nt + 31) >> 5;
  double A = a, B = y;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double pa = __shfl_up_sync(0xffffffffu, A, o), pb = __shfl_up_sync(0xffffffffu, B, o);
    if (lane >= o) {
      B = A * pb + B;
      A = A * pa;
    }
  }
  if (lane == 31) {
    sh_a[warp] = A;
    sh_b[warp] = B;
  }
  __syncthreads();
  if (warp == 0) {
    double wa = lane < nw ? sh_a[lane] : 1.0, wb = lane < nw ? sh_b[lane] : 0.0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double pa = __shfl_up_sync(0xffffffffu, wa, o), pb = __shfl_up_sync(0xffffffffu, wb, o);
      if (lane >= o) {
        wb = wa * pb + wb;
        wa = wa * pa;
      }
    }
    // exclusive: the composition of the preceding warps applied to 0
    const double ex = __shfl_up_sync(0xffffffffu, wb, 1);
    __syncwarp();
    if (lane < nw) sh_b[32 + lane] = lane == 0 ? 0.0 : ex;
  }
  __syncthreads();
  {
    // this thread's exclusive in-warp map applied to the warp's carry-in
    const double ea = __shfl_up_sync(0xffffffffu, A, 1), eb = __shfl_up_sync(0xffffffffu, B, 1);
    const double cw = sh_b[32 + warp];
    y = lane == 0 ? cw : ea * cw + eb;
  }
  __syncthreads();
  for (int i = lo; i < hi; i++) {
    y = __dadd_rn(__dmul_rn(y, s), __dmul_rn(v[i], om));
    v[i] = y;
  }
  __syncthreads();
}

// RangeFilter::apply (rangefilter.cpp:24-40): a sequential, data-dependent recurrence.
__device__ void range_seq(double* v, int n, double strength) {
  for (int i = 1; i < n - 1; i++) {
    double tc = (v[i - 1] + v[i + 1]) / 2;
    double d = (tc - v[i - 1]) * strength;
    if (v[i - 1] < v[i + 1]) {
      if (v[i] > v[i + 1] + d || v[i] < v[i - 1] - d) v[i] = tc;
    } else {
      if (v[i] < v[i + 1] + d || v[i] > v[i - 1] - d) v[i] = tc;
    }
  }
}

// The half-step solve of every group in phase kPhHalf runs as five launches: the per-column and
// per-frame set-up and the block assembly are spread over kSolveSplit CTAs per group
// (k_solve_prep, k_solve_planes, k_solve_expand), the steps that need the whole group in one CTA
// (compaction, the partitioned solve and the filters) run one 1024-thread CTA per group
// (k_solve_compact, k_solve_system). A single CTA per group spent most of its time in the
// independent per-node work, bound by one SM's global-memory queue.
//   blocksPresent / paramsUsed / errval (task_applyparameters.cuh:74-81, task_createparametermask.cuh,
//   task_calcerrval.cu:185), the filter switch-off (mainiteration.cpp:246-256), compaction
//   (task_generatesubsparseoffset.cu), the block-tridiagonal normal equations
//   (task_filldiagonals.cu:47-159, task_filljtr.cu:3-58) solved exactly in FP64, the solver's
//   filter (smearingfilter.cpp, rangefilter.cpp), the expansion with fixed knots
//   (task_expandresults.cu:9-36) and the line-search start.
constexpr int kSolveSplit = 32;     // CTAs per group of the parallel phases
constexpr int kSolvePrepThreads = 256;

// A group solves in this cycle: its half-step starts (no line search of it still runs).
__device__ __forceinline__ bool solve_starts(const GroupCtl& C) { return C.phase == kPhHalf && C.ls_state == 0; }

// Block presence, parameter use, knot copies, line-search state, errval of the active frames and
// the committed knots (grid: kSolveSplit x groups).
__global__ void __launch_bounds__(kSolvePrepThreads) k_solve_prep(const GroupDesc* __restrict__ gds,
                                                                  const GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.y];
  const GroupCtl& C = ctl[blockIdx.y];
  if (!solve_starts(C)) return;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
  const int W = G.W, N = G.N, nF = G.nF, fW = G.fW, shift = C.shift;
  // a column's block is present with enough valid pixels; a knot is used when a block next to it is
  for (int c = gt; c < fW; c += gn) {
    const bool present = G.asmcnt[c] >= G.min_points[c % W];
    G.blocks_present[c] = present;
    const int f = c / W;
    if (!frame_active(G, f, shift)) {
      // TimedMainIteration clears paramsUsed before every half-step (timedmainiteration.cpp:50), so
      // the knots of inactive frames are unused; MainIteration leaves their last use
      if (G.flags & kFlagTimeSub) G.params_used[c] = 0;
      continue;
    }
    const bool before = c > 0 && G.asmcnt[c - 1] >= G.min_points[(c - 1) % W];
    G.params_used[c] = present || before;
  }
  if (gt == 0) G.blocks_present[N - 1] = 0;
  // knot copies: kmask of every frame, kdiff of the active ones (the state the line search starts
  // from); line-search state
  const int W1 = W + 1;
  for (int idx = gt; idx < nF * W1; idx += gn) {
    const int f = idx / W1, k = idx - f * W1;
    const double x = G.p[(size_t)f * W + k], y = G.p[(size_t)N + (size_t)f * W + k];
    double* km = G.kmask + (size_t)f * 2 * W1;
    km[k] = x;
    km[W1 + k] = y;
    if (frame_active(G, f, shift)) {
      double* kd = G.kdiff + (size_t)f * 2 * W1;
      kd[k] = x;
      kd[W1 + k] = y;
    }
  }
  for (int f = gt; f < nF; f += gn) {
    G.fstate[f] = frame_active(G, f, shift) ? 2 : 0;  // searching once the step is known
    G.ls_trials[f] = 0;
  }
  // errval of the active frames (task_calcerrval.cu:185), a warp per frame
  {
    const int lane = threadIdx.x & 31;
    for (int f = gt >> 5; f < nF; f += gn >> 5) {
      if (!frame_active(G, f, shift)) continue;
      const double* ks = G.p + (size_t)f * W;
      double e = 0, rg = 0;
      int n = 0;
      for (int cc = lane; cc < W; cc += 32) {
        e += G.asmsum[(size_t)(f * W + cc) * kCsStride + kCsSsd];
        n += G.asmcnt[f * W + cc];
        if (G.lambda != 0.0) {  // knot-difference regulariser (extension); the right boundary is ks[W]
          const double dx = ks[cc + 1] - ks[cc], dy = ks[N + cc + 1] - ks[N + cc];
          rg += dx * dx + dy * dy;
        }
      }
      e = warp_sum(e);
      n = warp_sum(n);
      rg = warp_sum(rg);
      if (lane == 0) G.errval[shift * nF + f] = (G.lambda != 0.0) ? (e + G.lambda * rg) / (double)n : e / (double)n;
    }
  }
  for (int i = gt; i < 2 * N; i += gn) G.p_snap[i] = G.p[i];
}

// Filter switch-off, line-search start, compaction and the solver's coupling state (one CTA per
// group). Marks the groups that solve in this cycle (solve_now) for the launches that follow.
__global__ void __launch_bounds__(kSolveThreads) k_solve_compact(const GroupDesc* __restrict__ gds,
                                                                 GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  const bool starts = solve_starts(C);
  __syncthreads();  // every thread has read the phase before thread 0 changes the state below
  if (threadIdx.x == 0) C.solve_now = starts ? 1 : 0;
  // the first iteration's clock starts at its first solve (flags T and t)
  if (threadIdx.x == 0 && starts && G.o_iter_times && C.t_mark == 0) C.t_mark = device_clock_ns();
  if (!starts) return;
  const int t = threadIdx.x, nt = blockDim.x;
  const int N = G.N, nF = G.nF, shift = C.shift;
  __shared__ int sh_i[kSolveThreads];
  __shared__ int sh_h, sh_nact;
  __shared__ int sh_rebuild;
  if (t == 0) {
    if (C.n_filter_iter != 0 && C.iteration > C.n_filter_iter) {
      C.filter_active = 0;
      // TimedMainIteration keeps filterID here (timedmainiteration.cpp:97-105)
      if (!(G.flags & kFlagTimeSub)) C.filter_id = 0;
      C.n_filter_iter = 0;
    }
    sh_nact = 0;
  }
  __syncthreads();
  for (int f = t; f < nF; f += nt)
    if (frame_active(G, f, shift)) atomicAdd(&sh_nact, 1);
  __syncthreads();
  if (t == 0) {
    C.n_eval += sh_nact;
    C.passes[kAssemble] += nF;
    C.ls_state = 1;
    C.ls_pending = G.ls_rounds ? sh_nact : 0;  // frames whose line search starts (trial rounds)
  }

  // (2) compaction: list position of every used knot (paramsUsed[N-1] is never written, so it
  // keeps its zero fill: task_allocate.cu:223)
  {
    const int chunk = (N + nt - 1) / nt;
    const int lo = min(N, t * chunk), hi = min(N, lo + chunk);
    int cnt = 0;
    for (int k = lo; k < hi; k++) cnt += G.params_used[k] ? 1 : 0;
    // exclusive scan of the chunk counts: warp scans, then a scan of the warp totals
    const int lane = t & 31, warp = t >> 5;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) sh_i[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int nw = nt >> 5;
      int w = lane < nw ? sh_i[lane] : 0, wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += v;
      }
      if (lane < nw) sh_i[32 + lane] = wi - w;
      if (lane == nw - 1) sh_h = wi;
    }
    __syncthreads();
    int pos = sh_i[32 + warp] + incl - cnt;
    for (int k = lo; k < hi; k++) {
      if (G.params_used[k]) {
        G.list[pos] = k;
        G.list[N + k] = pos;  // inverse map in the second half
        pos++;
      }
    }
  }
  __syncthreads();
  const int h = sh_h;
  if (t == 0) {
    C.n_used = 2 * h;
    sh_rebuild = (G.solver_id == 2) && (C.eig_size != 2 * h);  // eigensolve.cpp:12-20
    if (G.solver_id == 2) C.eig_size = 2 * h;
  }
  __syncthreads();
  if (sh_rebuild)
    for (int i = t; i < N; i += nt) G.eig_valid[i] = 0;
  __syncthreads();

}

// Blocks of the compact system and the coupling to the next list position, written in the plane
// layout of the partitioned solve (node i at PartLayout(h, kSolveThreads).pos_of(i)); one node per
// thread of kSolveSplit CTAs per group.
__global__ void __launch_bounds__(kSolvePrepThreads) k_solve_planes(const GroupDesc* __restrict__ gds,
                                                                    const GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.y];
  const GroupCtl& C = ctl[blockIdx.y];
  if (!C.solve_now) return;
  const int h = C.n_used >> 1, N = G.N, fW = G.fW;
  if (h <= 0) return;
  const double lam = G.lambda;
  const PartLayout PLy(h, kSolveThreads);
  double* const pl = G.cr;
  const bool natural = G.solver_id == 0;  // the ILU(0) walk reads the planes in list order
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < h; i += gridDim.x * blockDim.x) {
    {
      const size_t q = natural ? (size_t)i : PLy.pos_of(i);
      const int k = G.list[i];
      double d0 = 0, d1 = 0, d2 = 0, r0 = 0, r1 = 0;
      double2 o78 = make_double2(0, 0), o9 = make_double2(0, 0);
      if (k < fW) {
        const double2* a = reinterpret_cast<const double2*>(G.asmsum + (size_t)k * kCsStride);
        const double2 v01 = a[0], v23 = a[1], v1011 = a[5];
        o78 = a[3];
        o9 = a[4];
        d0 += v01.y; d1 += v23.x; d2 += v23.y;   // kCsAxx kCsAyy kCsAxy
        r0 += v1011.x; r1 += v1011.y;            // kCsJ1x kCsJ1y
      }
      if (k > 0) {
        const double2* b = reinterpret_cast<const double2*>(G.asmsum + (size_t)(k - 1) * kCsStride);
        const double2 v45 = b[2], v67 = b[3], v1213 = b[6];
        d0 += v45.x; d1 += v45.y; d2 += v67.x;   // kCsBxx kCsByy kCsBxy
        r0 += v1213.x; r1 += v1213.y;            // kCsJ2x kCsJ2y
      }
      M2 R = {0, 0, 0, 0};
      const bool fresh = (i + 1 < h) && (G.list[i + 1] == k + 1);
      if (fresh) {
        R = {o78.y, o9.y, o9.y, o9.x};  // (Oxx Oxy; Oxy Oyy)
        if (G.solver_id == 2) {
          double* e = G.eig_c + (size_t)i * 4;
          e[0] = R.a; e[1] = R.b; e[2] = R.c; e[3] = R.d;
          G.eig_valid[i] = 1;
        }
      } else if (G.solver_id == 2 && i + 1 < h && G.eig_valid[i]) {
        // SolverEigen keeps its matrix between solves while the used count is unchanged
        // (eigensolve.cpp:7-31): a coupling that is not written now keeps its last value.
        const double* e = G.eig_c + (size_t)i * 4;
        R = {e[0], e[1], e[2], e[3]};
      }
      if (lam != 0.0) {
        const int deg = (k > 0) + (k < N - 1);
        d0 += lam * deg;
        d1 += lam * deg;
        const double* p = G.p;
        r0 -= lam * (deg * p[k] - (k > 0 ? p[k - 1] : 0) - (k < N - 1 ? p[k + 1] : 0));
        r1 -= lam * (deg * p[N + k] - (k > 0 ? p[N + k - 1] : 0) - (k < N - 1 ? p[N + k + 1] : 0));
        if (fresh) {
          R.a -= lam;
          R.d -= lam;
        }
      }
      pl[(size_t)kPD0 * h + q] = d0;
      pl[(size_t)kPD1 * h + q] = d1;
      pl[(size_t)kPD2 * h + q] = d2;
      pl[(size_t)kPR0 * h + q] = R.a;
      pl[(size_t)kPR1 * h + q] = R.b;
      pl[(size_t)kPR2 * h + q] = R.c;
      pl[(size_t)kPR3 * h + q] = R.d;
      pl[(size_t)kPB0 * h + q] = r0;
      pl[(size_t)kPB1 * h + q] = r1;
    }
  }
}

// Solver id 0: the reference's cuSPARSE path (cusparsesolver.cu:119-158), an incomplete LU
// factorisation without fill, ILU(0), of the compact system in [x_0..x_{h-1}, y_0..y_{h-1}] order
// (rows and their columns sorted, task_filldiagonals.cu:185-214), then the unit-lower and the upper
// triangular solve. Each row's pattern is its 2x2 diagonal block and, where list positions i and
// i+1 are consecutive knots (a "fresh" coupling), the coupling block: row x_i holds x_{i-1}, x_i,
// x_{i+1}, y_{i-1}, y_i, y_{i+1}; row y_i the same columns. Row by row (IKJ order) the x rows
// reduce to a tridiagonal LU whose updates of the y columns are kept where the pattern has them
// (the update of (x_i, y_{i-2}) is dropped); each y row eliminates x_{i-1}, x_i, x_{i+1} and
// y_{i-1} in column order. The recurrences run along the whole knot chain, so one thread walks
// them; the updates are unfused multiply and subtract, as the reference's libraries and the
// host-compiled oracle evaluate them. Inputs: the planes of k_solve_planes in list order (plane f
// at f * h); scratch: 11 h doubles at ilu; solution into xo[0..h) and yo[0..h).
__device__ void ilu0_solve_seq(const double* __restrict__ pl, int h, const int* __restrict__ list,
                               double* __restrict__ ilu, double* __restrict__ xo, double* __restrict__ yo) {
  const double* Dxx = pl + (size_t)kPD0 * h;
  const double* Dyy = pl + (size_t)kPD1 * h;
  const double* Dxy = pl + (size_t)kPD2 * h;
  const double* c0 = pl + (size_t)kPR0 * h;  // (x_i, x_{i+1})
  const double* c2 = pl + (size_t)kPR1 * h;  // (x_i, y_{i+1})
  const double* c3 = pl + (size_t)kPR2 * h;  // (y_i, x_{i+1})
  const double* c1 = pl + (size_t)kPR3 * h;  // (y_i, y_{i+1})
  const double* bx = pl + (size_t)kPB0 * h;
  const double* by = pl + (size_t)kPB1 * h;
  double* uxx = ilu;          // U (x_i, x_i)
  double* uxyp = uxx + h;     // U (x_i, y_{i-1})
  double* uxy = uxyp + h;     // U (x_i, y_i)
  double* lx = uxy + h;       // L (x_i, x_{i-1})
  double* l1 = lx + h;        // L (y_i, x_{i-1})
  double* l2 = l1 + h;        // L (y_i, x_i)
  double* l3 = l2 + h;        // L (y_i, x_{i+1})
  double* l4 = l3 + h;        // L (y_i, y_{i-1})
  double* uyy = l4 + h;       // U (y_i, y_i)
  double* uyn = uyy + h;      // U (y_i, y_{i+1})
  double* zx = uyn + h;       // L z = b, x half (the y half goes to yo first)
  auto fresh = [&](int i) { return i >= 0 && i + 1 < h && list[i + 1] == list[i] + 1; };
  auto sub = [](double a, double b, double c) { return __dsub_rn(a, __dmul_rn(b, c)); };
  // x rows: lower entry x_{i-1}; upper entries of row x_{i-1}: x_i, y_{i-2} (not in row x_i),
  // y_{i-1}, y_i
  for (int i = 0; i < h; i++) {
    double a_xx = Dxx[i], a_xyp = 0.0, a_xy = Dxy[i], l = 0.0;
    if (fresh(i - 1)) {
      a_xyp = c3[i - 1];
      l = __ddiv_rn(c0[i - 1], uxx[i - 1]);
      a_xx = sub(a_xx, l, c0[i - 1]);
      a_xyp = sub(a_xyp, l, uxy[i - 1]);
      a_xy = sub(a_xy, l, c2[i - 1]);
    }
    lx[i] = l;
    uxx[i] = a_xx;
    uxyp[i] = a_xyp;
    uxy[i] = a_xy;
  }
  // y rows: lower entries x_{i-1}, x_i, x_{i+1}, y_{i-1} in column order
  for (int i = 0; i < h; i++) {
    const bool fp = fresh(i - 1), fn = fresh(i);
    double a2 = Dxy[i], a3 = fn ? c3[i] : 0.0, a4 = fp ? c1[i - 1] : 0.0, ayy = Dyy[i], ayn = fn ? c1[i] : 0.0;
    double q1 = 0.0, q3 = 0.0, q4 = 0.0;
    if (fp) {  // row x_{i-1}: x_i, y_{i-1}, y_i
      q1 = __ddiv_rn(c2[i - 1], uxx[i - 1]);
      a2 = sub(a2, q1, c0[i - 1]);
      a4 = sub(a4, q1, uxy[i - 1]);
      ayy = sub(ayy, q1, c2[i - 1]);
    }
    const double q2 = __ddiv_rn(a2, uxx[i]);  // row x_i: x_{i+1}, y_{i-1}, y_i, y_{i+1}
    if (fn) a3 = sub(a3, q2, c0[i]);
    if (fp) a4 = sub(a4, q2, uxyp[i]);
    ayy = sub(ayy, q2, uxy[i]);
    if (fn) ayn = sub(ayn, q2, c2[i]);
    if (fn) {  // row x_{i+1}: y_i, y_{i+1}
      q3 = __ddiv_rn(a3, uxx[i + 1]);
      ayy = sub(ayy, q3, uxyp[i + 1]);
      ayn = sub(ayn, q3, uxy[i + 1]);
    }
    if (fp) {  // row y_{i-1}: y_i
      q4 = __ddiv_rn(a4, uyy[i - 1]);
      ayy = sub(ayy, q4, uyn[i - 1]);
    }
    l1[i] = q1; l2[i] = q2; l3[i] = q3; l4[i] = q4;
    uyy[i] = ayy;
    uyn[i] = ayn;
  }
  // L z = b (unit diagonal), entries in column order
  for (int i = 0; i < h; i++) zx[i] = fresh(i - 1) ? sub(bx[i], lx[i], zx[i - 1]) : bx[i];
  for (int i = 0; i < h; i++) {
    const bool fp = fresh(i - 1), fn = fresh(i);
    double acc = by[i];
    if (fp) acc = sub(acc, l1[i], zx[i - 1]);
    acc = sub(acc, l2[i], zx[i]);
    if (fn) acc = sub(acc, l3[i], zx[i + 1]);
    if (fp) acc = sub(acc, l4[i], yo[i - 1]);
    yo[i] = acc;
  }
  // U v = z, entries from the last column down
  for (int i = h - 1; i >= 0; i--) {
    double acc = yo[i];
    if (fresh(i)) acc = sub(acc, uyn[i], yo[i + 1]);
    yo[i] = __ddiv_rn(acc, uyy[i]);
  }
  for (int i = h - 1; i >= 0; i--) {
    const bool fp = fresh(i - 1), fn = fresh(i);
    double acc = zx[i];
    if (fn) acc = sub(acc, c2[i], yo[i + 1]);
    acc = sub(acc, uxy[i], yo[i]);
    if (fp) acc = sub(acc, uxyp[i], yo[i - 1]);
    if (fn) acc = sub(acc, c0[i], xo[i + 1]);
    xo[i] = __ddiv_rn(acc, uxx[i]);
  }
}

// The partitioned FP64 solve, the solver's filter and the median of flag R (one CTA per group).
__global__ void __launch_bounds__(kSolveThreads) k_solve_system(const GroupDesc* __restrict__ gds,
                                                                GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  if (!C.solve_now) return;
  const int t = threadIdx.x, nt = blockDim.x;
  const int h = C.n_used >> 1;
  __shared__ double sh_a[kSolveThreads], sh_b[kSolveThreads];

  // (4) FP64 solve into the compact step [x_0..x_h-1, y_0..y_h-1]: ILU(0) for solver id 0, else the
  // exact partitioned block-tridiagonal solve
  extern __shared__ double sh_red[];  // kSolveThreads x kPartSmemStride
  if (G.solver_id == 0) {
    if (t == 0 && h > 0) ilu0_solve_seq(G.cr, h, G.list, G.ilu, G.ndp, G.ndp + h);
    __syncthreads();
  } else {
    part_solve(G.cr, h, sh_red, G.ndp, 1, G.ndp + h, 1);
  }
  // (6) the solver's filter on the x half and the y half (eigensolver.cu:54-55)
  if (C.filter_active) {
    if (C.filter_kind == 1) {
      smear_scan(G.ndp, h, G.filter_strength, sh_a, sh_b);
      smear_scan(G.ndp + h, h, G.filter_strength, sh_a, sh_b);
    } else {
      if (t == 0) range_seq(G.ndp, h, G.filter_strength);
      if (t == 32) range_seq(G.ndp + h, h, G.filter_strength);
      __syncthreads();
    }
  }
  // (7) 3-tap median of each half (flag R), out of place, ends kept
  if (G.flags & kFlagMedianBefore) {
    double* tmp = G.cr;  // free after the solve
    for (int i = t; i < 2 * h; i += nt) tmp[i] = G.ndp[i];
    __syncthreads();
    for (int i = t; i < 2 * h; i += nt) {
      int base = i < h ? 0 : h, j = i - base;
      if (j == 0 || j == h - 1) continue;
      double a = tmp[i], b = tmp[i - 1], c = tmp[i + 1];
      int k = 1 * ((b >= a && b < c) || (b <= a && b > c)) + 2 * ((c >= a && c < b) || (c >= b && c < a));
      G.ndp[i] = k == 0 ? a : (k == 1 ? b : c);
    }
    __syncthreads();
  }
}

// Expansion of the step with the red/green fixed knots (kSolveSplit CTAs per group).
__global__ void __launch_bounds__(kSolvePrepThreads) k_solve_expand(const GroupDesc* __restrict__ gds,
                                                                    const GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.y];
  const GroupCtl& C = ctl[blockIdx.y];
  if (!C.solve_now) return;
  const int N = G.N, h = C.n_used >> 1, shift = C.shift;
  const int half = G.group_size >> 1;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < 2 * N; idx += gridDim.x * blockDim.x) {
    int j = idx >= N ? idx - N : idx;
    bool fixed = (((idx + 1) - shift * half) % G.group_size) == 0;
    if (fixed) continue;
    G.delta_p[idx] = G.params_used[j] ? G.ndp[(idx >= N ? h : 0) + G.list[N + j]] : 0.0;
  }
}

// After the line search of a half-step (task_linesearch.cu:158-169, mainiteration.cpp:266-284), a
// CTA per group: thread 0 runs the control; with flag t the CTA then copies the chain into the
// half-step's rgParams slot (timedmainiteration.cpp:124).
constexpr int kAfterLsThreads = 128;
__global__ void __launch_bounds__(kAfterLsThreads) k_after_ls(const GroupDesc* __restrict__ gds,
                                                              GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  __shared__ int sh_slot;
  if (threadIdx.x == 0) {
    sh_slot = -1;
    if (C.phase == kPhHalf && C.ls_state == 1 && C.ls_pending == 0) {
      C.ls_state = 0;
      double e0 = 0, e1 = 0;
      for (int i = 0; i < G.nF; i++) {
        e0 += G.errval[i];
        e1 += G.errval[i + G.nF];
      }
      bool imp = C.shift ? (e0 > e1) : (e0 < e1);
      C.improved = C.improved && imp;
      // TimedMainIteration runs its retry as iteration + 1 (timedmainiteration.cpp:141); slots past
      // its 2 max_iter are not written (the reference's buffer has 2 max_iter slots)
      const int slot = C.shift + 2 * (C.iteration - 1 + C.retry);
      if ((G.flags & kFlagTimeSub) && G.o_rg_params && slot < 2 * G.max_iter) sh_slot = slot;
      if (C.shift == 0) {
        C.shift = 1;
      } else {
        C.shift = 0;
        if (!C.improved && C.n_filter_iter != 0) {  // retry this iteration without the filter
          C.filter_active = 0;
          C.n_filter_iter = 0;
          C.improved = 1;
          C.retry = 1;
          // TimedMainIteration zeroes filterID here (timedmainiteration.cpp:136); MainIteration
          // does not (mainiteration.cpp:96-106)
          if (G.flags & kFlagTimeSub) C.filter_id = 0;
        } else {
          C.exec_result = C.improved;
          C.phase = kPhIterEnd;
          C.retry = 0;
          C.par_sel ^= G.dparity != nullptr;  // the correlation pass's parity bitmap is the current one
        }
      }
    }
  }
  __syncthreads();
  const int slot = sh_slot;
  if (slot < 0) return;
  const int P = 2 * G.N;
  double* dst = G.o_rg_params + (size_t)slot * P;
  for (int i = threadIdx.x; i < P; i += blockDim.x) dst[i] = G.p[i];
}

__device__ inline double pearson(double n, double sd, double si, double sdd, double sii, double sdi) {
  double ma = sd / n, mb = si / n;
  double a = sdd - 2 * ma * sd + n * ma * ma;
  double b = sii - 2 * mb * si + n * mb * mb;
  double q = sdi - mb * sd - ma * si + n * ma * mb;
  return q / sqrt(a * b);
}

// Partial sums of the global correlation (task_correlation.cu:62-99) over the per-column sums, for
// groups in kPhIterEnd: kIterSplit CTAs per group, each writing its 7 sums and valid count to
// G.cr[8 * blockIdx.x ...] (the solve's plane memory, free between the solve and the next one).
constexpr int kIterSplit = 32;
__global__ void __launch_bounds__(256) k_iter_sums(const GroupDesc* __restrict__ gds,
                                                   const GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.y];
  if (ctl[blockIdx.y].phase != kPhIterEnd) return;
  const int t = threadIdx.x;
  __shared__ double sh[8][8];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int c = blockIdx.x * blockDim.x + t; c < G.fW; c += gridDim.x * blockDim.x) {
    const double* s = G.colsum + (size_t)c * kCsStride;
    v[0] += s[kCsSumD]; v[1] += s[kCsSetN]; v[2] += s[kCsSetD]; v[3] += s[kCsSetDD];
    v[4] += s[kCsSetI]; v[5] += s[kCsSetII]; v[6] += s[kCsSetDI];
    v[7] += (double)G.colcnt[c];
  }
  for (int k = 0; k < 8; k++) v[k] = warp_sum(v[k]);
  if ((t & 31) == 0)
    for (int k = 0; k < 8; k++) sh[k][t >> 5] = v[k];
  __syncthreads();
  if (t < 8) {
    double a = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) a += sh[t][w];
    G.cr[8 * blockIdx.x + t] = a;
  }
}

// End of an iteration (task.cpp:281-373) for groups in kPhIterEnd, after k_eval<kCorr> and
// k_iter_sums.
__global__ void __launch_bounds__(kSolveThreads) k_iter_end(const GroupDesc* __restrict__ gds, GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  if (C.phase != kPhIterEnd) return;
  const int t = threadIdx.x, nt = blockDim.x, W = G.W, N = G.N, nF = G.nF;
  __shared__ int sh_action;
  // global correlation from the partial sums, combined in a fixed order
  if (t == 0) {
    double a[7] = {0, 0, 0, 0, 0, 0, 0};
    double nd = 0;
    for (int b = 0; b < kIterSplit; b++) {
      for (int k = 0; k < 7; k++) a[k] += G.cr[8 * b + k];
      nd += G.cr[8 * b + 7];
    }
    const long long nn = (long long)nd;
    double A = *G.sum_image / (double)nn, B = a[0] / (double)nn;
    double S = a[1];
    double assq = a[3] - 2 * A * a[2] + S * A * A;
    double bssq = a[5] - 2 * B * a[4] + S * B * B;
    double q = a[6] - B * a[2] - A * a[4] + S * A * B;
    C.corr = q / sqrt(assq * bssq);
  }
  __syncthreads();
  const int it = C.iteration;
  const double corr = C.corr;
  if (t == 0) C.passes[kCorr] += nF;
  if (G.o_all_params && it <= G.max_iter)
    for (int i = t; i < 2 * N; i += nt) G.o_all_params[(size_t)(it - 1) * 2 * N + i] = G.p[i];
  if (t == 0 && (G.flags & kFlagIterCorr) && G.o_iter_corr && it <= G.max_iter) G.o_iter_corr[it - 1] = corr;
  if (G.flags & kFlagFrameCorr) {  // task.cpp:287-306, a warp per frame
    const int lane = t & 31;
    for (int f = t >> 5; f < nF; f += nt >> 5) {
      double s5[5] = {0, 0, 0, 0, 0};
      double nf = 0;
      for (int cc = lane; cc < W; cc += 32) {
        const double* s = G.colsum + (size_t)(f * W + cc) * kCsStride;
        for (int k = 0; k < 5; k++) s5[k] += s[kCsFrD + k];
        nf += G.colcnt[f * W + cc];
      }
      for (int k = 0; k < 5; k++) s5[k] = warp_sum(s5[k]);
      nf = warp_sum(nf);
      if (lane == 0) {
        const double r = pearson(nf, s5[0], s5[1], s5[2], s5[3], s5[4]);
        G.o_frame_corr[f] = r;  // mem->corr
        if (G.o_frame_corr_hist && it <= G.max_iter) G.o_frame_corr_hist[(size_t)(it - 1) * nF + f] = r;
      }
    }
  }
  __syncthreads();
  if (t == 0) {
    int action;  // 0 next iteration, 1 next iteration without pLast update, 2 stop
    double d = corr - C.correlation;
    if (d < G.corr_inc_thr) {
      C.stop_reason = kStopCorrInc;
      action = 2;
    } else if (d < G.filter_corr_thr && C.filter_id != 0) {
      C.filter_active = 0;
      C.n_filter_iter = 0;
      C.filter_id = 0;
      action = 1;
    } else if (!C.exec_result) {
      C.stop_reason = kStopMovement;
      action = 2;
    } else if (G.max_iter == it) {
      C.stop_reason = kStopIterLimit;
      action = 2;
    } else if (C.correlation >= G.halt_corr) {
      C.stop_reason = kStopHaltCorr;
      action = 2;
    } else {
      C.correlation = corr;
      action = 0;
    }
    sh_action = action;
    // iteration times (flags T and t): not saved for an iteration that ends in the filter's
    // switch-off (task.cpp:323 continues before :358-360); every iteration restarts the clock
    if (G.o_iter_times) {
      const unsigned long long now = device_clock_ns();
      if (action != 1 && it <= G.max_iter) G.o_iter_times[it - 1] = (double)(now - C.t_mark) * 1e-9;
      C.t_mark = now;
    }
  }
  __syncthreads();
  const int action = sh_action;
  if (action == 0) {
    for (int i = t; i < 2 * N; i += nt) G.p_last[i] = G.p[i];
    if (G.flags & kFlagMaskInactive) {  // task_maskinactive.cu:3-25 (reads mem->corr)
      for (int i = t; i < 2 * G.n_rg; i += nt) G.grp_active[i] = 0;
      __syncthreads();
      const int hg = G.group_size >> 1;
      for (int idx = t; idx < G.fW; idx += nt) {
        int f = idx / W;
        if (G.o_frame_corr[f] < G.halt_corr) {
          int a = idx / G.group_size;
          if (a < 2 * G.n_rg) G.grp_active[a] = 1;
          if (idx < hg || idx >= G.fW - hg) continue;
          int b = (idx - hg) / G.group_size + G.n_rg;
          if (b < 2 * G.n_rg) G.grp_active[b] = 1;
        }
      }
    }
    if ((G.flags & kFlagIterErrvals) && G.o_iter_errvals && it <= G.max_iter)
      for (int i = t; i < nF; i += nt) {  // (2 max_iter) x nF column-major (task.cpp:362-372)
        G.o_iter_errvals[(size_t)(2 * (it - 1)) + (size_t)i * 2 * G.max_iter] = G.errval[i];
        G.o_iter_errvals[(size_t)(2 * (it - 1) + 1) + (size_t)i * 2 * G.max_iter] = G.errval[nF + i];
      }
  }
  __syncthreads();
  if (action == 2) {
    if (it == 1)
      for (int i = t; i < 2 * N; i += nt) G.p_last[i] = G.p[i];
    // the final hd_calculateGroupErrvals(mem, 0) recomputes the difference image of active frames
    const int W2 = 2 * (W + 1);
    for (int i = t; i < nF * W2; i += nt) {
      const int f = i / W2;
      if (frame_active(G, f, 0)) G.kdiff[i] = G.kmask[i];
    }
    __syncthreads();
    if (t == 0) C.phase = kPhFinal;
  } else if (t == 0) {
    C.iteration = it + 1;
    C.shift = 0;
    C.improved = 1;
    C.phase = kPhHalf;
  }
}

// Outputs of a finished group (task.cpp:381-411, :202-219), after k_eval<kFinal>.
__global__ void __launch_bounds__(kSolveThreads) k_final(const GroupDesc* __restrict__ gds, GroupCtl* __restrict__ ctl,
                                               int* __restrict__ n_done) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  if (C.phase != kPhFinal) return;
  const int t = threadIdx.x, nt = blockDim.x, W = G.W, N = G.N, nF = G.nF;
  __shared__ int sh_nact;
  if (t == 0) sh_nact = 0;
  __syncthreads();
  const int lane = t & 31;
  for (int f = t >> 5; f < nF; f += nt >> 5) {  // a warp per frame
    double s5[5] = {0, 0, 0, 0, 0}, ssd = 0;
    double nf = 0;
    for (int cc = lane; cc < W; cc += 32) {
      const double* s = G.colsum + (size_t)(f * W + cc) * kCsStride;
      for (int k = 0; k < 5; k++) s5[k] += s[kCsFrD + k];
      ssd += s[kCsFinalSsd];
      nf += G.colcnt[f * W + cc];
    }
    for (int k = 0; k < 5; k++) s5[k] = warp_sum(s5[k]);
    ssd = warp_sum(ssd);
    nf = warp_sum(nf);
    const double* ks = G.p + (size_t)f * W;
    const double rg = G.lambda != 0.0 ? frame_reg_warp(ks, W, N, ks[W], ks[N + W]) : 0.0;
    if (lane == 0) {
      if (frame_active(G, f, 0)) {
        double val = ssd / nf;
        if (G.lambda != 0.0) val = (ssd + G.lambda * rg) / nf;
        G.errval[f] = val;
        atomicAdd(&sh_nact, 1);
      }
      // with flag c the last iteration's frame correlations stand (task.cpp:392-395)
      if (!(G.flags & kFlagFrameCorr)) G.o_frame_corr[f] = pearson(nf, s5[0], s5[1], s5[2], s5[3], s5[4]);
      G.o_residrms[f] = sqrt(G.errval[f]);
    }
  }
  // ParameterOrganizer::organize1D2 (parameterorganizer.cpp:57-98): the last knot of each frame
  // repeats knot W-1
  for (int i = t; i < (W + 1) * nF; i += nt) {
    int f = i / (W + 1), k = i - f * (W + 1);
    int src = f * W + (k < W ? k : W - 1);
    if (G.o_dx) G.o_dx[i] = G.p_last[src];
    if (G.o_dy) G.o_dy[i] = G.p_last[N + src];
    if (G.o_frame_params) {  // nF x 2(W+1), column-major
      G.o_frame_params[(size_t)k * nF + f] = G.p_last[src];
      G.o_frame_params[(size_t)(k + W + 1) * nF + f] = G.p_last[N + src];
    }
  }
  if (G.o_raw)
    for (int i = t; i < 2 * N; i += nt) G.o_raw[i] = G.p_last[i];
  // blocksused of the caller (steady_scan.m:264-265): a block column with a valid pixel in the
  // final mask, whose per-column count the final pass left in colcnt
  if (G.o_blocks_used)
    for (int c = t; c < G.fW; c += nt) G.o_blocks_used[c] = G.colcnt[c] > 0 ? 1 : 0;
  __syncthreads();
  if (t == 0) {
    C.n_eval += sh_nact;
    C.passes[kFinal] += nF;
    C.phase = kPhDone;
    atomicAdd(n_done, 1);
  }
}

}  // namespace ss
