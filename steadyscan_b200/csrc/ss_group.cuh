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

// Standalone solve of a block-tridiagonal system given as diag (n x 3: xx yy xy), coupling
// ((n-1) x 4: [[c0 c2] [c3 c1]] between block i and i+1) and rhs (n x 2) into x (n x 2), with
// the caller's workspace cr (n x kCrStride doubles). One CTA.
__global__ void __launch_bounds__(kSolveThreads) k_block_tridiag(int n, const double* __restrict__ diag,
                                                                 const double* __restrict__ coupling,
                                                                 const double* __restrict__ rhs,
                                                                 double* __restrict__ x, double* __restrict__ cr) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double* q = cr + (size_t)i * kCrStride;
    q[0] = diag[3 * i]; q[1] = diag[3 * i + 1]; q[2] = diag[3 * i + 2];
    if (i > 0) {  // L_i = R_{i-1}^T
      const double* c = coupling + 4 * (size_t)(i - 1);
      q[3] = c[0]; q[4] = c[3]; q[5] = c[2]; q[6] = c[1];
    } else {
      q[3] = q[4] = q[5] = q[6] = 0.0;
    }
    if (i + 1 < n) {
      const double* c = coupling + 4 * (size_t)i;
      q[7] = c[0]; q[8] = c[2]; q[9] = c[3]; q[10] = c[1];
    } else {
      q[7] = q[8] = q[9] = q[10] = 0.0;
    }
    q[11] = rhs[2 * i];
    q[12] = rhs[2 * i + 1];
  }
  __syncthreads();
  cr_solve(cr, n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    x[2 * i] = cr[(size_t)i * kCrStride + 11];
    x[2 * i + 1] = cr[(size_t)i * kCrStride + 12];
  }
}

// Knot-difference regulariser of frame f (extension; lambda = 0 reproduces the reference): sum of
// |k_{t+1}-k_t|^2 over its W edges, own knots from own (+N for y), right boundary (bx, by).
__device__ inline double frame_reg(const double* own, int W, int N, double bx, double by) {
  double r = 0;
  for (int t = 0; t < W; t++) {
    double x0 = own[t], y0 = own[t + N];
    double x1 = t + 1 < W ? own[t + 1] : bx, y1 = t + 1 < W ? own[t + 1 + N] : by;
    r += (x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0);
  }
  return r;
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
  sh_a[t] = a;
  sh_b[t] = y;
  __syncthreads();
  if (t == 0) {
    double carry = 0.0;
    for (int k = 0; k < nt; k++) {
      double nc = sh_a[k] * carry + sh_b[k];
      sh_b[k] = carry;  // carry-in of chunk k
      carry = nc;
    }
  }
  __syncthreads();
  y = sh_b[t];
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

// Half-step set-up and solve for every group in phase kPhHalf (one CTA per group):
//   blocksPresent / paramsUsed / errval (task_applyparameters.cuh:74-81, task_createparametermask.cuh,
//   task_calcerrval.cu:185), the filter switch-off (mainiteration.cpp:246-256), compaction
//   (task_generatesubsparseoffset.cu), the block-tridiagonal normal equations
//   (task_filldiagonals.cu:47-159, task_filljtr.cu:3-58) solved exactly in FP64, the solver's
//   filter (smearingfilter.cpp, rangefilter.cpp), the expansion with fixed knots
//   (task_expandresults.cu:9-36) and the line-search start.
__global__ void __launch_bounds__(kSolveThreads) k_solve(const GroupDesc* __restrict__ gds, GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  if (C.phase != kPhHalf) return;
  const int t = threadIdx.x, nt = blockDim.x;
  const int W = G.W, N = G.N, nF = G.nF, fW = G.fW, shift = C.shift;
  __shared__ double sh_a[kSolveThreads], sh_b[kSolveThreads];
  __shared__ int sh_i[kSolveThreads];
  __shared__ int sh_h, sh_nact;

  __shared__ int sh_rebuild;
  if (t == 0) {
    if (C.n_filter_iter != 0 && C.iteration > C.n_filter_iter) {
      C.filter_active = 0;
      C.filter_id = 0;
      C.n_filter_iter = 0;
    }
    sh_nact = 0;
  }
  // (1) block presence for all columns; parameter use and errval for active frames
  for (int c = t; c < fW; c += nt) G.blocks_present[c] = G.colcnt[c] >= G.min_points[c % W];
  if (t == 0) G.blocks_present[N - 1] = 0;
  __syncthreads();
  for (int c = t; c < fW; c += nt) {
    int f = c / W;
    if (!frame_active(G, f, shift)) continue;
    G.params_used[c] = (c == 0) ? G.blocks_present[0] : (G.blocks_present[c] | G.blocks_present[c - 1]);
  }
  for (int f = t; f < nF; f += nt) {
    bool act = frame_active(G, f, shift);
    const double* ks = G.p + (size_t)f * W;
    double* km = G.kmask + (size_t)f * 2 * (W + 1);
    double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
    for (int k = 0; k <= W; k++) {
      km[k] = ks[k];
      km[W + 1 + k] = ks[N + k];
      if (act) {
        kd[k] = ks[k];
        kd[W + 1 + k] = ks[N + k];
      }
    }
    G.fstate[f] = act ? 2 : 0;  // searching once the step is known
    G.ls_trials[f] = 0;
    if (!act) continue;
    double e = 0;
    long long n = 0;
    for (int cc = 0; cc < W; cc++) {
      e += G.colsum[(size_t)(f * W + cc) * kCsStride + kCsSsd];
      n += G.colcnt[f * W + cc];
    }
    double val = e / (double)n;
    if (G.lambda != 0.0) val = (e + G.lambda * frame_reg(ks, W, N, ks[W], ks[N + W])) / (double)n;
    G.errval[shift * nF + f] = val;
    atomicAdd(&sh_nact, 1);
  }
  for (int i = t; i < 2 * N; i += nt) G.p_snap[i] = G.p[i];
  __syncthreads();
  if (t == 0) {
    C.n_eval += sh_nact;
    C.passes[kAssemble] += nF;
    atomicAdd(G.searching, sh_nact);  // frames whose line search starts (trial rounds)
  }

  // (2) compaction: list position of every used knot (paramsUsed[N-1] is never written, so it
  // keeps its zero fill: task_allocate.cu:223)
  {
    const int chunk = (N + nt - 1) / nt;
    const int lo = min(N, t * chunk), hi = min(N, lo + chunk);
    int cnt = 0;
    for (int k = lo; k < hi; k++) cnt += G.params_used[k] ? 1 : 0;
    sh_i[t] = cnt;
    __syncthreads();
    if (t == 0) {
      int run = 0;
      for (int k = 0; k < nt; k++) {
        int v = sh_i[k];
        sh_i[k] = run;
        run += v;
      }
      sh_h = run;
    }
    __syncthreads();
    int pos = sh_i[t];
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

  // (3) blocks of the compact system; coupling to the next list position
  const double lam = G.lambda;
  for (int i = t; i < h; i += nt) {
    int k = G.list[i];
    const double* a = G.colsum + (size_t)k * kCsStride;
    double* n = G.cr + (size_t)i * kCrStride;
    double d0 = 0, d1 = 0, d2 = 0, r0 = 0, r1 = 0;
    if (k < fW) {
      d0 += a[kCsAxx]; d1 += a[kCsAyy]; d2 += a[kCsAxy];
      r0 += a[kCsJ1x]; r1 += a[kCsJ1y];
    }
    if (k > 0) {
      const double* b = G.colsum + (size_t)(k - 1) * kCsStride;
      d0 += b[kCsBxx]; d1 += b[kCsByy]; d2 += b[kCsBxy];
      r0 += b[kCsJ2x]; r1 += b[kCsJ2y];
    }
    M2 R = {0, 0, 0, 0};
    bool fresh = (i + 1 < h) && (G.list[i + 1] == k + 1);
    if (fresh) {
      R = {a[kCsOxx], a[kCsOxy], a[kCsOxy], a[kCsOyy]};
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
      int deg = (k > 0) + (k < N - 1);
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
    n[0] = d0; n[1] = d1; n[2] = d2;
    n[7] = R.a; n[8] = R.b; n[9] = R.c; n[10] = R.d;
    n[11] = r0; n[12] = r1;
  }
  __syncthreads();
  for (int i = t; i < h; i += nt) {
    double* n = G.cr + (size_t)i * kCrStride;
    if (i > 0) {
      const double* pr = G.cr + (size_t)(i - 1) * kCrStride;
      n[3] = pr[7]; n[4] = pr[9]; n[5] = pr[8]; n[6] = pr[10];  // L_i = R_{i-1}^T
    } else {
      n[3] = n[4] = n[5] = n[6] = 0;
    }
  }
  __syncthreads();

  // (4) FP64 block cyclic reduction
  cr_solve(G.cr, h);
  // (5) compact step [x_0..x_h-1, y_0..y_h-1]
  for (int i = t; i < h; i += nt) {
    G.ndp[i] = G.cr[(size_t)i * kCrStride + 11];
    G.ndp[h + i] = G.cr[(size_t)i * kCrStride + 12];
  }
  __syncthreads();
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
  // (8) expansion with the red/green fixed knots
  const int half = G.group_size >> 1;
  for (int idx = t; idx < 2 * N; idx += nt) {
    int j = idx >= N ? idx - N : idx;
    bool fixed = (((idx + 1) - shift * half) % G.group_size) == 0;
    if (fixed) continue;
    G.delta_p[idx] = G.params_used[j] ? G.ndp[(idx >= N ? h : 0) + G.list[N + j]] : 0.0;
  }
}

// After the line search of a half-step (task_linesearch.cu:158-169, mainiteration.cpp:266-284).
__global__ void k_after_ls(const GroupDesc* __restrict__ gds, GroupCtl* __restrict__ ctl, int n_groups) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_groups) return;
  const GroupDesc& G = gds[g];
  GroupCtl& C = ctl[g];
  if (C.phase != kPhHalf) return;
  double e0 = 0, e1 = 0;
  for (int i = 0; i < G.nF; i++) {
    e0 += G.errval[i];
    e1 += G.errval[i + G.nF];
  }
  bool imp = C.shift ? (e0 > e1) : (e0 < e1);
  C.improved = C.improved && imp;
  if (C.shift == 0) {
    C.shift = 1;
    return;
  }
  C.shift = 0;
  if (!C.improved && C.n_filter_iter != 0) {  // retry this iteration without the filter
    C.filter_active = 0;
    C.n_filter_iter = 0;
    C.improved = 1;
    return;
  }
  C.exec_result = C.improved;
  C.phase = kPhIterEnd;
}

__device__ inline double pearson(double n, double sd, double si, double sdd, double sii, double sdi) {
  double ma = sd / n, mb = si / n;
  double a = sdd - 2 * ma * sd + n * ma * ma;
  double b = sii - 2 * mb * si + n * mb * mb;
  double q = sdi - mb * sd - ma * si + n * ma * mb;
  return q / sqrt(a * b);
}

// End of an iteration (task.cpp:281-373) for groups in kPhIterEnd, after k_eval<kCorr>.
__global__ void __launch_bounds__(kSolveThreads) k_iter_end(const GroupDesc* __restrict__ gds, GroupCtl* __restrict__ ctl) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  if (C.phase != kPhIterEnd) return;
  const int t = threadIdx.x, nt = blockDim.x, W = G.W, N = G.N, nF = G.nF;
  __shared__ double sh[8][kSolveThreads / 32];
  __shared__ long long sh_n[kSolveThreads / 32];
  __shared__ int sh_action;
  // global correlation (task_correlation.cu:62-99) from the per-column sums
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  long long n = 0;
  for (int c = t; c < G.fW; c += nt) {
    const double* s = G.colsum + (size_t)c * kCsStride;
    v[0] += s[kCsSumD]; v[1] += s[kCsSetN]; v[2] += s[kCsSetD]; v[3] += s[kCsSetDD];
    v[4] += s[kCsSetI]; v[5] += s[kCsSetII]; v[6] += s[kCsSetDI];
    n += G.colcnt[c];
  }
  for (int k = 0; k < 7; k++) v[k] = warp_sum(v[k]);
  n = (long long)warp_sum((int)n);
  if ((t & 31) == 0) {
    for (int k = 0; k < 7; k++) sh[k][t >> 5] = v[k];
    sh_n[t >> 5] = n;
  }
  __syncthreads();
  if (t == 0) {
    double a[7] = {0, 0, 0, 0, 0, 0, 0};
    long long nn = 0;
    for (int w = 0; w < nt / 32; w++) {
      for (int k = 0; k < 7; k++) a[k] += sh[k][w];
      nn += sh_n[w];
    }
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
  if (G.flags & kFlagFrameCorr) {  // task.cpp:287-306
    for (int f = t; f < nF; f += nt) {
      double s5[5] = {0, 0, 0, 0, 0};
      double nf = 0;
      for (int cc = 0; cc < W; cc++) {
        const double* s = G.colsum + (size_t)(f * W + cc) * kCsStride;
        for (int k = 0; k < 5; k++) s5[k] += s[kCsFrD + k];
        nf += G.colcnt[f * W + cc];
      }
      double r = pearson(nf, s5[0], s5[1], s5[2], s5[3], s5[4]);
      G.o_frame_corr[f] = r;  // mem->corr
      if (G.o_frame_corr_hist && it <= G.max_iter) G.o_frame_corr_hist[(size_t)(it - 1) * nF + f] = r;
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
    for (int f = t; f < nF; f += nt) {
      if (!frame_active(G, f, 0)) continue;
      double* km = G.kmask + (size_t)f * 2 * (W + 1);
      double* kd = G.kdiff + (size_t)f * 2 * (W + 1);
      for (int k = 0; k < 2 * (W + 1); k++) kd[k] = km[k];
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
__global__ void __launch_bounds__(256) k_final(const GroupDesc* __restrict__ gds, GroupCtl* __restrict__ ctl,
                                               int* __restrict__ n_done) {
  const GroupDesc& G = gds[blockIdx.x];
  GroupCtl& C = ctl[blockIdx.x];
  if (C.phase != kPhFinal) return;
  const int t = threadIdx.x, nt = blockDim.x, W = G.W, N = G.N, nF = G.nF;
  __shared__ int sh_nact;
  if (t == 0) sh_nact = 0;
  __syncthreads();
  for (int f = t; f < nF; f += nt) {
    double s5[5] = {0, 0, 0, 0, 0}, ssd = 0;
    double nf = 0;
    for (int cc = 0; cc < W; cc++) {
      const double* s = G.colsum + (size_t)(f * W + cc) * kCsStride;
      for (int k = 0; k < 5; k++) s5[k] += s[kCsFrD + k];
      ssd += s[kCsFinalSsd];
      nf += G.colcnt[f * W + cc];
    }
    if (frame_active(G, f, 0)) {
      double val = ssd / nf;
      if (G.lambda != 0.0) {
        const double* ks = G.p + (size_t)f * W;
        val = (ssd + G.lambda * frame_reg(ks, W, N, ks[W], ks[N + W])) / nf;
      }
      G.errval[f] = val;
      atomicAdd(&sh_nact, 1);
    }
    G.o_frame_corr[f] = pearson(nf, s5[0], s5[1], s5[2], s5[3], s5[4]);
    G.o_residrms[f] = sqrt(G.errval[f]);
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
  __syncthreads();
  if (t == 0) {
    C.n_eval += sh_nact;
    C.passes[kFinal] += nF;
    C.phase = kPhDone;
    atomicAdd(n_done, 1);
  }
}

}  // namespace ss
