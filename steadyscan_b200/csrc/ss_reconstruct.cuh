// Reconstruction of motion-corrected frames on the GPU: invert_bilinear_sampling of the
// reference's MATLAB driver (steady_scan.m:290-404), for the frames of one set at a time.
//
// Per frame (a template of th x tw pixels, np = th tw, column-major; data pixels of the cropped
// frame at template coordinates x, y of the frame's knots, steady_scan.m:452-453):
//  * constraints (bilinear_map_linear_constraints, :438-499): every data pixel strictly inside the
//    template adds w_c d to wy and w_c w_c' to ww at its four corners (FP64; MATLAB's sparse sums).
//    ww is kept as a forward stencil: per pixel p its diagonal and its entries with p + 1 (S),
//    p + th - 1 (NE), p + th (E), p + th + 1 (SE); the pair (p, q) of a data pixel's corners is
//    always one of these (a pair across a column boundary needs a corner outside the template);
//  * first guess (resample_frame / pushgrid, :562-599): FP32 push-grid z / n. The reference's
//    z(i) = z(i) + v statements do not accumulate repeated indices: for each statement the data
//    pixel with the largest column-major index among those naming a pixel stands (a pass that
//    records it, then a pass in which it alone adds), and the eight statements keep their order;
//  * system (:319-341, calc_interactions :501-523): mask = column sum of ww > 0 and a finite guess;
//    Q = ww + regfac GtG (GtG the adjacent-difference Laplacian, vertical pairs weighted vfac^2,
//    imageadjdiffquadmat :406-436) with the rows and columns of unmasked pixels zeroed; in FP32
//    R = Q(p,p), the neighbour terms Q(p,q) / R for the eight neighbours N NE E SE S SW W NW within
//    the reference's finders' bounds (calc_indices :645-723; the SE finder's strict "< np" drops
//    one real neighbour, reproduced), L = wy(p) / R (0 where not finite);
//  * iteration (:364-389): sweeps over the colours A B C D of the 2 x 2 pattern [A B; C D],
//    x(p) = L(p) - sum_j x(q_j) Rmat_j(p) in FP32 with the eight terms summed in order; every
//    n-th sweep the energy x'Qx - 2 Le x (FP64 quadratic form of the FP32 iterate, FP32 linear
//    term, compared in FP32) stops the frame when it did not decrease, the output being the
//    iterate of the last check that decreased it (zeros if none did); n is the interval the
//    previous frame's sweep count gave (:391).
// Frames run in parallel: the sweeps do not depend on n, and the host re-runs a frame whose
// interval, recomputed from its predecessor's sweep count, differs from the one it ran with.
#pragma once

#include "ss_common.cuh"

namespace ss {

constexpr int kRcStencil = 5;  // diagonal, S, NE, E, SE
constexpr int kRcParts = 64;   // partial-sum CTAs per frame of the energy

// Per-frame buffers of a chunk of frames (device pointers; [frame * np + p] unless noted).
struct RcBufs {
  int th, tw, np, hd, wd, nk;  // template size, data frame size, knots per frame
  double* wy;       // np
  double* ww;       // np x kRcStencil, pixel-major
  float* z;         // np: push-grid sums, then the first guess
  float* cnt;       // np: push-grid weights
  int* last_z;      // np
  int* last_n;      // np
  uint8_t* mask;    // np
  float* coef;      // np x 10: R, Rmat[8], L
  float* le;        // np: single(Lfull) of masked pixels, else 0
  float* x;         // np
  float* xo;        // np
  double* part;     // frames x kRcParts x 2: energy partial sums (FP64 quadratic, FP32-valued linear)
  float* part_l;    // frames x kRcParts
};

// Template coordinates of data pixel q (column-major in hd x wd) of frame f (steady_scan.m:452-453).
__device__ __forceinline__ void rc_coords(const double* __restrict__ bx, const double* __restrict__ by,
                                          const double* __restrict__ tf, const int* __restrict__ pk,
                                          const double* __restrict__ dxk, const double* __restrict__ dyk, int q,
                                          double& x, double& y) {
  const int k = pk[q] - 1;
  const double f = tf[q], c = 1.0 - f;
  x = bx[q] + dxk[k] * c + dxk[k + 1] * f;
  y = by[q] + dyk[k] * c + dyk[k + 1] * f;
}

template <class DataT>
__global__ void __launch_bounds__(256) k_rc_constraints(RcBufs b, const void* __restrict__ data, int f0, int nf,
                                                        const double* __restrict__ bx, const double* __restrict__ by,
                                                        const double* __restrict__ tf, const int* __restrict__ pk,
                                                        const double* __restrict__ dxk, const double* __restrict__ dyk) {
  const size_t per = (size_t)b.hd * b.wd, total = per * nf;
  const double eps = 2.220446049250313e-16;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(e / per), q = (int)(e - (size_t)f * per);
    double x, y;
    rc_coords(bx, by, tf, pk, dxk + (size_t)(f0 + f) * b.nk, dyk + (size_t)(f0 + f) * b.nk, q, x, y);
    if (!(x > 1 + eps && x < b.tw - eps && y > 1 + eps && y < b.th - eps)) continue;
    const double xi = floor(x), yi = floor(y), xf = x - xi, yf = y - yi;
    const int p0 = (int)yi - 1 + b.th * ((int)xi - 1);  // corner (y, x), 0-based
    const double d = to_double(reinterpret_cast<const DataT*>(data)[(size_t)(f0 + f) * per + q]);
    const double xc = 1 - xf, yc = 1 - yf;
    const double w[4] = {xc * yc, xc * yf, xf * yc, xf * yf};  // (y,x) (y+1,x) (y,x+1) (y+1,x+1)
    const int pc[4] = {p0, p0 + 1, p0 + b.th, p0 + b.th + 1};
    double* wy = b.wy + (size_t)f * b.np;
    double* ww = b.ww + (size_t)f * b.np * kRcStencil;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      atomicAdd(wy + pc[c], w[c] * d);
      atomicAdd(ww + (size_t)pc[c] * kRcStencil + 0, w[c] * w[c]);
    }
    atomicAdd(ww + (size_t)pc[0] * kRcStencil + 1, w[0] * w[1]);  // (y,x)-(y+1,x): S
    atomicAdd(ww + (size_t)pc[2] * kRcStencil + 1, w[2] * w[3]);  // (y,x+1)-(y+1,x+1): S
    atomicAdd(ww + (size_t)pc[0] * kRcStencil + 3, w[0] * w[2]);  // E
    atomicAdd(ww + (size_t)pc[1] * kRcStencil + 3, w[1] * w[3]);  // E
    atomicAdd(ww + (size_t)pc[0] * kRcStencil + 4, w[0] * w[3]);  // SE
    atomicAdd(ww + (size_t)pc[1] * kRcStencil + 2, w[1] * w[2]);  // (y+1,x)-(y,x+1): NE
  }
}

// One push-grid statement pair (step s of 4): z at corner offset oz, n at corner offset on; phase 0
// records the last data pixel naming each pixel, phase 1 lets it add.
template <class DataT>
__global__ void __launch_bounds__(256) k_rc_pushgrid(RcBufs b, const void* __restrict__ data, int f0, int nf, int s,
                                                     int phase, const double* __restrict__ bx,
                                                     const double* __restrict__ by, const double* __restrict__ tf,
                                                     const int* __restrict__ pk, const double* __restrict__ dxk,
                                                     const double* __restrict__ dyk) {
  const size_t per = (size_t)b.hd * b.wd, total = per * nf;
  // statement orders (steady_scan.m:589-598): z at (y,x) (y+1,x) (y,x+1) (y+1,x+1); n at
  // (y+1,x) (y,x+1) (y,x) (y+1,x+1); corner c: offset {0, 1, th, th+1}[c]
  const int cz = s, cn = (s == 0) ? 1 : (s == 1) ? 2 : (s == 2) ? 0 : 3;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(e / per), q = (int)(e - (size_t)f * per);
    double x, y;
    rc_coords(bx, by, tf, pk, dxk + (size_t)(f0 + f) * b.nk, dyk + (size_t)(f0 + f) * b.nk, q, x, y);
    if (!(x >= 1 && x < b.tw && y >= 1 && y < b.th)) continue;
    const double xi = floor(x), yi = floor(y), xf = x - xi, yf = y - yi;
    const int p0 = (int)yi - 1 + b.th * ((int)xi - 1);
    const int off[4] = {0, 1, b.th, b.th + 1};
    const double wc[4] = {(1 - xf) * (1 - yf), (1 - xf) * yf, xf * (1 - yf), xf * yf};
    const int tz = p0 + off[cz], tn = p0 + off[cn];
    int* lz = b.last_z + (size_t)f * b.np;
    int* ln = b.last_n + (size_t)f * b.np;
    if (phase == 0) {
      atomicMax(lz + tz, q);
      atomicMax(ln + tn, q);
    } else {
      const float d = (float)to_double(reinterpret_cast<const DataT*>(data)[(size_t)(f0 + f) * per + q]);
      if (lz[tz] == q) b.z[(size_t)f * b.np + tz] += (float)wc[cz] * d;
      if (ln[tn] == q) b.cnt[(size_t)f * b.np + tn] += (float)wc[cn];
    }
  }
}

__global__ void k_rc_fill_int(int* p, size_t n, int v) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) p[e] = v;
}

// ww entry of the pair (p, q), q - p one of the stencil offsets or their negatives (0 otherwise).
__device__ __forceinline__ double rc_ww(const double* __restrict__ ww, int th, int np, int p, int q) {
  const int lo = p < q ? p : q, d = p < q ? q - p : p - q;
  if (lo < 0 || lo + d >= np) return 0.0;
  int s = -1;
  if (d == 0) s = 0;
  else if (d == 1) s = 1;
  else if (d == th - 1) s = 2;
  else if (d == th) s = 3;
  else if (d == th + 1) s = 4;
  return s < 0 ? 0.0 : ww[(size_t)lo * kRcStencil + s];
}

// Mask (column sums of ww > 0 and a finite first guess) and the first iterate of every pixel.
__global__ void __launch_bounds__(256) k_rc_mask(RcBufs b, int nf) {
  const size_t total = (size_t)b.np * nf;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(e / b.np), p = (int)(e - (size_t)f * b.np);
    const double* ww = b.ww + (size_t)f * b.np * kRcStencil;
    const int th = b.th;
    const int nb[9] = {p, p - 1, p + 1, p - th + 1, p + th - 1, p - th, p + th, p - th - 1, p + th + 1};
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 9; j++) s += rc_ww(ww, th, b.np, p, nb[j]);
    const float iv = b.z[e] / b.cnt[e];
    b.mask[e] = (s > 0.0 && !isnan(iv)) ? 1 : 0;
    b.x[e] = isnan(iv) ? 0.0f : iv;
    b.xo[e] = 0.0f;
  }
}

// Q(p, q) of the masked system: ww + regfac GtG (vertical pairs vfac^2), rows and columns of
// unmasked pixels zero. Diagonal for q == p.
__device__ __forceinline__ double rc_q(const RcBufs& b, const double* ww, const uint8_t* mk, int p, int q, double regfac,
                                       double vf2) {
  if (!mk[p] || !mk[q]) return 0.0;
  const int th = b.th, r = p % th, c = p / th;
  double reg = 0.0;
  if (q == p) {
    const int nh = (c > 0) + (c < b.tw - 1), nv = (r > 0) + (r < th - 1);
    reg = regfac * ((double)nh + (double)nv * vf2);
  } else if ((q == p + 1 && r < th - 1) || (q == p - 1 && r > 0)) {
    reg = -regfac * vf2;
  } else if (q == p + th || q == p - th) {
    reg = -regfac;
  }
  return rc_ww(ww, th, b.np, p, q) + reg;
}

// FP32 coefficients of every pixel: R, the eight neighbour terms, L; and Le.
__global__ void __launch_bounds__(256) k_rc_coef(RcBufs b, int nf, double regfac, double vf2) {
  const size_t total = (size_t)b.np * nf;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(e / b.np), p = (int)(e - (size_t)f * b.np);
    const double* ww = b.ww + (size_t)f * b.np * kRcStencil;
    const uint8_t* mk = b.mask + (size_t)f * b.np;
    const int th = b.th, np = b.np, i = p + 1;  // 1-based, as the finders
    const float R = (float)rc_q(b, ww, mk, p, p, regfac, vf2);
    float* cf = b.coef + e * 10;
    cf[0] = R;
    // N NE E SE S SW W NW (steady_scan.m:677-723), 1-based candidates and their bounds
    const int cand[8] = {i - 1, i + th - 1, i + th, i + th + 1, i + 1, i - th + 1, i - th, i - th - 1};
    const bool ok[8] = {(i - 1) % th != 0, ((i + th - 1) % th != 0) && (i + th - 1 < np), i + th <= np,
                        (i % th != 0) && (i + th + 1 < np), i % th != 0, (i % th != 0) && (i - th + 1 > 0),
                        i - th > 0, i - th - 1 > 0};
#pragma unroll
    for (int j = 0; j < 8; j++) {
      float t = 0.0f;
      if (R != 0.0f && ok[j]) t = (float)rc_q(b, ww, mk, p, cand[j] - 1, regfac, vf2) / R;
      cf[1 + j] = t;
    }
    const float lf = mk[p] ? (float)b.wy[e] : 0.0f;
    float L = lf / R;
    if (!isfinite(L)) L = 0.0f;
    cf[9] = L;
    b.le[e] = lf;
  }
}

// One colour sweep of the frames still running (state[f] == 1).
__global__ void __launch_bounds__(256) k_rc_sweep(RcBufs b, int colour, const int* __restrict__ state) {
  const int f = blockIdx.y;
  if (state[f] != 1) return;
  const int th = b.th, tw = b.tw;
  const int rh = (th + 1 - (colour >> 1)) >> 1, cw = (tw + 1 - (colour & 1)) >> 1;  // rows / columns of the colour
  const int per = rh * cw;
  float* x = b.x + (size_t)f * b.np;
  const float* cf0 = b.coef + (size_t)f * b.np * 10;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < per; k += gridDim.x * blockDim.x) {
    const int r = 2 * (k % rh) + (colour >> 1), c = 2 * (k / rh) + (colour & 1);
    const int p = r + th * c;
    const float* cf = cf0 + (size_t)p * 10;
    const int q[8] = {p - 1, p + th - 1, p + th, p + th + 1, p + 1, p - th + 1, p - th, p - th - 1};
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int qq = (q[j] >= 0 && q[j] < b.np) ? q[j] : 0;  // absent neighbours: index 1 in the reference
      const float t = x[qq] * cf[1 + j];
      s = j == 0 ? t : s + t;
    }
    x[p] = cf[9] - s;
  }
}

// Energy partial sums of the frames due for a check: sum over masked p of x_p (Q x)_p (FP64) and
// of Le_p x_p (FP32), kRcParts CTAs per frame over fixed pixel ranges.
__global__ void __launch_bounds__(256) k_rc_energy(RcBufs b, int nf, const int* __restrict__ due, double regfac,
                                                   double vf2) {
  const int f = blockIdx.y;
  if (!due[f]) return;
  const int th = b.th, np = b.np;
  const double* ww = b.ww + (size_t)f * np * kRcStencil;
  const uint8_t* mk = b.mask + (size_t)f * np;
  const float* x = b.x + (size_t)f * np;
  const float* le = b.le + (size_t)f * np;
  const int per = (np + kRcParts - 1) / kRcParts, a = blockIdx.x * per, e = min(np, a + per);
  double qs = 0.0;
  float ls = 0.0f;
  for (int p = a + threadIdx.x; p < e; p += blockDim.x) {
    if (!mk[p]) continue;
    const double xp = (double)x[p];
    double qx = rc_q(b, ww, mk, p, p, regfac, vf2) * xp;
    const int nb[8] = {p - 1, p + 1, p - th + 1, p + th - 1, p - th, p + th, p - th - 1, p + th + 1};
#pragma unroll
    for (int j = 0; j < 8; j++)
      if (nb[j] >= 0 && nb[j] < np) qx += rc_q(b, ww, mk, p, nb[j], regfac, vf2) * (double)x[nb[j]];
    qs += xp * qx;
    ls += le[p] * x[p];
  }
  __shared__ double sq[256];
  __shared__ float sl[256];
  sq[threadIdx.x] = qs;
  sl[threadIdx.x] = ls;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sq[threadIdx.x] += sq[threadIdx.x + o];
      sl[threadIdx.x] += sl[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    b.part[((size_t)f * kRcParts + blockIdx.x)] = sq[0];
    b.part_l[(size_t)f * kRcParts + blockIdx.x] = sl[0];
  }
}

// The check of every due frame (a thread per frame): the energy from its partial sums in a fixed
// order; a frame whose energy did not decrease stops, else its iterate becomes the output candidate
// (copied by k_rc_keep). eo[f] starts as the energy of the first iterate (check number 0).
__global__ void k_rc_check(int nf, const int* __restrict__ due, int* __restrict__ state, float* __restrict__ eo,
                           int* __restrict__ keep, const double* __restrict__ part, const float* __restrict__ part_l,
                           int first, int it, int* __restrict__ iters) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  keep[f] = 0;
  if (!due[f]) return;
  double q = 0.0;
  float l = 0.0f;
  for (int i = 0; i < kRcParts; i++) {
    q += part[(size_t)f * kRcParts + i];
    l += part_l[(size_t)f * kRcParts + i];
  }
  const float e = (float)(q - 2.0 * (double)l);
  if (first) {
    eo[f] = e;
    return;
  }
  if (eo[f] <= e) {
    state[f] = 2;  // stopped
    iters[f] = it;
  } else {
    eo[f] = e;
    keep[f] = 1;
  }
}

// Frames due for a check after sweep `it`: running, and `it` a multiple of their interval.
__global__ void k_rc_due(int nf, const int* __restrict__ state, const int* __restrict__ interval, int it,
                         int* __restrict__ due) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < nf) due[f] = state[f] == 1 && it % interval[f] == 0;
}

// Masked pixels of every frame (a frame with none is skipped, as the reference's `continue`); grid
// (blocks, frames), one atomic per CTA.
__global__ void __launch_bounds__(256) k_rc_count(RcBufs b, int* __restrict__ count) {
  const int f = blockIdx.y;
  const uint8_t* mk = b.mask + (size_t)f * b.np;
  int c = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < b.np; p += gridDim.x * blockDim.x) c += mk[p] ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  __shared__ int sc[8];
  if ((threadIdx.x & 31) == 0) sc[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sc[w];
    if (t) atomicAdd(count + f, t);
  }
}

// The candidate iterate of the frames whose check kept the sweep: xo = x; grid (blocks, frames).
__global__ void __launch_bounds__(256) k_rc_keep(RcBufs b, const int* __restrict__ keep) {
  const int f = blockIdx.y;
  if (!keep[f]) return;
  const size_t o = (size_t)f * b.np;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < b.np; p += gridDim.x * blockDim.x) b.xo[o + p] = b.x[o + p];
}

// Output of a finished frame: its candidate iterate, NaN outside the mask.
template <class OutT>
__global__ void __launch_bounds__(256) k_rc_out(RcBufs b, int nf, OutT* __restrict__ out, uint8_t* __restrict__ mk_out,
                                                const int* __restrict__ skip) {
  const size_t total = (size_t)b.np * nf;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const bool m = b.mask[e] && !skip[e / b.np];
    out[e] = m ? (OutT)b.xo[e] : (OutT)NAN;
    if (mk_out) mk_out[e] = m ? 1 : 0;
  }
}

}  // namespace ss
