// Post-estimate validity of the recording-level estimate (ss_estimate_displacements).
//
// The reference's MATLAB driver turns each set's raw MEX outputs into the recording's result
// (estimate_displacements, steady_scan.m:246-284): it keeps every frame of the set but the last
// (the overlap frame that the next set estimates again), finds the blocks with a valid pixel in the
// set's final mask (blocksused, :264-265), marks a frame with none failed with a NaN correlation
// (:269-273), repeats the knots of the first and last used block over the unused blocks before and
// after them (extend_firstandlast, :277-281, :615-623) and marks the frame failed when its
// correlation is below corr_thresh (:283). Here one CTA per set applies these rules, a warp per
// frame, on the batch's device outputs and scatters the result into the recording's arrays.
#pragma once

#include "ss_common.cuh"

namespace ss {

// Frames of one set in the recording: the set's first frame and the frames it keeps.
struct SetSpan {
  int first, keep;
};

__global__ void __launch_bounds__(256) k_post_estimate(const GroupDesc* __restrict__ gds, const GroupCtl* __restrict__ ctl,
                                                       const SetSpan* __restrict__ sets, double corr_thresh,
                                                       double minblockfrac, double* __restrict__ dx,
                                                       double* __restrict__ dy, double* __restrict__ corr,
                                                       double* __restrict__ iters, double* __restrict__ residrms,
                                                       uint8_t* __restrict__ failed, uint8_t* __restrict__ used_out) {
  const GroupDesc& G = gds[blockIdx.x];
  const SetSpan sp = sets[blockIdx.x];
  const int W = G.W, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const double it = (double)ctl[blockIdx.x].iteration;
  for (int f = threadIdx.x >> 5; f < sp.keep; f += nw) {
    const size_t j = (size_t)sp.first + f;  // frame of the recording
    int lo = W, hi = -1;                    // first and last used block
    for (int b = lane; b < W; b += 32) {
      const bool u = G.colcnt[(size_t)f * W + b] > 0;
      if (used_out) used_out[j * W + b] = u ? 1 : 0;
      if (u) {
        lo = min(lo, b);
        hi = max(hi, b);
      }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    const bool any = hi >= 0;
    const bool extend = any && (lo > 0 || hi < W - 1);
    const double* sx = G.o_dx + (size_t)f * (W + 1);
    const double* sy = G.o_dy + (size_t)f * (W + 1);
    for (int k = lane; k <= W; k += 32) {
      const int src = extend ? (k < lo ? lo : (k > hi ? hi : k)) : k;
      dx[j * (W + 1) + k] = sx[src];
      dy[j * (W + 1) + k] = sy[src];
    }
    if (lane == 0) {
      const double c = G.o_frame_corr[f];
      corr[j] = any ? c : (double)NAN;
      // numel(blocksused) / (nknots - 1): the block count over itself, as the reference divides it
      failed[j] = (!any || !(c >= corr_thresh) || (double)W / (double)W < minblockfrac) ? 1 : 0;
      iters[j] = it;
      residrms[j] = G.o_residrms[f];
    }
  }
}

__global__ void k_fill_nan_u8(double* __restrict__ d, size_t nd, uint8_t* __restrict__ b, size_t nb) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nd; i += (size_t)gridDim.x * blockDim.x)
    d[i] = (double)NAN;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nb; i += (size_t)gridDim.x * blockDim.x)
    b[i] = 0;
}

}  // namespace ss
