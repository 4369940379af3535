// Tile schedules of the evaluation launches.
//
// An evaluation tile is one block column of one chunk of G.frames_per_cta consecutive frames of a
// group. Before each evaluation launch one CTA of k_schedule lists the (group, frame chunk) entries
// that have work in that launch (the group's phase for the mode; for a trial round, a frame of the
// chunk still searching), each standing for the group's W tiles, with the prefix sum of their tiles.
// The evaluation kernels then run as a grid of resident CTAs that take tiles from the list through
// an atomic counter, so a launch costs in proportion to the work left, not to the batch's size:
// late trial rounds of a ragged batch, where a few long searches remain, launch no idle CTAs.
// Results do not depend on the order in which tiles run (per-column sums land in their own slots
// and each frame's decision reads them in column order).
#pragma once

#include "ss_common.cuh"

namespace ss {

constexpr int kSchedThreads = 1024;

// Schedule buffer: header, then group[cap], chunk[cap], prefix[cap + 1] (cap = the batch's chunks).
enum SchedHeader : int { kSchTiles = 0, kSchEntries = 1, kSchNext = 2, kSchHdr = 4 };

__host__ __device__ constexpr size_t sched_ints(int cap) { return (size_t)kSchHdr + 3 * (size_t)cap + 1; }

// Whether a group has tiles in an evaluation launch of MODE (the phase tests of the evaluation
// kernels; a trial round also needs a frame still searching).
template <int MODE>
__device__ __forceinline__ bool group_has_work(const GroupCtl& C) {
  if (MODE == kFinal) return C.phase == kPhFinal;
  if (C.phase != kPhHalf) return false;
  if (MODE == kAssemble) return C.ls_state == 0;  // not while the group's line search runs
  if (MODE == kCorr) return C.shift == 1 && C.ls_state == 1 && C.ls_pending == 0;  // after shift 1's search
  return C.ls_state == 1 && C.ls_pending > 0;       // kTrial
}

// Builds the schedule of an evaluation launch of MODE (one CTA of kSchedThreads); returns the number
// of tiles listed in every thread.
template <int MODE>
__device__ __forceinline__ int build_schedule(const GroupDesc* __restrict__ gds, const GroupCtl* __restrict__ ctl,
                                              const int* __restrict__ chunk_group, int n_chunks,
                                              int* __restrict__ sched, int cap) {
  constexpr int kWarps = kSchedThreads / 32;
  __shared__ int s_e[kWarps], s_t[kWarps];
  __shared__ int s_base_e, s_base_t, s_sum_e, s_sum_t;
  int* grp = sched + kSchHdr;
  int* chk = grp + cap;
  int* pre = chk + cap;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) {
    s_base_e = 0;
    s_base_t = 0;
  }
  __syncthreads();
  for (int j0 = 0; j0 < n_chunks; j0 += kSchedThreads) {
    const int j = j0 + t;
    int g = -1, fb = 0, w = 0;
    if (j < n_chunks) {
      g = chunk_group[j];
      const GroupDesc& G = gds[g];
      fb = j - G.chunk_base;
      bool on = group_has_work<MODE>(ctl[g]);
      if (on && MODE == kTrial) {
        const int f0 = fb * G.frames_per_cta, f1 = min(G.nF, f0 + G.frames_per_cta);
        on = false;
        for (int f = f0; f < f1 && !on; f++) on = (G.fstate[f] & 2) != 0;
      }
      w = on ? G.W : 0;
    }
    // exclusive scans of the entries and their tiles over the CTA
    const unsigned bal = __ballot_sync(0xffffffffu, w > 0);
    const int e_in = __popc(bal & ((1u << lane) - 1u));
    int w_inc = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, w_inc, o);
      if (lane >= o) w_inc += v;
    }
    if (lane == 31) {
      s_e[warp] = __popc(bal);
      s_t[warp] = w_inc;
    }
    __syncthreads();
    if (warp == 0) {
      const int e = s_e[lane], tt = s_t[lane];
      int ei = e, ti = tt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int a = __shfl_up_sync(0xffffffffu, ei, o), b = __shfl_up_sync(0xffffffffu, ti, o);
        if (lane >= o) {
          ei += a;
          ti += b;
        }
      }
      s_e[lane] = ei - e;
      s_t[lane] = ti - tt;
      if (lane == 31) {
        s_sum_e = ei;
        s_sum_t = ti;
      }
    }
    __syncthreads();
    if (w > 0) {
      const int e = s_base_e + s_e[warp] + e_in;
      grp[e] = g;
      chk[e] = fb;
      pre[e] = s_base_t + s_t[warp] + w_inc - w;
    }
    __syncthreads();
    if (t == 0) {
      s_base_e += s_sum_e;
      s_base_t += s_sum_t;
    }
    __syncthreads();
  }
  if (t == 0) {
    sched[kSchTiles] = s_base_t;
    sched[kSchEntries] = s_base_e;
    sched[kSchNext] = 0;
    pre[s_base_e] = s_base_t;
  }
  return s_base_t;
}

template <int MODE>
__global__ void __launch_bounds__(kSchedThreads) k_schedule(const GroupDesc* __restrict__ gds,
                                                            const GroupCtl* __restrict__ ctl,
                                                            const int* __restrict__ chunk_group, int n_chunks,
                                                            int* __restrict__ sched, int cap) {
  build_schedule<MODE>(gds, ctl, chunk_group, n_chunks, sched, cap);
}

// The CTA's next tile of a scheduled launch into s_tile = (group, block column, frame chunk); false
// (in every thread) when the list is exhausted. All threads call; s_tile is read until the caller's
// next __syncthreads.
__device__ __forceinline__ bool fetch_tile(int* __restrict__ sched, int cap, int* s_tile) {
  if (threadIdx.x == 0) {
    const int idx = atomicAdd(sched + kSchNext, 1);
    if (idx >= sched[kSchTiles]) {
      s_tile[0] = -1;
    } else {
      const int* grp = sched + kSchHdr;
      const int* chk = grp + cap;
      const int* pre = chk + cap;
      int lo = 0, hi = sched[kSchEntries] - 1;  // the last entry starting at or before idx
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= idx) lo = mid;
        else hi = mid - 1;
      }
      s_tile[0] = grp[lo];
      s_tile[1] = idx - pre[lo];
      s_tile[2] = chk[lo];
    }
  }
  __syncthreads();
  return s_tile[0] >= 0;
}

// ---------------------------------------------------------------------------------------------
// Trial-round schedule
//
// A trial round evaluates only the frames still searching, which late in a cycle are a few per
// group. Tiles of fixed frame chunks then leave most warps of a CTA idle, so the trial schedule
// lists the searching frames themselves: one CTA compacts them (in frame order, hence grouped by
// group) and cuts each group's run into entries of up to kTrialTileFrames consecutive listed frames,
// each standing for the group's W tiles (one block column each); a tile's warps take its frames in
// turn. Each tile stages one template window for its frames, so tiles of 32 frames spend a quarter
// of the staging of tiles of 8 (512x512 frames, 2-line knots, groups of 64: trial rounds 85 ms with
// 32 frames per tile, 94 ms with 8).

#ifndef SS_TRIAL_TILE_FRAMES
#define SS_TRIAL_TILE_FRAMES 32
#endif
constexpr int kTrialTileFrames = SS_TRIAL_TILE_FRAMES;

// Buffer: header, list[nf] (batch frame index of each searching frame), first[ng] and end[ng] (each
// group's run in the list), then grp[nf], pos[nf], cnt[nf] (entries) and prefix[nf + 1] (tiles).
enum TrialSchedHeader : int { kTsTiles = 0, kTsEntries = 1, kTsNext = 2, kTsHdr = 4 };

__host__ __device__ constexpr size_t tsched_ints(int n_frames, int n_groups) {
  return (size_t)kTsHdr + 5 * (size_t)n_frames + 2 * (size_t)n_groups + 1;
}

// CTA-wide exclusive scan of v (kSchedThreads threads); returns the thread's exclusive prefix and
// the CTA's total in *total (every thread).
__device__ __forceinline__ int cta_exclusive_scan(int v, int* total) {
  constexpr int kWarps = kSchedThreads / 32;
  __shared__ int s_w[kWarps];
  __shared__ int s_total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int w = s_w[lane];
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += u;
    }
    s_w[lane] = wi - w;
    if (lane == 31) s_total = wi;
  }
  __syncthreads();
  const int r = s_w[warp] + inc - v;
  *total = s_total;
  __syncthreads();  // s_w and s_total are reused by the next call
  return r;
}

// Builds the trial-round schedule (one CTA of kSchedThreads); returns the number of tiles in every
// thread. frame_group maps the batch's frame index to its group (frames of a group contiguous, from
// its frame_base).
__device__ __forceinline__ int build_trial_schedule(const GroupDesc* __restrict__ gds, const GroupCtl* __restrict__ ctl,
                                                    const int* __restrict__ frame_group, int n_frames, int n_groups,
                                                    int* __restrict__ ts) {
  int* list = ts + kTsHdr;
  int* first = list + n_frames;
  int* end = first + n_groups;
  int* grp = end + n_groups;
  int* pos = grp + n_frames;
  int* cnt = pos + n_frames;
  int* pre = cnt + n_frames;
  __shared__ int s_base, s_base2, s_tiles;
  if (threadIdx.x == 0) {
    s_base = 0;
    s_base2 = 0;
    s_tiles = 0;
  }
  __syncthreads();
  // the searching frames, compacted in frame order, and each group's run
  for (int j0 = 0; j0 < n_frames; j0 += kSchedThreads) {
    const int j = j0 + threadIdx.x;
    int g = -1, f = 0;
    bool s = false;
    if (j < n_frames) {
      g = frame_group[j];
      const GroupDesc& G = gds[g];
      f = j - G.frame_base;
      s = group_has_work<kTrial>(ctl[g]) && (G.fstate[f] & 2) != 0;
    }
    int total;
    const int p = s_base + cta_exclusive_scan(s ? 1 : 0, &total);
    if (s) list[p] = j;
    if (g >= 0 && f == 0) first[g] = p;
    if (g >= 0 && f == gds[g].nF - 1) end[g] = p + (s ? 1 : 0);
    if (threadIdx.x == 0) s_base += total;
    __syncthreads();
  }
  const int n_list = s_base;
  // entries: runs of up to kTrialTileFrames listed frames of one group
  for (int p0 = 0; p0 < n_list; p0 += kSchedThreads) {
    const int p = p0 + threadIdx.x;
    int g = -1, w = 0;
    bool start = false;
    if (p < n_list) {
      g = frame_group[list[p]];
      start = (p - first[g]) % kTrialTileFrames == 0;
      w = start ? gds[g].W : 0;
    }
    int total_e, total_t;
    const int e = s_base2 + cta_exclusive_scan(start ? 1 : 0, &total_e);
    const int tp = s_tiles + cta_exclusive_scan(w, &total_t);
    if (start) {
      grp[e] = g;
      pos[e] = p;
      cnt[e] = min(kTrialTileFrames, end[g] - p);
      pre[e] = tp;
    }
    if (threadIdx.x == 0) {
      s_base2 += total_e;
      s_tiles += total_t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ts[kTsTiles] = s_tiles;
    ts[kTsEntries] = s_base2;
    ts[kTsNext] = 0;
    pre[s_base2] = s_tiles;
  }
  return s_tiles;
}

__global__ void __launch_bounds__(kSchedThreads) k_trial_schedule(const GroupDesc* __restrict__ gds,
                                                                  const GroupCtl* __restrict__ ctl,
                                                                  const int* __restrict__ frame_group, int n_frames,
                                                                  int n_groups, int* __restrict__ ts) {
  build_trial_schedule(gds, ctl, frame_group, n_frames, n_groups, ts);
}

// The CTA's next trial tile into s_tile = (group, block column, list position of its first frame,
// frames); false (in every thread) when the list is exhausted. All threads call.
__device__ __forceinline__ bool fetch_trial_tile(int* __restrict__ ts, int n_frames, int n_groups, int* s_tile) {
  if (threadIdx.x == 0) {
    const int idx = atomicAdd(ts + kTsNext, 1);
    if (idx >= ts[kTsTiles]) {
      s_tile[0] = -1;
    } else {
      const int* grp = ts + kTsHdr + n_frames + 2 * n_groups;
      const int* pos = grp + n_frames;
      const int* cnt = pos + n_frames;
      const int* pre = cnt + n_frames;
      int lo = 0, hi = ts[kTsEntries] - 1;  // the last entry starting at or before idx
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= idx) lo = mid;
        else hi = mid - 1;
      }
      s_tile[0] = grp[lo];
      s_tile[1] = idx - pre[lo];
      s_tile[2] = pos[lo];
      s_tile[3] = cnt[lo];
    }
  }
  __syncthreads();
  return s_tile[0] >= 0;
}

// The tile's group descriptor into shared memory (all threads call; ends with __syncthreads), so
// the many descriptor reads of a tile are shared-memory loads rather than dependent global ones.
__device__ __forceinline__ void load_desc(const GroupDesc* __restrict__ src, GroupDesc* dst) {
  static_assert(sizeof(GroupDesc) % 8 == 0, "descriptor copied in 8-byte words");
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(GroupDesc) / 8); i += blockDim.x) d[i] = __ldg(s + i);
  __syncthreads();
}

}  // namespace ss
