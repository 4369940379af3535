// Host engine and C-ABI of the B200 align_group_to_template.
//
// A Batch owns the device state of one or more groups (each group is one align_group_to_template
// call's worth of frames) and runs them to completion together: every kernel covers all groups,
// and a device-side state machine per group (GroupCtl) decides what each group does next, so
// groups of different sizes and convergence speeds share launches.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <mutex>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

#include "ss_common.cuh"
#include "ss_engine.h"
#include "ss_eval.cuh"
#include "ss_group.cuh"
#include "ss_recording.cuh"
#include "ss_frontend.cuh"
#include "ss_reconstruct.cuh"
#include "steadyscan_b200.h"

namespace ss {

static thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
const char* last_error() { return g_err.c_str(); }

#define SS_CK(call)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      int code_ = (e_ == cudaErrorMemoryAllocation) ? SS_ERR_OUT_OF_MEMORY : SS_ERR_CUDA;    \
      return fail(code_, std::string(#call) + ": " + cudaGetErrorString(e_));                \
    }                                                                                        \
  } while (0)

// ---------------------------------------------------------------------------------------------
// set-up kernels

// Template quads from a column-major FP64 template (mexgateway.cpp:46 reads it column-major and
// the reference indexes it row-major, task_differenceimage.cuh:120).
template <class TplT>
__global__ void k_build_tquad(const double* __restrict__ T, int Ht, int Wt, TplT* __restrict__ q) {
  const size_t n = (size_t)(Ht - 1) * (Wt - 1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int iy = (int)(i / (Wt - 1)), ix = (int)(i % (Wt - 1));
    q[4 * i + 0] = (TplT)T[(size_t)ix * Ht + iy];
    q[4 * i + 1] = (TplT)T[(size_t)(ix + 1) * Ht + iy];
    q[4 * i + 2] = (TplT)T[(size_t)ix * Ht + iy + 1];
    q[4 * i + 3] = (TplT)T[(size_t)(ix + 1) * Ht + iy + 1];
  }
}

// FP32 template rows of `pitch` floats (zero padding) from the column-major FP64 template, the
// source of the shared-memory row windows of precision 'S'.
__global__ void k_build_tplain(const double* __restrict__ T, int Ht, int Wt, int pitch, float* __restrict__ out) {
  const size_t n = (size_t)Ht * pitch;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int iy = (int)(i / pitch), ix = (int)(i % pitch);
    out[i] = ix < Wt ? (float)T[(size_t)ix * Ht + iy] : 0.0f;
  }
}

// Gradient quads (xg[iy][ix], xg[iy+1][ix], yg[iy][ix], yg[iy][ix+1]) for caller gradients that
// are not the template's forward differences.
template <class TplT>
__global__ void k_build_gquad(const double* __restrict__ xg, const double* __restrict__ yg, int Ht, int Wt,
                              TplT* __restrict__ q) {
  const size_t n = (size_t)(Ht - 1) * (Wt - 1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int iy = (int)(i / (Wt - 1)), ix = (int)(i % (Wt - 1));
    q[4 * i + 0] = (TplT)xg[(size_t)ix * Ht + iy];
    q[4 * i + 1] = (TplT)xg[(size_t)ix * Ht + iy + 1];
    q[4 * i + 2] = (TplT)yg[(size_t)ix * Ht + iy];
    q[4 * i + 3] = (TplT)yg[(size_t)(ix + 1) * Ht + iy];
  }
}

// Sum of all frame samples of a group in two deterministic passes: kSumBlocks CTA partials over
// fixed contiguous ranges, then one CTA adds the partials in a fixed order.
constexpr int kSumBlocks = 296;
// Entries of output 10: TimedMainIteration's ten sub-functions, then the correlation and the
// iteration end's remainder, and two that the reference never writes (task.cpp:244).
constexpr int kFunctionTimes = 14;

// The library's stream-ordered memory pool of a device (defined with the per-call work memory).
static cudaMemPool_t work_pool(int device);

__device__ __forceinline__ double block_sum(double s) {
  __shared__ double sh[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  double v = 0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

template <class FrameT>
__global__ void __launch_bounds__(1024) k_sum_image(const void* __restrict__ img, size_t n, double* __restrict__ parts) {
  const size_t per = (n + gridDim.x - 1) / gridDim.x;
  const size_t a = blockIdx.x * per, e = a + per < n ? a + per : n;
  double s = 0;
  for (size_t i = a + threadIdx.x; i < e; i += blockDim.x) s += to_double(ld_frame<FrameT>(img, i));
  s = block_sum(s);
  if (threadIdx.x == 0) parts[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_sum_parts(const double* __restrict__ parts, int n, double* __restrict__ out) {
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += parts[i];
  s = block_sum(s);
  if (threadIdx.x == 0) *out = s;
}

__global__ void k_fill(double* p, size_t n, double v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

// The per-group state reset at the start of a run (task_allocate.cu:201-255) as one launch:
// blockIdx.y is the group, the CTAs of a row stride over its buffers. The knot buffers start as
// NaN (an all-invalid mask and a zero difference image until the first knots are written), no
// column keeps assembly sums of an earlier run, and the errvals start at the reference's fill.
__global__ void k_reset_groups(const GroupDesc* __restrict__ gd) {
  const GroupDesc& G = gd[blockIdx.y];
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
  const size_t N = G.N, nF = G.nF, mi = G.max_iter, nrg2 = 2 * (size_t)G.n_rg;
  const size_t nk = nF * 2 * (size_t)(G.W + 1), na = (size_t)G.fW * 8;
  for (size_t i = t0; i < 2 * N; i += st) {
    G.p[i] = G.p0[i];
    G.p_last[i] = 0.0;
    G.delta_p[i] = 0.0;
  }
  for (size_t i = t0; i < N; i += st) {
    G.params_used[i] = 0;
    G.blocks_present[i] = 0;
    G.eig_valid[i] = 0;
  }
  for (size_t i = t0; i <= nrg2; i += st) G.grp_active[i] = i < nrg2 ? 1 : 0;
  for (size_t i = t0; i < nF; i += st) {
    G.o_frame_corr[i] = 0.0;
    G.ls_done[i] = 0;
  }
  for (size_t i = t0; i < 2 * nF; i += st) G.errval[i] = kErrvalFill;
  for (size_t i = t0; i < nk; i += st) {
    G.kmask[i] = NAN;
    G.kdiff[i] = NAN;
  }
  for (size_t i = t0; i < na; i += st) G.asmk[i] = NAN;
  if (G.o_rg_params)
    for (size_t i = t0; i < 4 * N * mi; i += st) G.o_rg_params[i] = 0.0;
  if (G.o_iter_times)
    for (size_t i = t0; i < mi; i += st) G.o_iter_times[i] = 0.0;
}

// ---------------------------------------------------------------------------------------------
// kernel dispatch by (compute, frame type, template type)

// Identifier of the calling thread's current CUDA context, unique for the life of the process (the
// context the runtime creates after a cudaDeviceReset gets a new one); 0 when none is current or the
// driver does not report one. Read through the runtime's driver entry points (no link to libcuda).
static unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Opts a kernel into `bytes` of dynamic shared memory on the current device, once per device and
// context (the attribute does not survive a reset of the device's context).
template <class F>
static cudaError_t smem_attr(F* fn, int bytes) {
  static std::mutex mu;
  static std::set<std::tuple<int, unsigned long long, const void*>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const auto key = std::make_tuple(dev, current_context_id(), reinterpret_cast<const void*>(fn));
  std::lock_guard<std::mutex> lock(mu);
  if (std::get<1>(key) != 0 && done.count(key)) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.insert(key);
  return e;
}

// Dynamic shared memory for staging one block column's geometry (tfrac, basex, basey, the next
// column's tfrac and base_mask) in k_eval.
constexpr int kStageBytes = 96 * 1024;
// Shared memory for one template row window of a precision-'S' evaluation CTA (36 rows of a
// 512-pixel template): three resident assembly / correlation / final CTAs per SM, the register
// limit of those kernels (build-time tuning; the trial rounds use kTrialWinBytes).
#ifndef SS_EVAL_WIN_KB
#define SS_EVAL_WIN_KB 72
#endif
constexpr int kWinBytes = SS_EVAL_WIN_KB * 1024;
// Shared memory for the template rows of one line-search CTA (98 rows of a 512-pixel template;
// with the kernel's static shared memory one 1024-thread CTA per SM).
constexpr int kLsWinBytes = 196 * 1024;

// Grid of an evaluation launch: the CTAs of `fn` resident on the device at once with `smem` bytes,
// at most the batch's tiles (the CTAs take tiles from the launch's schedule until it is exhausted).
template <class F>
static int resident_grid(F* fn, int threads, size_t smem, int max_tiles) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, size_t>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return std::max(1, std::min(max_tiles, 148));
  const auto key = std::make_tuple(dev, reinterpret_cast<const void*>(fn), smem);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it == cache.end()) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) per_sm = 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    it = cache.emplace(key, std::max(1, per_sm) * std::max(1, sms)).first;
  }
  return std::max(1, std::min(max_tiles, it->second));
}

using EvalFn = cudaError_t (*)(int mode, int max_tiles, cudaStream_t s, const GroupDesc* gd, int* sched, int cap,
                               const GroupCtl* ctl, int max_hb, int win_bytes);
using LsFn = cudaError_t (*)(int frames, cudaStream_t s, const GroupDesc* gd, const int* fg, GroupCtl* ctl,
                             int win_bytes);
using SumFn = void (*)(const void* img, size_t n, double* parts, double* out, cudaStream_t s);

template <class Acc, class FrameT, class TplT>
static cudaError_t eval_launch(int mode, int max_tiles, cudaStream_t s, const GroupDesc* gd, int* sched, int cap,
                               const GroupCtl* ctl, int max_hb, int win_bytes) {
  constexpr int kMaxDyn = kStageBytes + kWinBytes + 64;
  cudaError_t ae = smem_attr(k_eval<Acc, FrameT, TplT, kAssemble>, kMaxDyn);
  if (ae == cudaSuccess) ae = smem_attr(k_eval<Acc, FrameT, TplT, kFinal>, kMaxDyn);
  if (ae == cudaSuccess) ae = smem_attr(k_eval<Acc, FrameT, TplT, kCorr>, kMaxDyn);
  if (ae != cudaSuccess) return ae;
  const int rows = stage_bytes<Acc>(max_hb) <= (size_t)kStageBytes ? max_hb : 0;
  if (sizeof(Acc) != 4) win_bytes = 0;
  win_bytes = std::min(win_bytes, kWinBytes) & ~15;
  // the window's mbarrier, geometry staging (16-byte multiple), then the template window
  const size_t smem = 16 + (rows ? stage_bytes<Acc>(rows) : 0) + (size_t)win_bytes;
  const int th = 32 * kEvalWarps;
  auto* fa = k_eval<Acc, FrameT, TplT, kAssemble>;
  auto* fc = k_eval<Acc, FrameT, TplT, kCorr>;
  auto* ff = k_eval<Acc, FrameT, TplT, kFinal>;
  // grids first (the occupancy queries are cached: none runs while a graph is captured)
  const int ga = resident_grid(fa, th, smem, max_tiles), gc = resident_grid(fc, th, smem, max_tiles),
            gf = resident_grid(ff, th, smem, max_tiles);
  if (max_tiles <= 0) return cudaSuccess;
  if (mode == kAssemble) fa<<<ga, th, smem, s>>>(gd, sched, cap, ctl, rows, win_bytes);
  else if (mode == kCorr) fc<<<gc, th, smem, s>>>(gd, sched, cap, ctl, rows, win_bytes);
  else ff<<<gf, th, smem, s>>>(gd, sched, cap, ctl, rows, win_bytes);
  return cudaGetLastError();
}

template <class Acc, class FrameT, class TplT>
static cudaError_t ls_launch(int frames, cudaStream_t s, const GroupDesc* gd, const int* fg, GroupCtl* ctl,
                             int win_bytes) {
  if (sizeof(Acc) != 4) win_bytes = 0;
  win_bytes = std::min(win_bytes, kLsWinBytes) & ~15;
  if (win_bytes) {
    cudaError_t ae = smem_attr(k_linesearch<Acc, FrameT, TplT>, kLsWinBytes + 16);
    if (ae != cudaSuccess) return ae;
  }
  if (frames <= 0) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(frames * kLsCluster, 1, 1);
  cfg.blockDim = dim3(LsShape<Acc>::threads, 1, 1);
  cfg.dynamicSmemBytes = win_bytes ? (size_t)win_bytes + 16 : 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kLsCluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_linesearch<Acc, FrameT, TplT>, gd, fg, ctl, win_bytes);
}

using RoundFn = cudaError_t (*)(int max_tiles, cudaStream_t s, const GroupDesc* gd, int* tsched, int n_frames,
                                int n_groups, GroupCtl* ctl, int win_bytes);

// One line-search trial round of precision 'S' over the tiles of the round's trial schedule
// (tsched of a batch of n_frames frames in n_groups groups).
template <class FrameT, class TplT>
static cudaError_t round_launch(int max_tiles, cudaStream_t s, const GroupDesc* gd, int* tsched, int n_frames,
                                int n_groups, GroupCtl* ctl, int win_bytes) {
  auto* fn = k_trial_round<FrameT, TplT>;
  cudaError_t ae = smem_attr(fn, kTrialWinBytes + 16);
  if (ae != cudaSuccess) return ae;
  win_bytes = std::min(win_bytes, kTrialWinBytes) & ~15;
  const size_t smem = 16 + (size_t)win_bytes;
  const int th = 32 * kEvalWarps;
  const int grid = resident_grid(fn, th, smem, max_tiles);  // cached before any capture
  if (max_tiles <= 0) return cudaSuccess;
  fn<<<grid, th, smem, s>>>(gd, tsched, n_frames, n_groups, ctl, win_bytes);
  return cudaGetLastError();
}

// The trial schedule of the next round (one CTA).
static cudaError_t trial_sched_launch(cudaStream_t s, const GroupDesc* gd, const GroupCtl* ctl, const int* frame_group,
                                      int n_frames, int n_groups, int* tsched) {
  k_trial_schedule<<<1, kSchedThreads, 0, s>>>(gd, ctl, frame_group, n_frames, n_groups, tsched);
  return cudaGetLastError();
}

// The schedule of an evaluation launch of `mode` (one CTA).
static cudaError_t sched_launch(int mode, cudaStream_t s, const GroupDesc* gd, const GroupCtl* ctl,
                                const int* chunk_group, int n_chunks, int* sched) {
  if (mode == kAssemble) k_schedule<kAssemble><<<1, kSchedThreads, 0, s>>>(gd, ctl, chunk_group, n_chunks, sched, n_chunks);
  else if (mode == kTrial) k_schedule<kTrial><<<1, kSchedThreads, 0, s>>>(gd, ctl, chunk_group, n_chunks, sched, n_chunks);
  else if (mode == kCorr) k_schedule<kCorr><<<1, kSchedThreads, 0, s>>>(gd, ctl, chunk_group, n_chunks, sched, n_chunks);
  else k_schedule<kFinal><<<1, kSchedThreads, 0, s>>>(gd, ctl, chunk_group, n_chunks, sched, n_chunks);
  return cudaGetLastError();
}

struct KernelSet {
  EvalFn eval;
  LsFn ls;
  RoundFn round;  // precision 'S' only
};
template <class FrameT>
static void sum_launch(const void* img, size_t n, double* parts, double* out, cudaStream_t s) {
  k_sum_image<FrameT><<<kSumBlocks, 1024, 0, s>>>(img, n, parts);
  k_sum_parts<<<1, 256, 0, s>>>(parts, kSumBlocks, out);
}

template <class Acc, class FrameT, class TplT>
static KernelSet kset() {
  if constexpr (sizeof(Acc) == 4)
    return {eval_launch<Acc, FrameT, TplT>, ls_launch<Acc, FrameT, TplT>, round_launch<FrameT, TplT>};
  else
    return {eval_launch<Acc, FrameT, TplT>, ls_launch<Acc, FrameT, TplT>, nullptr};
}

static KernelSet pick_kernels(int compute, int fdt, int tdt) {
  if (compute == 0) {
    switch (fdt) {
      case SS_F64: return kset<double, double, double>();
      case SS_F32: return kset<double, float, double>();
      case SS_U16: return kset<double, uint16_t, double>();
      case SS_F16: return kset<double, __half, double>();
    }
  } else if (tdt == SS_F16) {
    switch (fdt) {
      case SS_F64: return kset<float, double, __half>();
      case SS_F32: return kset<float, float, __half>();
      case SS_U16: return kset<float, uint16_t, __half>();
      case SS_F16: return kset<float, __half, __half>();
    }
  } else {
    switch (fdt) {
      case SS_F64: return kset<float, double, float>();
      case SS_F32: return kset<float, float, float>();
      case SS_U16: return kset<float, uint16_t, float>();
      case SS_F16: return kset<float, __half, float>();
    }
  }
  return {nullptr, nullptr};
}
static SumFn pick_sum(int fdt) {
  switch (fdt) {
    case SS_F64: return sum_launch<double>;
    case SS_F32: return sum_launch<float>;
    case SS_U16: return sum_launch<uint16_t>;
    case SS_F16: return sum_launch<__half>;
  }
  return nullptr;
}

static size_t dtype_size(int dt) {
  switch (dt) {
    case SS_F64: return 8;
    case SS_F32: return 4;
    case SS_U16: return 2;
    case SS_F16: return 2;
    case SS_U8: return 1;
    case SS_I32: return 4;
  }
  return 0;
}

// ---------------------------------------------------------------------------------------------
// host-side conversion of small inputs

static double elem_as_double(const ss_matrix& m, size_t i) {
  const char* b = static_cast<const char*>(m.data);
  switch (m.dtype) {
    case SS_F64: return reinterpret_cast<const double*>(b)[i];
    case SS_F32: return reinterpret_cast<const float*>(b)[i];
    case SS_U16: return reinterpret_cast<const uint16_t*>(b)[i];
    case SS_U8: return reinterpret_cast<const uint8_t*>(b)[i];
    case SS_I32: return reinterpret_cast<const int32_t*>(b)[i];
    case SS_F16: {
      uint16_t h = reinterpret_cast<const uint16_t*>(b)[i];
      int e = (h >> 10) & 31, mnt = h & 1023;
      double v = e == 0 ? std::ldexp((double)mnt, -24) : (e == 31 ? (mnt ? NAN : INFINITY)
                                                                : std::ldexp((double)(mnt | 1024), e - 25));
      return (h & 0x8000) ? -v : v;
    }
  }
  return NAN;
}

static int host_doubles(const ss_matrix& m, const char* name, std::vector<double>& out) {
  if (m.location != SS_HOST) return fail(SS_ERR_INVALID_ARGUMENT, std::string(name) + " must be host memory");
  if (!m.data && m.rows * m.cols > 0) return fail(SS_ERR_INVALID_ARGUMENT, std::string(name) + " is NULL");
  if (dtype_size(m.dtype) == 0) return fail(SS_ERR_INVALID_ARGUMENT, std::string(name) + ": unknown dtype");
  size_t n = (size_t)(m.rows * m.cols);
  out.resize(n);
  if (m.dtype == SS_F64) {  // one type test per matrix, not per element
    if (n) std::memcpy(out.data(), m.data, n * sizeof(double));
  } else if (m.dtype == SS_F32) {
    const float* p = static_cast<const float*>(m.data);
    for (size_t i = 0; i < n; i++) out[i] = (double)p[i];
  } else {
    for (size_t i = 0; i < n; i++) out[i] = elem_as_double(m, i);
  }
  return SS_OK;
}

// A host matrix read as doubles: the caller's own array when it holds doubles (no copy), else a
// converted copy. It is read only while the batch prepares, when the call's inputs are valid.
struct HostDoubles {
  const double* ext = nullptr;
  std::vector<double> own;
  size_t n = 0;
  const double* data() const { return ext ? ext : own.data(); }
  size_t size() const { return n; }
};

static int host_doubles(const ss_matrix& m, const char* name, HostDoubles& out) {
  out.ext = nullptr;
  out.own.clear();
  out.n = 0;
  if (m.location == SS_HOST && m.dtype == SS_F64 && m.data) {
    out.ext = static_cast<const double*>(m.data);
    out.n = (size_t)(m.rows * m.cols);
    return SS_OK;
  }
  int rc = host_doubles(m, name, out.own);
  out.n = out.own.size();
  return rc;
}

static int parse_flags(const char* flags, int& compute, int& bits) {
  if (!flags) return fail(SS_ERR_INVALID_ARGUMENT, "flags is NULL");
  compute = -1;
  bits = 0;
  for (const char* c = flags; *c; c++) {
    switch (*c) {
      case 'D': compute = 0; break;
      case 'S': compute = 1; break;
      case 'M': bits |= kFlagMaskInactive; break;
      case 'C': bits |= kFlagIterCorr; break;
      case 'c': bits |= kFlagFrameCorr; break;
      case 'e': bits |= kFlagIterErrvals; break;
      case 'R': bits |= kFlagMedianBefore; break;
      case 'P': bits |= kFlagRawParams; break;
      case 'p': bits |= kFlagFrameOrdered; break;
      case 'T': bits |= kFlagTimeExec; break;
      case 't': bits |= kFlagTimeSub; break;
      default: break;  // I F W w G E r f V: printing and debug switches
    }
  }
  if (compute < 0)
    return fail(SS_ERR_INVALID_ARGUMENT, "invalid precision type! use 'S' for single-precision and 'D' for double-precision");
  return SS_OK;
}

// ---------------------------------------------------------------------------------------------
// Batch

// Source index of template and geometry buffers that a resident session holds.
constexpr int kFromSession = -2;

// Run counters of a batch on the device (and their pinned host copy).
enum RunCounter {
  kCtrMaxTrials = 0,  // most trials of a line search that ended in the cycle (host-driven cycles)
  kCtrDone = 1,       // groups that have finished
  kCtrCycles = 2,     // cycles run by the graph
  kCtrRound = 3,      // trial rounds of the graph's current cycle
  kCtrRounds = 4,     // trial rounds run by the graph
  kCtrBound = 5,      // bit 0: the graph stopped at the cycle bound; bit 1: a cycle hit its round bound
  kCtrWaiting = 6,    // groups whose streamed frames have not arrived (k_join)
  kCounters = 8
};

struct HostGroup {
  const ss_inputs* in = nullptr;
  int compute = 0, flags = 0;
  int Hb = 0, W = 0, nF = 0, fW = 0, N = 0, Ht = 0, Wt = 0, group_size = 0, n_rg = 0;
  int frame_dt = SS_F64, tpl_dt = SS_F64;
  bool grad_derived = true, frac_uniform = true;
  HostDoubles templ, xg, yg, frac, bx, by, ex, ey;  // ex, ey: the initial knots
  std::vector<float> frac_f, bx_f, by_f;  // precision 'S' geometry
  std::vector<float> yrange;              // per block column [min, max] of basey over valid rows
  int frames_per_cta = 32;
  int tpl_src = -1, geo_src = -1;         // earlier group whose template / geometry buffers are shared,
                                          // or kFromSession
  const GroupDesc* ses_gd = nullptr;      // resident session buffers (kFromSession)
  const HostGroup* ses_hg = nullptr;
  int geo_k = 0, geo_L = 0;               // affine geometry (0: tables)
  double geo_ax = 0, geo_bx = 0, geo_ay = 0, geo_by = 0, geo_fs = 0;
  std::vector<uint8_t> bmask;
  std::vector<int32_t> minp;
  const void* frames_dev = nullptr;  // caller device pointer when bm_data is on the device
  size_t frame_bytes = 0;
  // device pointers
  double* d_templ_stage = nullptr;
  double* d_xg_stage = nullptr;
  double* d_yg_stage = nullptr;
  double* d_sum = nullptr;
  double* d_p0 = nullptr;
  void* d_image = nullptr;
  // streamed frames (Batch::set_stream_frames): the frames and their image sum in the batch's early
  // buffer, uploaded while the host prepares the rest
  void* early_image = nullptr;
  double* early_sum = nullptr;
};

static void detect_affine_geometry(HostGroup& g);

static int validate_group(const ss_inputs* in, HostGroup& g) {
  if (!in) return fail(SS_ERR_INVALID_ARGUMENT, "inputs is NULL");
  int rc = parse_flags(in->flags, g.compute, g.flags);
  if (rc) return rc;
  g.in = in;
  g.Ht = (int)in->template_image.rows;
  g.Wt = (int)in->template_image.cols;
  if (g.Ht < 2 || g.Wt < 2) return fail(SS_ERR_INVALID_ARGUMENT, "template_image must be at least 2 x 2");
  if (in->xgrad.rows != g.Ht || in->xgrad.cols != g.Wt || in->ygrad.rows != g.Ht || in->ygrad.cols != g.Wt)
    return fail(SS_ERR_INVALID_ARGUMENT, "xgrad and ygrad must match template_image");
  g.Hb = (int)in->basex.rows;  // frameH, frameW from basex (mexgateway.cpp:176-177)
  g.W = (int)in->basex.cols;
  if (g.Hb < 1 || g.W < 1) return fail(SS_ERR_INVALID_ARGUMENT, "basex is empty");
  const ss_matrix* geo[3] = {&in->tfrac, &in->basey, &in->base_mask};
  const char* geon[3] = {"tfrac", "basey", "base_mask"};
  for (int i = 0; i < 3; i++)
    if (geo[i]->rows != g.Hb || geo[i]->cols != g.W)
      return fail(SS_ERR_INVALID_ARGUMENT, std::string(geon[i]) + " must match basex");
  g.nF = in->n_frames;
  if (g.nF < 1) return fail(SS_ERR_INVALID_ARGUMENT, "n_frames must be positive");
  g.fW = g.W * g.nF;
  if (in->frames_per_cta < 0 || in->frames_per_cta > kMaxChunk)
    return fail(SS_ERR_INVALID_ARGUMENT, "frames_per_cta must be 0 or 1..64");
  if (in->frames_per_cta > 0) {
    g.frames_per_cta = in->frames_per_cta;
  } else {  // frame chunks of the evaluation tiles: at most 32 frames, as even as the group allows
    const int chunks = (g.nF + 31) / 32;
    g.frames_per_cta = (g.nF + chunks - 1) / chunks;
  }
  g.N = g.fW + 1;
  if ((long long)g.Hb * g.fW > (1LL << 31) - 1) return fail(SS_ERR_INVALID_ARGUMENT, "too many pixels in one group");
  if (in->bm_data.rows != g.Hb || in->bm_data.cols != g.fW)
    return fail(SS_ERR_INVALID_ARGUMENT, "bm_data must be frameH x (frameW * n_frames)");
  g.frame_dt = in->bm_data.dtype;
  if (!(g.frame_dt == SS_F64 || g.frame_dt == SS_F32 || g.frame_dt == SS_U16 || g.frame_dt == SS_F16))
    return fail(SS_ERR_INVALID_ARGUMENT, "bm_data dtype must be f64, f32, u16 or f16");
  if (!in->bm_data.data) return fail(SS_ERR_INVALID_ARGUMENT, "bm_data is NULL");
  // known here, before the host inputs load: streamed uploads start right after validation
  g.frame_bytes = (size_t)g.Hb * g.fW * dtype_size(g.frame_dt);
  g.frames_dev = in->bm_data.location == SS_DEVICE ? in->bm_data.data : nullptr;
  if (in->est_dx_knots.rows * in->est_dx_knots.cols != (int64_t)(g.W + 1) * g.nF ||
      in->est_dy_knots.rows * in->est_dy_knots.cols != (int64_t)(g.W + 1) * g.nF)
    return fail(SS_ERR_INVALID_ARGUMENT, "est_dx_knots and est_dy_knots must hold (frameW + 1) x n_frames values");
  if (in->min_points_per_block.rows * in->min_points_per_block.cols < g.W)
    return fail(SS_ERR_INVALID_ARGUMENT, "min_points_per_block needs at least frameW entries");
  if (g.W > kMaxFrameW) return fail(SS_ERR_INVALID_ARGUMENT, "frameW exceeds the supported maximum of 2048");
  g.group_size = in->group_size;
  if (g.group_size <= 0 || g.group_size % g.W != 0)
    return fail(SS_ERR_INVALID_ARGUMENT, "group_size must be a positive multiple of frameW");
  g.n_rg = g.fW / g.group_size;
  if (in->max_iter < 1) return fail(SS_ERR_INVALID_ARGUMENT, "max_iter must be positive");
  if (in->solver_id < 0 || in->solver_id > 2)
    return fail(SS_ERR_INVALID_ARGUMENT, "invalid solver id\n0:CuSparse solver\n1:CuSolver solver\n2:Eigen solver");
  int fsel = in->filter_id & (0 - (in->max_filter_iterations != 0));  // task.cpp:54
  if (fsel < 0 || fsel > 2)
    return fail(SS_ERR_INVALID_ARGUMENT, "invalid filter ID\n0: disable filter\n1: smearingfiter\n2:rangefilter");
  if (!(in->linesearch_reduction_multiplier > 0.0 && in->linesearch_reduction_multiplier < 1.0))
    return fail(SS_ERR_INVALID_ARGUMENT, "linesearch_reduction_multiplier must be in (0, 1)");
  g.tpl_dt = g.compute == 0 ? SS_F64 : (in->template_storage == SS_F16 ? SS_F16 : SS_F32);
  return SS_OK;
}

static bool same_matrix(const ss_matrix& a, const ss_matrix& b) {
  return a.data == b.data && a.rows == b.rows && a.cols == b.cols && a.dtype == b.dtype && a.location == b.location;
}

// Groups that pass the same host buffers for template and gradients, or for the scan geometry,
// share one conversion and one device copy (typically all sets of one recording).
static void find_shared_inputs(std::vector<HostGroup>& hg) {
  for (size_t i = 0; i < hg.size(); i++) {
    const ss_inputs* a = hg[i].in;
    for (size_t j = 0; j < i; j++) {
      const ss_inputs* b = hg[j].in;
      if (hg[i].tpl_src == -1 && hg[j].tpl_src == -1 && same_matrix(a->template_image, b->template_image) &&
          same_matrix(a->xgrad, b->xgrad) && same_matrix(a->ygrad, b->ygrad))
        hg[i].tpl_src = (int)j;
      if (hg[i].geo_src == -1 && hg[j].geo_src == -1 && same_matrix(a->tfrac, b->tfrac) &&
          same_matrix(a->basex, b->basex) && same_matrix(a->basey, b->basey) &&
          same_matrix(a->base_mask, b->base_mask) && same_matrix(a->min_points_per_block, b->min_points_per_block))
        hg[i].geo_src = (int)j;
    }
  }
}

static int load_host_inputs(std::vector<HostGroup>& all, size_t gi) {
  HostGroup& g = all[gi];
  const ss_inputs* in = g.in;
  int rc;
  if (g.tpl_src == -1) {
    if ((rc = host_doubles(in->template_image, "template_image", g.templ))) return rc;
    if ((rc = host_doubles(in->xgrad, "xgrad", g.xg))) return rc;
    if ((rc = host_doubles(in->ygrad, "ygrad", g.yg))) return rc;
  }
  HostDoubles tmp;
  if (g.geo_src == -1) {
    if ((rc = host_doubles(in->tfrac, "tfrac", g.frac))) return rc;
    if ((rc = host_doubles(in->basex, "basex", g.bx))) return rc;
    if ((rc = host_doubles(in->basey, "basey", g.by))) return rc;
    if ((rc = host_doubles(in->base_mask, "base_mask", tmp))) return rc;
    g.bmask.resize(tmp.size());
    const double* mk = tmp.data();
    for (size_t i = 0; i < tmp.size(); i++) g.bmask[i] = mk[i] != 0.0;
    if ((rc = host_doubles(in->min_points_per_block, "min_points_per_block", tmp))) return rc;
    g.minp.resize(g.W);
    const double* mp = tmp.data();
    for (int i = 0; i < g.W; i++) g.minp[i] = (int32_t)mp[i];  // static_cast<int> (mexconverter.cpp:97)
  }
  if ((rc = host_doubles(in->est_dx_knots, "est_dx_knots", g.ex))) return rc;
  if ((rc = host_doubles(in->est_dy_knots, "est_dy_knots", g.ey))) return rc;
  if (g.tpl_src == -1) {
    // gradients that are exactly the template's forward differences are re-derived on the device
    const double* T = g.templ.data();
    const double* X = g.xg.data();
    const double* Y = g.yg.data();
    g.grad_derived = true;
    for (int c = 0; c + 1 < g.Wt && g.grad_derived; c++)
      for (int r = 0; r < g.Ht; r++) {
        double d = T[(size_t)(c + 1) * g.Ht + r] - T[(size_t)c * g.Ht + r];
        if (!(X[(size_t)c * g.Ht + r] == d)) { g.grad_derived = false; break; }
      }
    for (int c = 0; c < g.Wt && g.grad_derived; c++)
      for (int r = 0; r + 1 < g.Ht; r++) {
        double d = T[(size_t)c * g.Ht + r + 1] - T[(size_t)c * g.Ht + r];
        if (!(Y[(size_t)c * g.Ht + r] == d)) { g.grad_derived = false; break; }
      }
  } else {
    g.grad_derived = g.tpl_src == kFromSession ? g.ses_hg->grad_derived : all[g.tpl_src].grad_derived;
  }
  if (g.geo_src == -1) {
    g.frac_uniform = true;
    const double* F = g.frac.data();
    for (int c = 1; c < g.W && g.frac_uniform; c++)
      for (int r = 0; r < g.Hb; r++)
        if (std::memcmp(&F[(size_t)c * g.Hb + r], &F[r], sizeof(double)) != 0) { g.frac_uniform = false; break; }
    if (g.compute == 1 && g.frac_uniform) detect_affine_geometry(g);
  } else {
    const HostGroup& s = g.geo_src == kFromSession ? *g.ses_hg : all[g.geo_src];
    g.frac_uniform = s.frac_uniform;
    g.geo_k = s.geo_k; g.geo_L = s.geo_L;
    g.geo_ax = s.geo_ax; g.geo_bx = s.geo_bx; g.geo_ay = s.geo_ay; g.geo_by = s.geo_by; g.geo_fs = s.geo_fs;
  }
  return SS_OK;
}

// Recognises the geometry that steady_scan.m:787-827 builds for unidirectional scanning with an
// integer number of lines per knot dividing 32 and no cropping: block row r = j*k + l is pixel j
// of line cc*k + l, basex and basey are affine in j and in the line, and tfrac = (l*L + j + 1/2) /
// (k*L). Every table entry is checked; any mismatch keeps the tables.
static void detect_affine_geometry(HostGroup& g) {
  g.geo_k = 0;
  const int Hb = g.Hb, W = g.W;
  for (int k = 1; k <= 32; k <<= 1) {
    if (Hb % k) continue;
    const int L = Hb / k;
    if (L < 2 || (k > 1 && W < 1)) continue;
    const double fs = 1.0 / ((double)k * L);
    const double* BX = g.bx.data();
    const double* BY = g.by.data();
    const double* FR = g.frac.data();
    const uint8_t* MK = g.bmask.data();
    const double bx0 = BX[0], ax = BX[k] - BX[0];
    const double by0 = BY[0];
    const double ay = (k > 1) ? BY[1] - BY[0] : (W > 1 ? BY[Hb] - BY[0] : 1.0);
    auto near = [](double a, double b) { return std::fabs(a - b) <= 1e-9 * std::max(1.0, std::fabs(b)); };
    bool ok = true;
    // block row r = j * k + l: pixel j of line cc * k + l
    for (int cc = 0; cc < W && ok; cc++)
      for (int j = 0; j < L && ok; j++) {
        const double x = ax * j + bx0;
        for (int l = 0; l < k; l++) {
          const size_t i = (size_t)cc * Hb + (size_t)j * k + l;
          const double f = ((double)l * L + j + 0.5) * fs;
          const double y = ay * ((double)cc * k + l) + by0;
          if (!MK[i] || !near(f, FR[i]) || !near(x, BX[i]) || !near(y, BY[i])) {
            ok = false;
            break;
          }
        }
      }
    if (ok) {
      g.geo_k = k;
      g.geo_L = L;
      g.geo_ax = ax; g.geo_bx = bx0; g.geo_ay = ay; g.geo_by = by0; g.geo_fs = fs;
      return;
    }
  }
}

// Arena carving: every sub-buffer 256-byte aligned.
struct Carve {
  size_t off = 0;
  char* base = nullptr;
  template <class T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += n * sizeof(T);
    return p;
  }
};

struct Batch::Impl {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int compute = 0, frame_dt = SS_F64, tpl_dt = SS_F64;
  std::vector<HostGroup> hg;
  std::vector<GroupDesc> gd;
  std::vector<ss_outputs*> outs;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  bool external_arena = false;
  GroupDesc* d_gd = nullptr;
  GroupCtl* d_ctl = nullptr;
  int* d_chunk_group = nullptr;  // group of each frame chunk (the schedules' source)
  int* d_sched = nullptr;        // the schedule of the next evaluation launch (ss_sched.cuh)
  int* d_tsched = nullptr;       // the trial schedule of the next trial round (ss_sched.cuh)
  int* d_frame_group = nullptr;
  int* d_counters = nullptr;  // kCounters run counters (kCtr*)
  int* d_err = nullptr;       // device error word (bit 0: a shared-memory staging copy timed out)
  unsigned long long* d_staging = nullptr;  // staging counters of the run
  double* d_sum_parts = nullptr;            // partial sums of k_sum_image
  unsigned long long h_staging[kStagingCounters] = {};
  int win_bytes = 0;          // template window bytes per assembly/final CTA (0: no windows)
  int ls_win_bytes = 0;       // template window bytes per line-search CTA (0: no windows)
  int* h_counters = nullptr;  // pinned
  int n_tiles = 0, n_chunks = 0, n_frames_total = 0;
  int n_trial_tiles = 0;  // most tiles a trial round can have
  int max_hb = 0;  // largest block height among groups whose geometry k_eval stages in shared memory
  KernelSet ks = {nullptr, nullptr, nullptr};
  SumFn sum = nullptr;
  std::vector<GroupCtl> h_ctl;
  double init_ms = 0, run_ms = 0;
  int cycles = 0, rounds = 0, launches = 0;
  // optional CUDA-event timing of the evaluation kernels, per EvalMode
  bool timing = false;
  std::vector<cudaEvent_t> events;
  std::vector<int> event_mode;
  size_t event_used = 0;
  double eval_ms[4] = {0, 0, 0, 0};
  // streamed frame uploads (set_stream_frames): the upload stream, its start event, and a ready
  // flag per group written after the group's frames and image sum
  bool stream_req = false;
  cudaStream_t up_stream = nullptr;
  cudaEvent_t ev_up = nullptr;
  int* d_ready = nullptr;
  void* early = nullptr;  // streamed frames, their image sums, sum scratch and ready flags (pool)
  bool pool_arena = false;  // the arena comes from the library's memory pool
  // flag t: CUDA-event timing of the stages, summed into the reference's sub-function slots
  // (output 10, timedmainiteration.cpp:45-143 and task.cpp:293-356); the interval from a mark to the
  // next one counts for the first mark's slot (-1: not counted)
  bool ftime = false;
  std::vector<cudaEvent_t> fevents;
  std::vector<int> fslot;
  size_t fused = 0;
  double ftimes[kFunctionTimes] = {};
  // non-blocking cycle state: 0 prepared, 1 ready to launch a cycle, 2 cycle in flight, 3 finished
  int state = 0;
  int cur_rounds = 0;
  long long cycle_no = 0, max_cycles = 0;
  cudaEvent_t ev_cycle = nullptr;
  std::chrono::steady_clock::time_point t_start;
  // the whole run as one CUDA graph (device-side loops over cycles and trial rounds)
  bool use_graph = true;
  bool graph_run = false;  // the run in flight was launched as the graph
  cudaGraphExec_t run_exec = nullptr;
  cudaStream_t cap_stream = nullptr;

  void fmark(int slot) {
    if (!ftime) return;
    if (fused == fevents.size()) {
      for (int k = 0; k < 64; k++) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        fevents.push_back(e);
        fslot.push_back(-1);
      }
    }
    cudaEventRecord(fevents[fused], stream);
    fslot[fused++] = slot;
  }

  void eval_timed(int mode) {
    if (mode == kTrial && ks.round)
      trial_sched_launch(stream, d_gd, d_ctl, d_frame_group, n_frames_total, (int)gd.size(), d_tsched);
    else if (mode != kTrial)
      sched_launch(mode, stream, d_gd, d_ctl, d_chunk_group, n_chunks, d_sched);
    if (timing) {
      if (event_used + 2 > events.size()) {
        for (int k = 0; k < 64; k++) {
          cudaEvent_t e;
          cudaEventCreate(&e);
          events.push_back(e);
          event_mode.push_back(0);
        }
      }
      cudaEventRecord(events[event_used], stream);
    }
    if (mode == kTrial && ks.round)
      ks.round(n_trial_tiles, stream, d_gd, d_tsched, n_frames_total, (int)gd.size(), d_ctl, win_bytes);
    else if (mode == kTrial) ks.ls(n_frames_total, stream, d_gd, d_frame_group, d_ctl, ls_win_bytes);
    else ks.eval(mode, n_tiles, stream, d_gd, d_sched, n_chunks, d_ctl, max_hb, win_bytes);
    if (timing) {
      cudaEventRecord(events[event_used + 1], stream);
      event_mode[event_used] = mode;
      event_used += 2;
    }
  }
};

Batch::Batch() : d(new Impl) {}
Batch::~Batch() {
  if (d->stream && d->own_stream) cudaStreamSynchronize(d->stream);
  for (cudaEvent_t e : d->events) cudaEventDestroy(e);
  for (cudaEvent_t e : d->fevents) cudaEventDestroy(e);
  if (d->ev_cycle) cudaEventDestroy(d->ev_cycle);
  if (d->run_exec) cudaGraphExecDestroy(d->run_exec);
  if (d->cap_stream) cudaStreamDestroy(d->cap_stream);
  if (d->up_stream) {
    cudaStreamSynchronize(d->up_stream);
    if (d->early) {
      cudaFreeAsync(d->early, d->up_stream);
      cudaStreamSynchronize(d->up_stream);
    }
    cudaStreamDestroy(d->up_stream);
  }
  if (d->ev_up) cudaEventDestroy(d->ev_up);
  if (d->arena && !d->external_arena) {
    if (d->pool_arena) {
      cudaFreeAsync(d->arena, d->stream);
      cudaStreamSynchronize(d->stream);
    } else {
      cudaFree(d->arena);
    }
  }
  if (d->h_counters) cudaFreeHost(d->h_counters);
  if (d->stream && d->own_stream) cudaStreamDestroy(d->stream);
  delete d;
}

size_t Batch::arena_bytes() const { return d->arena_bytes; }
void Batch::set_stream_frames(bool on) { d->stream_req = on; }

// Lays out all device buffers of the batch; with base == nullptr only measures.
static void layout(Batch::Impl* b, char* base) {
  Carve cv;
  cv.base = base;
  const size_t tsz = dtype_size(b->tpl_dt);
  b->n_tiles = 0;
  b->n_trial_tiles = 0;
  b->n_chunks = 0;
  b->n_frames_total = 0;
  std::vector<GroupDesc>& gd = b->gd;
  gd.assign(b->hg.size(), GroupDesc{});
  b->d_err = cv.take<int>(1);
  b->d_counters = cv.take<int>(kCounters);
  b->d_staging = cv.take<unsigned long long>(kStagingCounters);
  b->d_sum_parts = cv.take<double>(kSumBlocks);
  if (!b->early) b->d_ready = b->stream_req ? cv.take<int>(std::max<size_t>(1, b->hg.size())) : nullptr;
  b->win_bytes = 0;
  b->ls_win_bytes = 0;
  for (size_t i = 0; i < b->hg.size(); i++) {
    HostGroup& g = b->hg[i];
    GroupDesc& G = gd[i];
    G.Hb = g.Hb; G.W = g.W; G.nF = g.nF; G.fW = g.fW; G.N = g.N; G.Ht = g.Ht; G.Wt = g.Wt;
    G.group_size = g.group_size; G.n_rg = g.n_rg;
    G.chunk_base = b->n_chunks;
    G.frames_per_cta = g.frames_per_cta;
    G.geo_k = g.geo_k;
    G.geo_L = g.geo_L;
    G.geo_ax = (float)g.geo_ax; G.geo_bx = (float)g.geo_bx; G.geo_ay = (float)g.geo_ay; G.geo_by = (float)g.geo_by;
    G.geo_fs = (float)g.geo_fs;
    b->n_tiles += g.W * ((g.nF + g.frames_per_cta - 1) / g.frames_per_cta);
    b->n_trial_tiles += g.W * ((g.nF + kTrialTileFrames - 1) / kTrialTileFrames);
    b->n_chunks += (g.nF + g.frames_per_cta - 1) / g.frames_per_cta;
    if (!(b->compute == 1 && g.geo_k > 0)) b->max_hb = std::max(b->max_hb, g.Hb);  // affine: no tables
    G.frame_base = b->n_frames_total;
    b->n_frames_total += g.nF;
    const ss_inputs* in = g.in;
    G.max_iter = in->max_iter; G.solver_id = in->solver_id; G.max_filter_iter = in->max_filter_iterations;
    G.filter_id = in->filter_id; G.flags = g.flags; G.frac_uniform = g.frac_uniform ? 1 : 0;
    G.move_thresh = in->move_thresh; G.halt_corr = in->halt_correlation;
    G.corr_inc_thr = in->correlation_increase_threshold; G.filter_strength = in->filter_strength;
    G.filter_corr_thr = in->filter_deactivation_threshold; G.lambda = in->lambda;
    G.ls_mult = in->linesearch_reduction_multiplier;
    const size_t hbw = (size_t)g.Hb * g.W, npx = (size_t)g.Hb * g.fW, N = g.N, nF = g.nF;
    const size_t nq = (size_t)(g.Ht - 1) * (g.Wt - 1);
    if (g.geo_src != -1) {  // shared with an earlier group or held by a session
      const GroupDesc& S = g.geo_src == kFromSession ? *g.ses_gd : gd[g.geo_src];
      G.frac = S.frac; G.basex = S.basex; G.basey = S.basey;
      G.frac_f = S.frac_f; G.basex_f = S.basex_f; G.basey_f = S.basey_f;
      G.base_mask = S.base_mask; G.min_points = S.min_points;
      G.col_yrange = S.col_yrange;
    } else {
      G.frac = cv.take<double>(hbw);
      G.basex = cv.take<double>(hbw);
      G.basey = cv.take<double>(hbw);
      if (b->compute == 1) {
        G.frac_f = cv.take<float>(hbw);
        G.basex_f = cv.take<float>(hbw);
        G.basey_f = cv.take<float>(hbw);
      } else {
        G.frac_f = G.basex_f = G.basey_f = nullptr;
      }
      G.base_mask = cv.take<uint8_t>(hbw);
      G.min_points = cv.take<int>(g.W);
      G.col_yrange = b->compute == 1 ? cv.take<float>(2 * (size_t)g.W) : nullptr;
    }
    G.err = b->d_err;
    G.ls_rounds = b->compute == 1 ? 1 : 0;
    G.ls_max_trials = b->d_counters;
    G.staging = b->d_staging;
    g.d_image = (g.frames_dev || g.early_image) ? nullptr : cv.take<char>(g.frame_bytes);
    G.image = g.frames_dev ? g.frames_dev : (g.early_image ? g.early_image : g.d_image);
    {
      const size_t fsz = dtype_size(g.frame_dt);
      G.pair_ok = (b->compute == 1 && g.geo_k > 0 && g.Hb % 64 == 0 &&
                   reinterpret_cast<uintptr_t>(G.image) % (2 * fsz) == 0) ? 1 : 0;
      G.quad_ok = (G.pair_ok && fsz == 2 && g.geo_k <= 2 && g.Hb % 256 == 0 &&
                   reinterpret_cast<uintptr_t>(G.image) % 16 == 0) ? 1 : 0;
    }
    if (g.tpl_src != -1) {
      const GroupDesc& S = g.tpl_src == kFromSession ? *g.ses_gd : gd[g.tpl_src];
      G.tquad = S.tquad;
      G.gquad = S.gquad;
      G.tplain = S.tplain;
      G.tpitch = S.tpitch;
    } else {
      G.tquad = cv.take<char>(nq * 4 * tsz);
      G.gquad = g.grad_derived ? nullptr : cv.take<char>(nq * 4 * tsz);
      // precision 'S' with an FP32 template and derived gradients samples row windows in shared
      // memory: rows padded to 16 bytes for the bulk copies
      G.tpitch = (g.Wt + 3) & ~3;
      // (the layout's measuring pass takes no memory: decide by the condition, not by the pointer)
      const bool rows = b->compute == 1 && b->tpl_dt == SS_F32 && g.grad_derived && 2 * G.tpitch * 4 <= kWinBytes;
      G.tplain = rows ? cv.take<float>((size_t)g.Ht * G.tpitch) : nullptr;
      g.d_templ_stage = cv.take<double>((size_t)g.Ht * g.Wt);
      if (!g.grad_derived) {
        g.d_xg_stage = cv.take<double>((size_t)g.Ht * g.Wt);
        g.d_yg_stage = cv.take<double>((size_t)g.Ht * g.Wt);
      }
    }
    if (G.tplain) b->win_bytes = kWinBytes;  // the line search runs from the global template
    g.d_sum = g.early_sum ? g.early_sum : cv.take<double>(1);
    G.sum_image = g.d_sum;
    g.d_p0 = cv.take<double>(2 * N);
    G.p0 = g.d_p0;
    G.p = cv.take<double>(2 * N);
    G.p_last = cv.take<double>(2 * N);
    G.p_snap = cv.take<double>(2 * N);
    G.delta_p = cv.take<double>(2 * N);
    G.ndp = cv.take<double>(2 * N);
    G.colsum = cv.take<double>((size_t)g.fW * kCsStride);
    G.colcnt = cv.take<int>(g.fW);
    G.asmsum = cv.take<double>((size_t)g.fW * kCsStride);
    G.asmcnt = cv.take<int>(g.fW);
    G.asmk = cv.take<double>((size_t)g.fW * 8);
    G.params_used = cv.take<uint8_t>(N);
    G.blocks_present = cv.take<uint8_t>(N);
    G.grp_active = cv.take<uint8_t>(2 * (size_t)g.n_rg + 1);
    G.errval = cv.take<double>(2 * nF);
    G.kmask = cv.take<double>(nF * 2 * (g.W + 1));
    G.kdiff = cv.take<double>(nF * 2 * (g.W + 1));
    // written by every correlation pass before a stale frame reads it: no initial value
    G.dparity = (g.flags & kFlagMaskInactive) ? cv.take<uint32_t>(2 * (size_t)g.fW * ((g.Hb + 31) / 32)) : nullptr;
    G.fstate = cv.take<uint8_t>(nF);
    G.ls_trials = cv.take<int>(nF);
    G.ls_done = cv.take<int>(nF);
    G.eig_c = cv.take<double>(4 * N);
    G.eig_valid = cv.take<uint8_t>(N);
    G.list = cv.take<int>(2 * N);
    // the solve's planes; between solves, the partial sums of the iteration end (k_iter_sums)
    G.cr = cv.take<double>(std::max<size_t>((size_t)kCrStride * N, 8 * (size_t)kIterSplit));
    G.ilu = in->solver_id == 0 ? cv.take<double>(11 * N) : nullptr;
    const ss_outputs* o = b->outs[i];
    const int mi = in->max_iter;
    G.o_frame_corr = cv.take<double>(nF);
    G.o_residrms = cv.take<double>(nF);
    G.o_dx = cv.take<double>((g.W + 1) * nF);
    G.o_dy = cv.take<double>((g.W + 1) * nF);
    G.o_iter_corr = (o && o->iteration_corr) ? cv.take<double>(mi) : nullptr;
    G.o_frame_corr_hist = (o && o->frame_corr_history) ? cv.take<double>((size_t)mi * nF) : nullptr;
    G.o_iter_errvals = (o && o->iteration_errvals) ? cv.take<double>((size_t)2 * mi * nF) : nullptr;
    G.o_all_params = (o && o->all_params) ? cv.take<double>((size_t)2 * N * mi) : nullptr;
    G.o_frame_params = (o && o->frame_params) ? cv.take<double>(2 * (size_t)(g.W + 1) * nF) : nullptr;
    G.o_raw = (o && o->raw_params) ? cv.take<double>(2 * N) : nullptr;
    G.o_mask = (o && o->mask) ? cv.take<uint8_t>(npx) : nullptr;
    G.o_blocks_used = (o && o->blocks_used) ? cv.take<uint8_t>(g.fW) : nullptr;
    const bool timed = g.flags & kFlagTimeSub, exec_timed = g.flags & kFlagTimeExec;
    G.o_rg_params = (o && o->rg_params && timed) ? cv.take<double>((size_t)2 * N * 2 * mi) : nullptr;
    G.o_iter_times = (o && o->iteration_times && timed && exec_timed) ? cv.take<double>(mi) : nullptr;
    if (timed && o && o->function_times) b->ftime = true;
  }
  b->d_gd = cv.take<GroupDesc>(gd.size());
  b->d_ctl = cv.take<GroupCtl>(gd.size());
  b->d_chunk_group = cv.take<int>(std::max(1, b->n_chunks));
  b->d_sched = cv.take<int>(sched_ints(b->n_chunks));
  b->d_tsched = cv.take<int>(tsched_ints(b->n_frames_total, (int)gd.size()));
  b->d_frame_group = cv.take<int>(std::max(1, b->n_frames_total));
  b->arena_bytes = cv.off + 256;
}

__global__ void k_set_flag(int* __restrict__ flag) { *flag = 1; }

// Streamed frames: as soon as the groups are validated, one pool allocation on the upload stream
// holds every host-resident group's frames (256-byte aligned), their image sums, the sums' scratch
// and the ready flags; the upload stream then copies each group's frames, sums them and sets its
// flag, in group order, while the host prepares the rest of the batch. Groups whose frames are on
// the device only get their flag. ev_up, recorded right after the allocation, orders the buffer
// before the batch stream's work.
static int start_frame_uploads(Batch::Impl* b, int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SS_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(SS_ERR_INVALID_ARGUMENT, "gpu_device_id out of range");
  SS_CK(cudaSetDevice(device));
  SumFn sum = pick_sum(b->hg[0].frame_dt);
  if (!sum) return fail(SS_ERR_INVALID_ARGUMENT, "unsupported frame dtype");
  const size_t n = b->hg.size();
  auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
  size_t bytes = up(n * sizeof(int)) + up(kSumBlocks * sizeof(double)) + up(n * sizeof(double));
  for (const HostGroup& g : b->hg) {
    if (g.frame_bytes == 0 || g.frame_bytes != (size_t)g.Hb * g.fW * dtype_size(g.frame_dt))
      return fail(SS_ERR_INVALID_ARGUMENT, "streamed frames: group not validated");
    if (!g.frames_dev) bytes += up(g.frame_bytes);
  }
  SS_CK(cudaStreamCreateWithFlags(&b->up_stream, cudaStreamNonBlocking));
  SS_CK(cudaEventCreateWithFlags(&b->ev_up, cudaEventDisableTiming));
  cudaMemPool_t pool = work_pool(device);
  if (!pool) return fail(SS_ERR_OUT_OF_MEMORY, "no device memory pool");
  if (cudaMallocFromPoolAsync(&b->early, bytes, pool, b->up_stream) != cudaSuccess)
    return fail(SS_ERR_OUT_OF_MEMORY, "device memory for the streamed frames");
  SS_CK(cudaEventRecord(b->ev_up, b->up_stream));
  char* p = static_cast<char*>(b->early);
  b->d_ready = reinterpret_cast<int*>(p);
  p += up(n * sizeof(int));
  double* parts = reinterpret_cast<double*>(p);
  p += up(kSumBlocks * sizeof(double));
  double* sums = reinterpret_cast<double*>(p);
  p += up(n * sizeof(double));
  SS_CK(cudaMemsetAsync(b->d_ready, 0, n * sizeof(int), b->up_stream));
  for (size_t i = 0; i < n; i++) {
    HostGroup& g = b->hg[i];
    if (!g.frames_dev) {
      g.early_image = p;
      g.early_sum = sums + i;
      p += up(g.frame_bytes);
      SS_CK(cudaMemcpyAsync(g.early_image, g.in->bm_data.data, g.frame_bytes, cudaMemcpyHostToDevice, b->up_stream));
      sum(g.early_image, (size_t)g.Hb * g.fW, parts, g.early_sum, b->up_stream);
    }
    k_set_flag<<<1, 1, 0, b->up_stream>>>(b->d_ready + i);
  }
  SS_CK(cudaGetLastError());
  return SS_OK;
}

// ParameterOrganizer::organize2D1 (parameterorganizer.cpp:31-55): the initial knots of every frame
// as the group's parameter vector (x then y; a frame's last knot and the next frame's first become
// one parameter at their mean).
static void organize_p0(const HostGroup& g, double* p0) {
  const double* ex = g.ex.data();
  const double* ey = g.ey.data();
  std::memset(p0, 0, 2 * (size_t)g.N * sizeof(double));
  for (int f = 0; f < g.nF; f++) {
    int j = f * g.W + (f != 0);
    for (int i = (f != 0); i < g.W; i++, j++) {
      p0[j] = ex[(size_t)f * (g.W + 1) + i];
      p0[j + g.N] = ey[(size_t)f * (g.W + 1) + i];
    }
    if (f < g.nF - 1) {
      p0[j] = (ex[(size_t)f * (g.W + 1) + g.W] + ex[(size_t)(f + 1) * (g.W + 1)]) / 2;
      p0[j + g.N] = (ey[(size_t)f * (g.W + 1) + g.W] + ey[(size_t)(f + 1) * (g.W + 1)]) / 2;
    } else {
      p0[j] = ex[(size_t)f * (g.W + 1) + g.W];
      p0[j + g.N] = ey[(size_t)f * (g.W + 1) + g.W];
    }
  }
}

// Page-locked host staging for a batch's small uploads (geometry, template, initial knots,
// descriptors): one buffer per process, held by one batch at a time from its first staged copy
// until the batch's stream has drained, so those copies run as DMA from page-locked memory rather
// than through the driver's pageable path (which stalls behind streamed frame uploads). A copy
// that does not fit goes the pageable way; the buffer then grows to the batch's total for the
// next batch. A batch on a borrowed stream, which does not drain it, copies the pageable way.
static std::mutex g_stage_mu;
static char* g_stage = nullptr;
static size_t g_stage_cap = 0;
constexpr size_t kStageItemMax = size_t(16) << 20;  // larger copies (frames, masks) go direct
constexpr size_t kStageMax = size_t(128) << 20;

struct Staging {
  std::unique_lock<std::mutex> lock;
  cudaStream_t stream = nullptr;
  size_t off = 0, want = 0;
  bool on = false;
  explicit Staging(cudaStream_t s, bool enable) : stream(s), on(enable) {
    if (on) lock = std::unique_lock<std::mutex>(g_stage_mu);
  }
  // staging space for n bytes (16-byte aligned), or null when it does not fit
  void* take(size_t n) {
    if (!on || n > kStageItemMax) return nullptr;
    const size_t m = (n + 15) & ~size_t(15);
    want += m;
    if (off + m > g_stage_cap) return nullptr;
    void* p = g_stage + off;
    off += m;
    return p;
  }
  // host-to-device copy of n bytes through the staging buffer when it has room
  cudaError_t put(void* dst, const void* src, size_t n) {
    if (!n) return cudaSuccess;
    void* p = take(n);
    if (p) {
      std::memcpy(p, src, n);
      src = p;
    }
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, stream);
  }
  // after the stream has drained: grows the buffer when the batch wanted more
  void release() {
    if (!on) return;
    if (want > g_stage_cap && g_stage_cap < kStageMax) {
      if (g_stage) cudaFreeHost(g_stage);
      g_stage = nullptr;
      g_stage_cap = 0;
      const size_t cap = std::min(want + want / 4, kStageMax);
      if (cudaHostAlloc((void**)&g_stage, cap, cudaHostAllocPortable) == cudaSuccess) g_stage_cap = cap;
      else g_stage = nullptr;
      cudaGetLastError();  // a failed allocation leaves the pageable path; clear its error
    }
    on = false;
    lock.unlock();
  }
  ~Staging() {
    if (!on) return;
    cudaStreamSynchronize(stream);  // an early return: no copy may still read the buffer
    on = false;
    lock.unlock();
  }
};

int Batch::prepare(int n, const ss_inputs* in, ss_outputs* out, void* external, size_t external_bytes,
                   const Batch* const* sessions, bool measure_only, void* borrow_stream) {
  Impl* b = d;
  if (n < 1) return fail(SS_ERR_INVALID_ARGUMENT, "no groups");
  b->hg.assign(n, HostGroup{});
  b->outs.assign(n, nullptr);
  for (int i = 0; i < n; i++) {
    int rc = validate_group(&in[i], b->hg[i]);
    if (rc) return rc;
    b->outs[i] = out ? &out[i] : nullptr;
    if (sessions && sessions[i]) {  // template and geometry resident in a session
      const Impl* S = sessions[i]->d;
      if (S->hg.empty()) return fail(SS_ERR_INVALID_ARGUMENT, "session is not prepared");
      const HostGroup& sh = S->hg[0];
      HostGroup& g = b->hg[i];
      if (sh.Ht != g.Ht || sh.Wt != g.Wt || sh.Hb != g.Hb || sh.W != g.W)
        return fail(SS_ERR_INVALID_ARGUMENT, "group and session differ in template or frame geometry");
      if (sh.compute != g.compute || sh.tpl_dt != g.tpl_dt || S->device != in[i].gpu_device_id)
        return fail(SS_ERR_INVALID_ARGUMENT, "group and session differ in precision, template storage or device");
      g.tpl_src = g.geo_src = kFromSession;
      g.ses_gd = &S->gd[0];
      g.ses_hg = &sh;
    }
    if (i > 0) {
      const HostGroup& a = b->hg[0];
      const HostGroup& c = b->hg[i];
      if (c.compute != a.compute || c.frame_dt != a.frame_dt || c.tpl_dt != a.tpl_dt ||
          in[i].gpu_device_id != in[0].gpu_device_id)
        return fail(SS_ERR_INVALID_ARGUMENT, "all groups of a batch need the same precision, frame dtype and device");
    }
  }
  if (b->stream_req && !measure_only) {  // the frames travel while the host prepares the rest
    int rc = start_frame_uploads(b, in[0].gpu_device_id);
    if (rc) return rc;
  }
  find_shared_inputs(b->hg);
  for (int i = 0; i < n; i++) {
    int rc = load_host_inputs(b->hg, i);
    if (rc) return rc;
  }
  b->compute = b->hg[0].compute;
  b->frame_dt = b->hg[0].frame_dt;
  b->tpl_dt = b->hg[0].tpl_dt;
  b->ks = pick_kernels(b->compute, b->frame_dt, b->tpl_dt);
  b->sum = pick_sum(b->frame_dt);
  if (!b->ks.eval || !b->sum) return fail(SS_ERR_INVALID_ARGUMENT, "unsupported dtype combination");
  if (measure_only) {
    layout(b, nullptr);
    return SS_OK;
  }

  auto t0 = std::chrono::steady_clock::now();
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SS_ERR_NO_DEVICE, "no CUDA device");
  b->device = in[0].gpu_device_id;
  if (b->device < 0 || b->device >= ndev) return fail(SS_ERR_INVALID_ARGUMENT, "gpu_device_id out of range");
  SS_CK(cudaSetDevice(b->device));
  if (borrow_stream) {  // a server slot: the server's stream, no blocking
    b->stream = static_cast<cudaStream_t>(borrow_stream);
    b->own_stream = false;
  } else {
    SS_CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  // the early buffer was allocated on the upload stream: order it before this stream's work (the
  // event precedes the uploads, which the ready flags order)
  if (b->early) SS_CK(cudaStreamWaitEvent(b->stream, b->ev_up, 0));
  layout(b, nullptr);
  if (external) {
    if (external_bytes < b->arena_bytes) return fail(SS_ERR_OUT_OF_MEMORY, "external arena too small");
    b->arena = external;
    b->external_arena = true;
  } else {
    cudaMemPool_t pool = work_pool(b->device);
    if (!pool) return fail(SS_ERR_OUT_OF_MEMORY, "no device memory pool");
    if (cudaMallocFromPoolAsync(&b->arena, b->arena_bytes, pool, b->stream) != cudaSuccess)
      return fail(SS_ERR_OUT_OF_MEMORY, "device arena");
    b->pool_arena = true;
  }
  char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(b->arena) + 255) & ~uintptr_t(255));
  layout(b, base);
  b->init_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

  // uploads
  cudaStream_t s = b->stream;
  Staging stg(s, b->own_stream);
  std::vector<int> chunk_group(std::max(1, b->n_chunks)), frame_group(std::max(1, b->n_frames_total));
  for (size_t i = 0; i < b->hg.size(); i++) {
    HostGroup& g = b->hg[i];
    GroupDesc& G = b->gd[i];
    const size_t hbw = (size_t)g.Hb * g.W;
    if (g.geo_src == -1) {
      SS_CK(stg.put((void*)G.frac, g.frac.data(), hbw * 8));
      SS_CK(stg.put((void*)G.basex, g.bx.data(), hbw * 8));
      SS_CK(stg.put((void*)G.basey, g.by.data(), hbw * 8));
      if (b->compute == 1) {  // precision 'S' geometry, converted straight into the staging buffer
        const double* src[3] = {g.frac.data(), g.bx.data(), g.by.data()};
        const float* dst[3] = {G.frac_f, G.basex_f, G.basey_f};
        std::vector<float>* keep[3] = {&g.frac_f, &g.bx_f, &g.by_f};
        for (int a = 0; a < 3; a++) {
          float* h = static_cast<float*>(stg.take(hbw * 4));
          if (!h) {
            keep[a]->resize(hbw);
            h = keep[a]->data();
          }
          for (size_t e = 0; e < hbw; e++) h[e] = (float)src[a][e];
          SS_CK(cudaMemcpyAsync((void*)dst[a], h, hbw * 4, cudaMemcpyHostToDevice, s));
        }
      }
      SS_CK(stg.put((void*)G.base_mask, g.bmask.data(), hbw));
      SS_CK(stg.put((void*)G.min_points, g.minp.data(), g.W * 4));
      if (G.col_yrange) {  // [min, max] of basey over the valid rows of each block column
        const double* BY = g.by.data();
        g.yrange.assign(2 * (size_t)g.W, 0.0f);
        for (int c = 0; c < g.W; c++) {
          double lo = INFINITY, hi = -INFINITY;
          for (int r = 0; r < g.Hb; r++) {
            const size_t i = (size_t)c * g.Hb + r;
            if (!g.bmask[i]) continue;
            lo = std::min(lo, BY[i]);
            hi = std::max(hi, BY[i]);
          }
          g.yrange[2 * c] = (float)lo;
          g.yrange[2 * c + 1] = (float)hi;
        }
        SS_CK(stg.put((void*)G.col_yrange, g.yrange.data(), g.yrange.size() * 4));
      }
    }
    const bool streamed = g.early_image != nullptr;  // uploaded by start_frame_uploads
    if (!g.frames_dev && !streamed)
      SS_CK(cudaMemcpyAsync(g.d_image, g.in->bm_data.data, g.frame_bytes, cudaMemcpyHostToDevice, s));
    {  // the initial parameter vector, organised straight into the staging buffer
      const size_t np = 2 * (size_t)g.N;
      double* h = static_cast<double*>(stg.take(np * 8));
      std::vector<double> p0;
      if (!h) {
        p0.resize(np);
        h = p0.data();
      }
      organize_p0(g, h);
      SS_CK(cudaMemcpyAsync(g.d_p0, h, np * 8, cudaMemcpyHostToDevice, s));
    }
    if (g.tpl_src == -1) {
      SS_CK(stg.put(g.d_templ_stage, g.templ.data(), g.templ.size() * 8));
      if (!g.grad_derived) {
        SS_CK(stg.put(g.d_xg_stage, g.xg.data(), g.xg.size() * 8));
        SS_CK(stg.put(g.d_yg_stage, g.yg.data(), g.yg.size() * 8));
      }
    }
    const int nb = 148 * 4;
    if (g.tpl_src != -1) {
      // template quads shared with an earlier group or held by a session
    } else if (b->tpl_dt == SS_F64) {
      k_build_tquad<double><<<nb, 256, 0, s>>>(g.d_templ_stage, g.Ht, g.Wt, (double*)G.tquad);
      if (!g.grad_derived)
        k_build_gquad<double><<<nb, 256, 0, s>>>(g.d_xg_stage, g.d_yg_stage, g.Ht, g.Wt, (double*)G.gquad);
    } else if (b->tpl_dt == SS_F32) {
      k_build_tquad<float><<<nb, 256, 0, s>>>(g.d_templ_stage, g.Ht, g.Wt, (float*)G.tquad);
      if (G.tplain) k_build_tplain<<<nb, 256, 0, s>>>(g.d_templ_stage, g.Ht, g.Wt, G.tpitch, (float*)G.tplain);
      if (!g.grad_derived)
        k_build_gquad<float><<<nb, 256, 0, s>>>(g.d_xg_stage, g.d_yg_stage, g.Ht, g.Wt, (float*)G.gquad);
    } else {
      k_build_tquad<__half><<<nb, 256, 0, s>>>(g.d_templ_stage, g.Ht, g.Wt, (__half*)G.tquad);
      if (!g.grad_derived)
        k_build_gquad<__half><<<nb, 256, 0, s>>>(g.d_xg_stage, g.d_yg_stage, g.Ht, g.Wt, (__half*)G.gquad);
    }
    SS_CK(cudaGetLastError());
    if (!streamed) b->sum(G.image, (size_t)g.Hb * g.fW, b->d_sum_parts, g.d_sum, s);
    SS_CK(cudaGetLastError());
    const int nchunks = (g.nF + g.frames_per_cta - 1) / g.frames_per_cta;
    for (int t = 0; t < nchunks; t++) chunk_group[G.chunk_base + t] = (int)i;
    for (int f = 0; f < g.nF; f++) frame_group[G.frame_base + f] = (int)i;
  }
  SS_CK(stg.put(b->d_gd, b->gd.data(), b->gd.size() * sizeof(GroupDesc)));
  SS_CK(stg.put(b->d_chunk_group, chunk_group.data(), chunk_group.size() * 4));
  SS_CK(stg.put(b->d_frame_group, frame_group.data(), frame_group.size() * 4));
  // pageable sources are staged before the copies return; an own stream is also drained, after
  // which the staging buffer is free for the next batch
  if (b->own_stream) SS_CK(cudaStreamSynchronize(s));
  stg.release();
  return SS_OK;
}

// Resets the iteration state of every group to the call's start (task_allocate.cu:201-255).
static int reset_state(Batch::Impl* b) {
  cudaStream_t s = b->stream;
  b->h_ctl.assign(b->gd.size(), GroupCtl{});
  // the device buffers of every group (d_gd is on the device since the batch was prepared)
  const int nG = (int)b->gd.size();
  for (int g0 = 0; g0 < nG; g0 += 65535)
    k_reset_groups<<<dim3(16, std::min(nG - g0, 65535)), 256, 0, s>>>(b->d_gd + g0);
  SS_CK(cudaGetLastError());
  for (size_t i = 0; i < b->gd.size(); i++) {
    const HostGroup& g = b->hg[i];
    GroupCtl& C = b->h_ctl[i];
    std::memset(&C, 0, sizeof(C));
    C.phase = b->stream_req && !g.frames_dev ? kPhWait : kPhHalf;
    C.iteration = 1;
    C.improved = 1;
    C.stop_reason = kStopError;
    C.eig_size = -1;
    const ss_inputs* in = g.in;
    C.filter_id = in->filter_id;
    C.n_filter_iter = in->max_filter_iterations;
    int fsel = in->filter_id & (0 - (in->max_filter_iterations != 0));  // task.cpp:54-70
    if (fsel == 0) {
      C.filter_active = 0;
      C.n_filter_iter = 0;
    } else {
      C.filter_active = 1;
      C.filter_kind = fsel;
    }
  }
  SS_CK(cudaMemcpyAsync(b->d_ctl, b->h_ctl.data(), b->h_ctl.size() * sizeof(GroupCtl), cudaMemcpyHostToDevice, s));
  SS_CK(cudaMemsetAsync(b->d_counters, 0, kCounters * sizeof(int), s));
  SS_CK(cudaMemsetAsync(b->d_err, 0, sizeof(int), s));
  SS_CK(cudaMemsetAsync(b->d_staging, 0, kStagingCounters * sizeof(unsigned long long), s));
  return SS_OK;
}

// Dynamic shared memory of k_solve_system and k_block_tridiag: the separator system of the partitioned
// solve and the partitions' first-interior relations.
constexpr size_t kSolveSmem = (size_t)kSolveThreads * kPartSmemStride * sizeof(double);

// The half-step solve of every group in phase kPhHalf: set-up over kSolveSplit CTAs per group,
// compaction in one CTA, the blocks over kSolveSplit CTAs, the partitioned solve and filters in one
// CTA, the expansion over kSolveSplit CTAs (ss_group.cuh).
static void solve_launch(cudaStream_t s, const GroupDesc* gd, GroupCtl* ctl, int nG) {
  const dim3 split(kSolveSplit, nG);
  k_solve_prep<<<split, kSolvePrepThreads, 0, s>>>(gd, ctl);
  k_solve_compact<<<nG, kSolveThreads, 0, s>>>(gd, ctl);
  k_solve_planes<<<split, kSolvePrepThreads, 0, s>>>(gd, ctl);
  k_solve_system<<<nG, kSolveThreads, kSolveSmem, s>>>(gd, ctl);
  k_solve_expand<<<split, kSolvePrepThreads, 0, s>>>(gd, ctl);
}

// Opts k_block_tridiag into kSolveSmem of dynamic shared memory.
static cudaError_t block_tridiag_attr() { return smem_attr(k_block_tridiag, (int)kSolveSmem); }

// Trial rounds per cycle of the precision 'S' line search: the first cycle's, and the range of the
// later ones (set from the longest search that ended in the cycle before).
constexpr int kFirstRounds = 8, kMinRounds = 3, kMaxRounds = 16;

// Groups whose streamed frames have arrived (ready flag, written on the upload stream after the
// frames and their image sum) join the run at the start of the cycle; ctr[kCtrWaiting] counts those
// still waiting. One CTA.
__global__ void __launch_bounds__(1024) k_join(GroupCtl* __restrict__ ctl, const int* __restrict__ ready, int n_groups,
                                               int* __restrict__ ctr) {
  int waiting = 0;
  for (int g = threadIdx.x; g < n_groups; g += blockDim.x) {
    if (ctl[g].phase != kPhWait) continue;
    if (ld_acquire(ready + g)) ctl[g].phase = kPhHalf;
    else waiting++;
  }
  for (int o = 16; o > 0; o >>= 1) waiting += __shfl_xor_sync(0xffffffffu, waiting, o);
  __shared__ int sw[32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = waiting;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sw[w];
    ctr[kCtrWaiting] = t;
  }
}


// Enqueues one cycle of every group's state machine on the batch stream (assembly, solve, trial
// rounds or the cluster line search, correlation, iteration end, final pass) and the copy of the
// cycle's counters to pinned memory.
static int enqueue_cycle(Batch::Impl* b) {
  cudaStream_t s = b->stream;
  const int nG = (int)b->gd.size();
  // flag t's sub-function slots (output 10): 1 applyParameters, here with the errval, gradient and
  // JᵀJ / Jᵀr sums of the same pass; 2 the group errvals and parameter mask; 4 the compaction;
  // 5 the system's blocks (fillDiagonals, fillJtr); 7 the solve and its filter; 8 the expansion;
  // 9 the line search; 10 the correlation; 11 the rest of the iteration end
  if (b->d_ready) k_join<<<1, 1024, 0, s>>>(b->d_ctl, b->d_ready, nG, b->d_counters);
  b->fmark(1);
  b->eval_timed(kAssemble);
  if (b->ftime) {
    const dim3 split(kSolveSplit, nG);
    b->fmark(2);
    k_solve_prep<<<split, kSolvePrepThreads, 0, s>>>(b->d_gd, b->d_ctl);
    b->fmark(4);
    k_solve_compact<<<nG, kSolveThreads, 0, s>>>(b->d_gd, b->d_ctl);
    b->fmark(5);
    k_solve_planes<<<split, kSolvePrepThreads, 0, s>>>(b->d_gd, b->d_ctl);
    b->fmark(7);
    k_solve_system<<<nG, kSolveThreads, kSolveSmem, s>>>(b->d_gd, b->d_ctl);
    b->fmark(8);
    k_solve_expand<<<split, kSolvePrepThreads, 0, s>>>(b->d_gd, b->d_ctl);
  } else {
    solve_launch(s, b->d_gd, b->d_ctl, nG);
  }
  SS_CK(cudaGetLastError());
  b->fmark(9);
  if (b->ks.round) {
    // trial rounds without a host round trip: as many as the longest search of the previous
    // cycle took; a search that needs more continues in the next cycle (its group skips
    // assembly and solve until it has finished)
    SS_CK(cudaMemsetAsync(b->d_counters, 0, sizeof(int), s));
    for (int r = 0; r < b->cur_rounds; r++) b->eval_timed(kTrial);
    b->fmark(10);
    b->eval_timed(kCorr);  // correlation sums after the second half-step
    b->fmark(9);
  } else {
    b->eval_timed(kTrial);  // line search (and, after shift 1, the correlation sums)
  }
  SS_CK(cudaGetLastError());
  k_after_ls<<<nG, kAfterLsThreads, 0, s>>>(b->d_gd, b->d_ctl);
  b->fmark(10);
  k_iter_sums<<<dim3(kIterSplit, nG), 256, 0, s>>>(b->d_gd, b->d_ctl);
  b->fmark(11);
  k_iter_end<<<nG, kSolveThreads, 0, s>>>(b->d_gd, b->d_ctl);
  b->fmark(-1);
  b->eval_timed(kFinal);
  k_final<<<nG, kSolveThreads, 0, s>>>(b->d_gd, b->d_ctl, b->d_counters + 1);
  SS_CK(cudaGetLastError());
  SS_CK(cudaMemcpyAsync(b->h_counters, b->d_counters, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  return SS_OK;
}

// Launches one cycle and records the cycle event. No host synchronisation.
static int launch_cycle(Batch::Impl* b) {
  b->cycles++;
  b->rounds += b->ks.round ? b->cur_rounds : 1;
  // schedules and evaluation passes (2 each), the solve (5), after-ls, iteration end (2), final; the
  // line search (precision 'D') or the correlation pass and two launches per trial round ('S')
  b->launches += b->ks.round ? 2 * b->cur_rounds + 15 : 14;
  int rc = enqueue_cycle(b);
  if (rc) return rc;
  if (!b->ev_cycle) SS_CK(cudaEventCreateWithFlags(&b->ev_cycle, cudaEventDisableTiming));
  SS_CK(cudaEventRecord(b->ev_cycle, b->stream));
  return SS_OK;
}

// ---------------------------------------------------------------------------------------------
// The whole run as one CUDA graph: a WHILE node over cycles whose body is the cycle, and inside it
// (precision 'S') a WHILE node over trial rounds. One-thread control kernels set both conditions
// from the groups' state on the device, so the run needs no host round trip until every group has
// stopped. Both loops are bounded by counters (cycles by the batch's cycle bound, rounds per cycle
// by kGraphRounds, after which a search continues in the next cycle).

constexpr int kGraphRounds = 64;

// Schedule of the next trial round and the condition of the trial-round loop: another round while
// a frame is searching and the cycle is under its round bound. `first` starts the cycle's count.
__global__ void __launch_bounds__(kSchedThreads) k_sched_rounds(const GroupDesc* __restrict__ gds,
                                                                const GroupCtl* __restrict__ ctl,
                                                                const int* __restrict__ frame_group, int n_frames,
                                                                int n_groups, int* __restrict__ tsched,
                                                                int* __restrict__ ctr, int first,
                                                                cudaGraphConditionalHandle h) {
  const int tiles = build_trial_schedule(gds, ctl, frame_group, n_frames, n_groups, tsched);
  if (threadIdx.x == 0) {
    if (first) ctr[kCtrRound] = 0;
    const bool more = tiles > 0 && ctr[kCtrRound] < kGraphRounds;
    if (more) {
      ctr[kCtrRound]++;
      ctr[kCtrRounds]++;
    } else if (tiles > 0) {
      ctr[kCtrBound] |= 2;
    }
    cudaGraphSetConditional(h, more ? 1u : 0u);
  }
}

// Condition of the cycle loop: another cycle while a group is running, up to `max_cycles`. A cycle
// in which every running group still waits for its frames does not count toward the bound.
__global__ void k_cycle_ctl(int* __restrict__ ctr, int n_groups, int max_cycles, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  const bool idle = ctr[kCtrWaiting] > 0 && ctr[kCtrWaiting] + ctr[kCtrDone] >= n_groups;
  const int c = idle ? ctr[kCtrCycles] : ++ctr[kCtrCycles];
  const bool running = ctr[kCtrDone] < n_groups;
  if (running && c >= max_cycles) ctr[kCtrBound] |= 1;
  cudaGraphSetConditional(h, running && c < max_cycles ? 1u : 0u);
}

// Adds a WHILE node after the work captured so far on `s` and makes it the capture's dependency;
// returns its body graph.
static int capture_while(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t n_deps = 0;
  SS_CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &n_deps));
  if (st != cudaStreamCaptureStatusActive) return fail(SS_ERR_CUDA, "run graph: stream is not capturing");
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  SS_CK(cudaGraphAddNode(&node, g, deps, n_deps, &p));
  *body = p.conditional.phGraph_out[0];
  SS_CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return SS_OK;
}

// Opts every kernel of the run into its shared memory before capture (no attribute calls inside).
static int prime_attributes(Batch::Impl* b) {
  SS_CK(smem_attr(k_solve_system, (int)kSolveSmem));
  SS_CK(b->ks.eval(kAssemble, 0, b->stream, b->d_gd, b->d_sched, b->n_chunks, b->d_ctl, b->max_hb, b->win_bytes));
  if (b->ks.round)
    SS_CK(b->ks.round(0, b->stream, b->d_gd, b->d_tsched, b->n_frames_total, (int)b->gd.size(), b->d_ctl,
                      b->win_bytes));
  else SS_CK(b->ks.ls(0, b->stream, b->d_gd, b->d_frame_group, b->d_ctl, b->ls_win_bytes));
  return SS_OK;
}

static int build_run_graph(Batch::Impl* b) {
  int rc = prime_attributes(b);
  if (rc) return rc;
  if (!b->cap_stream) SS_CK(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
  cudaStream_t s = b->cap_stream;
  const int nG = (int)b->gd.size();
  // two half-steps per iteration, a line search of up to kTrialCap trials each
  int max_iter = 1;
  for (auto& g : b->hg) max_iter = std::max(max_iter, g.in->max_iter);
  const int max_cycles = 4 * (max_iter + 2) * (1 + kTrialCap / kGraphRounds) + 16;
  cudaGraph_t top = nullptr, body = nullptr, rounds_body = nullptr;
  SS_CK(cudaGraphCreate(&top, 0));
  struct GraphGuard {
    cudaGraph_t g;
    ~GraphGuard() { cudaGraphDestroy(g); }
  } guard{top};
  cudaGraphConditionalHandle h_cycle = 0, h_round = 0;
  SS_CK(cudaGraphConditionalHandleCreate(&h_cycle, top, 1, cudaGraphCondAssignDefault));
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  // top: counters, the cycle loop, the counters to the host
  SS_CK(cudaStreamBeginCaptureToGraph(s, top, nullptr, nullptr, 0, mode));
  cudaMemsetAsync(b->d_counters + kCtrCycles, 0, (kCtrWaiting - kCtrCycles + 1) * sizeof(int), s);
  rc = capture_while(s, h_cycle, &body);
  cudaMemcpyAsync(b->h_counters, b->d_counters, kCounters * sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaGraph_t out = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &out);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("run graph: ") + cudaGetErrorString(e));
  // one cycle
  if (b->ks.round) SS_CK(cudaGraphConditionalHandleCreate(&h_round, body, 0, 0));
  SS_CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, mode));
  int* sc = b->d_sched;
  const int nc = b->n_chunks;
  if (b->d_ready) k_join<<<1, 1024, 0, s>>>(b->d_ctl, b->d_ready, nG, b->d_counters);
  sched_launch(kAssemble, s, b->d_gd, b->d_ctl, b->d_chunk_group, nc, sc);
  b->ks.eval(kAssemble, b->n_tiles, s, b->d_gd, sc, nc, b->d_ctl, b->max_hb, b->win_bytes);
  solve_launch(s, b->d_gd, b->d_ctl, nG);
  if (b->ks.round) {
    k_sched_rounds<<<1, kSchedThreads, 0, s>>>(b->d_gd, b->d_ctl, b->d_frame_group, b->n_frames_total, nG,
                                               b->d_tsched, b->d_counters, 1, h_round);
    rc = capture_while(s, h_round, &rounds_body);
    if (!rc) {
      sched_launch(kCorr, s, b->d_gd, b->d_ctl, b->d_chunk_group, nc, sc);
      b->ks.eval(kCorr, b->n_tiles, s, b->d_gd, sc, nc, b->d_ctl, b->max_hb, b->win_bytes);
    }
  } else {
    b->ks.ls(b->n_frames_total, s, b->d_gd, b->d_frame_group, b->d_ctl, b->ls_win_bytes);
  }
  k_after_ls<<<nG, kAfterLsThreads, 0, s>>>(b->d_gd, b->d_ctl);
  k_iter_sums<<<dim3(kIterSplit, nG), 256, 0, s>>>(b->d_gd, b->d_ctl);
  k_iter_end<<<nG, kSolveThreads, 0, s>>>(b->d_gd, b->d_ctl);
  sched_launch(kFinal, s, b->d_gd, b->d_ctl, b->d_chunk_group, nc, sc);
  b->ks.eval(kFinal, b->n_tiles, s, b->d_gd, sc, nc, b->d_ctl, b->max_hb, b->win_bytes);
  k_final<<<nG, kSolveThreads, 0, s>>>(b->d_gd, b->d_ctl, b->d_counters + kCtrDone);
  k_cycle_ctl<<<1, 32, 0, s>>>(b->d_counters, nG, max_cycles, h_cycle);
  e = cudaStreamEndCapture(s, &out);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("run graph cycle: ") + cudaGetErrorString(e));
  // one trial round
  if (b->ks.round) {
    SS_CK(cudaStreamBeginCaptureToGraph(s, rounds_body, nullptr, nullptr, 0, mode));
    b->ks.round(b->n_trial_tiles, s, b->d_gd, b->d_tsched, b->n_frames_total, nG, b->d_ctl, b->win_bytes);
    k_sched_rounds<<<1, kSchedThreads, 0, s>>>(b->d_gd, b->d_ctl, b->d_frame_group, b->n_frames_total, nG,
                                               b->d_tsched, b->d_counters, 0, h_round);
    e = cudaStreamEndCapture(s, &out);
    if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("run graph rounds: ") + cudaGetErrorString(e));
  }
  SS_CK(cudaGetLastError());
  SS_CK(cudaGraphInstantiate(&b->run_exec, top, 0));
  return SS_OK;
}

// Launches the whole run as the graph and records the cycle event.
static int launch_run_graph(Batch::Impl* b) {
  if (!b->run_exec) {
    int rc = build_run_graph(b);
    if (rc) return rc;
  }
  SS_CK(cudaGraphLaunch(b->run_exec, b->stream));
  if (!b->ev_cycle) SS_CK(cudaEventCreateWithFlags(&b->ev_cycle, cudaEventDisableTiming));
  SS_CK(cudaEventRecord(b->ev_cycle, b->stream));
  b->graph_run = true;
  return SS_OK;
}

int Batch::start() {
  Impl* b = d;
  b->t_start = std::chrono::steady_clock::now();
  SS_CK(cudaSetDevice(b->device));
  if (!b->h_counters) SS_CK(cudaHostAlloc(&b->h_counters, (kCounters + 1) * sizeof(int), cudaHostAllocDefault));
  SS_CK(smem_attr(k_solve_system, (int)kSolveSmem));
  int rc = reset_state(b);
  if (rc) return rc;
  b->cycles = 0;
  b->rounds = 0;
  b->launches = 0;
  b->event_used = 0;
  b->fused = 0;
  b->cur_rounds = kFirstRounds;
  b->cycle_no = 0;
  b->graph_run = false;
  b->state = 1;
  int max_iter = 1;
  for (auto& g : b->hg) max_iter = std::max(max_iter, g.in->max_iter);
  // two half-steps per iteration, a line search of up to kTrialCap trials each
  b->max_cycles = 4LL * (max_iter + 2) * (1 + kTrialCap / kMinRounds) + 16;
  return SS_OK;
}

int Batch::step() {
  Impl* b = d;
  if (b->state != 1) return fail(SS_ERR_INVALID_ARGUMENT, "batch: step() needs start() and a finished cycle");
  SS_CK(cudaSetDevice(b->device));
  int rc = b->use_graph && !b->timing && !b->ftime ? launch_run_graph(b) : launch_cycle(b);
  if (rc) return rc;
  b->state = 2;
  return SS_OK;
}

// Completion of the batch: final state, error word and staging counters on the host.
static int finish_run(Batch::Impl* b) {
  if (b->up_stream) SS_CK(cudaStreamSynchronize(b->up_stream));
  SS_CK(cudaMemcpyAsync(b->h_ctl.data(), b->d_ctl, b->h_ctl.size() * sizeof(GroupCtl), cudaMemcpyDeviceToHost,
                        b->stream));
  SS_CK(cudaMemcpyAsync(b->h_counters + kCounters, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  SS_CK(cudaMemcpyAsync(b->h_staging, b->d_staging, sizeof(b->h_staging), cudaMemcpyDeviceToHost, b->stream));
  SS_CK(cudaStreamSynchronize(b->stream));
  if (b->h_counters[kCounters] & 1) return fail(SS_ERR_CUDA, "a shared-memory staging copy did not complete in time");
  for (int k = 0; k < kFunctionTimes; k++) b->ftimes[k] = 0;
  for (size_t k = 0; k + 1 < b->fused; k++) {
    if (b->fslot[k] < 0) continue;
    float ms = 0;
    SS_CK(cudaEventElapsedTime(&ms, b->fevents[k], b->fevents[k + 1]));
    b->ftimes[b->fslot[k]] += ms * 1e-3;
  }
  for (int m = 0; m < 4; m++) b->eval_ms[m] = 0;
  for (size_t k = 0; k < b->event_used; k += 2) {
    float ms = 0;
    SS_CK(cudaEventElapsedTime(&ms, b->events[k], b->events[k + 1]));
    b->eval_ms[b->event_mode[k]] += ms;
  }
  b->run_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - b->t_start).count();
  return SS_OK;
}

int Batch::poll() {
  Impl* b = d;
  if (b->state == 3) return 2;
  if (b->state != 2) return fail(SS_ERR_INVALID_ARGUMENT, "batch: poll() without a cycle in flight");
  cudaError_t q = cudaEventQuery(b->ev_cycle);
  if (q == cudaErrorNotReady) return 0;
  if (q != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cycle: ") + cudaGetErrorString(q));
  if (b->graph_run) {
    const int* c = b->h_counters;
    b->graph_run = false;
    b->cycles = c[kCtrCycles];
    b->rounds = b->ks.round ? c[kCtrRounds] : c[kCtrCycles];
    // per cycle: schedules and evaluation passes, the solve (5), after-ls, iteration end (2), final,
    // cycle control, and the line search (precision 'D') or the first round schedule and the
    // correlation pass (precision 'S'); two launches per trial round
    b->launches = b->ks.round ? 17 * c[kCtrCycles] + 2 * c[kCtrRounds] : 15 * c[kCtrCycles];
    if (c[kCtrBound] & 1) return fail(SS_ERR_CUDA, "alignment did not finish within the iteration bound");
    b->state = 3;
    int rc = finish_run(b);
    return rc ? rc : 2;
  }
  if (b->h_counters[1] >= (int)b->gd.size()) {
    b->state = 3;
    int rc = finish_run(b);
    return rc ? rc : 2;
  }
  if (b->h_counters[0] > 0) b->cur_rounds = std::min(kMaxRounds, std::max(kMinRounds, b->h_counters[0]));
  if (++b->cycle_no >= b->max_cycles) return fail(SS_ERR_CUDA, "alignment did not finish within the iteration bound");
  b->state = 1;
  return 1;
}

int Batch::run() {
  int rc = start();
  if (rc) return rc;
  for (;;) {
    if ((rc = step())) return rc;
    SS_CK(cudaStreamSynchronize(d->stream));
    rc = poll();
    if (rc < 0) return rc;
    if (rc == 2) return SS_OK;
  }
}

// Resets the batch's groups to their initial state (the start of a server slot; waits on an own
// stream).
int Batch::reset() {
  Impl* b = d;
  SS_CK(cudaSetDevice(b->device));
  int rc = reset_state(b);
  if (rc) return rc;
  if (b->own_stream) SS_CK(cudaStreamSynchronize(b->stream));
  return SS_OK;
}

void Batch::set_timing(bool on) { d->timing = on; }
void Batch::set_graph(bool on) { d->use_graph = on; }

void Batch::stats(ss_batch_stats* st) const {
  std::memset(st, 0, sizeof(*st));
  st->n_groups = (int32_t)d->gd.size();
  st->cycles = d->cycles;
  st->linesearch_rounds = d->rounds;
  st->kernel_launches = d->launches;
  for (const GroupCtl& C : d->h_ctl)
    for (int m = 0; m < 4; m++) st->frame_passes[m] += C.passes[m];
  for (int m = 0; m < 4; m++) st->eval_ms[m] = d->eval_ms[m];
  st->arena_bytes = (int64_t)d->arena_bytes;
  st->run_ms = d->run_ms;
  for (int i = 0; i < 6; i++) st->staging[i] = (int64_t)d->h_staging[i];
  st->assembly_columns_kept = (int64_t)d->h_staging[6];
}

int Batch::collect() {
  Impl* b = d;
  cudaStream_t s = b->stream;
  // outputs come back through the page-locked staging buffer where it has room (copied out after
  // the stream has drained), else straight into the caller's arrays
  Staging stg(s, b->own_stream);
  struct Pending {
    void* dst;
    const void* src;
    size_t n;
  };
  std::vector<Pending> pend;
  auto get = [&](void* dst, const void* src, size_t n) -> cudaError_t {
    if (!n) return cudaSuccess;
    void* p = stg.take(n);
    if (!p) return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s);
    pend.push_back({dst, p, n});
    return cudaMemcpyAsync(p, src, n, cudaMemcpyDeviceToHost, s);
  };
  SS_CK(cudaMemcpyAsync(b->h_ctl.data(), b->d_ctl, b->h_ctl.size() * sizeof(GroupCtl), cudaMemcpyDeviceToHost, s));
  for (size_t i = 0; i < b->gd.size(); i++) {
    ss_outputs* o = b->outs[i];
    if (!o) continue;
    const HostGroup& g = b->hg[i];
    const GroupDesc& G = b->gd[i];
    const size_t nF = g.nF, nk = (size_t)(g.W + 1) * nF;
    const bool frame_ordered = g.flags & kFlagFrameOrdered;
    if (o->dx_knots && !frame_ordered) SS_CK(get(o->dx_knots, G.o_dx, nk * 8));
    if (o->dy_knots && !frame_ordered) SS_CK(get(o->dy_knots, G.o_dy, nk * 8));
    if (o->frame_corr) SS_CK(get(o->frame_corr, G.o_frame_corr, nF * 8));
    if (o->residrms) SS_CK(get(o->residrms, G.o_residrms, nF * 8));
    if (o->mask) SS_CK(get(o->mask, G.o_mask, (size_t)g.Hb * g.fW));
    if (o->blocks_used) SS_CK(get(o->blocks_used, G.o_blocks_used, g.fW));
    const size_t mi = g.in->max_iter;
    if (o->iteration_corr) SS_CK(get(o->iteration_corr, G.o_iter_corr, mi * 8));
    if (o->frame_corr_history)
      SS_CK(get(o->frame_corr_history, G.o_frame_corr_hist, mi * nF * 8));
    if (o->iteration_errvals)
      SS_CK(get(o->iteration_errvals, G.o_iter_errvals, 2 * mi * nF * 8));
    if (o->all_params) SS_CK(get(o->all_params, G.o_all_params, 2 * (size_t)g.N * mi * 8));
    if (o->frame_params && frame_ordered)
      SS_CK(get(o->frame_params, G.o_frame_params, 2 * nk * 8));
    if (o->raw_params && (g.flags & kFlagRawParams))
      SS_CK(get(o->raw_params, G.o_raw, 2 * (size_t)g.N * 8));
    // outputs 9, 10, 14: zeros where the flags do not produce them
    if (o->rg_params) {
      if (G.o_rg_params)
        SS_CK(get(o->rg_params, G.o_rg_params, (size_t)2 * g.N * 2 * mi * 8));
      else
        std::memset(o->rg_params, 0, (size_t)2 * g.N * 2 * mi * 8);
    }
    if (o->iteration_times) {
      if (G.o_iter_times) SS_CK(get(o->iteration_times, G.o_iter_times, mi * 8));
      else std::memset(o->iteration_times, 0, mi * 8);
    }
    if (o->function_times)
      for (int k = 0; k < kFunctionTimes; k++)
        o->function_times[k] = (g.flags & kFlagTimeSub) ? b->ftimes[k] : 0.0;
  }
  SS_CK(cudaStreamSynchronize(s));
  for (const Pending& q : pend) std::memcpy(q.dst, q.src, q.n);
  stg.release();
  for (size_t i = 0; i < b->gd.size(); i++) {
    ss_outputs* o = b->outs[i];
    if (!o) continue;
    const GroupCtl& C = b->h_ctl[i];
    if (o->iter_used) *o->iter_used = C.iteration;
    if (o->device_init_time) *o->device_init_time = b->init_ms / 1000.0;
    o->stop_reason = C.stop_reason;
    o->trial_cap_hit = C.cap_hit;
    o->n_frame_passes = C.n_eval;
  }
  return SS_OK;
}

// ---------------------------------------------------------------------------------------------
// Continuous batching: a table of group slots served by one launch sequence per cycle

struct Server::Impl {
  struct Slot {
    Batch* batch = nullptr;  // the group's buffers (its arena) and host metadata
    bool active = false;
    bool joining = false;    // admitted since the last cycle was launched
    int tiles = 0, chunks = 0, frames = 0, trial_tiles = 0;
    GroupCtl init;           // initial control state, uploaded when the slot joins
  };
  int device = 0, capacity = 0;
  cudaStream_t stream = nullptr;         // the cycles
  cudaStream_t upload_stream = nullptr;  // admissions: uploads and resets that need not wait for a cycle
  cudaEvent_t ev_upload = nullptr;
  bool configured = false;
  int compute = 0, frame_dt = 0, tpl_dt = 0;
  KernelSet ks = {nullptr, nullptr, nullptr};
  int max_hb = 0, win_bytes = 0, ls_win_bytes = 0;
  std::vector<Slot> slots;
  std::vector<GroupDesc> h_gd;
  GroupCtl* h_ctl = nullptr;  // pinned: the slots' control state after each cycle
  GroupDesc* d_gd = nullptr;
  GroupCtl* d_ctl = nullptr;
  int* d_chunk_group = nullptr;
  int* d_sched = nullptr;
  int* d_tsched = nullptr;
  int* d_frame_group = nullptr;
  int chunk_cap = 0, frame_cap = 0, n_tiles = 0, n_chunks = 0, n_frames = 0, n_trial_tiles = 0;
  std::vector<int> cg, fg;
  int* d_counters = nullptr;  // [0] most trials of a search that ended in the cycle, [1] finished groups
  int* h_counters = nullptr;  // pinned
  int* d_err = nullptr;
  unsigned long long* d_staging = nullptr;
  cudaEvent_t ev = nullptr;
  bool dirty = false, in_flight = false;
  int cur_rounds = kFirstRounds;
  long long cycles = 0;
};

Server::Server() : d(new Impl) {}
Server::~Server() {
  Impl* v = d;
  if (v->stream) cudaStreamSynchronize(v->stream);
  if (v->upload_stream) cudaStreamSynchronize(v->upload_stream);
  for (auto& sl : v->slots) {
    delete sl.batch;
    sl.batch = nullptr;
  }
  if (v->ev) cudaEventDestroy(v->ev);
  if (v->ev_upload) cudaEventDestroy(v->ev_upload);
  if (v->upload_stream) cudaStreamDestroy(v->upload_stream);
  cudaFree(v->d_gd);
  cudaFree(v->d_ctl);
  cudaFree(v->d_chunk_group);
  cudaFree(v->d_sched);
  cudaFree(v->d_tsched);
  cudaFree(v->d_frame_group);
  cudaFree(v->d_counters);
  cudaFree(v->d_err);
  cudaFree(v->d_staging);
  if (v->h_ctl) cudaFreeHost(v->h_ctl);
  if (v->h_counters) cudaFreeHost(v->h_counters);
  if (v->stream) cudaStreamDestroy(v->stream);
  delete v;
}

int Server::create(int capacity, int device) {
  Impl* v = d;
  if (capacity < 1) return fail(SS_ERR_INVALID_ARGUMENT, "server capacity must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SS_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(SS_ERR_INVALID_ARGUMENT, "device out of range");
  v->device = device;
  v->capacity = capacity;
  SS_CK(cudaSetDevice(device));
  SS_CK(cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking));
  SS_CK(cudaStreamCreateWithFlags(&v->upload_stream, cudaStreamNonBlocking));
  SS_CK(cudaEventCreateWithFlags(&v->ev, cudaEventDisableTiming));
  SS_CK(cudaEventCreateWithFlags(&v->ev_upload, cudaEventDisableTiming));
  v->slots.assign(capacity, Impl::Slot{});
  v->h_gd.assign(capacity, GroupDesc{});
  SS_CK(cudaHostAlloc(&v->h_ctl, capacity * sizeof(GroupCtl), cudaHostAllocDefault));
  SS_CK(cudaHostAlloc(&v->h_counters, 4 * sizeof(int), cudaHostAllocDefault));
  SS_CK(cudaMalloc(&v->d_gd, capacity * sizeof(GroupDesc)));
  SS_CK(cudaMalloc(&v->d_ctl, capacity * sizeof(GroupCtl)));
  SS_CK(cudaMalloc(&v->d_counters, 4 * sizeof(int)));
  SS_CK(cudaMalloc(&v->d_err, sizeof(int)));
  SS_CK(cudaMalloc(&v->d_staging, kStagingCounters * sizeof(unsigned long long)));
  SS_CK(cudaMemset(v->d_counters, 0, 4 * sizeof(int)));
  SS_CK(cudaMemset(v->d_err, 0, sizeof(int)));
  SS_CK(cudaMemset(v->d_staging, 0, kStagingCounters * sizeof(unsigned long long)));
  // empty slots are in the done phase: every kernel passes them by
  for (int k = 0; k < capacity; k++) {
    std::memset(&v->h_ctl[k], 0, sizeof(GroupCtl));
    v->h_ctl[k].phase = kPhDone;
  }
  SS_CK(cudaMemcpy(v->d_ctl, v->h_ctl, capacity * sizeof(GroupCtl), cudaMemcpyHostToDevice));
  SS_CK(cudaMemset(v->d_gd, 0, capacity * sizeof(GroupDesc)));
  return SS_OK;
}

int Server::admit(const ss_inputs* in, ss_outputs* out, const Batch* session, void* arena, size_t arena_bytes,
                  int* slot_out) {
  Impl* v = d;
  if (!in || !slot_out) return fail(SS_ERR_INVALID_ARGUMENT, "bad admit arguments");
  int slot = -1;
  for (int k = 0; k < v->capacity; k++)
    if (!v->slots[k].batch) {
      slot = k;
      break;
    }
  if (slot < 0) return fail(SS_ERR_BUSY, "every server slot is taken");
  if (in->gpu_device_id != v->device) return fail(SS_ERR_INVALID_ARGUMENT, "group and server differ in device");
  Batch* b = new Batch;
  const Batch* ses[1] = {session};
  int rc = b->prepare(1, in, out, arena, arena_bytes, ses, false, v->upload_stream);
  if (!rc) rc = b->reset();
  if (rc) {
    delete b;
    return rc;
  }
  Batch::Impl* bi = b->d;
  if (!v->configured) {
    v->compute = bi->compute;
    v->frame_dt = bi->frame_dt;
    v->tpl_dt = bi->tpl_dt;
    v->ks = bi->ks;
    v->configured = true;
  } else if (bi->compute != v->compute || bi->frame_dt != v->frame_dt || bi->tpl_dt != v->tpl_dt) {
    delete b;
    return fail(SS_ERR_INVALID_ARGUMENT, "all groups of a server need the same precision, frame and template types");
  }
  v->max_hb = std::max(v->max_hb, bi->max_hb);
  v->win_bytes = std::max(v->win_bytes, bi->win_bytes);
  v->ls_win_bytes = std::max(v->ls_win_bytes, bi->ls_win_bytes);
  Impl::Slot& sl = v->slots[slot];
  sl.batch = b;
  sl.joining = true;
  sl.active = true;
  const HostGroup& g = bi->hg[0];
  sl.chunks = (g.nF + g.frames_per_cta - 1) / g.frames_per_cta;
  sl.tiles = g.W * sl.chunks;
  sl.trial_tiles = g.W * ((g.nF + kTrialTileFrames - 1) / kTrialTileFrames);
  sl.frames = g.nF;
  GroupDesc G = bi->gd[0];
  G.err = v->d_err;
  G.staging = v->d_staging;
  G.ls_max_trials = v->d_counters;
  v->h_gd[slot] = G;
  sl.init = bi->h_ctl[0];  // not into h_ctl: a cycle in flight still copies into it
  v->dirty = true;
  *slot_out = slot;
  return SS_OK;
}

// Tile and frame tables over the active slots, descriptors and the joining slots' control state.
static int server_tables(Server::Impl* v) {
  cudaStream_t s = v->stream;
  v->n_tiles = 0;
  v->n_trial_tiles = 0;
  v->n_chunks = 0;
  v->n_frames = 0;
  for (int k = 0; k < v->capacity; k++) {
    auto& sl = v->slots[k];
    if (!sl.active) continue;
    v->h_gd[k].chunk_base = v->n_chunks;
    v->h_gd[k].frame_base = v->n_frames;
    v->n_tiles += sl.tiles;
    v->n_trial_tiles += sl.trial_tiles;
    v->n_chunks += sl.chunks;
    v->n_frames += sl.frames;
  }
  if (v->n_chunks > v->chunk_cap || v->n_frames > v->frame_cap) {  // between cycles: nothing in flight
    SS_CK(cudaStreamSynchronize(s));
    cudaFree(v->d_chunk_group);
    cudaFree(v->d_sched);
    cudaFree(v->d_tsched);
    cudaFree(v->d_frame_group);
    v->chunk_cap = std::max(2 * v->chunk_cap, v->n_chunks);
    v->frame_cap = std::max(2 * v->frame_cap, v->n_frames);
    SS_CK(cudaMalloc(&v->d_chunk_group, (size_t)v->chunk_cap * sizeof(int)));
    SS_CK(cudaMalloc(&v->d_sched, sched_ints(v->chunk_cap) * sizeof(int)));
    SS_CK(cudaMalloc(&v->d_tsched, tsched_ints(v->frame_cap, v->capacity) * sizeof(int)));
    SS_CK(cudaMalloc(&v->d_frame_group, (size_t)v->frame_cap * sizeof(int)));
  }
  v->cg.assign(std::max(1, v->n_chunks), 0);
  v->fg.assign(std::max(1, v->n_frames), 0);
  for (int k = 0; k < v->capacity; k++) {
    auto& sl = v->slots[k];
    if (!sl.active) continue;
    for (int t = 0; t < sl.chunks; t++) v->cg[v->h_gd[k].chunk_base + t] = k;
    for (int f = 0; f < sl.frames; f++) v->fg[v->h_gd[k].frame_base + f] = k;
  }
  // pageable sources are staged before the copies return
  SS_CK(cudaMemcpyAsync(v->d_gd, v->h_gd.data(), v->capacity * sizeof(GroupDesc), cudaMemcpyHostToDevice, s));
  if (v->n_chunks)
    SS_CK(cudaMemcpyAsync(v->d_chunk_group, v->cg.data(), v->n_chunks * sizeof(int), cudaMemcpyHostToDevice, s));
  if (v->n_frames)
    SS_CK(cudaMemcpyAsync(v->d_frame_group, v->fg.data(), v->n_frames * sizeof(int), cudaMemcpyHostToDevice, s));
  for (int k = 0; k < v->capacity; k++) {
    auto& sl = v->slots[k];
    if (!sl.joining) continue;
    SS_CK(cudaMemcpyAsync(v->d_ctl + k, &sl.init, sizeof(GroupCtl), cudaMemcpyHostToDevice, s));
    sl.joining = false;
  }
  v->dirty = false;
  return SS_OK;
}

int Server::step() {
  Impl* v = d;
  if (v->in_flight) return fail(SS_ERR_INVALID_ARGUMENT, "server: a cycle is in flight");
  SS_CK(cudaSetDevice(v->device));
  if (v->dirty) {
    // joining groups' uploads and resets come first
    SS_CK(cudaEventRecord(v->ev_upload, v->upload_stream));
    SS_CK(cudaStreamWaitEvent(v->stream, v->ev_upload, 0));
    int rc = server_tables(v);
    if (rc) return rc;
  }
  if (v->n_tiles == 0) return SS_OK;  // nothing to run
  cudaStream_t s = v->stream;
  const int nG = v->capacity;
  SS_CK(smem_attr(k_solve_system, (int)kSolveSmem));
  v->cycles++;
  int* sc = v->d_sched;
  const int nc = v->n_chunks;
  sched_launch(kAssemble, s, v->d_gd, v->d_ctl, v->d_chunk_group, nc, sc);
  v->ks.eval(kAssemble, v->n_tiles, s, v->d_gd, sc, nc, v->d_ctl, v->max_hb, v->win_bytes);
  solve_launch(s, v->d_gd, v->d_ctl, nG);
  if (v->ks.round) {
    SS_CK(cudaMemsetAsync(v->d_counters, 0, sizeof(int), s));
    for (int r = 0; r < v->cur_rounds; r++) {
      trial_sched_launch(s, v->d_gd, v->d_ctl, v->d_frame_group, v->n_frames, nG, v->d_tsched);
      v->ks.round(v->n_trial_tiles, s, v->d_gd, v->d_tsched, v->n_frames, nG, v->d_ctl, v->win_bytes);
    }
    sched_launch(kCorr, s, v->d_gd, v->d_ctl, v->d_chunk_group, nc, sc);
    v->ks.eval(kCorr, v->n_tiles, s, v->d_gd, sc, nc, v->d_ctl, v->max_hb, v->win_bytes);
  } else {
    v->ks.ls(v->n_frames, s, v->d_gd, v->d_frame_group, v->d_ctl, v->ls_win_bytes);
  }
  k_after_ls<<<nG, kAfterLsThreads, 0, s>>>(v->d_gd, v->d_ctl);
  k_iter_sums<<<dim3(kIterSplit, nG), 256, 0, s>>>(v->d_gd, v->d_ctl);
  k_iter_end<<<nG, kSolveThreads, 0, s>>>(v->d_gd, v->d_ctl);
  sched_launch(kFinal, s, v->d_gd, v->d_ctl, v->d_chunk_group, nc, sc);
  v->ks.eval(kFinal, v->n_tiles, s, v->d_gd, sc, nc, v->d_ctl, v->max_hb, v->win_bytes);
  k_final<<<nG, kSolveThreads, 0, s>>>(v->d_gd, v->d_ctl, v->d_counters + 1);
  SS_CK(cudaGetLastError());
  SS_CK(cudaMemcpyAsync(v->h_counters, v->d_counters, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  SS_CK(cudaMemcpyAsync(v->h_ctl, v->d_ctl, nG * sizeof(GroupCtl), cudaMemcpyDeviceToHost, s));
  SS_CK(cudaEventRecord(v->ev, s));
  v->in_flight = true;
  return SS_OK;
}

int Server::poll(int* done, int max_done, int* n_done) {
  Impl* v = d;
  *n_done = 0;
  if (v->in_flight) {
    cudaError_t q = cudaEventQuery(v->ev);
    if (q == cudaErrorNotReady) return 0;
    if (q != cudaSuccess) return fail(SS_ERR_CUDA, std::string("server cycle: ") + cudaGetErrorString(q));
    v->in_flight = false;
    int err = 0;
    SS_CK(cudaMemcpy(&err, v->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err & 1) return fail(SS_ERR_CUDA, "a shared-memory staging copy did not complete in time");
    if (v->h_counters[0] > 0) v->cur_rounds = std::min(kMaxRounds, std::max(kMinRounds, v->h_counters[0]));
  }
  for (int k = 0; k < v->capacity && *n_done < max_done; k++) {
    auto& sl = v->slots[k];
    if (!sl.active || sl.joining || v->h_ctl[k].phase != kPhDone) continue;
    // the group has stopped: its control state to its own batch, then its outputs to the host
    Batch::Impl* bi = sl.batch->d;
    SS_CK(cudaMemcpy(bi->d_ctl, v->d_ctl + k, sizeof(GroupCtl), cudaMemcpyDeviceToDevice));
    int rc = sl.batch->collect();
    if (rc) return rc;
    delete sl.batch;
    sl = Impl::Slot{};
    v->dirty = true;
    done[(*n_done)++] = k;
  }
  return 1;
}

int Server::active() const {
  int n = 0;
  for (auto& sl : d->slots) n += sl.active ? 1 : 0;
  return n;
}

// ---------------------------------------------------------------------------------------------
// Recording-level estimate (the caller loop of steady_scan.m:157-288)

int recording_sets(int n_frames, int frames_per_set, int min_frames_per_set, int* first, int* count, int max_sets,
                   int* n_sets) {
  if (n_frames < 1) return fail(SS_ERR_INVALID_ARGUMENT, "recording has no frames");
  if (frames_per_set < 1) return fail(SS_ERR_INVALID_ARGUMENT, "frames_per_set must be positive");
  if (min_frames_per_set < 0) return fail(SS_ERR_INVALID_ARGUMENT, "min_frames_per_set must not be negative");
  // set_start = 1:frames_per_set:nframes, then nframes + 1 (steady_scan.m:97-99, 1-based); the
  // size rebalancing of the last two sets (:101-106) changes set_size, which the estimate loop
  // does not read: set iset covers set_start(iset) : min(set_start(iset + 1), nframes) (:220)
  int k = 0;
  for (int s = 1; s <= n_frames; s += frames_per_set, k++) {
    const int next = s + frames_per_set <= n_frames ? s + frames_per_set : n_frames + 1;
    const int end = std::min(next, n_frames);
    if (k < max_sets) {
      if (first) first[k] = s - 1;
      if (count) count[k] = end - s + 1;
    }
  }
  if (n_sets) *n_sets = k;
  return SS_OK;
}

int estimate_displacements(const ss_recording* rec, ss_recording_outputs* out) {
  if (!rec || !out) return fail(SS_ERR_INVALID_ARGUMENT, "recording or outputs is NULL");
  const ss_inputs& g = rec->group;
  const int n = g.n_frames;
  const int64_t Hb = g.basex.rows, W = g.basex.cols;
  if (n < 1 || Hb < 1 || W < 1) return fail(SS_ERR_INVALID_ARGUMENT, "recording has no frames or no blocks");
  if (g.bm_data.rows != Hb || g.bm_data.cols != W * n)
    return fail(SS_ERR_INVALID_ARGUMENT, "bm_data must be frameH x (frameW * n_frames)");
  const size_t esz = dtype_size(g.bm_data.dtype);
  if (!esz || !g.bm_data.data) return fail(SS_ERR_INVALID_ARGUMENT, "bm_data is NULL or of an unknown dtype");
  int n_sets = 0;
  int rc = recording_sets(n, rec->frames_per_set, rec->min_frames_per_set, nullptr, nullptr, 0, &n_sets);
  if (rc) return rc;
  std::vector<int> first(n_sets), count(n_sets);
  recording_sets(n, rec->frames_per_set, rec->min_frames_per_set, first.data(), count.data(), n_sets, &n_sets);
  // initial knots: the first columns for every set (the reference), or each set's own
  const int64_t est_vals = std::min(g.est_dx_knots.rows * g.est_dx_knots.cols, g.est_dy_knots.rows * g.est_dy_knots.cols);
  const size_t ex_sz = dtype_size(g.est_dx_knots.dtype), ey_sz = dtype_size(g.est_dy_knots.dtype);
  if (!ex_sz || !ey_sz || g.est_dx_knots.location != SS_HOST || g.est_dy_knots.location != SS_HOST)
    return fail(SS_ERR_INVALID_ARGUMENT, "est_dx_knots and est_dy_knots must be host matrices of a known dtype");
  std::vector<ss_inputs> ins(n_sets, g);
  for (int s = 0; s < n_sets; s++) {
    ss_inputs& in = ins[s];
    in.n_frames = count[s];
    const char* base = static_cast<const char*>(g.bm_data.data);
    in.bm_data.data = base + (size_t)first[s] * W * Hb * esz;
    in.bm_data.cols = W * count[s];
    const int64_t col0 = rec->per_set_estimates ? first[s] : 0;
    if ((col0 + count[s]) * (W + 1) > est_vals)
      return fail(SS_ERR_INVALID_ARGUMENT, "est_dx_knots / est_dy_knots hold too few columns for the sets");
    in.est_dx_knots = {static_cast<const char*>(g.est_dx_knots.data) + (size_t)col0 * (W + 1) * ex_sz, W + 1, count[s],
                       g.est_dx_knots.dtype, SS_HOST};
    in.est_dy_knots = {static_cast<const char*>(g.est_dy_knots.data) + (size_t)col0 * (W + 1) * ey_sz, W + 1, count[s],
                       g.est_dy_knots.dtype, SS_HOST};
  }
  Batch b;
  if ((rc = b.prepare(n_sets, ins.data(), nullptr, nullptr, 0))) return rc;
  if ((rc = b.run())) return rc;
  Batch::Impl* bi = b.d;
  cudaStream_t s = bi->stream;
  // the recording's outputs on the device: NaN / 0 where no set estimates a frame
  const size_t nk = (size_t)(W + 1) * n, nd = 2 * nk + 3 * (size_t)n, nb = (size_t)n + (size_t)W * n;
  std::vector<SetSpan> spans(n_sets);
  for (int k = 0; k < n_sets; k++) spans[k] = {first[k], count[k] - 1};
  char* buf = nullptr;
  const size_t span_off = (nd * 8 + nb + 255) & ~size_t(255);
  SS_CK(cudaMalloc(&buf, span_off + spans.size() * sizeof(SetSpan)));
  struct Free {
    char* p;
    ~Free() { cudaFree(p); }
  } guard{buf};
  double* d_dx = reinterpret_cast<double*>(buf);
  double* d_dy = d_dx + nk;
  double* d_corr = d_dy + nk;
  double* d_it = d_corr + n;
  double* d_rr = d_it + n;
  uint8_t* d_failed = reinterpret_cast<uint8_t*>(d_rr + n);
  uint8_t* d_used = d_failed + n;
  SetSpan* d_spans = reinterpret_cast<SetSpan*>(buf + span_off);
  k_fill_nan_u8<<<148, 256, 0, s>>>(d_dx, nd, d_failed, nb);
  SS_CK(cudaMemcpyAsync(d_spans, spans.data(), spans.size() * sizeof(SetSpan), cudaMemcpyHostToDevice, s));
  k_post_estimate<<<n_sets, 256, 0, s>>>(bi->d_gd, bi->d_ctl, d_spans, rec->corr_thresh, rec->minblockfrac, d_dx, d_dy,
                                         d_corr, d_it, d_rr, d_failed, d_used);
  SS_CK(cudaGetLastError());
  if (out->dx_knots) SS_CK(cudaMemcpyAsync(out->dx_knots, d_dx, nk * 8, cudaMemcpyDeviceToHost, s));
  if (out->dy_knots) SS_CK(cudaMemcpyAsync(out->dy_knots, d_dy, nk * 8, cudaMemcpyDeviceToHost, s));
  if (out->corr) SS_CK(cudaMemcpyAsync(out->corr, d_corr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  if (out->iter_used) SS_CK(cudaMemcpyAsync(out->iter_used, d_it, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  if (out->residrms) SS_CK(cudaMemcpyAsync(out->residrms, d_rr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  if (out->failed) SS_CK(cudaMemcpyAsync(out->failed, d_failed, (size_t)n, cudaMemcpyDeviceToHost, s));
  if (out->blocks_used) SS_CK(cudaMemcpyAsync(out->blocks_used, d_used, (size_t)W * n, cudaMemcpyDeviceToHost, s));
  SS_CK(cudaStreamSynchronize(s));
  out->n_sets = n_sets;
  return SS_OK;
}

int Batch::cycles() const { return d->cycles; }
int Batch::rounds() const { return d->rounds; }
int Batch::n_groups() const { return (int)d->gd.size(); }
const GroupCtl* Batch::host_ctl() const { return d->h_ctl.data(); }
void* Batch::stream() const { return d->stream; }

}  // namespace ss

// ---------------------------------------------------------------------------------------------
// Caller-side preparation of frames (ss_frontend.cuh)

namespace ss {

// The library's memory pool of a device for the work memory of synchronous calls: stream-ordered
// allocations whose freed memory the pool keeps for the next call (no cudaMalloc / cudaFree, and no
// device-wide synchronisation, per call once a call of that size has run).
static cudaMemPool_t work_pool(int device) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(device);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[device] = pool;
  return pool;
}

// Device allocations and a stream of one synchronous call, released into the device's work pool
// when it returns (the stream drained first). The stream must exist before the first take().
struct CallMem {
  std::vector<void*> ptrs;
  cudaStream_t s = nullptr;
  cudaMemPool_t pool = nullptr;
  CallMem() = default;
  CallMem(const CallMem&) = delete;
  CallMem& operator=(const CallMem&) = delete;
  ~CallMem() {
    for (void* q : ptrs) cudaFreeAsync(q, s);
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
  template <class T>
  T* take(size_t count) {
    if (!s) return nullptr;
    if (!pool) {
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess || !(pool = work_pool(dev))) return nullptr;
    }
    void* q = nullptr;
    if (cudaMallocFromPoolAsync(&q, std::max<size_t>(1, count) * sizeof(T), pool, s) != cudaSuccess) return nullptr;
    ptrs.push_back(q);
    return static_cast<T*>(q);
  }
};

// Normalised taps of one axis of the reference's periodic Gaussian (steady_scan.m:628-633): the
// weights at circular distance 0..R in a period of `period` samples, divided by the axis' sum over
// the whole period (the 2-D normalisation is the product of the two axes' sums).
static std::vector<double> blur_taps(double sd, int period, int* r_out) {
  auto g = [&](int d) {
    const double c = (double)std::min(d, period - d);
    return std::exp(-c * c / (2.0 * sd * sd));
  };
  double sum = 0.0;
  for (int d = 0; d < period; d++) sum += g(d);
  const int R = std::min((int)std::ceil(9.6 * sd), (period - 1) / 2);
  std::vector<double> t((size_t)R + 1);
  for (int d = 0; d <= R; d++) t[d] = g(d) / sum;
  *r_out = R;
  return t;
}

template <class T>
__global__ void k_to_f64(const void* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = to_double(reinterpret_cast<const T*>(in)[e]);
}

template <class InT>
static void fe_blur(const void* in, double* w1, double* w2, int h, int w, int n, int ph, int pw, const double* ty,
                    int ry, const double* tx, int rx, cudaStream_t s) {
  const dim3 grid((h + 255) / 256, w, n);
  k_blur_pass<InT, 0><<<grid, 256, 0, s>>>(in, w1, h, w, ph, ty, ry);
  k_blur_pass<double, 1><<<grid, 256, 0, s>>>(w1, w2, h, w, pw, tx, rx);
}

template <class InT>
static void fe_gather(const void* in, int out_dt, void* out, int h, int w, int n, int r0, int c0, int hc,
                      const int* gather, int hb, int nb, cudaStream_t s) {
  const int g = 148 * 8;
  if (out_dt == SS_F64) k_block_gather<InT, double><<<g, 256, 0, s>>>(in, (double*)out, h, w, n, r0, c0, hc, gather, hb, nb);
  else if (out_dt == SS_F32) k_block_gather<InT, float><<<g, 256, 0, s>>>(in, (float*)out, h, w, n, r0, c0, hc, gather, hb, nb);
  else k_block_gather<InT, uint16_t><<<g, 256, 0, s>>>(in, (uint16_t*)out, h, w, n, r0, c0, hc, gather, hb, nb);
}

int prepare_frames(const ss_prep_frames* p) {
  if (!p) return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: no arguments");
  const int n = p->n_frames;
  const int64_t h = p->frames.rows;
  if (n < 1 || h < 1 || p->frames.cols % n != 0 || !p->frames.data)
    return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: frames must be H x (W * n_frames)");
  const int64_t w = p->frames.cols / n;
  const int* cr = p->cropping;
  if (cr[0] < 0 || cr[1] < 0 || cr[2] < 0 || cr[3] < 0 || cr[0] + cr[1] >= w || cr[2] + cr[3] >= h)
    return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: cropping leaves no pixel");
  const int64_t hc = h - cr[2] - cr[3], wc = w - cr[0] - cr[1];
  const int hb = p->block_h, nbk = p->n_blocks;
  if (!p->gather || hb < 1 || nbk < 1) return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: empty block map");
  for (int64_t i = 0; i < (int64_t)hb * nbk; i++)
    if (p->gather[i] < -1 || p->gather[i] >= hc * wc)
      return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: block map index outside the cropped frame");
  const ss_matrix& o = p->out;
  if (o.location != SS_DEVICE || !o.data || o.rows != hb || o.cols != (int64_t)nbk * n)
    return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: out must be block_h x (n_blocks * n_frames) on the device");
  const bool blur = p->pregauss > 0.0, med = p->mednorm != 0;
  if (o.dtype != SS_F64 && o.dtype != SS_F32 && o.dtype != SS_U16)
    return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: out must be SS_F64, SS_F32 or SS_U16");
  if (o.dtype == SS_U16 && (p->frames.dtype != SS_U16 || blur || med))
    return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: SS_U16 output only copies SS_U16 frames without prefilter");
  const int fdt = p->frames.dtype;
  if (fdt != SS_F64 && fdt != SS_F32 && fdt != SS_U16 && fdt != SS_F16)
    return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: frames must be SS_F64, SS_F32, SS_U16 or SS_F16");
  if (blur && !(p->pregauss < 3989.0))
    return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: pregauss must be below 3989");
  if (blur && w > 65535) return fail(SS_ERR_INVALID_ARGUMENT, "prepare_frames: the blur takes frames of at most 65535 columns");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SS_ERR_NO_DEVICE, "no CUDA device");
  if (p->gpu_device_id < 0 || p->gpu_device_id >= ndev) return fail(SS_ERR_INVALID_ARGUMENT, "gpu_device_id out of range");
  SS_CK(cudaSetDevice(p->gpu_device_id));

  // padded periods and taps of the blur (steady_scan.m:627-633)
  int ry = 0, rx = 0, ph = 0, pw = 0;
  std::vector<double> ty, tx;
  if (blur) {
    const double sd = p->pregauss;
    const int L = (int)std::ceil(std::sqrt((2.0 * sd * sd) * std::log(10000.0 / (std::sqrt(2.0 * M_PI) * sd))));
    ph = (int)h + L;
    pw = (int)w + L;
    ty = blur_taps(sd, ph, &ry);
    tx = blur_taps(sd, pw, &rx);
  }
  const size_t fsz = dtype_size(fdt), osz = dtype_size(o.dtype), npx = (size_t)h * w;
  // frames per pass: about 1 GB of FP64 work memory, and the blur grid's z extent
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>({(size_t)n, ((size_t)1 << 30) / (16 * npx), (size_t)65535}));
  CallMem m;
  SS_CK(cudaStreamCreateWithFlags(&m.s, cudaStreamNonBlocking));
  cudaStream_t s = m.s;
  int* d_gather = m.take<int>((size_t)hb * nbk);
  double* d_taps = blur ? m.take<double>(ty.size() + tx.size()) : nullptr;
  void* d_raw = p->frames.location == SS_HOST ? m.take<char>(fsz * npx * chunk) : nullptr;
  double* w1 = (blur || med) ? m.take<double>(npx * chunk) : nullptr;
  double* w2 = blur ? m.take<double>(npx * chunk) : nullptr;
  double* d_med = med ? m.take<double>(chunk) : nullptr;
  if (!d_gather || (blur && !d_taps) || (p->frames.location == SS_HOST && !d_raw) || ((blur || med) && !w1) ||
      (blur && !w2) || (med && !d_med))
    return fail(SS_ERR_OUT_OF_MEMORY, "prepare_frames: work memory");
  SS_CK(cudaMemcpyAsync(d_gather, p->gather, (size_t)hb * nbk * sizeof(int), cudaMemcpyHostToDevice, s));
  if (blur) {
    SS_CK(cudaMemcpyAsync(d_taps, ty.data(), ty.size() * 8, cudaMemcpyHostToDevice, s));
    SS_CK(cudaMemcpyAsync(d_taps + ty.size(), tx.data(), tx.size() * 8, cudaMemcpyHostToDevice, s));
  }
  const int r0 = cr[2], c0 = cr[0];
  const int g = 148 * 8;
  for (int f0 = 0; f0 < n; f0 += chunk) {
    const int c = std::min(chunk, n - f0);
    const char* src = static_cast<const char*>(p->frames.data) + fsz * npx * f0;
    if (d_raw) {
      SS_CK(cudaMemcpyAsync(d_raw, src, fsz * npx * c, cudaMemcpyHostToDevice, s));
      src = static_cast<const char*>(d_raw);
    }
    const void* cur = src;
    int cur_dt = fdt;
    if (blur) {  // prefilter_foralignment's blur, then its samples in FP64
      const double* dty = d_taps;
      const double* dtx = d_taps + ty.size();
      if (fdt == SS_F64) fe_blur<double>(src, w1, w2, (int)h, (int)w, c, ph, pw, dty, ry, dtx, rx, s);
      else if (fdt == SS_F32) fe_blur<float>(src, w1, w2, (int)h, (int)w, c, ph, pw, dty, ry, dtx, rx, s);
      else if (fdt == SS_U16) fe_blur<uint16_t>(src, w1, w2, (int)h, (int)w, c, ph, pw, dty, ry, dtx, rx, s);
      else fe_blur<__half>(src, w1, w2, (int)h, (int)w, c, ph, pw, dty, ry, dtx, rx, s);
      cur = w2;
      cur_dt = SS_F64;
    } else if (med) {  // the median division works on FP64 samples
      if (fdt == SS_F64) k_to_f64<double><<<g, 256, 0, s>>>(src, w1, npx * c);
      else if (fdt == SS_F32) k_to_f64<float><<<g, 256, 0, s>>>(src, w1, npx * c);
      else if (fdt == SS_U16) k_to_f64<uint16_t><<<g, 256, 0, s>>>(src, w1, npx * c);
      else k_to_f64<__half><<<g, 256, 0, s>>>(src, w1, npx * c);
      cur = w1;
      cur_dt = SS_F64;
    }
    if (med) {
      double* x = const_cast<double*>(static_cast<const double*>(cur));
      k_frame_median<double><<<c, 1024, 0, s>>>(x, npx, d_med);
      k_frame_divide<<<g, 256, 0, s>>>(x, npx, npx * c, d_med);
    }
    void* dst = static_cast<char*>(const_cast<void*>(o.data)) + osz * (size_t)hb * nbk * f0;
    if (cur_dt == SS_F64) fe_gather<double>(cur, o.dtype, dst, (int)h, (int)w, c, r0, c0, (int)hc, d_gather, hb, nbk, s);
    else if (cur_dt == SS_F32) fe_gather<float>(cur, o.dtype, dst, (int)h, (int)w, c, r0, c0, (int)hc, d_gather, hb, nbk, s);
    else if (cur_dt == SS_U16) fe_gather<uint16_t>(cur, o.dtype, dst, (int)h, (int)w, c, r0, c0, (int)hc, d_gather, hb, nbk, s);
    else fe_gather<__half>(cur, o.dtype, dst, (int)h, (int)w, c, r0, c0, (int)hc, d_gather, hb, nbk, s);
    SS_CK(cudaGetLastError());
  }
  SS_CK(cudaStreamSynchronize(s));
  return SS_OK;
}

// ---------------------------------------------------------------------------------------------
// Reconstruction (ss_reconstruct.cuh)

// The error-check interval that follows a frame of `iter` sweeps (steady_scan.m:391):
// int32(max(1, min(10, sqrt(single(iter))))), int32 rounding halves away from zero.
static int rc_interval(int iter) {
  const float v = std::max(1.0f, std::min(10.0f, std::sqrt((float)iter)));
  return (int)std::floor((double)v + 0.5);
}

static bool host_f64(const ss_matrix& m, int64_t rows, int64_t cols, std::vector<double>& out) {
  if (m.location != SS_HOST || !m.data || m.rows != rows || m.cols != cols) return false;
  const size_t n = (size_t)rows * cols;
  out.resize(n);
  if (m.dtype == SS_F64) std::memcpy(out.data(), m.data, n * 8);
  else if (m.dtype == SS_F32) for (size_t i = 0; i < n; i++) out[i] = static_cast<const float*>(m.data)[i];
  else if (m.dtype == SS_I32) for (size_t i = 0; i < n; i++) out[i] = static_cast<const int32_t*>(m.data)[i];
  else return false;
  return true;
}

int reconstruct_frames(const ss_reconstruct* r) {
  if (!r) return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: no arguments");
  const int n = r->n_frames, th = r->template_h, tw = r->template_w;
  const int64_t hd = r->basex.rows, wd = r->basex.cols;
  if (n < 1 || th < 2 || tw < 2 || hd < 1 || wd < 1)
    return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: empty frames or template");
  const int64_t np64 = (int64_t)th * tw;
  if (np64 > (1LL << 30) || hd * wd > (1LL << 30)) return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: too large");
  const int np = (int)np64;
  const ss_matrix& fr = r->frames;
  if (!fr.data || fr.rows != hd || fr.cols != wd * n || (fr.dtype != SS_F32 && fr.dtype != SS_F64))
    return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: frames must be FP32 or FP64 h x (w * n_frames)");
  const int nk = (int)r->dx_knots.rows;
  std::vector<double> bx, by, tf, pkd, dxk, dyk;
  if (!host_f64(r->basex, hd, wd, bx) || !host_f64(r->basey, hd, wd, by) || !host_f64(r->tfrac, hd, wd, tf) ||
      !host_f64(r->prevknotind, hd, wd, pkd))
    return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: basex, basey, tfrac, prevknotind must be h x w in host memory");
  if (nk < 2 || !host_f64(r->dx_knots, nk, n, dxk) || !host_f64(r->dy_knots, nk, n, dyk))
    return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: dx_knots, dy_knots must be nknots x n_frames in host memory");
  std::vector<int> pk(pkd.size());
  for (size_t i = 0; i < pkd.size(); i++) {
    pk[i] = (int)pkd[i];
    if (!(pkd[i] >= 1 && pkd[i] <= nk - 1) || pk[i] != pkd[i])
      return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: prevknotind must be integers in 1..nknots-1");
  }
  const ss_matrix& o = r->out;
  if (!o.data || o.rows != th || o.cols != (int64_t)tw * n || (o.dtype != SS_F32 && o.dtype != SS_F64))
    return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: out must be FP32 or FP64 template_h x (template_w * n_frames)");
  if (!(r->regfac >= 0.0) || !(r->pixel_aspect_ratio > 0.0))
    return fail(SS_ERR_INVALID_ARGUMENT, "reconstruct: regfac >= 0 and pixel_aspect_ratio > 0 required");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SS_ERR_NO_DEVICE, "no CUDA device");
  if (r->gpu_device_id < 0 || r->gpu_device_id >= ndev) return fail(SS_ERR_INVALID_ARGUMENT, "gpu_device_id out of range");
  SS_CK(cudaSetDevice(r->gpu_device_id));

  const int chunk = std::min(n, 64);
  const size_t px = (size_t)hd * wd, fsz = fr.dtype == SS_F64 ? 8 : 4, osz = o.dtype == SS_F64 ? 8 : 4;
  CallMem m;
  SS_CK(cudaStreamCreateWithFlags(&m.s, cudaStreamNonBlocking));
  cudaStream_t s = m.s;
  double* d_bx = m.take<double>(px);
  double* d_by = m.take<double>(px);
  double* d_tf = m.take<double>(px);
  int* d_pk = m.take<int>(px);
  double* d_dxk = m.take<double>((size_t)nk * n);
  double* d_dyk = m.take<double>((size_t)nk * n);
  const void* d_data = fr.data;
  if (fr.location == SS_HOST) {
    void* q = m.take<char>(fsz * px * n);
    if (q) SS_CK(cudaMemcpyAsync(q, fr.data, fsz * px * n, cudaMemcpyHostToDevice, s));
    d_data = q;
  }
  RcBufs b{};
  b.th = th;
  b.tw = tw;
  b.np = np;
  b.hd = (int)hd;
  b.wd = (int)wd;
  b.nk = nk;
  const size_t cnp = (size_t)chunk * np;
  b.wy = m.take<double>(cnp);
  b.ww = m.take<double>(cnp * kRcStencil);
  b.z = m.take<float>(cnp);
  b.cnt = m.take<float>(cnp);
  b.last_z = m.take<int>(cnp);
  b.last_n = m.take<int>(cnp);
  b.mask = m.take<uint8_t>(cnp);
  b.coef = m.take<float>(cnp * 10);
  b.le = m.take<float>(cnp);
  b.x = m.take<float>(cnp);
  b.xo = m.take<float>(cnp);
  b.part = m.take<double>((size_t)chunk * kRcParts);
  b.part_l = m.take<float>((size_t)chunk * kRcParts);
  int* d_state = m.take<int>(chunk);
  int* d_due = m.take<int>(chunk);
  int* d_keep = m.take<int>(chunk);
  int* d_iters = m.take<int>(chunk);
  int* d_interval = m.take<int>(chunk);
  int* d_count = m.take<int>(chunk);
  int* d_skip = m.take<int>(chunk);
  float* d_eo = m.take<float>(chunk);
  void* d_out = o.location == SS_DEVICE ? const_cast<void*>(o.data) : m.take<char>(osz * cnp);
  uint8_t* d_mk = r->mask ? m.take<uint8_t>(cnp) : nullptr;
  if (!d_bx || !d_by || !d_tf || !d_pk || !d_dxk || !d_dyk || !d_data || !b.wy || !b.ww || !b.z || !b.cnt ||
      !b.last_z || !b.last_n || !b.mask || !b.coef || !b.le || !b.x || !b.xo || !b.part || !b.part_l || !d_state ||
      !d_due || !d_keep || !d_iters || !d_interval || !d_count || !d_skip || !d_eo || !d_out || (r->mask && !d_mk))
    return fail(SS_ERR_OUT_OF_MEMORY, "reconstruct: work memory");
  SS_CK(cudaMemcpyAsync(d_bx, bx.data(), px * 8, cudaMemcpyHostToDevice, s));
  SS_CK(cudaMemcpyAsync(d_by, by.data(), px * 8, cudaMemcpyHostToDevice, s));
  SS_CK(cudaMemcpyAsync(d_tf, tf.data(), px * 8, cudaMemcpyHostToDevice, s));
  SS_CK(cudaMemcpyAsync(d_pk, pk.data(), px * 4, cudaMemcpyHostToDevice, s));
  SS_CK(cudaMemcpyAsync(d_dxk, dxk.data(), (size_t)nk * n * 8, cudaMemcpyHostToDevice, s));
  SS_CK(cudaMemcpyAsync(d_dyk, dyk.data(), (size_t)nk * n * 8, cudaMemcpyHostToDevice, s));
  const double regfac = r->regfac, vfac = 1.0 / r->pixel_aspect_ratio, vf2 = vfac * vfac;
  const int g = 148 * 8;

  // Frames [a, a + nf) of the set with check intervals iv[0..nf): their sweeps to completion, their
  // outputs into the chunk slots 0..nf; per-frame sweep counts (0: skipped) into it_out.
  auto run = [&](int a, int nf, const std::vector<int>& iv, std::vector<int>& it_out) -> int {
    const size_t fnp = (size_t)nf * np;
    SS_CK(cudaMemsetAsync(b.wy, 0, fnp * 8, s));
    SS_CK(cudaMemsetAsync(b.ww, 0, fnp * kRcStencil * 8, s));
    SS_CK(cudaMemsetAsync(b.z, 0, fnp * 4, s));
    SS_CK(cudaMemsetAsync(b.cnt, 0, fnp * 4, s));
    SS_CK(cudaMemsetAsync(d_count, 0, nf * 4, s));
    SS_CK(cudaMemsetAsync(d_iters, 0, nf * 4, s));
    if (fr.dtype == SS_F64)
      k_rc_constraints<double><<<g, 256, 0, s>>>(b, d_data, a, nf, d_bx, d_by, d_tf, d_pk, d_dxk, d_dyk);
    else
      k_rc_constraints<float><<<g, 256, 0, s>>>(b, d_data, a, nf, d_bx, d_by, d_tf, d_pk, d_dxk, d_dyk);
    for (int st = 0; st < 4; st++) {
      k_rc_fill_int<<<g, 256, 0, s>>>(b.last_z, fnp, -1);
      k_rc_fill_int<<<g, 256, 0, s>>>(b.last_n, fnp, -1);
      for (int ph = 0; ph < 2; ph++) {
        if (fr.dtype == SS_F64)
          k_rc_pushgrid<double><<<g, 256, 0, s>>>(b, d_data, a, nf, st, ph, d_bx, d_by, d_tf, d_pk, d_dxk, d_dyk);
        else
          k_rc_pushgrid<float><<<g, 256, 0, s>>>(b, d_data, a, nf, st, ph, d_bx, d_by, d_tf, d_pk, d_dxk, d_dyk);
      }
    }
    k_rc_mask<<<g, 256, 0, s>>>(b, nf);
    k_rc_coef<<<g, 256, 0, s>>>(b, nf, regfac, vf2);
    const dim3 fg(std::max(1, g / nf), nf);  // per-frame grids: at most g CTAs (one wave) over the frames
    k_rc_count<<<fg, 256, 0, s>>>(b, d_count);
    SS_CK(cudaGetLastError());
    std::vector<int> count(nf), state(nf), due(nf);
    SS_CK(cudaMemcpyAsync(count.data(), d_count, nf * 4, cudaMemcpyDeviceToHost, s));
    SS_CK(cudaStreamSynchronize(s));
    int running = 0;
    for (int f = 0; f < nf; f++) {
      state[f] = count[f] > 0 ? 1 : 3;
      due[f] = state[f] == 1;
      running += due[f];
    }
    SS_CK(cudaMemcpyAsync(d_state, state.data(), nf * 4, cudaMemcpyHostToDevice, s));
    SS_CK(cudaMemcpyAsync(d_due, due.data(), nf * 4, cudaMemcpyHostToDevice, s));
    SS_CK(cudaMemcpyAsync(d_interval, iv.data(), nf * 4, cudaMemcpyHostToDevice, s));
    std::vector<int> skip(nf);
    for (int f = 0; f < nf; f++) skip[f] = state[f] == 3;
    SS_CK(cudaMemcpyAsync(d_skip, skip.data(), nf * 4, cudaMemcpyHostToDevice, s));
    const dim3 eg(kRcParts, nf);
    const int cb = (nf + 127) / 128;
    k_rc_energy<<<eg, 256, 0, s>>>(b, nf, d_due, regfac, vf2);
    k_rc_check<<<cb, 128, 0, s>>>(nf, d_due, d_state, d_eo, d_keep, b.part, b.part_l, 1, 0, d_iters);
    const int kMaxSweeps = 1 << 22;
    for (int it = 1; running > 0; it++) {
      if (it > kMaxSweeps) return fail(SS_ERR_CUDA, "reconstruct: the energy kept decreasing over 4M sweeps");
      for (int colour = 0; colour < 4; colour++) k_rc_sweep<<<fg, 256, 0, s>>>(b, colour, d_state);
      k_rc_due<<<cb, 128, 0, s>>>(nf, d_state, d_interval, it, d_due);
      k_rc_energy<<<eg, 256, 0, s>>>(b, nf, d_due, regfac, vf2);
      k_rc_check<<<cb, 128, 0, s>>>(nf, d_due, d_state, d_eo, d_keep, b.part, b.part_l, 0, it, d_iters);
      k_rc_keep<<<fg, 256, 0, s>>>(b, d_keep);
      if (it % 8 == 0) {
        SS_CK(cudaMemcpyAsync(state.data(), d_state, nf * 4, cudaMemcpyDeviceToHost, s));
        SS_CK(cudaStreamSynchronize(s));
        running = 0;
        for (int f = 0; f < nf; f++) running += state[f] == 1;
      }
    }
    SS_CK(cudaGetLastError());
    it_out.resize(nf);
    SS_CK(cudaMemcpyAsync(it_out.data(), d_iters, nf * 4, cudaMemcpyDeviceToHost, s));
    char* dst = o.location == SS_DEVICE ? static_cast<char*>(d_out) + osz * (size_t)a * np : static_cast<char*>(d_out);
    if (o.dtype == SS_F64) k_rc_out<double><<<g, 256, 0, s>>>(b, nf, (double*)dst, d_mk, d_skip);
    else k_rc_out<float><<<g, 256, 0, s>>>(b, nf, (float*)dst, d_mk, d_skip);
    SS_CK(cudaStreamSynchronize(s));
    return SS_OK;
  };

  int carried = 1;  // the interval entering the next frame; 1 at the start of a call
  std::vector<int> last_iters;
  for (int f0 = 0; f0 < n; f0 += chunk) {
    const int F = std::min(chunk, n - f0);
    std::vector<int> guess(F, 10), iters(F, 0);
    guess[0] = carried;
    int start = 0;
    while (start < F) {
      std::vector<int> iv(guess.begin() + start, guess.end()), got;
      int rc = run(f0 + start, F - start, iv, got);
      if (rc) return rc;
      // the chain of intervals from `start`: frames up to the first mismatch ran with their own
      int cur = guess[start], bad = -1;
      for (int i = start; i < F; i++) {
        if (guess[i] != cur) {
          bad = i;
          break;
        }
        iters[i] = got[i - start];
        if (iters[i] > 0) cur = rc_interval(iters[i]);  // skipped frames keep the interval
      }
      const int good_end = bad < 0 ? F : bad;
      // outputs of the settled frames [start, good_end) to the host
      if (o.location == SS_HOST && good_end > start)
        SS_CK(cudaMemcpy(static_cast<char*>(const_cast<void*>(o.data)) + osz * (size_t)(f0 + start) * np,
                         d_out, osz * (size_t)(good_end - start) * np, cudaMemcpyDeviceToHost));
      if (r->mask && good_end > start)
        SS_CK(cudaMemcpy(r->mask + (size_t)(f0 + start) * np, d_mk, (size_t)(good_end - start) * np,
                         cudaMemcpyDeviceToHost));
      if (bad < 0) {
        carried = cur;
        break;
      }
      // re-run from the first frame that ran with another interval, with the intervals this run's
      // sweep counts give (its own is now exact)
      guess[bad] = cur;
      int g2 = cur;
      for (int i = bad + 1; i < F; i++) {
        const int prev = got[i - 1 - start];
        if (prev > 0) g2 = rc_interval(prev);
        guess[i] = g2;
      }
      start = bad;
    }
    if (r->iterations)
      for (int i = 0; i < F; i++) r->iterations[f0 + i] = iters[i];
  }
  return SS_OK;
}

}  // namespace ss

// ---------------------------------------------------------------------------------------------
// C ABI

extern "C" {

int ss_align_groups(int32_t n_groups, const ss_inputs* in, ss_outputs* out) {
  auto t0 = std::chrono::steady_clock::now();
  if (!in || n_groups < 1) return ss::fail(SS_ERR_INVALID_ARGUMENT, "no groups");
  ss::Batch b;
  b.set_stream_frames(true);  // frames of later groups upload while earlier groups run
  int rc = b.prepare(n_groups, in, out, nullptr, 0);
  if (!rc) rc = b.run();
  if (!rc) rc = b.collect();
  if (rc) return rc;
  double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (out)
    for (int i = 0; i < n_groups; i++) out[i].elapsed_ms = ms;
  ss::g_err.clear();
  return SS_OK;
}

int ss_align_group_to_template(const ss_inputs* in, ss_outputs* out) { return ss_align_groups(1, in, out); }

struct ss_batch {
  ss::Batch b;
};

struct ss_server {
  ss::Server v;
};

struct ss_session {
  ss::Batch b;
  std::vector<double> zeros, kx, ky;
};

int ss_batch_create(int32_t n_groups, const ss_inputs* in, ss_outputs* out, ss_batch** batch) {
  if (!batch || !in || n_groups < 1) return ss::fail(SS_ERR_INVALID_ARGUMENT, "bad batch arguments");
  *batch = nullptr;
  ss_batch* h = new ss_batch;
  int rc = h->b.prepare(n_groups, in, out, nullptr, 0);
  if (rc) {
    delete h;
    return rc;
  }
  *batch = h;
  return SS_OK;
}

int ss_session_create(const ss_inputs* proto, ss_session** session) {
  if (!proto || !session) return ss::fail(SS_ERR_INVALID_ARGUMENT, "bad session arguments");
  *session = nullptr;
  const int64_t hb = proto->basex.rows, w = proto->basex.cols;
  if (hb < 1 || w < 1) return ss::fail(SS_ERR_INVALID_ARGUMENT, "basex is empty");
  ss_session* h = new ss_session;
  // a one-frame group of zeros carries the session's template and geometry into device memory
  ss_inputs in = *proto;
  h->zeros.assign((size_t)hb * w, 0.0);
  h->kx.assign((size_t)w + 1, 0.0);
  h->ky.assign((size_t)w + 1, 0.0);
  in.n_frames = 1;
  in.bm_data = {h->zeros.data(), hb, w, SS_F64, SS_HOST};
  in.est_dx_knots = {h->kx.data(), w + 1, 1, SS_F64, SS_HOST};
  in.est_dy_knots = {h->ky.data(), w + 1, 1, SS_F64, SS_HOST};
  int rc = h->b.prepare(1, &in, nullptr, nullptr, 0);
  if (rc) {
    delete h;
    return rc;
  }
  *session = h;
  return SS_OK;
}

void ss_session_destroy(ss_session* session) { delete session; }

static std::vector<const ss::Batch*> session_list(int32_t n, ss_session* const* sessions) {
  std::vector<const ss::Batch*> v((size_t)n, nullptr);
  if (sessions)
    for (int32_t i = 0; i < n; i++) v[i] = sessions[i] ? &sessions[i]->b : nullptr;
  return v;
}

int ss_batch_measure(int32_t n_groups, const ss_inputs* in, ss_outputs* out, ss_session* const* sessions,
                     int64_t* arena_bytes) {
  if (!in || n_groups < 1 || !arena_bytes) return ss::fail(SS_ERR_INVALID_ARGUMENT, "bad batch arguments");
  ss::Batch b;
  const auto ses = session_list(n_groups, sessions);
  int rc = b.prepare(n_groups, in, out, nullptr, 0, ses.data(), true);
  if (rc) return rc;
  *arena_bytes = (int64_t)b.arena_bytes();
  return SS_OK;
}

int ss_batch_create_ex(int32_t n_groups, const ss_inputs* in, ss_outputs* out, ss_session* const* sessions,
                       void* arena, int64_t arena_bytes, ss_batch** batch) {
  if (!batch || !in || n_groups < 1 || (arena && arena_bytes <= 0))
    return ss::fail(SS_ERR_INVALID_ARGUMENT, "bad batch arguments");
  *batch = nullptr;
  ss_batch* h = new ss_batch;
  const auto ses = session_list(n_groups, sessions);
  int rc = h->b.prepare(n_groups, in, out, arena, arena ? (size_t)arena_bytes : 0, ses.data());
  if (rc) {
    delete h;
    return rc;
  }
  *batch = h;
  return SS_OK;
}

int ss_batch_start(ss_batch* batch) {
  if (!batch) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch is NULL");
  return batch->b.start();
}

int ss_batch_step(ss_batch* batch) {
  if (!batch) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch is NULL");
  return batch->b.step();
}

int ss_batch_poll(ss_batch* batch) {
  if (!batch) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch is NULL");
  return batch->b.poll();
}

int ss_server_create(int32_t capacity, int32_t device, ss_server** server) {
  if (!server) return ss::fail(SS_ERR_INVALID_ARGUMENT, "server is NULL");
  *server = nullptr;
  ss_server* h = new ss_server;
  int rc = h->v.create(capacity, device);
  if (rc) {
    delete h;
    return rc;
  }
  *server = h;
  return SS_OK;
}

int ss_server_admit(ss_server* server, const ss_inputs* in, ss_outputs* out, ss_session* session, void* arena,
                    int64_t arena_bytes, int32_t* slot) {
  if (!server || !slot || (arena && arena_bytes <= 0)) return ss::fail(SS_ERR_INVALID_ARGUMENT, "bad admit arguments");
  int k = -1;
  int rc = server->v.admit(in, out, session ? &session->b : nullptr, arena, arena ? (size_t)arena_bytes : 0, &k);
  *slot = k;
  return rc;
}

int ss_server_step(ss_server* server) {
  if (!server) return ss::fail(SS_ERR_INVALID_ARGUMENT, "server is NULL");
  return server->v.step();
}

int ss_server_poll(ss_server* server, int32_t* done_slots, int32_t max_done, int32_t* n_done) {
  if (!server || !n_done || (max_done > 0 && !done_slots)) return ss::fail(SS_ERR_INVALID_ARGUMENT, "bad poll arguments");
  int n = 0;
  int rc = server->v.poll(done_slots, max_done, &n);
  *n_done = n;
  return rc;
}

int32_t ss_server_active(const ss_server* server) { return server ? server->v.active() : 0; }

void ss_server_destroy(ss_server* server) { delete server; }

int ss_batch_run(ss_batch* batch) {
  if (!batch) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch is NULL");
  return batch->b.run();
}

int ss_batch_collect(ss_batch* batch) {
  if (!batch) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch is NULL");
  return batch->b.collect();
}

int ss_batch_set_timing(ss_batch* batch, int32_t on) {
  if (!batch) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch is NULL");
  batch->b.set_timing(on != 0);
  return SS_OK;
}

int ss_batch_set_graph(ss_batch* batch, int32_t on) {
  if (!batch) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch is NULL");
  batch->b.set_graph(on != 0);
  return SS_OK;
}

int ss_batch_stats_get(const ss_batch* batch, ss_batch_stats* stats) {
  if (!batch || !stats) return ss::fail(SS_ERR_INVALID_ARGUMENT, "batch or stats is NULL");
  batch->b.stats(stats);
  return SS_OK;
}

void* ss_batch_stream(const ss_batch* batch) { return batch ? batch->b.stream() : nullptr; }

}  // extern "C"

namespace ss {

// Workspace of ss_solve_block_tridiagonal_noalloc: the cyclic-reduction nodes of up to
// kNoAllocMaxBlocks blocks (3.4 MB). It is file-scope device memory, so every GPU that loads this
// library holds it until the process exits. Its host-side name is only a handle; the device
// address comes from cudaGetSymbolAddress, looked up on the first call per device and context
// below (a context created after cudaDeviceReset has its own copy of the array at its own address).
constexpr int kNoAllocMaxBlocks = 32768;
static __device__ __align__(256) double g_noalloc_work[(size_t)kNoAllocMaxBlocks * kCrStride];

struct NoAllocSlot {
  unsigned long long ctx = 0;  // context the address belongs to (0: not looked up)
  double* addr = nullptr;
};
static std::mutex g_noalloc_mu;
static NoAllocSlot g_noalloc_addr[128];  // per device ordinal

// Device address of g_noalloc_work on the current device and context, looked up on the first call
// in that context.
static int noalloc_workspace(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 128) return fail(SS_ERR_NO_DEVICE, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot& slot = g_noalloc_addr[dev];
  const unsigned long long ctx = current_context_id();
  if (!slot.addr || ctx == 0 || slot.ctx != ctx) {
    double* p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_work);
    if (e != cudaSuccess || !p)
      return fail(SS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    slot.addr = p;
    slot.ctx = current_context_id();  // the lookup makes the device's context current if none was
  }
  *out = slot.addr;
  return SS_OK;
}

}  // namespace ss

extern "C" {

int ss_solve_block_tridiagonal_noalloc(int32_t n, const double* diag, const double* coupling, const double* rhs,
                                       double* x, void* stream) {
  if (n < 1 || !diag || !rhs || !x || (n > 1 && !coupling))
    return ss::fail(SS_ERR_INVALID_ARGUMENT, "ss_solve_block_tridiagonal_noalloc: bad arguments");
  if (n > ss::kNoAllocMaxBlocks)
    return ss::fail(SS_ERR_INVALID_ARGUMENT, "ss_solve_block_tridiagonal_noalloc: n = " + std::to_string(n) +
                                                 " exceeds the fixed workspace of " +
                                                 std::to_string(ss::kNoAllocMaxBlocks) + " blocks");
  double* work = nullptr;
  int rc = ss::noalloc_workspace(&work);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // every node of the workspace that the solve reads is written first by k_block_tridiag
  cudaError_t ea = ss::block_tridiag_attr();
  if (ea != cudaSuccess) return ss::fail(SS_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ea));
  ss::k_block_tridiag<<<1, ss::kSolveThreads, ss::kSolveSmem, s>>>(n, diag, coupling, rhs, x, work);
  cudaError_t e = cudaGetLastError();
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e != cudaSuccess || e2 != cudaSuccess)
    return ss::fail(SS_ERR_CUDA, std::string("ss_solve_block_tridiagonal_noalloc: ") +
                                     cudaGetErrorString(e != cudaSuccess ? e : e2));
  ss::g_err.clear();
  return SS_OK;
}

int ss_solve_block_tridiagonal(int32_t n, const double* diag, const double* coupling, const double* rhs, double* x,
                               void* stream) {
  if (n < 1 || !diag || !rhs || !x || (n > 1 && !coupling))
    return ss::fail(SS_ERR_INVALID_ARGUMENT, "ss_solve_block_tridiagonal: bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* work = nullptr;
  cudaError_t e = cudaMallocAsync(&work, (size_t)n * ss::kCrStride * sizeof(double), s);
  if (e != cudaSuccess) return ss::fail(SS_ERR_OUT_OF_MEMORY, std::string("workspace: ") + cudaGetErrorString(e));
  cudaError_t ea = ss::block_tridiag_attr();
  if (ea != cudaSuccess) return ss::fail(SS_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ea));
  ss::k_block_tridiag<<<1, ss::kSolveThreads, ss::kSolveSmem, s>>>(n, diag, coupling, rhs, x, work);
  e = cudaGetLastError();
  cudaError_t e2 = cudaFreeAsync(work, s);
  cudaError_t e3 = cudaStreamSynchronize(s);
  if (e != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
    return ss::fail(SS_ERR_CUDA, std::string("ss_solve_block_tridiagonal: ") +
                                     cudaGetErrorString(e != cudaSuccess ? e : (e2 != cudaSuccess ? e2 : e3)));
  ss::g_err.clear();
  return SS_OK;
}

int ss_estimate_displacements(const ss_recording* rec, ss_recording_outputs* out) {
  int rc = ss::estimate_displacements(rec, out);
  if (!rc) ss::g_err.clear();
  return rc;
}

int ss_recording_sets(int32_t n_frames, int32_t frames_per_set, int32_t min_frames_per_set, int32_t* first,
                      int32_t* count, int32_t max_sets, int32_t* n_sets) {
  int rc = ss::recording_sets(n_frames, frames_per_set, min_frames_per_set, first, count, max_sets, n_sets);
  if (!rc) ss::g_err.clear();
  return rc;
}

int ss_reconstruct_frames(const ss_reconstruct* r) {
  int rc = ss::reconstruct_frames(r);
  if (!rc) ss::g_err.clear();
  return rc;
}

int ss_prepare_frames(const ss_prep_frames* p) {
  int rc = ss::prepare_frames(p);
  if (!rc) ss::g_err.clear();
  return rc;
}

void ss_batch_destroy(ss_batch* batch) { delete batch; }

const char* ss_last_error(void) { return ss::last_error(); }

int32_t ss_abi_version(void) { return SS_ABI_VERSION; }

}  // extern "C"
