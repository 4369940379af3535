/* Force-included by the host build of the reference's task layer (oracle/_ref/run, made by
 * run_transform.py): TEST INFRASTRUCTURE ONLY, for pinning the oracle's Gauss-Newton trajectory to
 * the reference's own code. No GPU is involved.
 *
 * The real CUDA headers give the types and declarations; hostcuda.cpp defines the few runtime,
 * cuSPARSE and cuSOLVER entry points the task layer calls, on host memory. A kernel launch
 * (SS_LAUNCH) runs the grid's blocks one after another; each block's threads are cooperative
 * fibers that run in thread order up to the next __syncthreads() (or lock-step read), so block
 * barriers and shared memory behave as on the device. The reference's configuration headers are
 * replaced: no MATLAB, no Eigen (localdependencies.h is skipped), Thrust on its CPP backend.
 */
#ifndef SS_HOSTCUDA_H_
#define SS_HOSTCUDA_H_

#ifndef _DEBUG
#define _DEBUG 1
#endif
#define LOCALDEPENDENCIES_H_ /* no Eigen or MATLAB include paths */

#include <cuda_runtime.h>

#include <thrust/count.h> /* named by task_correlation.cu:80 without its header */

#include <cmath>
#include <cstddef>
#include <cstring>
#include <functional>
#include <iostream> /* std::cout in cudahelper.cu */

struct ss_dim3 {
  unsigned int x, y, z;
};
extern ss_dim3 ss_threadIdx, ss_blockIdx, ss_blockDim, ss_gridDim;
#define threadIdx ss_threadIdx
#define blockIdx ss_blockIdx
#define blockDim ss_blockDim
#define gridDim ss_gridDim

/* block barrier of the running block's fibers */
void ss_syncthreads();
#define __syncthreads() ss_syncthreads()

/* shared memory: a static shared by the block's fibers; the dynamic buffer is one global array */
#define SS_SHARED static
#define SS_EXTERN_SHARED extern
extern char s_mem[];

inline ss_dim3 ss_dim(unsigned int v) { return ss_dim3{v, 1, 1}; }
inline ss_dim3 ss_dim(int v) { return ss_dim3{(unsigned int)v, 1, 1}; }
inline ss_dim3 ss_dim(long v) { return ss_dim3{(unsigned int)v, 1, 1}; }
inline ss_dim3 ss_dim(unsigned long v) { return ss_dim3{(unsigned int)v, 1, 1}; }
inline ss_dim3 ss_dim(const dim3& d) { return ss_dim3{d.x, d.y, d.z}; }

/* runs `body` for every thread of a grid of `g` blocks of `b` threads */
void ss_launch(ss_dim3 g, ss_dim3 b, const std::function<void()>& body);
#define SS_LAUNCH(g, b, smem, call) ss_launch(ss_dim(g), ss_dim(b), [&]() { call; })

/* Called by the rewritten host launcher of d_linesearch (defined in refrun.cpp). */
template <typename T>
struct DeviceMemory;
template <class T>
void ss_refrun_sync_boundary(DeviceMemory<T>& mem);

/* A read of block-wide state that the reference's threads read and then change without a barrier
 * in between (a warp in lock step reads before any of its threads writes): the value is read,
 * then every thread of the block reaches this point before any goes on. */
void ss_lockstep_point();
template <class T>
inline T ss_lockstep_read(const T& v) {
  T r = v;
  ss_lockstep_point();
  return r;
}

#endif
