/* Force-included shim that lets g++ compile the reference's race-free CUDA device functions and
 * host classes as plain host code, for pinning the oracle: TEST INFRASTRUCTURE ONLY.
 *
 * CUDA qualifiers become no-ops, the thread/block indices become globals that the wrapper sets
 * while it walks the launch grid in order, and the few CUDA runtime and library types that the
 * reference's headers name are stubbed. No GPU is involved.
 */
#ifndef SS_REF_PIN_SHIM_H_
#define SS_REF_PIN_SHIM_H_

#ifndef _DEBUG
#define _DEBUG 1 /* debug.h: keeps the MATLAB (mex.h) code paths out */
#endif
#define CUDAINCLUDES_H_ /* the reference's cudaincludes.h is replaced by the lines below */
#define CUDAHELPER_CUH_

#include <cstddef>
#include <cstring>
#include <cmath>
#include <cfloat>
#include <climits>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline

struct ss_pin_dim3 { unsigned int x, y, z; };
extern ss_pin_dim3 blockIdx, blockDim, threadIdx, gridDim;
inline void __syncthreads() {}

typedef void* cusparseHandle_t;
typedef void* cusolverSpHandle_t;
typedef void* cusparseMatDescr_t;
typedef int cudaError_t;
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2,
                      cudaMemcpyDeviceToDevice = 3 };
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
    std::memcpy(d, s, n);
    return 0;
}

#define IDX2C(i, j, ld) (((j) * (ld)) + (i))
#define IDX2R(i, j, ld) (((i) * (ld)) + (j))
#define THREADS_PER_BLOCK 256

#endif
