// Shared helpers of libincrmt_gpu: status handling, launch geometry and
// block reductions.
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdarg>
#include <string>
#include "incrmt.h"

namespace incrmt {

/** Records the calling thread's last error message. */
void set_error(const char *fmt, ...);

/** Converts a CUDA error into INCRMT_ERR_CUDA / INCRMT_ERR_OOM with a message. */
int cuda_status(cudaError_t e, const char *what, const char *file, int line);

#define INCRMT_CK(expr)                                                        \
    do {                                                                       \
        cudaError_t e_ = (expr);                                               \
        if (e_ != cudaSuccess) return incrmt::cuda_status(e_, #expr, __FILE__, __LINE__); \
    } while (0)

/** Checks the launch that was just issued. */
#define INCRMT_CKL(what)                                                       \
    do {                                                                       \
        cudaError_t e_ = cudaGetLastError();                                   \
        if (e_ != cudaSuccess) return incrmt::cuda_status(e_, what, __FILE__, __LINE__); \
    } while (0)

/** Number of streaming multiprocessors of a B200. Grids of grid-stride
 * kernels are sized in multiples of it. */
constexpr int kB200SMs = 148;

inline int cdiv(long a, long b) { return static_cast<int>((a + b - 1) / b); }

/** Sum over a block of 256 threads; the result is valid in thread 0. */
template <class T>
__device__ __forceinline__ T block_sum_256(T v) {
    __shared__ T warp_part[8];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_part[w] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x < 8) t = warp_part[threadIdx.x];
    if (w == 0) {
        for (int o = 4; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;
}

}  // namespace incrmt
