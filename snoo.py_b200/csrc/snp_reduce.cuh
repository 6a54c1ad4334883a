// Device helpers shared by the Krylov engines: Dirichlet mask test and deterministic
// last-block reductions (every block writes its partial sum, the block that takes the last
// ticket of an atomicInc counter reduces them in a fixed order; nobody waits).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "snp_common.cuh"

namespace snp {

__device__ __forceinline__ bool is_free(const uint8_t *free_mask, int64_t i) { return free_mask == nullptr || free_mask[i]; }

// True in every thread of the block that took the last ticket (the counter wraps to 0).
__device__ __forceinline__ bool last_block(unsigned int *counter) {
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int t = atomicInc(counter, gridDim.x - 1);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return s_last;
}

// Sum of `part[i * width + comp]` over i < nparts; valid in thread 0.
template <typename T>
__device__ double reduce_parts(const T *part, int nparts, int width, int comp, double *sh) {
    double v = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) v += (double)__ldcg(part + (int64_t)i * width + comp);
    v = block_sum(v, sh);
    return v;
}

// Sum of two per-thread values over the block; results valid in thread 0.
__device__ __forceinline__ void block_sum2(double &a, double &b, double (*sh)[32]) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = a;
        sh[1][wid] = b;
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    a = (threadIdx.x < nw) ? sh[0][threadIdx.x] : 0.0;
    b = (threadIdx.x < nw) ? sh[1][threadIdx.x] : 0.0;
    if (wid == 0) {
        a = warp_sum(a);
        b = warp_sum(b);
    }
}

}  // namespace snp
