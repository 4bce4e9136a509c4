// qmb_lanczos.cuh -- device reductions shared by the Lanczos engines.
#pragma once
#include "qmb_scalar.cuh"

namespace qmb {

// Sum over the block; valid in thread 0.  Fixed shuffle tree, so the result
// depends only on the per-thread inputs (deterministic).
__device__ __forceinline__ double block_sum(double v, double* red /* >= 32 */) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        s = l < nw ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    return s;
}

// Grid-wide deterministic reduction: every block publishes its partial, the
// last block to arrive sums the partials in block order and returns true in
// all of its threads with the total in *total (thread 0).  counter is reset.
__device__ __forceinline__ bool grid_reduce(double v, double* partials, unsigned* counter,
                                            double* red, double* total) {
    __shared__ bool last;
    double b = block_sum(v, red);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = b;
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) s += __ldcg(partials + i);
    s = block_sum(s, red);
    if (threadIdx.x == 0) {
        *total = s;
        *counter = 0;
    }
    return true;
}

}  // namespace qmb
