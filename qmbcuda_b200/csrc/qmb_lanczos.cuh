// qmb_lanczos.cuh -- device reductions shared by the Lanczos engines.
#pragma once
#include <cstdlib>
#include "qmb_scalar.cuh"

namespace qmb {

// Gap cap of an FP64 restart from an FP32 Ritz vector, relative to |theta|.
// Two levels closer than the FP32 phase resolves (about 1e-6 |theta|) look
// like one Ritz value there, so the FP32 gap to the next visible level says
// nothing about them: the restart's Ritz vector can be a blend c1 u1 + c2 u2
// of the pair, with a residual of |c1 c2| times their splitting and an
// energy between the two.  The restart bounds its energy error with a gap of
// at most cap |theta|, so it accepts only residuals below sqrt(tol cap) |theta|
// and keeps going until such a pair separates, unless the FP32 vector holds
// almost none of the lower level (|c1 / c2| below about that bound over the
// splitting).  On an L=20 pair split by 1.2e-7 |theta|, 256 start vectors:
// 8 end on the upper level at cap 1e-4, 32 at 1e-3, 1 at 1e-5, none at 1e-6,
// against 126 without a cap; the L=20 batch solve takes 119, 111, 131 and
// 105 ms at caps 1e-4, 1e-3, 1e-5 and none.
constexpr double kRestartGapCap = 1e-4;

// The cap in effect: QMB_RESTART_GAP_CAP=x (x > 0) replaces the default.
inline double restart_gap_cap() {
    const char* e = std::getenv("QMB_RESTART_GAP_CAP");
    const double v = e ? std::atof(e) : 0.0;
    return v > 0.0 ? v : kRestartGapCap;
}

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
