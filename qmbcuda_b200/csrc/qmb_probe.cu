// qmb_probe.cu -- a measurement entry point: the device's bandwidth for the
// access pattern of the batched product's gathers (whole rows of a
// [row][set] vector, read at scattered rows of a buffer that stays in L2),
// with nothing else in the kernel.  The batched H*v kernel is compared with
// it beside the HBM copy bandwidth: its x gathers can go no faster than this.
#include <cuda_runtime.h>

#include <algorithm>

#include "qmb_common.cuh"

namespace qmb {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeUnroll = 8;

__device__ __forceinline__ uint32_t probe_hash(uint32_t a) {
    a ^= a >> 16;
    a *= 0x7feb352du;
    a ^= a >> 15;
    a *= 0x846ca68bu;
    a ^= a >> 16;
    return a;
}

// A row group of row_u4 threads (one 16-byte word of the row each) gathers
// `per_group` rows chosen by a hash, kProbeUnroll loads in flight per thread.
__global__ void __launch_bounds__(kProbeThreads) k_gather_probe(const uint4* __restrict__ x, uint32_t rows,
                                                                 int row_u4, int64_t per_group,
                                                                 float* __restrict__ sink) {
    const int RG = kProbeThreads / row_u4;
    const int rg = threadIdx.x / row_u4, t = threadIdx.x % row_u4;
    if (rg >= RG) return;
    const uint32_t grp = blockIdx.x * RG + rg;
    float acc = 0.0f;
    for (int64_t i = 0; i < per_group; i += kProbeUnroll) {
        uint4 v[kProbeUnroll];
#pragma unroll
        for (int u = 0; u < kProbeUnroll; ++u) {
            const uint32_t row = probe_hash(grp * 0x9e3779b9u + (uint32_t)(i + u)) % rows;
            v[u] = x[(size_t)row * row_u4 + t];
        }
#pragma unroll
        for (int u = 0; u < kProbeUnroll; ++u)
            acc += __uint_as_float(v[u].x) + __uint_as_float(v[u].y) + __uint_as_float(v[u].z) +
                   __uint_as_float(v[u].w);
    }
    if (acc == 1.0e30f) sink[blockIdx.x] = acc;  // keeps the loads; the buffer is zero
}

}  // namespace
}  // namespace qmb

using namespace qmb;

extern "C" qmb_status qmb_l2_gather_probe(int64_t rows, int row_bytes, int64_t gathers, double* gbs, double* ms) {
    return guarded([&] {
        QMB_REQUIRE(gbs && ms, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(rows >= 1 && rows <= (1ll << 31), QMB_ERR_INVALID, "rows must be in 1..2^31");
        QMB_REQUIRE(row_bytes >= 16 && row_bytes <= 16 * kProbeThreads && row_bytes % 16 == 0 &&
                        (kProbeThreads / (row_bytes / 16)) * (row_bytes / 16) == kProbeThreads,
                    QMB_ERR_INVALID, "row_bytes must be 16 * a power of two, at most 4096");
        QMB_REQUIRE(gathers >= 1, QMB_ERR_INVALID, "gathers must be positive");
        int dev = 0, sms = 0;
        QMB_CUDA_TRY(cudaGetDevice(&dev));
        QMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int row_u4 = row_bytes / 16;
        const int RG = kProbeThreads / row_u4;
        int per_sm = 0;
        QMB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather_probe, kProbeThreads, 0));
        const int blocks = std::max(1, per_sm) * sms;
        const int64_t groups = (int64_t)blocks * RG;
        int64_t per_group = (gathers + groups - 1) / groups;
        per_group = (per_group + kProbeUnroll - 1) / kProbeUnroll * kProbeUnroll;
        DevBuf<uint4> x((size_t)rows * row_u4);
        x.zero();
        DevBuf<float> sink(blocks);
        cudaEvent_t e0, e1;
        QMB_CUDA_TRY(cudaEventCreate(&e0));
        QMB_CUDA_TRY(cudaEventCreate(&e1));
        struct EG { cudaEvent_t a, b; ~EG() { cudaEventDestroy(a); cudaEventDestroy(b); } } eg{e0, e1};
        float best = 1e30f;
        for (int rep = 0; rep < 6; ++rep) {
            QMB_CUDA_TRY(cudaEventRecord(e0));
            k_gather_probe<<<blocks, kProbeThreads>>>(x.p, (uint32_t)rows, row_u4, per_group, sink.p);
            QMB_CUDA_TRY(cudaEventRecord(e1));
            QMB_CUDA_TRY(cudaEventSynchronize(e1));
            check_launch("k_gather_probe");
            float t = 0.0f;
            QMB_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
            if (rep > 0) best = std::min(best, t);  // the first launch warms L2
        }
        *ms = best;
        *gbs = (double)groups * per_group * row_bytes / (best * 1e-3) / 1e9;
    });
}
