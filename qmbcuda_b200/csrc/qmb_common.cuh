// qmb_common.cuh -- shared device/host helpers of libqmb_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "qmb_b200.h"

namespace qmb {

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
qmb_status fail(qmb_status s, const std::string& msg);

struct Error {
    qmb_status code;
    std::string msg;
};

#define QMB_CUDA_TRY(expr)                                                                   \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess)                                                               \
            throw ::qmb::Error{_e == cudaErrorMemoryAllocation ? QMB_ERR_NOMEM : QMB_ERR_CUDA, \
                               std::string(#expr) + ": " + cudaGetErrorString(_e)};          \
    } while (0)

#define QMB_REQUIRE(cond, code, msg)                 \
    do {                                             \
        if (!(cond)) throw ::qmb::Error{code, msg};  \
    } while (0)

// Runs f, converting exceptions into a status.
template <class F>
qmb_status guarded(F&& f) {
    try {
        f();
        return QMB_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return fail(QMB_ERR_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(QMB_ERR_INVALID, e.what());
    }
}

// ------------------------------------------------------------ device memory
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        QMB_CUDA_TRY(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void zero(cudaStream_t st = 0) { QMB_CUDA_TRY(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
    void upload(const T* h, size_t count, cudaStream_t st = 0) {
        QMB_CUDA_TRY(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    void download(T* h, size_t count, cudaStream_t st = 0) const {
        QMB_CUDA_TRY(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, st));
    }
};

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
            throw Error{QMB_ERR_NO_DEVICE, "no CUDA device is visible"};
        QMB_REQUIRE(dev >= 0 && dev < n, QMB_ERR_INVALID, "device ordinal out of range");
        cudaGetDevice(&prev);
        QMB_CUDA_TRY(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

inline void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error{QMB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

// ---------------------------------------------------------------- binomials
uint64_t host_binom(int n, int k);

// Next string with the same popcount (Gosper's hack); s != 0.
__host__ __device__ __forceinline__ uint64_t next_comb(uint64_t s) {
    uint64_t c = s & (~s + 1);
    uint64_t r = s + c;
    return (((r ^ s) >> 2) / c) | r;
}

// ----------------------------------------------------------- group elements
// An element maps bit q to bit perm[q], optionally followed by inversion of
// all L bits.  When every site map is a lattice translation of a torus whose
// rows are W consecutive bits, the map is a rotation of the rows plus a
// rotation inside every row; those run as a few word operations.  Otherwise
// each element uses a table of 16 entries per 4-bit chunk.
struct GroupDev {
    int L;
    int G;           // site maps
    int n_ext;       // G or 2G (with inversion)
    int structured;  // 1: rotations, 0: nibble tables
    int W;           // row width in bits (structured)
    int n_chunks;    // ceil(L/4) (tables)
    uint64_t mask;   // low L bits
    uint64_t row_lo_mask[65];  // unused slots zero; see apply_rot
    const uint8_t* rot_row;    // [G] row rotation (bits, multiple of W)
    const uint8_t* rot_in;     // [G] rotation inside rows (bits)
    const uint64_t* tables;    // [G][n_chunks][16]
};

__device__ __forceinline__ uint64_t rotl_bits(uint64_t x, int r, int L, uint64_t mask) {
    if (r == 0) return x;
    return ((x << r) | (x >> (L - r))) & mask;
}

// Rotation by c bits inside each W-bit row of an L-bit word (L multiple of W).
// lo = bits whose in-row position is < W - c (they move up by c), the rest
// wrap to the bottom of their row.
__device__ __forceinline__ uint64_t rot_rows(uint64_t x, int c, int W, uint64_t lo) {
    if (c == 0) return x;
    return ((x & lo) << c) | ((x & ~lo) >> (W - c));
}

}  // namespace qmb
