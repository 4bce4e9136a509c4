/*
 * ref_gpu_harness.cu -- runs the reference's own GPU Lanczos,
 * LanczosEigVals_CUDA<T> (exact_diagonalization/lanczos.cu:128-317), compiled
 * unmodified for sm_100a together with the kernels and library wrappers it
 * calls (exact_diagonalization/utils.cu, cuda_wrappers/CudaWrappers.cu,
 * utils/misc_funcs_gpu.cu, utils/print_funcs.cu) by oracle/Makefile into
 * oracle/_ref/libqmb_ref_gpu.so.  TEST INFRASTRUCTURE ONLY: the comparator
 * that tests/ hold the engine's reference-layout Lanczos against; never
 * linked into the product.
 *
 * Allocation padding.  init_random_vec (utils/misc_funcs_gpu.cu:31-52) tests
 * `id > nobv`, so it also writes element nobv of the start vector and of the
 * curandState array, both allocated by LanczosEigVals_CUDA and
 * LanczosEigenStateFromSeed with exactly nobv elements (lanczos.cu:156-164,
 * 49-55).  The library is linked with --wrap=cudaMalloc: every cudaMalloc
 * made from the reference's objects (thrust's vectors included) goes through
 * __wrap_cudaMalloc below, which asks for kPad more bytes, so those one-past
 * writes land inside their own allocation.  qmb_refgpu_padded_allocs()
 * counts the padded calls; qmb_refgpu_probe_alloc() lets a host without a
 * GPU check that thrust's allocations take this path.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>
#include <thrust/complex.h>
#include <thrust/device_vector.h>

#include "exact_diagonalization/lanczos.h"

using complex_th = thrust::complex<float>;

static constexpr size_t kPad = 1024;  // >= one float2 and one 48-byte curandState
static long long g_padded = 0;

extern "C" cudaError_t __real_cudaMalloc(void** p, size_t n);
extern "C" cudaError_t __wrap_cudaMalloc(void** p, size_t n) {
    ++g_padded;
    return __real_cudaMalloc(p, n + kPad);
}

extern "C" long long qmb_refgpu_padded_allocs() { return g_padded; }

/* A thrust device vector of 16 floats, as the reference's Lanczos allocates
 * them: 0 when it was allocated, 1 when the allocation failed (no device). */
extern "C" int qmb_refgpu_probe_alloc() {
    try {
        thrust::device_vector<float> v(16);
        return 0;
    } catch (...) {
        cudaGetLastError();
        return 1;
    }
}

/* pow2ceil (utils/misc_funcs.cu, which needs Armadillo and is not built):
 * the next power of two >= v.  LanczosEigVals_CUDA only prints it. */
int pow2ceil(uint32_t v) {
    uint32_t p = 1;
    while (p < v && p) p <<= 1;
    return (int)p;
}

/* LanczosEigVals_CUDA<T> on a reference-layout ELL given in host memory
 * (ind [nobv*max_terms], val [nobv*max_terms] float or interleaved complex,
 * track [nobv]): the tables are copied to the device (padded allocations),
 * the reference solves with NStates = 1, exportKrylovVec = true and the
 * given checkEigState, and E, the NIter Krylov coefficients and the returned
 * residual come back.  Returns 0, or the CUDA error code of a failed copy. */
extern "C" int qmb_refgpu_lanczos(int is_complex, int n_iter, int nobv, int max_terms, long long seed,
                                  const uint32_t* ind, const float* val, const int16_t* track,
                                  int check_eig_state, float* E, float* krylov, float* residual) {
    const size_t ne = (size_t)nobv * max_terms;
    const size_t vs = is_complex ? 2 * sizeof(float) : sizeof(float);
    uint32_t* d_ind = nullptr;
    void* d_val = nullptr;
    short* d_tr = nullptr;
    cudaError_t e = cudaMalloc((void**)&d_ind, ne * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_val, ne * vs);
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_tr, (size_t)nobv * sizeof(short));
    if (e == cudaSuccess) e = cudaMemcpy(d_ind, ind, ne * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_val, val, ne * vs, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_tr, track, (size_t)nobv * sizeof(short), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        std::vector<float> kv(n_iter, 0.0f);
        float r;
        if (is_complex)
            r = LanczosEigVals_CUDA<complex_th>(E, 1, n_iter, nobv, max_terms, seed, d_ind,
                                                static_cast<complex_th*>(d_val), d_tr, kv.data(), true,
                                                check_eig_state != 0);
        else
            r = LanczosEigVals_CUDA<float>(E, 1, n_iter, nobv, max_terms, seed, d_ind,
                                           static_cast<float*>(d_val), d_tr, kv.data(), true,
                                           check_eig_state != 0);
        if (krylov) std::memcpy(krylov, kv.data(), sizeof(float) * n_iter);
        if (residual) *residual = r;
        e = cudaDeviceSynchronize();
    }
    cudaFree(d_ind);
    cudaFree(d_val);
    cudaFree(d_tr);
    std::fflush(stdout);
    return (int)e;
}
