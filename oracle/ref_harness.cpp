/*
 * ref_harness.cpp -- drives the reference's own kernels and model classes,
 * compiled for the host from the unmodified sources (oracle/Makefile), so the
 * oracle can be checked against the reference itself.  TEST INFRASTRUCTURE
 * ONLY: called from tests/, tests/golden/make_golden.py and bench.py's
 * reference / cpu_baseline legs; never linked into the product.
 *
 * A "launch" runs every (block, thread) of the grid sequentially.  The
 * emulated kernels are the per-thread kernels of
 * exact_diagonalization/utils.cu, none of which uses shared memory or
 * intra-block synchronisation, so a sequential run computes what the GPU
 * computes; where threads race (ComputeOrbitIndices) the sequential order
 * keeps the last writer.  Kernel call sequences mirror the reference drivers
 * with the cited lines.
 */
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <thrust/complex.h>
#include <curand_kernel.h>

#include "exact_diagonalization/utils.h"
#include "utils/misc_funcs_gpu.h"
#include "lattice_models/T_standard.h"

using cf = thrust::complex<float>;

extern "C" void qmb_ref_set_thread(unsigned block, unsigned thread, unsigned block_dim,
                                   unsigned grid_dim);

template <class F>
static void launch(long long n_threads, unsigned block, F&& body) {
    if (n_threads <= 0) return;
    unsigned grid = (unsigned)((n_threads + block - 1) / block);
    for (unsigned b = 0; b < grid; ++b)
        for (unsigned t = 0; t < block; ++t) {
            qmb_ref_set_thread(b, t, block, grid);
            body();
        }
}

extern "C" int ref_rank(uint32_t s, int k) { return GetIndexInHilbertSubspace(s, k); }

extern "C" double ref_nchoosek_dev(double n, double k) { return NChoosek2_dev(n, k); }

/* Basis (BuildBasisStates order) for uint32 states. */
static std::vector<uint32_t> basis(int L, int k) {
    std::vector<uint32_t> out;
    for (uint64_t i = 0; i < (1ull << L); ++i)
        if (__builtin_popcountll(i) == k) out.push_back((uint32_t)i);
    return out;
}

/* BuildSRStates (exact_diagonalization/HeisenbergHamAbelianSymms_CUDA.cu:340-427)
 * for char type T.  Outputs: reps as sector ranks [R], SRS orbit table [R*G],
 * norms [R*NIr], orbit_indices [2N].  Returns R (or -R if reps_cap too small). */
template <class T>
static int build_srs(int L, int k, int G, const uint32_t* group_el, int NIr, const T* chars,
                     uint32_t* reps_out, int reps_cap, uint32_t* srs_out, float* norms_out,
                     uint32_t* orbit_out) {
    std::vector<uint32_t> bas = basis(L, k);
    int N = (int)bas.size();
    std::vector<uint32_t> ge(group_el, group_el + (size_t)G * L);
    std::vector<T> ch(chars, chars + (size_t)NIr * G);
    std::vector<uint32_t> srs((size_t)N * G), srs_min(N);
    const int th = 32;  /* threads_GS (HeisenbergHamAbelianSymms_CUDA.cu:43) */
    launch((long long)N * G, th, [&] { SetUpSRS(bas.data(), srs.data(), ge.data(), N, G, L, k); });
    launch(N, th, [&] { SolveSRS_min(srs.data(), srs_min.data(), N, G); });
    std::sort(srs_min.begin(), srs_min.end());
    int R = (int)(std::unique(srs_min.begin(), srs_min.end()) - srs_min.begin());
    launch((long long)R * G, th, [&] {
        SetUpSRS_from_indices(srs_min.data(), srs.data(), ge.data(), R, G, L, k, bas.data());
    });
    std::vector<float> norms((size_t)R * NIr);
    launch((long long)R * NIr, th, [&] {
        ComputeSRSNorms<T>(norms.data(), srs.data(), ch.data(), R, NIr, G, bas.data());
    });
    std::vector<uint32_t> oi((size_t)2 * N, 0);
    launch((long long)R * G, th, [&] { ComputeOrbitIndices(oi.data(), R, G, srs.data(), k); });
    if (R > reps_cap) return -R;
    std::memcpy(reps_out, srs_min.data(), sizeof(uint32_t) * R);
    if (srs_out) std::memcpy(srs_out, srs.data(), sizeof(uint32_t) * (size_t)R * G);
    if (norms_out) std::memcpy(norms_out, norms.data(), sizeof(float) * (size_t)R * NIr);
    if (orbit_out) std::memcpy(orbit_out, oi.data(), sizeof(uint32_t) * 2 * (size_t)N);
    return R;
}

extern "C" int ref_build_srs_real(int L, int k, int G, const uint32_t* group_el, int NIr, const float* chars,
                       uint32_t* reps_out, int reps_cap, uint32_t* srs_out, float* norms_out,
                       uint32_t* orbit_out) {
    return build_srs<float>(L, k, G, group_el, NIr, chars, reps_out, reps_cap, srs_out, norms_out,
                            orbit_out);
}

extern "C" int ref_build_srs_complex(int L, int k, int G, const uint32_t* group_el, int NIr,
                          const float* chars_ri, uint32_t* reps_out, int reps_cap,
                          uint32_t* srs_out, float* norms_out, uint32_t* orbit_out) {
    return build_srs<cf>(L, k, G, group_el, NIr, reinterpret_cast<const cf*>(chars_ri), reps_out,
                         reps_cap, srs_out, norms_out, orbit_out);
}

/* BuildHamiltonianForAbelianGroup<T> over all R orbit rows, after the
 * fills of HeisenbergHamAbelianSymms_CUDA.cu:124-126 and the launch of
 * :131-136.  val is T[R*W] (complex as interleaved floats). */
template <class T>
static void ham_bonds(float jxy_w, float jz_w, int L, int k, int G, int R, const uint32_t* srs,
                      const uint32_t* orbit, int NIr, const T* chars, int alpha,
                      const float* norms, float tol, int T_size, const int* ti, const int* tj,
                      const T* tval, int W, uint32_t* ind, T* val, short* track) {
    std::vector<uint32_t> bas = basis(L, k);
    std::fill(ind, ind + (size_t)R * W, 0u);
    std::fill(val, val + (size_t)R * W, T(0));
    std::fill(track, track + R, (short)0);
    launch(R, 32, [&] {
        BuildHamiltonianForAbelianGroup<T>(
            jxy_w, jz_w, k, bas.data(), ind, val, track, W, R, const_cast<int*>(ti),
            const_cast<int*>(tj), const_cast<T*>(tval), T_size, const_cast<uint32_t*>(srs), G,
            const_cast<uint32_t*>(orbit), const_cast<T*>(chars), alpha, const_cast<float*>(norms),
            NIr, tol);
    });
}

extern "C" void ref_ham_bonds_real(float jxy_w, float jz_w, int L, int k, int G, int R, const uint32_t* srs,
                        const uint32_t* orbit, int NIr, const float* chars, int alpha,
                        const float* norms, float tol, int T_size, const int* ti, const int* tj,
                        const float* tval, int W, uint32_t* ind, float* val, short* track) {
    ham_bonds<float>(jxy_w, jz_w, L, k, G, R, srs, orbit, NIr, chars, alpha, norms, tol, T_size,
                     ti, tj, tval, W, ind, val, track);
}

extern "C" void ref_ham_bonds_complex(float jxy_w, float jz_w, int L, int k, int G, int R,
                           const uint32_t* srs, const uint32_t* orbit, int NIr,
                           const float* chars, int alpha, const float* norms, float tol,
                           int T_size, const int* ti, const int* tj, const float* tval, int W,
                           uint32_t* ind, float* val, short* track) {
    ham_bonds<cf>(jxy_w, jz_w, L, k, G, R, srs, orbit, NIr, reinterpret_cast<const cf*>(chars),
                  alpha, norms, tol, T_size, ti, tj, reinterpret_cast<const cf*>(tval), W, ind,
                  reinterpret_cast<cf*>(val), track);
}

/* BuildHamiltonianXXZForAbelianGroup<T> (launch of
 * HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:229-259).  op codes follow
 * OperatorType (quantum_operators/SingleParticleOperators.h:4). */
template <class T>
static void ham_terms(int L, int k, int G, int R, const uint32_t* srs, const uint32_t* orbit,
                      int NIr, const T* chars, int alpha, const float* norms, float tol,
                      int H_size, int H_col, const int* n_ops, const int* codes,
                      const int* sites, const T* scalars, int W, uint32_t* ind, T* val,
                      short* track) {
    std::vector<uint32_t> bas = basis(L, k);
    std::vector<OperatorType> dec((size_t)H_size * H_col);
    for (size_t i = 0; i < dec.size(); ++i) dec[i] = static_cast<OperatorType>(codes[i]);
    std::fill(ind, ind + (size_t)R * W, 0u);
    std::fill(val, val + (size_t)R * W, T(0));
    std::fill(track, track + R, (short)0);
    launch(R, 32, [&] {
        BuildHamiltonianXXZForAbelianGroup<T>(
            const_cast<T*>(scalars), dec.data(), const_cast<int*>(sites),
            const_cast<int*>(n_ops), H_size, H_col, k, bas.data(), ind, val, track, W, R,
            const_cast<uint32_t*>(srs), G, const_cast<uint32_t*>(orbit), const_cast<T*>(chars),
            alpha, const_cast<float*>(norms), NIr, tol);
    });
}

extern "C" void ref_ham_terms_real(int L, int k, int G, int R, const uint32_t* srs, const uint32_t* orbit,
                        int NIr, const float* chars, int alpha, const float* norms, float tol,
                        int H_size, int H_col, const int* n_ops, const int* codes,
                        const int* sites, const float* scalars, int W, uint32_t* ind,
                        float* val, short* track) {
    ham_terms<float>(L, k, G, R, srs, orbit, NIr, chars, alpha, norms, tol, H_size, H_col, n_ops,
                     codes, sites, scalars, W, ind, val, track);
}

extern "C" void ref_ham_terms_complex(int L, int k, int G, int R, const uint32_t* srs,
                           const uint32_t* orbit, int NIr, const float* chars, int alpha,
                           const float* norms, float tol, int H_size, int H_col, const int* n_ops,
                           const int* codes, const int* sites, const float* scalars, int W,
                           uint32_t* ind, float* val, short* track) {
    ham_terms<cf>(L, k, G, R, srs, orbit, NIr, reinterpret_cast<const cf*>(chars), alpha, norms,
                  tol, H_size, H_col, n_ops, codes, sites, reinterpret_cast<const cf*>(scalars), W,
                  ind, reinterpret_cast<cf*>(val), track);
}

/* BuildHoppingHam_v2 (launch of HeisenbergHam_CUDA.cu:110-112). */
extern "C" void ref_ham_nosym(float jxy_w, float jz_w, int L, int k, int T_size, const int* ti,
                   const int* tj, const float* tval, int W, uint32_t* ind, float* val,
                   short* track) {
    std::vector<uint32_t> bas = basis(L, k);
    int N = (int)bas.size();
    std::fill(ind, ind + (size_t)N * W, 0u);
    std::fill(val, val + (size_t)N * W, 0.0f);
    std::fill(track, track + N, (short)0);
    launch(N, 32, [&] {
        BuildHoppingHam_v2(jxy_w, jz_w, k, bas.data(), ind, val, track, W, N,
                           const_cast<int*>(ti), const_cast<int*>(tj), const_cast<float*>(tval),
                           T_size);
    });
}

/* The reference's only CPU H*v: SparseMatDenseVec_prod_EEL_host
 * (exact_diagonalization/utils.cu:649-670), FP32.  Called on contiguous
 * row blocks, one per host thread (its column indices are global, so a
 * block is an offset call). */
extern "C" void ref_spmv_host(const uint32_t* ind, const float* val, const short* track,
                              const float* x, float* y, int nobv, int W, int n_threads) {
    if (n_threads < 1) n_threads = 1;
    int chunk = (nobv + n_threads - 1) / n_threads;
    std::vector<std::thread> pool;
    for (int c = 0; c < n_threads; ++c) {
        int r0 = c * chunk;
        int r1 = std::min(nobv, r0 + chunk);
        if (r0 >= r1) break;
        pool.emplace_back([=] {
            SparseMatDenseVec_prod_EEL_host(const_cast<uint32_t*>(ind) + (size_t)r0 * W,
                                            const_cast<float*>(val) + (size_t)r0 * W,
                                            const_cast<short*>(track) + r0, const_cast<float*>(x),
                                            y + r0, r1 - r0, W);
        });
    }
    for (auto& t : pool) t.join();
}

/* One sweep of SparseMatDenseVec_prod_EEL_host (utils.cu:649-670) over
 * n_mats matrices with a single pool of host threads: thread c takes the
 * c-th contiguous row block of every matrix in turn, so thread start-up is
 * paid once per sweep rather than once per matrix. */
extern "C" void ref_spmv_host_sweep(int n_mats, const uint32_t* const* ind, const float* const* val,
                                    const short* const* track, const float* const* x,
                                    float* const* y, const int* nobv, const int* W,
                                    int n_threads) {
    if (n_threads < 1) n_threads = 1;
    std::vector<std::thread> pool;
    for (int c = 0; c < n_threads; ++c) {
        pool.emplace_back([=] {
            for (int m = 0; m < n_mats; ++m) {
                int chunk = (nobv[m] + n_threads - 1) / n_threads;
                int r0 = c * chunk;
                int r1 = std::min(nobv[m], r0 + chunk);
                if (r0 >= r1) continue;
                SparseMatDenseVec_prod_EEL_host(
                    const_cast<uint32_t*>(ind[m]) + (size_t)r0 * W[m],
                    const_cast<float*>(val[m]) + (size_t)r0 * W[m],
                    const_cast<short*>(track[m]) + r0, const_cast<float*>(x[m]), y[m] + r0,
                    r1 - r0, W[m]);
            }
        });
    }
    for (auto& t : pool) t.join();
}

/* SparseMatDenseVec_prod_EEL<T> emulated (utils.cu:601-624; launch shape of
 * lanczos.cu:149-150,212-213). */
extern "C" void ref_spmv_kernel_complex(const uint32_t* ind, const float* val, const short* track,
                             const float* x, float* y, int nobv, int W) {
    launch(nobv, 512, [&] {
        SparseMatDenseVec_prod_EEL<cf>(const_cast<uint32_t*>(ind),
                                       reinterpret_cast<cf*>(const_cast<float*>(val)),
                                       const_cast<short*>(track),
                                       reinterpret_cast<cf*>(const_cast<float*>(x)),
                                       reinterpret_cast<cf*>(y), nobv, W);
    });
}

/* init_random_vec<curandState, float> (utils/misc_funcs_gpu.cu:31-52) as
 * launched by lanczos.cu:165-166.  The kernel also writes element nobv
 * (its bound test is `id > nobv`), so both buffers here hold nobv + 1. */
extern "C" void ref_init_random_vec(long long seed, int nobv, float* out /* nobv */) {
    std::vector<curandState> st((size_t)nobv + 1);
    std::vector<float> v((size_t)nobv + 1, 1.0f);
    launch((long long)nobv + 1, 512, [&] {
        if (blockIdx.x * blockDim.x + threadIdx.x <= (unsigned)nobv)
            init_random_vec<curandState, float>(seed, st.data(), nobv, v.data());
    });
    std::memcpy(out, v.data(), sizeof(float) * nobv);
}

/* T_standard<T> pair list (lattice_models/T_standard.cu:12-147) and site
 * coordinates (Lattice::GetR1/GetR2). Returns the pair count or -count. */
template <class T>
static int tstandard(int N1, int N2, int M, const float* A, const float* rx, const float* ry,
                     int nJ, const T* J, const float* range, int intra, int inter, int cap,
                     int* ti, int* tj, T* tv, float* R1, float* R2) {
    LatticeGeometryInfo g;
    g.N1 = N1;
    g.N2 = N2;
    g.rx_alpha.assign(rx, rx + M);
    g.ry_alpha.assign(ry, ry + M);
    g.A_mat = {{A[0], A[1]}, {A[2], A[3]}};
    std::vector<T> Jv(J, J + nJ);
    std::vector<float> Rv(range, range + nJ);
    T_standard<T> t(g, Jv, Rv, intra, inter);
    std::vector<std::vector<T>> m = t.getTmat();
    int n = (int)m.size();
    std::vector<float> r1 = t.GetR1(), r2 = t.GetR2();
    if (R1) std::copy(r1.begin(), r1.end(), R1);
    if (R2) std::copy(r2.begin(), r2.end(), R2);
    if (n > cap) return -n;
    for (int i = 0; i < n; ++i) {
        ti[i] = (int)ExtReal(m[i][0]);
        tj[i] = (int)ExtReal(m[i][1]);
        tv[i] = m[i][2];
    }
    return n;
}

extern "C" int ref_tstandard_real(int N1, int N2, int M, const float* A, const float* rx, const float* ry,
                       int nJ, const float* J, const float* range, int intra, int inter, int cap,
                       int* ti, int* tj, float* tv, float* R1, float* R2) {
    return tstandard<float>(N1, N2, M, A, rx, ry, nJ, J, range, intra, inter, cap, ti, tj, tv, R1,
                            R2);
}

extern "C" int ref_tstandard_complex(int N1, int N2, int M, const float* A, const float* rx,
                          const float* ry, int nJ, const float* J, const float* range, int intra,
                          int inter, int cap, int* ti, int* tj, float* tv, float* R1,
                          float* R2) {
    return tstandard<cf>(N1, N2, M, A, rx, ry, nJ, reinterpret_cast<const cf*>(J), range, intra,
                         inter, cap, ti, tj, reinterpret_cast<cf*>(tv), R1, R2);
}


/* ExpecValArbOperatorAbelianIrrepProjHeisenbergZeroT<S> over all R orbit rows
 * (the launch of HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:574-594, 32
 * threads a block), then the reduction and the division by G of :596-597 as
 * a sequential complex<float> sum.  Operator tables in the driver's form
 * (:434-455): per factor an action (0 Sz, -1 lowering, +1 raising) and a
 * site (-1 in unused slots), scalars already conjugated.  chars is the
 * complex character table [NIr][G]; phi has R entries of S. */
template <class S>
static void expval(int L, int k, int G, int R, const uint32_t* srs, const uint32_t* orbit, int NIr,
                   const cf* chars, int alpha, const float* norms, float tol, int A_size, int A_col,
                   const int* n_ops, const int* actions, const int* sites, const cf* scalars,
                   const S* phi, float* out) {
    std::vector<uint32_t> bas = basis(L, k);
    std::vector<cf> a_exp(R, cf(0.0f, 0.0f));
    launch(R, 32, [&] {
        ExpecValArbOperatorAbelianIrrepProjHeisenbergZeroT<S>(
            const_cast<cf*>(scalars), const_cast<int*>(actions), const_cast<int*>(sites),
            const_cast<int*>(n_ops), A_col, R, const_cast<uint32_t*>(srs), G, k,
            const_cast<uint32_t*>(orbit), const_cast<cf*>(chars), alpha, const_cast<float*>(norms), NIr,
            tol, A_size, A_col, bas.data(), const_cast<S*>(phi), a_exp.data());
    });
    cf sum(0.0f, 0.0f);
    for (const cf& v : a_exp) sum = sum + v;
    sum = sum / (float)G;
    out[0] = sum.real();
    out[1] = sum.imag();
}

extern "C" void ref_expval_real(int L, int k, int G, int R, const uint32_t* srs, const uint32_t* orbit, int NIr,
                                const float* chars_ri, int alpha, const float* norms, float tol, int A_size,
                                int A_col, const int* n_ops, const int* actions, const int* sites,
                                const float* scalars_ri, const float* phi, float* out) {
    expval<float>(L, k, G, R, srs, orbit, NIr, reinterpret_cast<const cf*>(chars_ri), alpha, norms, tol, A_size,
                  A_col, n_ops, actions, sites, reinterpret_cast<const cf*>(scalars_ri), phi, out);
}

extern "C" void ref_expval_complex(int L, int k, int G, int R, const uint32_t* srs, const uint32_t* orbit,
                                   int NIr, const float* chars_ri, int alpha, const float* norms, float tol,
                                   int A_size, int A_col, const int* n_ops, const int* actions,
                                   const int* sites, const float* scalars_ri, const float* phi_ri, float* out) {
    expval<cf>(L, k, G, R, srs, orbit, NIr, reinterpret_cast<const cf*>(chars_ri), alpha, norms, tol, A_size,
               A_col, n_ops, actions, sites, reinterpret_cast<const cf*>(scalars_ri),
               reinterpret_cast<const cf*>(phi_ri), out);
}
