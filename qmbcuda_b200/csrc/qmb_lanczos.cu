// qmb_lanczos.cu -- ground-state Lanczos on one GPU.
//
// Replaces LanczosEigVals_CUDA / LanczosEigenStateFromSeed
// (exact_diagonalization/lanczos.cu:31-317).  The reference runs ~14 vector
// passes per step through thrust and cuBLAS (a handle created and destroyed
// per call, host-synchronising scalars).  Here one step is two kernels:
//   K1  y = H (w_j / beta_j) - beta_j v_{j-1};  v_j = w_j / beta_j;  alpha_j = <v_j, y>
//   K2  w_{j+1} = y - alpha_j v_j;  beta_{j+1} = ||w_{j+1}||
// with FP64 scalars kept on the device (deterministic last-block reductions)
// and the step index read from device memory, so a step is a replayable CUDA
// graph.  Optional full reorthogonalisation runs classical Gram-Schmidt
// passes against the stored Krylov basis.  The tridiagonal eigenproblem is
// solved on the host in FP64 every `check_every` steps.
#include <curand_kernel.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>

#include "qmb_ham.cuh"
#include "qmb_lanczos.cuh"
#include "qmb_tridiag.h"

namespace qmb {

constexpr int kLzBlock = 256;

// Kernels executed for the current qmb_lanczos call on this thread.
thread_local double g_lz_kernels = 0;

struct LzDev {
    double* alpha;      // [cap]
    double* beta;       // [cap + 1]
    int* iter;
    unsigned* counter;
    double* partials;   // [2 * max_blocks]
    double2* coefs;     // [cap + 1]
    double* cpart;      // [2 * max_blocks * (cap + 1)]
    double* scratch;    // [4]
};

__host__ __device__ inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double splitmix_uniform(uint64_t seed, uint64_t i) {
    uint64_t z = splitmix64(seed + i);
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// ----------------------------------------------------------------- kernels
// Start vector w_0 (unnormalised) and beta_0 = ||w_0||; resets the step.
// mode 0: uniform(-1,1) from splitmix64(seed + i) (complex: seed + 2i, 2i+1)
// mode 1: curand_init(seed + i, 0, 0) then curand_uniform (complex: two draws),
//         the start vector of init_random_vec (utils/misc_funcs_gpu.cu:31-52)
// mode 2: copy of `from`
template <class V, class P>
__global__ void k_lz_start(int64_t n, int mode, uint64_t seed, const P* __restrict__ from,
                           V* __restrict__ w0, LzDev d) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        V v;
        if (mode == 2) {
            v = cvt<V>(from[i]);
        } else if (mode == 1) {
            curandState st;
            curand_init((unsigned long long)(seed + (uint64_t)i), 0ull, 0ull, &st);
            float a = curand_uniform(&st);
            if constexpr (Sc<V>::cplx) {
                float b = curand_uniform(&st);
                v = Sc<V>::from(make_double2(a, b));
            } else {
                v = Sc<V>::from(make_double2(a, 0.0));
            }
        } else {
            if constexpr (Sc<V>::cplx)
                v = Sc<V>::from(make_double2(splitmix_uniform(seed, 2 * i), splitmix_uniform(seed, 2 * i + 1)));
            else
                v = Sc<V>::from(make_double2(splitmix_uniform(seed, i), 0.0));
        }
        w0[i] = v;
        acc += Sc<V>::abs2(v);
    }
    double tot;
    if (grid_reduce(acc, d.partials, d.counter, red, &tot) && threadIdx.x == 0) {
        d.beta[0] = sqrt(tot);
        *d.iter = 0;
    }
}

// K1: y = H w_j / beta_j - beta_j v_{j-1}; v_j = w_j / beta_j; alpha_j = Re <v_j, y>.
// Optionally psi += c_j v_j (eigenvector regeneration).
template <class Op, class V, class P>
__global__ void __launch_bounds__(kLzBlock, OpMinBlocks<Op>::value) k_lz_hv(Op op, V* __restrict__ wbuf, V* __restrict__ vring,
                                                    int K, LzDev d, const double* __restrict__ ritz,
                                                    P* __restrict__ psi) {
    extern __shared__ __align__(16) unsigned char smem_lz[];
    __shared__ double red[32];
    op.init(smem_lz);
    const int64_t n = op.n;
    const int j = *d.iter;
    const V* X = wbuf + (int64_t)(j & 1) * n;
    V* Y = wbuf + (int64_t)((j + 1) & 1) * n;
    V* Vc = vring + (int64_t)(j % K) * n;
    const V* Vp = vring + (int64_t)((j + K - 1) % K) * n;
    const double bj = d.beta[j];
    const double inv = 1.0 / bj;
    const double c = ritz ? ritz[j] : 0.0;
    double acc = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        V xr;
        V hx = op.row(r, X, xr);
        V vj = Sc<V>::scale(xr, inv);
        V y = Sc<V>::scale(hx, inv);
        if (j > 0) y = Sc<V>::sub(y, Sc<V>::scale(Vp[r], bj));
        Vc[r] = vj;
        Y[r] = y;
        acc += Sc<V>::re_conj_mul(vj, y);
        if (psi) psi[r] = Sc<P>::add(psi[r], Sc<P>::scale(cvt<P>(vj), c));
    }
    double tot;
    if (grid_reduce(acc, d.partials, d.counter, red, &tot) && threadIdx.x == 0) d.alpha[j] = tot;
}

// K2: w_{j+1} = y - alpha_j v_j; beta_{j+1} = ||w_{j+1}||; finalize advances the step.
template <class V>
__global__ void __launch_bounds__(kLzBlock) k_lz_update(int64_t n, V* __restrict__ wbuf,
                                                        const V* __restrict__ vring, int K,
                                                        LzDev d, int finalize) {
    __shared__ double red[32];
    const int j = *d.iter;
    V* Y = wbuf + (int64_t)((j + 1) & 1) * n;
    const V* Vc = vring + (int64_t)(j % K) * n;
    const double a = d.alpha[j];
    double acc = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        V y = Sc<V>::sub(Y[r], Sc<V>::scale(Vc[r], a));
        Y[r] = y;
        acc += Sc<V>::abs2(y);
    }
    double tot;
    if (grid_reduce(acc, d.partials, d.counter, red, &tot) && threadIdx.x == 0) {
        d.beta[j + 1] = sqrt(tot);
        if (finalize) *d.iter = j + 1;
    }
}

// Classical Gram-Schmidt with the Kahan-Parlett criterion ("twice is
// enough", as in the DGKS correction): with two passes requested, the second
// pass runs only when the first removed enough of w that its rounding can
// matter, ||w'|| < kReorthEta ||w||.  scratch[2] keeps ||w|| before the first
// pass and scratch[3] is 1 when the second pass must run.
constexpr double kReorthEta = 0.70710678118654752;

// Reorthogonalisation, dot half of a pass: coefs[i] = <v_i, w_{j+1}> for
// i <= j, kDotChunk basis vectors a sweep over the rows (w is read once per
// chunk): 16 for real and complex FP32 vectors, 8 for complex FP64.  Pass 0
// records ||w|| first; pass 1 returns at once when the first pass made it
// unnecessary.
template <class V>
__global__ void __launch_bounds__(kLzBlock) k_reorth_dots(int64_t n, const V* __restrict__ wbuf,
                                                          const V* __restrict__ vring, LzDev d, int pass) {
    constexpr int kDotChunk = sizeof(V) >= 16 ? 8 : 16;
    __shared__ double red[2 * kDotChunk * (kLzBlock / 32)];
    __shared__ bool last;
    const int j = *d.iter;
    if (pass == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) d.scratch[2] = d.beta[j + 1];
    } else if (d.scratch[3] == 0.0) {
        return;
    }
    const V* Y = wbuf + (int64_t)((j + 1) & 1) * n;
    const int nb = gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    for (int i0 = 0; i0 <= j; i0 += kDotChunk) {
        const int cnt = min(kDotChunk, j + 1 - i0);
        double re[kDotChunk], im[kDotChunk];
#pragma unroll
        for (int k = 0; k < kDotChunk; ++k) re[k] = im[k] = 0.0;
        for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
             r += (int64_t)gridDim.x * blockDim.x) {
            const V y = Y[r];
#pragma unroll
            for (int k = 0; k < kDotChunk; ++k)
                if (k < cnt) {
                    const V v = vring[(int64_t)(i0 + k) * n + r];
                    re[k] += Sc<V>::re_conj_mul(v, y);
                    if constexpr (Sc<V>::cplx) im[k] += Sc<V>::im_conj_mul(v, y);
                }
        }
#pragma unroll
        for (int k = 0; k < kDotChunk; ++k)
            for (int o = 16; o > 0; o >>= 1) {
                re[k] += __shfl_xor_sync(0xffffffffu, re[k], o);
                im[k] += __shfl_xor_sync(0xffffffffu, im[k], o);
            }
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < kDotChunk; ++k) {
                red[2 * (warp * kDotChunk + k)] = re[k];
                red[2 * (warp * kDotChunk + k) + 1] = im[k];
            }
        __syncthreads();
        if (threadIdx.x < cnt) {
            double bre = 0.0, bim = 0.0;
            for (int w = 0; w < n_warps; ++w) {
                bre += red[2 * (w * kDotChunk + threadIdx.x)];
                bim += red[2 * (w * kDotChunk + threadIdx.x) + 1];
            }
            d.cpart[2 * ((int64_t)(i0 + threadIdx.x) * nb + blockIdx.x)] = bre;
            d.cpart[2 * ((int64_t)(i0 + threadIdx.x) * nb + blockIdx.x) + 1] = bim;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned t = atomicAdd(d.counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block: one warp per coefficient sums the blocks' partials
    for (int i = warp; i <= j; i += n_warps) {
        double re = 0.0, im = 0.0;
        for (int b = lane; b < nb; b += 32) {
            re += __ldcg(d.cpart + 2 * ((int64_t)i * nb + b));
            im += __ldcg(d.cpart + 2 * ((int64_t)i * nb + b) + 1);
        }
        for (int o = 16; o > 0; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (lane == 0) d.coefs[i] = make_double2(re, im);
    }
    __syncthreads();
    if (threadIdx.x == 0) *d.counter = 0;
}

// Reorthogonalisation, update half of a pass: w_{j+1} -= sum_i coefs[i] v_i;
// beta_{j+1} = ||w_{j+1}||.  After pass 0, scratch[3] says whether pass 1
// runs (always when `selective` is 0); a skipped pass 1 only finalizes.
template <class V>
__global__ void __launch_bounds__(kLzBlock) k_reorth_update(int64_t n, V* __restrict__ wbuf,
                                                            const V* __restrict__ vring, LzDev d,
                                                            int finalize, int pass, int selective) {
    extern __shared__ __align__(16) unsigned char smem_ro[];
    __shared__ double red[32];
    double2* cf = reinterpret_cast<double2*>(smem_ro);
    const int j = *d.iter;
    if (pass == 1 && d.scratch[3] == 0.0) {
        if (finalize && blockIdx.x == 0 && threadIdx.x == 0) *d.iter = j + 1;
        return;
    }
    for (int i = threadIdx.x; i <= j; i += blockDim.x) cf[i] = d.coefs[i];
    __syncthreads();
    V* Y = wbuf + (int64_t)((j + 1) & 1) * n;
    double acc = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        V y = Y[r];
        // U basis rows loaded before their products are subtracted, so that
        // U loads per thread are in flight instead of one
        constexpr int U = sizeof(V) >= 16 ? 8 : 16;
        int i = 0;
        for (; i + U <= j + 1; i += U) {
            V v[U];
#pragma unroll
            for (int k = 0; k < U; ++k) v[k] = vring[(int64_t)(i + k) * n + r];
#pragma unroll
            for (int k = 0; k < U; ++k) y = Sc<V>::sub(y, Sc<V>::mul(Sc<V>::from(cf[i + k]), v[k]));
        }
        for (; i <= j; ++i) y = Sc<V>::sub(y, Sc<V>::mul(Sc<V>::from(cf[i]), vring[(int64_t)i * n + r]));
        Y[r] = y;
        acc += Sc<V>::abs2(y);
    }
    double tot;
    if (grid_reduce(acc, d.partials, d.counter, red, &tot) && threadIdx.x == 0) {
        const double b = sqrt(tot);
        d.beta[j + 1] = b;
        if (pass == 0) d.scratch[3] = (!selective || b < kReorthEta * d.scratch[2]) ? 1.0 : 0.0;
        if (finalize) *d.iter = j + 1;
    }
}

// psi = sum_i ritz[i] v_i over a stored basis.
template <class V, class P>
__global__ void k_ritz(int64_t n, const V* __restrict__ vring, int m,
                       const double* __restrict__ ritz, P* __restrict__ psi) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        P acc = Sc<P>::zero();
        // U basis rows in flight a thread, summed in index order
        constexpr int U = sizeof(V) >= 16 ? 8 : 16;
        int i = 0;
        for (; i + U <= m; i += U) {
            V v[U];
#pragma unroll
            for (int k = 0; k < U; ++k) v[k] = vring[(int64_t)(i + k) * n + r];
#pragma unroll
            for (int k = 0; k < U; ++k) acc = Sc<P>::add(acc, Sc<P>::scale(cvt<P>(v[k]), ritz[i + k]));
        }
        for (; i < m; ++i) acc = Sc<P>::add(acc, Sc<P>::scale(cvt<P>(vring[(int64_t)i * n + r]), ritz[i]));
        psi[r] = acc;
    }
}

// scratch[0] = ||H psi - theta psi||^2, scratch[1] = ||psi||^2.
template <class Op, class P>
__global__ void k_residual(Op op, const P* __restrict__ psi, double theta, LzDev d) {
    extern __shared__ __align__(16) unsigned char smem_rs[];
    __shared__ double red[32];
    op.init(smem_rs);
    double a = 0.0, b = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < op.n;
         r += (int64_t)gridDim.x * blockDim.x) {
        P xr;
        P hx = op.row(r, psi, xr);
        P res = Sc<P>::sub(hx, Sc<P>::scale(xr, theta));
        a += Sc<P>::abs2(res);
        b += Sc<P>::abs2(xr);
    }
    double ta, tb;
    bool la = grid_reduce(a, d.partials, d.counter, red, &ta);
    if (la && threadIdx.x == 0) d.scratch[0] = ta;
    __syncthreads();
    bool lb = grid_reduce(b, d.partials + gridDim.x, d.counter + 1, red, &tb);
    if (lb && threadIdx.x == 0) d.scratch[1] = tb;
}

// ------------------------------------------------------------------- host
// QMB_REORTH_ALWAYS=1: with two passes requested, always run the second one
// (by default it runs only when the Kahan-Parlett criterion asks for it).
static bool reorth_selective() {
    const char* e = std::getenv("QMB_REORTH_ALWAYS");
    return !(e && e[0] == '1');
}

static int lz_ring_max() {
    const char* e = std::getenv("QMB_LZ_RING_MAX");
    return e ? std::max(0, std::atoi(e)) : 0;
}

int lz_blocks() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * 4;
}

struct LzState {
    int cap = 0;
    int nb = 0;
    DevBuf<double> alpha, beta, partials, cpart, scratch;
    DevBuf<int> iter;
    DevBuf<unsigned> counter;
    DevBuf<double2> coefs;
    LzDev d{};
    void init(int cap_, int nb_, bool reorth) {
        cap = cap_;
        nb = nb_;
        alpha.alloc(cap + 1);
        beta.alloc(cap + 2);
        partials.alloc(2 * (size_t)nb);
        scratch.alloc(4);
        scratch.zero();
        iter.alloc(1);
        counter.alloc(2);
        counter.zero();
        iter.zero();
        coefs.alloc(reorth ? cap + 2 : 1);
        cpart.alloc(reorth ? 2 * (size_t)nb * (cap + 2) : 1);
        d.alpha = alpha.p;
        d.beta = beta.p;
        d.iter = iter.p;
        d.counter = counter.p;
        d.partials = partials.p;
        d.coefs = coefs.p;
        d.cpart = cpart.p;
        d.scratch = scratch.p;
    }
};

struct PhaseOut {
    int m = 0;            // Lanczos vectors used (tridiagonal size)
    double theta = 0.0;
    double est = 0.0;     // residual estimate beta_m |s_{m-1}|
    bool converged = false;
    bool stored = false;   // v_0 .. v_{m-1} are all in the ring (else the Ritz vector is regenerated)
    bool stalled = false;  // theta stopped moving at the FP32 floor
    double gap = 0.0;      // theta_2 - theta_1 of the last check
    std::vector<double> s_start;  // Ritz coefficients of the restart vector
    std::vector<double> a, e, s;
    int n_hv = 0;
};

// A typed view of a byte buffer that only grows: alloc(count) keeps the
// memory when it is large enough, so the handle's Lanczos buffers persist
// between solves instead of being allocated and freed (tens of ms for a
// stored basis of several GB) every time.
template <class V>
struct GrowBuf {
    DevBuf<unsigned char>* bytes;
    V* p = nullptr;
    explicit GrowBuf(DevBuf<unsigned char>* b) : bytes(b) {}
    void alloc(size_t count) {
        if (bytes->n < count * sizeof(V)) {
            bytes->release();
            bytes->alloc(count * sizeof(V));
        }
        p = reinterpret_cast<V*>(bytes->p);
    }
};

struct PhaseOpts {
    int* ring_hint = nullptr;  // in/out: stored-basis slots to start with
    int max_iter = 200;
    int min_iter = 1;
    double tol = 1e-12;       // <= 0: run exactly max_iter steps
    // stopping tests (any one suffices; all off when tol <= 0):
    double e_tol = 0.0;       // est^2 / gap <= e_tol |theta|  (energy error bound)
    double res_tol = 0.0;     // est <= res_tol |theta|        (residual of the Ritz pair)
    double stall_tol = 0.0;   // |d theta| <= stall_tol |theta| between checks
    double gap_in = 0.0;      // gap to use instead of theta_2 - theta_1 (> 0)
    int reorth = 0;           // CGS passes
    int check_every = 10;
    bool use_graph = true;
};

// Runs one Lanczos phase for operator op with vectors of type V.
// start_mode 0/1: generated from seed, 2: copied from `from` (type P).
// With `store` the basis is kept for the Ritz vector: the ring starts with
// the slots the hint asks for (the previous phase's steps plus a check block)
// and doubles, its filled slots copied over, before a block of steps would
// wrap it.  A ring that may not grow further (the doubled ring would not fit
// in free memory) wraps from then on and out.stored is false: the caller
// regenerates the basis for the Ritz vector.  Reorthogonalisation needs the
// whole basis, so its ring is allocated in full up front.
template <class Op, class V, class P>
PhaseOut run_phase(const Op& op, size_t op_smem, const PhaseOpts& po, int start_mode,
                   uint64_t seed, const P* from, bool store, GrowBuf<V>& vring, int& K,
                   GrowBuf<V>& wbuf, LzState& st, cudaStream_t s) {
    const int64_t n = op.n;
    PhaseOut out;
    const double gap_cap = restart_gap_cap();
    int cap = std::max(1, po.max_iter);
    const int K_full = store ? cap + 1 : 2;
    const int hint = po.ring_hint ? *po.ring_hint : 0;
    const int every_steps = std::max(1, po.check_every);
    // memory the ring may take: the ring kept from earlier solves (reused)
    // plus free memory, less a reserve for the vectors a solve allocates
    // besides (work vectors, start and Ritz vectors in the high precision)
    const size_t slot = (size_t)n * sizeof(V);
    const size_t reserve = 6 * (size_t)n * sizeof(P) + ((size_t)256 << 20);
    auto free_bytes = [&]() {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            (void)cudaGetLastError();
            return (size_t)0;
        }
        return fr;
    };
    K = store ? std::min(K_full, std::max({hint, 2 + every_steps, 32})) : 2;
    // a ring kept from an earlier solve is used to its full size
    if (store) K = std::min(K_full, std::max(K, (int)(vring.bytes->n / slot)));
    if (store && !po.reorth) {
        const size_t avail = vring.bytes->n + free_bytes();
        const int K_fit = avail > reserve ? (int)std::min<size_t>((avail - reserve) / slot, (size_t)K_full) : 0;
        K = std::min(K, K_fit);
        if (K < 2 + every_steps) {  // not even one block of steps: regenerate instead
            store = false;
            K = 2;
        }
    }
    // QMB_LZ_RING_MAX caps the ring (tests of the wrapping ring)
    const int ring_max = lz_ring_max();
    if (store && ring_max > 0) K = std::max(2, std::min(K, ring_max));
    if (po.reorth) K = K_full;
    bool wrapped = false;
    vring.alloc((size_t)K * n);
    wbuf.alloc(2 * (size_t)n);
    st.init(cap, lz_blocks(), po.reorth > 0);
    const int nb = st.nb;
    QMB_REQUIRE(po.reorth == 0 || store, QMB_ERR_INVALID, "reorthogonalisation needs the stored basis");

    g_lz_kernels += 1;
    k_lz_start<V, P><<<nb, kLzBlock, 0, s>>>(n, start_mode, seed, from, wbuf.p, st.d);
    check_launch("k_lz_start");

    const void* f1 = (const void*)k_lz_hv<Op, V, P>;
    set_group_smem_attr(f1, op_smem);
    size_t ro_smem = sizeof(double2) * (size_t)(cap + 2);
    if (po.reorth) set_group_smem_attr((const void*)k_reorth_update<V>, ro_smem);

    auto step = [&](cudaStream_t ss) {
        op.pre((const V*)wbuf.p, st.d.iter, ss);  // column-block passes or the matrix-free scaling, if any
        k_lz_hv<Op, V, P><<<nb, kLzBlock, op_smem, ss>>>(op, wbuf.p, vring.p, K, st.d, nullptr,
                                                         (P*)nullptr);
        k_lz_update<V><<<nb, kLzBlock, 0, ss>>>(n, wbuf.p, vring.p, K, st.d, po.reorth ? 0 : 1);
        for (int p = 0; p < po.reorth; ++p) {
            k_reorth_dots<V><<<nb, kLzBlock, 0, ss>>>(n, wbuf.p, vring.p, st.d, p);
            k_reorth_update<V><<<nb, kLzBlock, ro_smem, ss>>>(n, wbuf.p, vring.p, st.d,
                                                              p == po.reorth - 1 ? 1 : 0, p,
                                                              reorth_selective() ? 1 : 0);
        }
    };

    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    auto capture = [&]() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        if (!po.use_graph) return;
        QMB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        step(s);
        cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            exec = nullptr;
        }
        check_launch("lanczos step capture");
    };
    capture();

    std::vector<double> ha(cap + 1), hb(cap + 2);
    int done = 0;
    double theta_prev = 0.0;
    bool have_prev = false;
    const int every = std::max(1, po.check_every);
    while (done < cap) {
        int todo = std::min(every, cap - done);
        if (store && !wrapped && done + todo > K) {
            // steps done .. done+todo-1 write slots j: grow the ring first,
            // or let it wrap when the doubled ring does not fit
            const int K2 = std::min(K_full, std::max(2 * K, done + todo));
            // the grown ring is allocated while the current one is held
            if ((ring_max > 0 && K2 > ring_max) || (size_t)K2 * slot + reserve > free_bytes()) {
                wrapped = true;
            } else {
                DevBuf<unsigned char> grown;
                grown.alloc((size_t)K2 * n * sizeof(V));
                QMB_CUDA_TRY(cudaMemcpyAsync(grown.p, vring.p, (size_t)done * n * sizeof(V),
                                             cudaMemcpyDeviceToDevice, s));
                QMB_CUDA_TRY(cudaStreamSynchronize(s));
                std::swap(vring.bytes->p, grown.p);
                std::swap(vring.bytes->n, grown.n);
                vring.p = reinterpret_cast<V*>(vring.bytes->p);
                K = K2;
                capture();
            }
        }
        for (int t = 0; t < todo; ++t) {
            if (exec) QMB_CUDA_TRY(cudaGraphLaunch(exec, s));
            else step(s);
        }
        g_lz_kernels += (double)todo * (2 + 2 * po.reorth);
        check_launch("lanczos step");
        done += todo;
        out.n_hv += todo;
        QMB_CUDA_TRY(cudaMemcpyAsync(ha.data(), st.alpha.p, sizeof(double) * done,
                                     cudaMemcpyDeviceToHost, s));
        QMB_CUDA_TRY(cudaMemcpyAsync(hb.data(), st.beta.p, sizeof(double) * (done + 1),
                                     cudaMemcpyDeviceToHost, s));
        QMB_CUDA_TRY(cudaStreamSynchronize(s));
        // a (near) zero beta ends the Krylov space: keep the steps up to it
        bool breakdown = false;
        for (int i = done - todo; i < done; ++i) {
            double sc_i = std::fabs(ha[i]) + (i > 0 ? std::fabs(hb[i]) : 0.0) + 1e-300;
            if (!(hb[i + 1] > 1e-13 * sc_i)) {
                QMB_REQUIRE(std::isfinite(ha[i]), QMB_ERR_INVALID,
                            "non-finite Lanczos coefficient (check the Hamiltonian)");
                done = i + 1;
                breakdown = true;
                break;
            }
            QMB_REQUIRE(std::isfinite(ha[i]) && std::isfinite(hb[i + 1]), QMB_ERR_INVALID,
                        "non-finite Lanczos coefficient (check the Hamiltonian)");
        }
        // tridiagonal of the first `done` steps
        double theta = tridiag_min_eig(ha.data(), hb.data() + 1, done);
        std::vector<double> sv(done);
        tridiag_eigvec(ha.data(), hb.data() + 1, done, theta, sv.data());
        double est = hb[done] * std::fabs(sv[done - 1]);
        double scale = std::max(std::fabs(theta), 1e-300);
        if (breakdown) est = 0.0;
        out.m = done;
        out.theta = theta;
        out.est = est;
        out.s = sv;
        out.s_start = sv;
        // partner levels within 1e-4 |theta| (ghost copies excluded): their
        // Ritz vectors join the start of an FP64 restart
        for (int kth = 1; kth < std::min(done, 4); ++kth) {
            double tk = tridiag_eig(ha.data(), hb.data() + 1, done, kth);
            if (tk - theta > 1e-4 * std::max(std::fabs(theta), 1e-300)) break;
            if (tk - theta > 1e-10 * std::max(std::fabs(theta), 1e-300)) {
                std::vector<double> sk(done);
                tridiag_eigvec(ha.data(), hb.data() + 1, done, tk, sk.data());
                for (int i = 0; i < done; ++i) out.s_start[i] += sk[i];
            }
        }
        if (breakdown) {
            out.converged = true;
            break;
        }
        // gap to the next Ritz value that is not a copy of theta (ghosts)
        out.gap = 1e-10 * scale;
        for (int kth = 1; kth < std::min(done, 5); ++kth) {
            double tk = tridiag_eig(ha.data(), hb.data() + 1, done, kth);
            if (tk - theta > 1e-10 * scale) {
                out.gap = tk - theta;
                break;
            }
        }
        if (po.tol > 0 && done >= po.min_iter) {
            const double gap = po.gap_in > 0
                                   ? std::min({std::max(po.gap_in, 1e-10 * scale), gap_cap * scale, out.gap})
                                   : out.gap;
            // energy bound plus a settled theta (an unresolved close level
            // keeps theta moving while the gap estimate is too large)
            bool e_ok = po.e_tol > 0 && have_prev && est * est / gap <= po.e_tol * scale &&
                        std::fabs(theta - theta_prev) <= po.e_tol * scale;
            bool r_ok = po.res_tol > 0 && est <= po.res_tol * scale;
            bool stall = po.stall_tol > 0 && have_prev && est <= 1e-3 * scale &&
                         std::fabs(theta - theta_prev) <= po.stall_tol * scale;
            if (e_ok || r_ok || stall) {
                out.converged = true;
                out.stalled = stall && !(e_ok || r_ok);
                break;
            }
        }
        theta_prev = theta;
        have_prev = true;
    }
    if (po.tol <= 0) out.converged = true;
    out.stored = store && !wrapped;
    if (out.stored && po.ring_hint) *po.ring_hint = std::max(*po.ring_hint, out.m + 1 + every);
    out.a.assign(ha.begin(), ha.begin() + out.m);
    out.e.assign(hb.begin() + 1, hb.begin() + out.m);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    return out;
}

// psi = Ritz vector of a finished phase (stored basis, else regeneration).
template <class Op, class V, class P, class Buf>
void ritz_vector(const Op& op, size_t op_smem, const PhaseOut& ph, int start_mode, uint64_t seed,
                 const P* from, bool stored, Buf& vring, int K, Buf& wbuf,
                 LzState& st, P* psi, int& n_hv, cudaStream_t s, bool for_restart = false) {
    const int64_t n = op.n;
    DevBuf<double> ritz(ph.m);
    ritz.upload(for_restart ? ph.s_start.data() : ph.s.data(), ph.m, s);
    if (stored) {
        g_lz_kernels += 1;
        k_ritz<V, P><<<grid_for(n, 256), 256, 0, s>>>(n, vring.p, ph.m, ritz.p, psi);
        check_launch("k_ritz");
        QMB_CUDA_TRY(cudaStreamSynchronize(s));
        return;
    }
    // regenerate v_0..v_{m-1} with the same start; kernels are deterministic
    QMB_CUDA_TRY(cudaMemsetAsync(psi, 0, sizeof(P) * n, s));
    const int nb = st.nb;
    g_lz_kernels += 2 * ph.m;  // start, m products, m - 1 updates
    k_lz_start<V, P><<<nb, kLzBlock, 0, s>>>(n, start_mode, seed, from, wbuf.p, st.d);
    for (int j = 0; j < ph.m; ++j) {
        op.pre((const V*)wbuf.p, st.d.iter, s);
        k_lz_hv<Op, V, P><<<nb, kLzBlock, op_smem, s>>>(op, wbuf.p, vring.p, K, st.d, ritz.p, psi);
        if (j + 1 < ph.m) k_lz_update<V><<<nb, kLzBlock, 0, s>>>(n, wbuf.p, vring.p, K, st.d, 1);
        ++n_hv;
    }
    check_launch("regenerate");
    QMB_CUDA_TRY(cudaStreamSynchronize(s));
}

template <class Op, class P>
double residual_norm(const Op& op, size_t op_smem, const P* psi, double theta, LzState& st,
                     cudaStream_t s, double* psi_norm2) {
    set_group_smem_attr((const void*)k_residual<Op, P>, op_smem);
    g_lz_kernels += 1;
    op.pre(psi, (const int*)nullptr, s);
    k_residual<Op, P><<<st.nb, kLzBlock, op_smem, s>>>(op, psi, theta, st.d);
    check_launch("k_residual");
    double h[2];
    QMB_CUDA_TRY(cudaMemcpyAsync(h, st.scratch.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    QMB_CUDA_TRY(cudaStreamSynchronize(s));
    if (psi_norm2) *psi_norm2 = h[1];
    return std::sqrt(h[0] / std::max(h[1], 1e-300));
}

bool fits_device(size_t bytes) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return false;
    return bytes < fr * 0.6;
}

// Full solve for one storage / precision combination.
//   V32/V64: vector types of the low / high phase, Op32/Op64 the operators.
template <class Op32, class Op64, class V32, class V64>
void solve(qmb_ham_s* h, const Op32& op32, size_t sm32, const Op64& op64, size_t sm64,
           const qmb_lanczos_opts& o, qmb_lanczos_result* res, double* coeffs, int64_t n_coeffs) {
    cudaStream_t s;
    QMB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct SG { cudaStream_t s; ~SG() { cudaStreamDestroy(s); } } sg{s};
    cudaEvent_t e0, e1;
    QMB_CUDA_TRY(cudaEventCreate(&e0));
    QMB_CUDA_TRY(cudaEventCreate(&e1));
    struct EG { cudaEvent_t a, b; ~EG() { cudaEventDestroy(a); cudaEventDestroy(b); } } eg{e0, e1};
    QMB_CUDA_TRY(cudaEventRecord(e0, s));
    const int64_t n = h->n;
    std::memset(res, 0, sizeof(*res));
    res->ms_hv = -1;
    g_lz_kernels = 0;
    LzState st;
    PhaseOpts po;
    po.max_iter = o.max_iter;
    po.min_iter = std::max(1, o.min_iter);
    po.tol = o.tol;
    po.e_tol = o.tol;  // FP64: stop on the energy error bound
    po.reorth = o.reorth;
    po.check_every = o.check_every > 0 ? o.check_every : 10;
    const int cap = std::max(1, o.max_iter);
    int n_hv = 0;
    DevBuf<V64> psi(n);
    double theta = 0.0;
    int iters = 0;
    bool conv = false;
    PhaseOut last;

    // full FP64 solve from the seeded start vector
    po.ring_hint = &h->lz_ring_hint;
    auto fp64_solve = [&]() {
        bool store = o.reorth > 0 ? fits_device(sizeof(V64) * (size_t)(cap + 3) * n) : true;
        QMB_REQUIRE(o.reorth == 0 || store, QMB_ERR_NOMEM, "Krylov basis does not fit for reorthogonalisation");
        GrowBuf<V64> vr(&h->lz_ring), wb(&h->lz_wbuf);
        int K;
        last = run_phase<Op64, V64, V64>(op64, sm64, po, o.start, o.seed, nullptr, store, vr, K, wb, st, s);
        n_hv += last.n_hv;
        ritz_vector<Op64, V64, V64>(op64, sm64, last, o.start, o.seed, nullptr, last.stored, vr, K, wb, st,
                                    psi.p, n_hv, s);
        theta = last.theta;
        iters += last.m;
        conv = last.converged;
    };
    if (o.mode == QMB_MODE_FP64) {
        fp64_solve();
    } else {
        // low phase: FP32 vectors and values, FP64 scalars
        // FP32 vectors: Ritz values stop improving near 1e-7 relative
        PhaseOpts p1 = po;
        if (o.tol > 0) {  // tol <= 0 keeps the fixed step count
            if (o.mode == QMB_MODE_MIXED) {
                // accurate enough that the FP64 restart needs few steps
                p1.e_tol = 1e-9;
                p1.res_tol = 1e-6;
            } else {
                // FP32 only: stop at the FP32 floor
                p1.e_tol = 1e-7;
                p1.res_tol = 1e-6;
                p1.stall_tol = 2e-7;
            }
        }
        bool store = o.reorth > 0 ? fits_device(sizeof(V32) * (size_t)(cap + 3) * n) : true;
        QMB_REQUIRE(o.reorth == 0 || store, QMB_ERR_NOMEM, "Krylov basis does not fit for reorthogonalisation");
        PhaseOut ph1;
        {
            GrowBuf<V32> vr(&h->lz_ring), wb(&h->lz_wbuf);
            int K;
            ph1 = run_phase<Op32, V32, V64>(op32, sm32, p1, o.start, o.seed, nullptr, store, vr, K, wb, st, s);
            n_hv += ph1.n_hv;
            ritz_vector<Op32, V32, V64>(op32, sm32, ph1, o.start, o.seed, nullptr, ph1.stored, vr, K, wb,
                                        st, psi.p, n_hv, s, o.mode == QMB_MODE_MIXED);
        }
        res->E0_low = ph1.theta;
        res->iters_low = ph1.m;
        theta = ph1.theta;
        iters = ph1.m;
        conv = ph1.converged;
        last = ph1;
        if (o.mode == QMB_MODE_MIXED) {
            // FP64 restart from the FP32 Ritz vector
            PhaseOpts p2 = po;
            p2.max_iter = o.refine_max_iter > 0 ? o.refine_max_iter : 300;
            p2.min_iter = 2;
            p2.check_every = 4;
            p2.gap_in = ph1.gap;
            int cap2 = std::max(1, p2.max_iter);
            bool store2 = o.reorth > 0 ? fits_device(sizeof(V64) * (size_t)(cap2 + 3) * n) : true;
            DevBuf<V64> start(n);
            QMB_CUDA_TRY(cudaMemcpyAsync(start.p, psi.p, sizeof(V64) * n, cudaMemcpyDeviceToDevice, s));
            GrowBuf<V64> vr(&h->lz_ring), wb(&h->lz_wbuf);
            int K;
            PhaseOut ph2 = run_phase<Op64, V64, V64>(op64, sm64, p2, 2, 0, start.p, store2, vr, K,
                                                     wb, st, s);
            n_hv += ph2.n_hv;
            ritz_vector<Op64, V64, V64>(op64, sm64, ph2, 2, 0, start.p, ph2.stored, vr, K, wb, st,
                                        psi.p, n_hv, s);
            theta = ph2.theta;
            iters += ph2.m;
            conv = ph2.converged;
            last = ph2;
        }
    }
    double pn2 = 0;
    res->residual = residual_norm<Op64, V64>(op64, sm64, psi.p, theta, st, s, &pn2);
    ++n_hv;
    if (o.mode == QMB_MODE_MIXED && o.tol > 0) {
        // A restart whose Krylov residual estimate is far below the true FP64
        // residual has stagnated (its start vector lacked the ground state,
        // e.g. a level pair swapped by FP32 rounding): solve in FP64 instead.
        const double sc = std::max(std::fabs(theta), 1e-300);
        if (res->residual > 1e-7 * sc && res->residual > 100.0 * last.est) {
            fp64_solve();
            res->residual = residual_norm<Op64, V64>(op64, sm64, psi.p, theta, st, s, &pn2);
            ++n_hv;
        }
    }
    res->residual_ref = res->residual * std::sqrt(pn2) / (double)n;
    QMB_CUDA_TRY(cudaEventRecord(e1, s));
    QMB_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    res->ms_total = ms;
    res->E0 = theta;
    res->iters = iters;
    res->n_hv = n_hv;
    res->n_products = n_hv;
    res->n_launches = g_lz_kernels;
    res->converged = conv ? 1 : 0;
    if (o.mode == QMB_MODE_FP64) res->E0_low = theta;
    if (coeffs) {
        for (int64_t i = 0; i < n_coeffs; ++i) coeffs[i] = i < (int64_t)last.s.size() ? last.s[i] : 0.0;
    }
    if (o.want_vector) {
        h->psi.alloc(sizeof(V64) * n);
        QMB_CUDA_TRY(cudaMemcpy(h->psi.p, psi.p, sizeof(V64) * n, cudaMemcpyDeviceToDevice));
        h->psi_n = n;
    }
}

}  // namespace qmb

using namespace qmb;

extern "C" void qmb_lanczos_default_opts(qmb_lanczos_opts* o) {
    if (!o) return;
    o->mode = QMB_MODE_FP64;
    o->max_iter = 300;
    o->min_iter = 5;
    o->tol = 1e-12;
    o->reorth = 0;
    o->start = QMB_START_SPLITMIX;
    o->seed = 20261203ull;
    o->check_every = 10;
    o->hv = QMB_HV_STORED;
    o->refine_max_iter = 300;
    o->want_vector = 0;
}

extern "C" qmb_status qmb_lanczos(qmb_ham h, const qmb_lanczos_opts* opts, qmb_lanczos_result* res,
                                  double* krylov_coeffs, int64_t n_coeffs) {
    return guarded([&] {
        QMB_REQUIRE(h && opts && res, QMB_ERR_INVALID, "null argument");
        const qmb_lanczos_opts& o = *opts;
        QMB_REQUIRE(o.mode >= 0 && o.mode <= 2, QMB_ERR_INVALID, "unknown mode");
        QMB_REQUIRE(o.max_iter >= 1 && o.max_iter <= 4096, QMB_ERR_INVALID, "max_iter must be in 1..4096");
        QMB_REQUIRE(o.reorth >= 0 && o.reorth <= 2, QMB_ERR_INVALID, "reorth must be 0, 1 or 2");
        QMB_REQUIRE(o.start == QMB_START_SPLITMIX || o.start == QMB_START_CURAND, QMB_ERR_INVALID,
                    "unknown start-vector mode");
        QMB_REQUIRE(o.hv == QMB_HV_STORED || o.hv == QMB_HV_MATRIX_FREE, QMB_ERR_INVALID, "unknown hv");
        DeviceGuard dg(h->device);
        bool mf = o.hv == QMB_HV_MATRIX_FREE;
        bool need64 = o.mode != QMB_MODE_FP32;
        bool need32 = o.mode != QMB_MODE_FP64;
        if (!mf) {
            QMB_REQUIRE(!need64 || h->val64.p, QMB_ERR_INVALID, "handle holds no FP64 values");
            QMB_REQUIRE(!need32 || h->val32.p, QMB_ERR_INVALID, "handle holds no FP32 values");
        } else {
            mf_tables(h);
        }
        // operators: matrix-free, or the stored values in the coded layout
        // where one was built, else the plain sliced ELL; the low phase's
        // operator is unused in FP64 mode and stands in for the high one in
        // FP32 mode
        auto dispatch = [&](auto real_tag) {
            using R = decltype(real_tag);  // float or float2
            using D = typename std::conditional<std::is_same<R, float>::value, double, double2>::type;
            auto run = [&](const auto& a, size_t sa, const auto& b, size_t sb) {
                using A = typename std::decay<decltype(a)>::type;
                using B = typename std::decay<decltype(b)>::type;
                solve<A, B, R, D>(h, a, sa, b, sb, o, res, krylov_coeffs, n_coeffs);
            };
            auto op32 = [&](auto&& k) {
                if (h->cb32.nb > 0) k(h->cb<R>(), CbSellOp<R>::smem_bytes());
                else k(h->sell<R>(false), (size_t)0);
            };
            auto op64 = [&](auto&& k) {
                if (h->cb64.nb > 0) {
                    k(h->cb<D>(), CbSellOp<D>::smem_bytes());
                    return;
                }
                k(h->sell<D>(true), (size_t)0);
            };
            if (mf) {
                auto a = h->mf<R>();
                auto b = h->mf<D>();
                run(a, a.smem_bytes(), b, b.smem_bytes());
            } else if (!need32) {
                op64([&](const auto& b, size_t sb) { run(b, sb, b, sb); });
            } else if (!need64) {
                op32([&](const auto& a, size_t sa) { run(a, sa, a, sa); });
            } else {
                op32([&](const auto& a, size_t sa) { op64([&](const auto& b, size_t sb) { run(a, sa, b, sb); }); });
            }
        };
        if (h->cplx) dispatch(float2{});
        else dispatch(float{});
        if (!res->converged && o.tol > 0) throw Error{QMB_ERR_NOT_CONVERGED, "Lanczos did not reach the tolerance within max_iter"};
    });
}

extern "C" qmb_status qmb_ground_state(qmb_ham h, void* psi, int64_t n) {
    return guarded([&] {
        QMB_REQUIRE(h && psi, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(h->psi.p && h->psi_n == n, QMB_ERR_INVALID,
                    "no ground state kept (run qmb_lanczos with want_vector) or wrong length");
        DeviceGuard dg(h->device);
        QMB_CUDA_TRY(cudaMemcpy(psi, h->psi.p, h->psi.n, cudaMemcpyDeviceToHost));
    });
}

extern "C" qmb_status qmb_set_ground_state(qmb_ham h, const void* psi, int64_t n) {
    return guarded([&] {
        QMB_REQUIRE(h && psi, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(n == h->n, QMB_ERR_INVALID, "length differs from the handle's row count");
        DeviceGuard dg(h->device);
        const size_t bytes = (size_t)n * (h->cplx ? sizeof(double2) : sizeof(double));
        h->psi.alloc(bytes);
        QMB_CUDA_TRY(cudaMemcpy(h->psi.p, psi, bytes, cudaMemcpyHostToDevice));
        h->psi_n = n;
    });
}

// LanczosEigenStateFromSeed (exact_diagonalization/lanczos.cu:31-104): the
// Lanczos vectors of qmb_lanczos_ref_ell are regenerated from the same cuRAND
// start with the same kernels, so they are bit-identical to the solve's, and
// psi = sum_j c_j v_j accumulates in the caller's FP32 type.  Trailing zero
// coefficients (a solve that broke down early) end the regeneration there.
extern "C" qmb_status qmb_eigvec_from_seed_ref(long long seed, void* psi_dev, const float* krylov, int n_iter,
                                               int nobv, int max_terms, const uint32_t* ind_dev,
                                               const void* val_dev, const int16_t* track_dev, int is_complex) {
    return guarded([&] {
        QMB_REQUIRE(psi_dev && krylov && ind_dev && val_dev && track_dev, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(nobv >= 1 && max_terms >= 1 && n_iter >= 1 && n_iter <= 4096, QMB_ERR_INVALID, "bad sizes");
        int m = n_iter;
        while (m > 0 && krylov[m - 1] == 0.0f) --m;
        cudaStream_t s;
        QMB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct SG { cudaStream_t s; ~SG() { cudaStreamDestroy(s); } } sg{s};
        const size_t es = is_complex ? sizeof(float2) : sizeof(float);
        QMB_CUDA_TRY(cudaMemsetAsync(psi_dev, 0, es * (size_t)nobv, s));
        if (m == 0) {
            QMB_CUDA_TRY(cudaStreamSynchronize(s));
            return;
        }
        PhaseOut ph;
        ph.m = m;
        ph.s.assign(krylov, krylov + m);
        LzState st;
        st.init(m, lz_blocks(), false);
        int n_hv = 0;
        if (is_complex) {
            RefEllOp<float2> op{nobv, max_terms, ind_dev, (const float2*)val_dev, track_dev};
            DevBuf<float2> vr(2 * (size_t)nobv), wb(2 * (size_t)nobv);
            ritz_vector<RefEllOp<float2>, float2, float2>(op, 0, ph, QMB_START_CURAND, (uint64_t)seed, nullptr,
                                                          false, vr, 2, wb, st, (float2*)psi_dev, n_hv, s);
        } else {
            RefEllOp<float> op{nobv, max_terms, ind_dev, (const float*)val_dev, track_dev};
            DevBuf<float> vr(2 * (size_t)nobv), wb(2 * (size_t)nobv);
            ritz_vector<RefEllOp<float>, float, float>(op, 0, ph, QMB_START_CURAND, (uint64_t)seed, nullptr,
                                                       false, vr, 2, wb, st, (float*)psi_dev, n_hv, s);
        }
    });
}

extern "C" qmb_status qmb_lanczos_ref_ell(float* E, int n_iter, int nobv, int max_terms,
                                          long long seed, const uint32_t* ind_dev,
                                          const void* val_dev, const int16_t* track_dev,
                                          int is_complex, float* krylov_out, int check_eig_state,
                                          float* residual) {
    return guarded([&] {
        QMB_REQUIRE(E && ind_dev && val_dev && track_dev, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(nobv >= 1 && max_terms >= 1 && n_iter >= 1 && n_iter <= 4096, QMB_ERR_INVALID,
                    "bad sizes");
        int dev = 0;
        QMB_CUDA_TRY(cudaGetDevice(&dev));
        qmb_ham_s dummy;
        dummy.n = nobv;
        qmb_lanczos_opts o;
        qmb_lanczos_default_opts(&o);
        o.mode = QMB_MODE_FP32;
        o.max_iter = n_iter;
        o.tol = 0.0;
        o.start = QMB_START_CURAND;
        o.seed = (uint64_t)seed;
        o.check_every = o.max_iter;
        qmb_lanczos_result r;
        std::vector<double> cf(o.max_iter);
        if (is_complex) {
            RefEllOp<float2> op{nobv, max_terms, ind_dev, (const float2*)val_dev, track_dev};
            solve<RefEllOp<float2>, RefEllOp<float2>, float2, double2>(&dummy, op, 0, op, 0, o, &r, cf.data(), o.max_iter);
        } else {
            RefEllOp<float> op{nobv, max_terms, ind_dev, (const float*)val_dev, track_dev};
            solve<RefEllOp<float>, RefEllOp<float>, float, double>(&dummy, op, 0, op, 0, o, &r, cf.data(), o.max_iter);
        }
        *E = (float)r.E0;
        if (krylov_out)
            for (int i = 0; i < n_iter; ++i) krylov_out[i] = i < o.max_iter ? (float)cf[i] : 0.0f;
        if (residual) *residual = check_eig_state ? (float)r.residual_ref : 0.0f;
    });
}

// ------------------------------------------------------ no-allocation variant
// qmb_lanczos_ref_ell_noalloc: the computation of qmb_lanczos_ref_ell with
// every device buffer carved out of one file-scope static array, for callers
// that must not allocate device memory while they run: a serving loop that
// owns its memory budget up front, a process sharing the GPU under a hard
// memory cap, or code running next to a pooled allocator that must not see
// cudaMalloc/cudaFree traffic (which synchronises the device).
namespace qmb {
namespace {

constexpr int64_t kNaMaxRows = 262144;  // nobv limit
constexpr int kNaMaxIter = 1024;        // n_iter limit
constexpr int kNaMaxBlocks = 1024;      // reduction partials per grid
// vectors: 2 work + 2 basis vectors in FP32 and the FP64 Ritz vector, complex
constexpr size_t kNaVecBytes = (size_t)kNaMaxRows * (4 * sizeof(float2) + sizeof(double2));
// scalars: alpha, beta, Ritz coefficients, partials (2 grids), scratch, step, counters
constexpr size_t kNaScalarBytes = 64 * 1024;
constexpr size_t kNaScratchBytes = kNaVecBytes + kNaScalarBytes;  // 12 MiB + 64 KiB
static_assert(sizeof(double) * ((kNaMaxIter + 1) + (kNaMaxIter + 2) + kNaMaxIter + 2 * kNaMaxBlocks + 4) +
                      64 <= kNaScalarBytes,
              "scalar region too small");

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

std::mutex g_na_mutex;  // one caller at a time per process

// Host-side work arrays of a call (tridiagonal, Ritz coefficients and the
// tridiagonal solver's workspace, about 70 KB), kept off the caller's stack
// for callers on small-stack threads; g_na_mutex guards them.
struct NaHost {
    double ha[kNaMaxIter + 1], hb[kNaMaxIter + 2];
    double sv[kNaMaxIter], work[4 * kNaMaxIter], cf[kNaMaxIter];
    int iwork[kNaMaxIter];
};
NaHost g_na_host;

// The device address of the static scratch on the current device, looked up
// on every call (a device reset by the host application reloads the module,
// which may move it).  The first call on a device loads this module's device
// code.
unsigned char* na_scratch() {
    void* p = nullptr;
    cudaError_t ce = cudaGetSymbolAddress(&p, g_na_scratch);
    if (ce != cudaSuccess || !p) {
        cudaGetLastError();
        throw Error{QMB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(ce)};
    }
    return static_cast<unsigned char*>(p);
}

template <class V, class P>
void na_solve(unsigned char* base, const RefEllOp<V>& op, int n_iter, uint64_t seed, cudaStream_t s,
              double* E, double* coeffs, double* res_ref) {
    const int64_t n = op.n;
    const int nb = std::min(lz_blocks(), kNaMaxBlocks);
    // vector region
    V* wbuf = reinterpret_cast<V*>(base);
    V* vring = wbuf + 2 * n;
    P* psi = reinterpret_cast<P*>(base + (size_t)kNaMaxRows * 4 * sizeof(float2));
    // scalar region
    double* sc = reinterpret_cast<double*>(base + kNaVecBytes);
    LzDev d{};
    d.alpha = sc;
    d.beta = d.alpha + (kNaMaxIter + 1);
    double* ritz = d.beta + (kNaMaxIter + 2);
    d.partials = ritz + kNaMaxIter;
    d.scratch = d.partials + 2 * kNaMaxBlocks;
    d.iter = reinterpret_cast<int*>(d.scratch + 4);
    d.counter = reinterpret_cast<unsigned*>(d.iter + 4);
    d.coefs = nullptr;
    d.cpart = nullptr;
    const int K = 2;
    // the reduction counters must start at zero (an interrupted earlier call
    // may have left them set)
    QMB_CUDA_TRY(cudaMemsetAsync(d.counter, 0, 2 * sizeof(unsigned), s));

    k_lz_start<V, P><<<nb, kLzBlock, 0, s>>>(n, 1, seed, (const P*)nullptr, wbuf, d);
    for (int j = 0; j < n_iter; ++j) {
        k_lz_hv<RefEllOp<V>, V, P><<<nb, kLzBlock, 0, s>>>(op, wbuf, vring, K, d, nullptr, (P*)nullptr);
        k_lz_update<V><<<nb, kLzBlock, 0, s>>>(n, wbuf, vring, K, d, 1);
    }
    check_launch("noalloc lanczos steps");
    double* ha = g_na_host.ha;
    double* hb = g_na_host.hb;
    QMB_CUDA_TRY(cudaMemcpyAsync(ha, d.alpha, sizeof(double) * n_iter, cudaMemcpyDeviceToHost, s));
    QMB_CUDA_TRY(cudaMemcpyAsync(hb, d.beta, sizeof(double) * (n_iter + 1), cudaMemcpyDeviceToHost, s));
    QMB_CUDA_TRY(cudaStreamSynchronize(s));
    int m = n_iter;
    for (int i = 0; i < n_iter; ++i) {
        QMB_REQUIRE(std::isfinite(ha[i]) && std::isfinite(hb[i + 1]), QMB_ERR_INVALID,
                    "non-finite Lanczos coefficient (check the Hamiltonian)");
        double sc_i = std::fabs(ha[i]) + (i > 0 ? std::fabs(hb[i]) : 0.0) + 1e-300;
        if (!(hb[i + 1] > 1e-13 * sc_i)) {  // invariant subspace reached
            m = i + 1;
            break;
        }
    }
    double theta = tridiag_min_eig(ha, hb + 1, m);
    double* sv = g_na_host.sv;
    tridiag_eigvec_ws(ha, hb + 1, m, theta, sv, g_na_host.work, g_na_host.iwork);
    for (int i = 0; i < n_iter; ++i) coeffs[i] = i < m ? sv[i] : 0.0;
    *E = theta;
    if (!res_ref) return;
    // Ritz vector by regenerating v_0..v_{m-1} (same kernels, same order)
    QMB_CUDA_TRY(cudaMemcpyAsync(ritz, sv, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    QMB_CUDA_TRY(cudaMemsetAsync(psi, 0, sizeof(P) * n, s));
    k_lz_start<V, P><<<nb, kLzBlock, 0, s>>>(n, 1, seed, (const P*)nullptr, wbuf, d);
    for (int j = 0; j < m; ++j) {
        k_lz_hv<RefEllOp<V>, V, P><<<nb, kLzBlock, 0, s>>>(op, wbuf, vring, K, d, ritz, psi);
        if (j + 1 < m) k_lz_update<V><<<nb, kLzBlock, 0, s>>>(n, wbuf, vring, K, d, 1);
    }
    k_residual<RefEllOp<V>, P><<<nb, kLzBlock, 0, s>>>(op, psi, theta, d);
    check_launch("noalloc residual");
    double h[2];
    QMB_CUDA_TRY(cudaMemcpyAsync(h, d.scratch, sizeof(h), cudaMemcpyDeviceToHost, s));
    QMB_CUDA_TRY(cudaStreamSynchronize(s));
    double rn = std::sqrt(h[0] / std::max(h[1], 1e-300));
    *res_ref = rn * std::sqrt(h[1]) / (double)n;
}

}  // namespace
}  // namespace qmb

extern "C" qmb_status qmb_lanczos_ref_ell_noalloc(float* E, int n_iter, int nobv, int max_terms,
                                                  long long seed, const uint32_t* ind_dev,
                                                  const void* val_dev, const int16_t* track_dev,
                                                  int is_complex, float* krylov_out,
                                                  int check_eig_state, float* residual,
                                                  void* stream) {
    return guarded([&] {
        QMB_REQUIRE(E && ind_dev && val_dev && track_dev, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(nobv >= 1 && max_terms >= 1 && n_iter >= 1, QMB_ERR_INVALID, "bad sizes");
        QMB_REQUIRE(nobv <= kNaMaxRows, QMB_ERR_INVALID,
                    "nobv exceeds the 262144 rows of the static scratch (use qmb_lanczos_ref_ell)");
        QMB_REQUIRE(n_iter <= kNaMaxIter, QMB_ERR_INVALID,
                    "n_iter exceeds the 1024 steps of the static scratch (use qmb_lanczos_ref_ell)");
        std::lock_guard<std::mutex> lock(g_na_mutex);
        unsigned char* base = na_scratch();
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        double e0 = 0.0, rr = 0.0;
        double* cf = g_na_host.cf;
        double* want_res = (residual && check_eig_state) ? &rr : nullptr;
        if (is_complex) {
            RefEllOp<float2> op{nobv, max_terms, ind_dev, (const float2*)val_dev, track_dev};
            na_solve<float2, double2>(base, op, n_iter, (uint64_t)seed, s, &e0, cf, want_res);
        } else {
            RefEllOp<float> op{nobv, max_terms, ind_dev, (const float*)val_dev, track_dev};
            na_solve<float, double>(base, op, n_iter, (uint64_t)seed, s, &e0, cf, want_res);
        }
        *E = (float)e0;
        if (krylov_out)
            for (int i = 0; i < n_iter; ++i) krylov_out[i] = (float)cf[i];
        if (residual) *residual = check_eig_state ? (float)rr : 0.0f;
    });
}
