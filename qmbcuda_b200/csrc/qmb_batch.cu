// qmb_batch.cu -- many coupling sets x many sectors in one batched Lanczos.
//
// Extends the serial irrep loop of the reference driver
// (exact_diagonalization/HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:127-242),
// which rebuilds an ELL and runs one Lanczos per irrep.  Here a family
//   H(set, sector) = c_xy[set] * A_sector + c_z[set] * D_sector
// shares the sparsity and values of A (hopping) and D (diagonal) across all
// coupling sets.  Vectors are stored [sector][row][set] (set fastest), so the
// gather of x[col] for a whole warp is one contiguous run of n_sets elements:
// every load is coalesced and the matrix entries are warp-uniform broadcasts.
// A warp owns a row; lane l owns sets l*SPL .. l*SPL+SPL-1.  The Lanczos
// scalars are per (sector, set); the convergence test and the Ritz
// coefficients are computed on the device, one thread per problem.  Sectors
// whose problems have all converged leave the work list (their tiles return
// at once), and every step is a replayable CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <chrono>
#include <cstdio>
#include <cstdlib>

#include <cub/cub.cuh>

#include "qmb_ham.cuh"
#include "qmb_lanczos.cuh"

namespace qmb {

constexpr int kBThreads = 256;      // threads per block
constexpr int kBTile = 32;          // rows per work item

// Kernels of this file executed for the current batched call on this thread
// (launches, plus kernel nodes run by the CUDA graphs).
thread_local double g_kernels = 0;

// Non-owning view of device memory with DevBuf's helpers.
template <class T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    void zero(cudaStream_t st = 0) { QMB_CUDA_TRY(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
    void upload(const T* h, size_t count, cudaStream_t st = 0) {
        QMB_CUDA_TRY(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    void download(T* h, size_t count, cudaStream_t st = 0) const {
        QMB_CUDA_TRY(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, st));
    }
};

// Temporaries of a batched solve, kept for the next solve: ws_take() hands
// out the pool's buffers in call order and grows one only when a request is
// larger than it, so a solve that repeats an earlier one allocates nothing
// (no cudaMalloc / cudaFree, whose device-wide synchronisation and driver
// latency would otherwise sit inside the solve).
struct WsPool {
    std::vector<std::unique_ptr<DevBuf<unsigned char>>> bufs;
    size_t next = 0;
};
thread_local WsPool* g_ws = nullptr;  // pool of the solve running on this thread

template <class T>
static Buf<T> ws_take(size_t count) {
    if (count == 0) count = 1;
    QMB_REQUIRE(g_ws, QMB_ERR_INVALID, "internal: workspace taken outside a batched solve");
    WsPool& w = *g_ws;
    if (w.next == w.bufs.size()) w.bufs.emplace_back(new DevBuf<unsigned char>());
    DevBuf<unsigned char>& d = *w.bufs[w.next++];
    if (d.n < count * sizeof(T)) d.alloc(count * sizeof(T));
    return Buf<T>{reinterpret_cast<T*>(d.p), count};
}

struct BatchArgs {
    int n_sectors;
    int nsp;                     // padded sets: 32, 64, 128 or 256
    int n_groups;                // unused (1)
    const int* tile_sector;      // [n_tiles]
    const int* tile_row0;        // [n_tiles]
    const int64_t* sec_elem;     // [n_sectors+1] element offset (rows*nsp)
    const int64_t* sec_nrows;    // [n_sectors]
    const int64_t* row_ptr;      // concatenated CSR row pointers (global entry index)
    const int64_t* row_base;     // [n_sectors] index of the sector's first row in row_ptr
    const int64_t* row0;         // [n_sectors] index of the sector's first row in the diagonals
    const uint32_t* col;
    const void* val;             // double/double2/float/float2 per sector kind
    const void* dxy;             // diagonal of A  [rows]
    const void* dz;              // diagonal of D  [rows]
    const double* cxy;           // [nsp]
    const double* cz;            // [nsp]
    const int* active;           // [n_sectors]
    int max_tile_entries;        // largest CSR entry count of one work item
    int c_stride;                // couplings of sector s at cxy[s * c_stride + set] (0: shared)
};

// SPL consecutive sets of one row: one 4-, 8- or 16-byte access.
template <class V, int SPL>
struct alignas(sizeof(V) * SPL) Pack {
    V v[SPL];
};

struct BLz {
    double* alpha;      // [cap][n_prob]
    double* beta;       // [cap+1][n_prob]
    double* partials;   // [n_tiles][nsp]
    int* iter;
    int n_prob;
    unsigned* sec_ctr;       // [n_sectors] tiles finished in the current kernel
    const int* sec_tile0;    // [n_sectors]
    const int* sec_ntiles;   // [n_sectors]
    double gap_cap = kRestartGapCap;  // restart gap cap relative to |theta| (with a phase-1 gap)
};

// Called by every thread of a block after it wrote the partials of one tile
// of sector s.  The block that finishes the sector's last tile sums the
// sector's partials in tile order (deterministic) into out[s*nsp + set],
// optionally as a square root, and resets the sector counter.  Other blocks
// keep working on later sectors meanwhile.
__device__ __forceinline__ void sector_tail_reduce(const BatchArgs& a, const BLz& lz, int s,
                                                   double* __restrict__ out, bool take_sqrt) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned old = atomicAdd(lz.sec_ctr + s, 1u);
        last = (old == (unsigned)lz.sec_ntiles[s] - 1u);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        const int nsp = a.nsp, t0 = lz.sec_tile0[s], nt = lz.sec_ntiles[s];
        for (int set = threadIdx.x; set < nsp; set += blockDim.x) {
            double t = 0.0;
            for (int k = 0; k < nt; ++k) t += __ldcg(lz.partials + (int64_t)(t0 + k) * nsp + set);
            out[(int64_t)s * nsp + set] = take_sqrt ? sqrt(t) : t;
        }
        if (threadIdx.x == 0) lz.sec_ctr[s] = 0u;
    }
    __syncthreads();
}

// Batched H*v, and with `lanczos` the Lanczos step K1:
//   y = H w_j / beta_j - beta_j v_{j-1};  v_j = w_j / beta_j;  alpha partials per (tile, set)
// Thread layout: a row is handled by TPR = nsp/SPL threads (whole warps),
// thread t owns sets t*SPL .. t*SPL+SPL-1, so every gather of x[col] is one
// 16-byte access per thread and a contiguous nsp-element run per row.  The
// block's 256 threads form RG = 256/TPR row groups.  Blocks are persistent
// and take 32-row work items from a queue in sector order, so the rows in
// flight (and the vectors they gather) stay within about two sectors, which
// keeps the gathered x resident in L2.  ctr[0] is the queue head, ctr[1]
// counts retired blocks; the last block resets both.
//
// HOIST: the row's own x[r] and v_{j-1}[r] are loaded before its gathers
// instead of after them, so they travel with the first batch of gathers
// rather than adding a dependent round trip per row; the per-set constants of
// the tile (couplings, beta_j, 1/beta_j) and the alpha partials live in
// shared memory instead of registers, which leaves the registers to the
// gathers of the wider slices.
template <class V, int SPL, int UNR, int MINB, bool HOIST = false>
__global__ void __launch_bounds__(kBThreads, MINB) k_bhv(BatchArgs a, int n_tiles, unsigned* __restrict__ ctr,
                                                   const V* __restrict__ X0, V* __restrict__ Y0,
                                                   V* __restrict__ vring, int K, BLz lz,
                                                   const double* __restrict__ ritz, void* psi_v,
                                                   int lanczos) {
    using M = V;
    using PK = Pack<V, SPL>;
    __shared__ double red[kBThreads * SPL];
    __shared__ int s_tile;
    __shared__ int s_rp[kBTile + 1];
    __shared__ M s_dx[kBTile], s_dz[kBTile];
    extern __shared__ __align__(16) unsigned char s_dyn[];
    M* s_val = reinterpret_cast<M*>(s_dyn);                    // [max_tile_entries]
    uint32_t* s_col = reinterpret_cast<uint32_t*>(s_val + a.max_tile_entries);
    const int nsp = a.nsp;
    const int TPR = nsp / SPL;
    const int RG = kBThreads / TPR;
    const int rg = threadIdx.x / TPR, t = threadIdx.x % TPR, set0 = t * SPL;
    const int lane = threadIdx.x & 31;
    const int j = lanczos ? *lz.iter : 0;
    const int64_t tot = a.sec_elem[a.n_sectors];
    const M* val = reinterpret_cast<const M*>(a.val);
    const M* dxy = reinterpret_cast<const M*>(a.dxy);
    const M* dz = reinterpret_cast<const M*>(a.dz);
    using R = typename Sc<V>::real;
    R cx[SPL], cz[SPL];
    __shared__ R s_cst[HOIST ? 4 * 256 : 1];  // HOIST: cx, cz, beta_j, 1/beta_j per set (nsp <= 256)
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(ctr, 1u);
        __syncthreads();
        const int tile = s_tile;
        __syncthreads();
        if (tile >= n_tiles) break;
        const int s = a.tile_sector[tile];
        if (lanczos && !a.active[s]) continue;
        if constexpr (!HOIST) {
#pragma unroll
            for (int q = 0; q < SPL; ++q) {
                cx[q] = (R)a.cxy[(int64_t)s * a.c_stride + set0 + q];
                cz[q] = (R)a.cz[(int64_t)s * a.c_stride + set0 + q];
            }
        }
        const int64_t nrows = a.sec_nrows[s];
        const int64_t eo = a.sec_elem[s];
        const V* X = X0 + (lanczos ? (int64_t)(j & 1) * tot : 0) + eo;
        V* Y = Y0 + (lanczos ? (int64_t)((j + 1) & 1) * tot : 0) + eo;
        V* Vc = lanczos ? vring + (int64_t)(j % K) * tot + eo : nullptr;
        const V* Vp = lanczos ? vring + (int64_t)((j + K - 1) % K) * tot + eo : nullptr;
        const int prob0 = s * nsp + set0;
        R bj[SPL], inv[SPL];
        double apar[SPL];
        if constexpr (HOIST) {
            for (int i = threadIdx.x; i < nsp; i += blockDim.x) {
                const double b = lanczos ? lz.beta[(int64_t)j * lz.n_prob + s * nsp + i] : 1.0;
                s_cst[i] = (R)a.cxy[(int64_t)s * a.c_stride + i];
                s_cst[256 + i] = (R)a.cz[(int64_t)s * a.c_stride + i];
                s_cst[512 + i] = (R)b;
                s_cst[768 + i] = (R)(1.0 / b);
            }
#pragma unroll
            for (int q = 0; q < SPL; ++q) red[rg * nsp + set0 + q] = 0.0;
        } else {
#pragma unroll
            for (int q = 0; q < SPL; ++q) {
                const double b = lanczos ? lz.beta[(int64_t)j * lz.n_prob + prob0 + q] : 1.0;
                bj[q] = (R)b;
                inv[q] = (R)(1.0 / b);
                apar[q] = 0.0;
            }
        }
        const int64_t rb = a.row_base[s], d0 = a.row0[s];
        const int64_t r0 = a.tile_row0[tile];
        const int64_t r_end = min(nrows, r0 + kBTile);
        const int nr = (int)(r_end - r0);
        // stage the tile's CSR entries, row pointers and diagonals in shared
        // memory: one coalesced load instead of a dependent chain per row
        {
            const int64_t e0 = a.row_ptr[rb + r0];
            const int ne = (int)(a.row_ptr[rb + r_end] - e0);
            for (int i = threadIdx.x; i < ne; i += blockDim.x) {
                s_col[i] = __ldg(a.col + e0 + i);
                s_val[i] = __ldg(val + e0 + i);
            }
            for (int i = threadIdx.x; i <= nr; i += blockDim.x) s_rp[i] = (int)(a.row_ptr[rb + r0 + i] - e0);
            for (int i = threadIdx.x; i < nr; i += blockDim.x) {
                s_dx[i] = dxy[d0 + r0 + i];
                s_dz[i] = dz[d0 + r0 + i];
            }
        }
        __syncthreads();
        for (int64_t r = r0 + rg; r < r_end; r += RG) {
            V acc[SPL];
#pragma unroll
            for (int q = 0; q < SPL; ++q) acc[q] = Sc<V>::zero();
            const int p0 = s_rp[r - r0], p1 = s_rp[r - r0 + 1];
            PK xr, vp, vo, yo;
            if constexpr (HOIST) {
                xr = *reinterpret_cast<const PK*>(X + r * nsp + set0);
                if (lanczos && j > 0) vp = *reinterpret_cast<const PK*>(Vp + r * nsp + set0);
            }
            for (int k = p0; k < p1; k += UNR) {
                // issue the (up to) UNR gathers first, then the FMAs
                PK xv[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u)
                    if (k + u < p1) xv[u] = *reinterpret_cast<const PK*>(X + (int64_t)s_col[k + u] * nsp + set0);
#pragma unroll
                for (int u = 0; u < UNR; ++u)
                    if (k + u < p1) {
                        const M v = s_val[k + u];
#pragma unroll
                        for (int q = 0; q < SPL; ++q) acc[q] = Sc<V>::fma(v, xv[u].v[q], acc[q]);
                    }
            }
            if constexpr (!HOIST) {
                xr = *reinterpret_cast<const PK*>(X + r * nsp + set0);
                if (lanczos && j > 0) vp = *reinterpret_cast<const PK*>(Vp + r * nsp + set0);
            }
            const M dx = s_dx[r - r0], dzz = s_dz[r - r0];
#pragma unroll
            for (int q = 0; q < SPL; ++q) {
                R cxq, czq, bjq, invq;
                if constexpr (HOIST) {
                    cxq = s_cst[set0 + q];
                    czq = s_cst[256 + set0 + q];
                    bjq = s_cst[512 + set0 + q];
                    invq = s_cst[768 + set0 + q];
                } else {
                    cxq = cx[q];
                    czq = cz[q];
                    bjq = bj[q];
                    invq = inv[q];
                }
                V hx = Sc<V>::add(Sc<V>::scale(Sc<V>::fma(dx, xr.v[q], acc[q]), cxq),
                                  Sc<V>::scale(Sc<V>::mul(dzz, xr.v[q]), czq));
                if (!lanczos) {
                    yo.v[q] = hx;
                    continue;
                }
                V vj = Sc<V>::scale(xr.v[q], invq);
                V y = Sc<V>::scale(hx, invq);
                if (j > 0) y = Sc<V>::sub(y, Sc<V>::scale(vp.v[q], bjq));
                vo.v[q] = vj;
                yo.v[q] = y;
                if constexpr (HOIST) red[rg * nsp + set0 + q] += Sc<V>::re_conj_mul(vj, y);
                else apar[q] += Sc<V>::re_conj_mul(vj, y);
                const double crq = (psi_v && ritz) ? ritz[(int64_t)j * lz.n_prob + prob0 + q] : 0.0;
                if (crq != 0.0) {
                    const int64_t e = eo + r * nsp + set0 + q;
                    if constexpr (Sc<V>::cplx) {
                        double2* p2 = reinterpret_cast<double2*>(psi_v) + e;
                        double2 tv = cvt<double2>(vj);
                        p2->x += crq * tv.x;
                        p2->y += crq * tv.y;
                    } else {
                        reinterpret_cast<double*>(psi_v)[e] += crq * (double)vj;
                    }
                }
            }
            *reinterpret_cast<PK*>(Y + r * nsp + set0) = yo;
            if (lanczos) *reinterpret_cast<PK*>(Vc + r * nsp + set0) = vo;
        }
        if (lanczos) {
            if constexpr (!HOIST) {
#pragma unroll
                for (int q = 0; q < SPL; ++q) red[rg * nsp + set0 + q] = apar[q];
            }
            __syncthreads();
            for (int i = threadIdx.x; i < nsp; i += blockDim.x) {
                double tt = 0.0;
                for (int g = 0; g < RG; ++g) tt += red[g * nsp + i];
                lz.partials[(int64_t)tile * nsp + i] = tt;
            }
            sector_tail_reduce(a, lz, s, lz.alpha + (int64_t)j * lz.n_prob, false);
        } else {
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned d = atomicAdd(ctr + 1, 1u);
        if (d == gridDim.x - 1) {
            ctr[0] = 0u;
            ctr[1] = 0u;
            __threadfence();
        }
    }
}

// K2 (batched): w_{j+1} = y - alpha_j v_j; ||w_{j+1}||^2 partials.  One
// block per work item, thread t = set t (coalesced [row][set] runs).
template <class V>
__global__ void k_bupdate(BatchArgs a, int n_tiles, V* __restrict__ W0, const V* __restrict__ vring,
                          int K, BLz lz) {
    const int tile = blockIdx.x;
    const int set = threadIdx.x;
    if (tile >= n_tiles) return;
    const int s = a.tile_sector[tile];
    if (!a.active[s]) return;
    const int nsp = a.nsp;
    const int j = *lz.iter;
    const int64_t tot = a.sec_elem[a.n_sectors];
    const int64_t eo = a.sec_elem[s];
    V* Y = W0 + (int64_t)((j + 1) & 1) * tot + eo;
    const V* Vc = vring + (int64_t)(j % K) * tot + eo;
    if (set < nsp) {
        const double al = lz.alpha[(int64_t)j * lz.n_prob + s * nsp + set];
        double acc = 0.0;
        const int64_t r_end = min(a.sec_nrows[s], (int64_t)a.tile_row0[tile] + kBTile);
        for (int64_t r = a.tile_row0[tile]; r < r_end; ++r) {
            const int64_t e = r * nsp + set;
            V y = Sc<V>::sub(Y[e], Sc<V>::scale(Vc[e], al));
            Y[e] = y;
            acc += Sc<V>::abs2(y);
        }
        lz.partials[(int64_t)tile * nsp + set] = acc;
    }
    sector_tail_reduce(a, lz, s, lz.beta + (int64_t)(j + 1) * lz.n_prob, true);
}

// ||w0||^2 partials per (tile, set).
template <class V>
__global__ void k_bnorm0(BatchArgs a, int n_tiles, const V* __restrict__ W0, BLz lz) {
    const int tile = blockIdx.x;
    const int set = threadIdx.x;
    if (tile >= n_tiles || set >= a.nsp) return;
    const int s = a.tile_sector[tile];
    const int nsp = a.nsp;
    const V* X = W0 + a.sec_elem[s];
    double acc = 0.0;
    const int64_t r_end = min(a.sec_nrows[s], (int64_t)a.tile_row0[tile] + kBTile);
    for (int64_t r = a.tile_row0[tile]; r < r_end; ++r) acc += Sc<V>::abs2(X[r * nsp + set]);
    lz.partials[(int64_t)tile * nsp + set] = acc;
}

__global__ void k_badvance(BLz lz) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *lz.iter += 1;
}

// Start vectors (splitmix uniform(-1,1) or a copy) and beta_0 per problem.
// Per (tile, set) partial sums over a sector's rows of two vectors u, w:
// E == nullptr: part[0] = Re <u, w>, part[1] = ||u||^2;
// otherwise:    part[0] = ||w - E u||^2 (E per problem), part[1] = 0.
template <class V>
__global__ void k_bdot(BatchArgs a, int n_tiles, const V* __restrict__ u, const V* __restrict__ w,
                       const double* __restrict__ E, double* __restrict__ part) {
    const int tile = blockIdx.x;
    const int set = threadIdx.x;
    if (tile >= n_tiles || set >= a.nsp) return;
    const int s = a.tile_sector[tile];
    const int nsp = a.nsp;
    const int64_t eo = a.sec_elem[s];
    const double e = E ? E[s * nsp + set] : 0.0;
    double p0 = 0.0, p1 = 0.0;
    const int64_t r_end = min(a.sec_nrows[s], (int64_t)a.tile_row0[tile] + kBTile);
    for (int64_t r = a.tile_row0[tile]; r < r_end; ++r) {
        const V uu = u[eo + r * nsp + set], ww = w[eo + r * nsp + set];
        if (E) {
            p0 += Sc<V>::abs2(Sc<V>::sub(ww, Sc<V>::scale(uu, e)));
        } else {
            p0 += Sc<V>::re_conj_mul(uu, ww);
            p1 += Sc<V>::abs2(uu);
        }
    }
    const int64_t nt = n_tiles;
    part[(int64_t)tile * nsp + set] = p0;
    part[(nt + tile) * nsp + set] = p1;
}

// Sums the tile partials of every problem in tile order: out[k][p] for k < n_arr.
__global__ void k_bsum(BatchArgs a, int n_tiles, const int* __restrict__ sec_tile0,
                       const int* __restrict__ sec_ntiles, const double* __restrict__ part, int n_arr,
                       int n_prob, double* __restrict__ out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_prob; p += gridDim.x * blockDim.x) {
        int s = p / a.nsp, set = p % a.nsp;
        for (int k = 0; k < n_arr; ++k) {
            double t = 0.0;
            for (int i = 0; i < sec_ntiles[s]; ++i)
                t += part[((int64_t)k * n_tiles + sec_tile0[s] + i) * a.nsp + set];
            out[(int64_t)k * n_prob + p] = t;
        }
    }
}

// Rayleigh quotient of psi (E = <psi,H psi>/<psi,psi>) from s1, s2 in out.
__global__ void k_brq_energy(int n_prob, const double* __restrict__ sums, double* __restrict__ E) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_prob; p += gridDim.x * blockDim.x)
        E[p] = sums[p] / sums[n_prob + p];
}

// Accept a problem when its FP64 residual r satisfies r^2/gap <= tol |E| and
// r <= 1e-4 |E|; sectors with an unaccepted set stay active for the restart.
__global__ void k_brq_accept(BatchArgs a, int n_prob, int nsets, const double* __restrict__ E,
                             const double* __restrict__ r2, const double* __restrict__ psi2,
                             const double* __restrict__ gap, double tol, double gap_cap,
                             int* __restrict__ ok, int* __restrict__ active) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_prob; p += gridDim.x * blockDim.x) {
        int s = p / a.nsp, set = p % a.nsp;
        double sc = fmax(fabs(E[p]), 1e-300);
        double r = sqrt(r2[p] / fmax(psi2[p], 1e-300));
        // the FP32 phase's gap, capped as in the restart (a pair of levels
        // it did not separate would otherwise pass as converged)
        double g = fmin(fmax(gap[p], 1e-10 * sc), gap_cap * sc);
        bool acc = r <= 1e-4 * sc && r * r / g <= tol * sc;
        ok[p] = acc ? 1 : 0;
        if (!acc && set < nsets) atomicOr(active + s, 1);
    }
}

template <class V>
__global__ void k_bstart(BatchArgs a, int64_t tot, int mode, uint64_t seed, const void* from,
                         V* __restrict__ w0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot;
         i += (int64_t)gridDim.x * blockDim.x) {
        V v;
        if (mode == 2) {
            if constexpr (Sc<V>::cplx) v = cvt<V>(reinterpret_cast<const double2*>(from)[i]);
            else v = cvt<V>(reinterpret_cast<const double*>(from)[i]);
        } else {
            auto u = [&](uint64_t k) {
                uint64_t z = seed + k + 0x9E3779B97F4A7C15ull;
                z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
                z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
                z ^= z >> 31;
                return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
            };
            if constexpr (Sc<V>::cplx) v = Sc<V>::from(make_double2(u(2 * i), u(2 * i + 1)));
            else v = Sc<V>::from(make_double2(u(i), 0.0));
        }
        w0[i] = v;
    }
}

__global__ void k_bbeta0(BatchArgs a, const int* __restrict__ sec_tile0,
                         const int* __restrict__ sec_ntiles, BLz lz) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < lz.n_prob; p += gridDim.x * blockDim.x) {
        int s = p / a.nsp, set = p % a.nsp;
        double t = 0.0;
        int t0 = sec_tile0[s], nt = sec_ntiles[s];
        for (int k = 0; k < nt; ++k) t += lz.partials[(int64_t)(t0 + k) * a.nsp + set];
        lz.beta[p] = sqrt(t);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *lz.iter = 0;
}

// Lowest Ritz value of every problem by Sturm bisection on its tridiagonal
// (m_p steps).  Marks converged problems and deactivates finished sectors.
__device__ double bis_kth(const double* al, const double* be, int n_prob, int p, int m, int kth) {
    double lo = al[p], hi = al[p];
    for (int i = 0; i < m; ++i) {
        double a = al[(int64_t)i * n_prob + p];
        double r = (i > 0 ? fabs(be[(int64_t)i * n_prob + p]) : 0.0) +
                   (i < m - 1 ? fabs(be[(int64_t)(i + 1) * n_prob + p]) : 0.0);
        lo = fmin(lo, a - r);
        hi = fmax(hi, a + r);
    }
    double span = fmax(fabs(lo), fabs(hi));
    lo -= 1e-12 * span + 1e-300;
    hi += 1e-12 * span + 1e-300;
    for (int it = 0; it < 200; ++it) {
        double x = 0.5 * (lo + hi);
        if (x <= lo || x >= hi) break;
        int cnt = 0;
        double d = al[p] - x;
        if (d < 0) ++cnt;
        for (int i = 1; i < m; ++i) {
            if (fabs(d) < 1e-290) d = d < 0 ? -1e-290 : 1e-290;
            double e = be[(int64_t)i * n_prob + p];
            d = al[(int64_t)i * n_prob + p] - x - e * e / d;
            if (d < 0) ++cnt;
        }
        if (cnt >= kth + 1) hi = x;
        else lo = x;
        if (hi - lo <= 4.5e-16 * fmax(fabs(lo), fabs(hi))) break;
    }
    return 0.5 * (lo + hi);
}

__device__ double bis_min(const double* al, const double* be, int n_prob, int p, int m) {
    return bis_kth(al, be, n_prob, p, m, 0);
}

// Last component of the unit eigenvector of T_m for eigenvalue th: inverse
// iteration with LDL^T of T - th I (tiny pivots replaced), scratch [i][p].
__device__ double last_ritz_component(const BLz& lz, int p, int m, double th, double* L,
                                      double* D, double* x) {
    const int np = lz.n_prob;
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(lz.alpha[(int64_t)i * np + p] - th));
    double tiny = 1e-15 * fmax(scale, 1e-300);
    double d = lz.alpha[p] - th;
    for (int i = 0; i < m; ++i) {
        if (i > 0) {
            double e = lz.beta[(int64_t)i * np + p];
            double l = e / D[(int64_t)(i - 1) * np + p];
            L[(int64_t)(i - 1) * np + p] = l;
            d = lz.alpha[(int64_t)i * np + p] - th - l * e;
        }
        if (fabs(d) < tiny) d = d < 0 ? -tiny : tiny;
        D[(int64_t)i * np + p] = d;
    }
    for (int i = 0; i < m; ++i) x[(int64_t)i * np + p] = 1.0;
    double last = 0.0;
    for (int it = 0; it < 2; ++it) {
        for (int i = 1; i < m; ++i)
            x[(int64_t)i * np + p] -= L[(int64_t)(i - 1) * np + p] * x[(int64_t)(i - 1) * np + p];
        for (int i = 0; i < m; ++i) x[(int64_t)i * np + p] /= D[(int64_t)i * np + p];
        for (int i = m - 2; i >= 0; --i)
            x[(int64_t)i * np + p] -= L[(int64_t)i * np + p] * x[(int64_t)(i + 1) * np + p];
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += x[(int64_t)i * np + p] * x[(int64_t)i * np + p];
        nrm = sqrt(nrm);
        for (int i = 0; i < m; ++i) x[(int64_t)i * np + p] /= nrm;
        last = x[(int64_t)(m - 1) * np + p];
    }
    return last;
}

// Number of eigenvalues of the m x m tridiagonal (a, b) below x: sign
// changes of the characteristic-polynomial sequence
//   P_0 = 1, P_1 = a_0 - x, P_i = (a_{i-1} - x) P_{i-1} - b_{i-1}^2 P_{i-2}
// (Sturm).  The pair is rescaled by a power of two when it leaves
// [2^-400, 2^400], which keeps every ratio P_i / P_{i-1} exact; a zero P_i
// is replaced by a tiny value of the previous sign (ratio +tiny, the usual
// perturbation of the LDL^T count).  b2[i] = b_i^2 for i >= 1.
__device__ __forceinline__ int sturm_count_poly(const double* __restrict__ a, const double* __restrict__ b2,
                                                int m, double x) {
    double p0 = 1.0, p1 = a[0] - x;
    if (p1 == 0.0) p1 = 1e-300;
    int cnt = p1 < 0.0;
    for (int i = 1; i < m; ++i) {
        double pn = fma(a[i] - x, p1, -b2[i] * p0);
        if (pn == 0.0) pn = p1 * 0x1p-200;
        cnt += (pn < 0.0) != (p1 < 0.0);
        p0 = p1;
        p1 = pn;
        const double s = fabs(p1);
        if (s > 0x1p400 || s < 0x1p-400) {
            int e;
            frexp(p1, &e);
            p0 = ldexp(p0, -e);
            p1 = ldexp(p1, -e);
        }
    }
    return cnt;
}

// k-th smallest eigenvalue (k = 0 lowest) by 33-section: every lane counts at
// one of 32 interior points of [lo, hi] (count(lo) <= k < count(hi) on entry)
// and the bracket shrinks to the sub-interval where the count passes k.
// Stops when the width is <= rtol * max(|lo|, |hi|) + atol or stops shrinking.
__device__ double warp_kth_eig(const double* a, const double* b2, int m, int k, double lo, double hi,
                               double rtol, double atol) {
    const int lane = threadIdx.x & 31;
    for (int round = 0; round < 64; ++round) {
        const double w = hi - lo;
        if (!(w > rtol * fmax(fabs(lo), fabs(hi)) + atol)) break;
        const double x = lo + w * (double)(lane + 1) * (1.0 / 33.0);
        const int c = sturm_count_poly(a, b2, m, x);
        const unsigned ge = __ballot_sync(0xffffffffu, c >= k + 1);
        const int f = ge ? __ffs(ge) - 1 : 32;
        const double xf = __shfl_sync(0xffffffffu, x, f < 32 ? f : 31);
        const double xl = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
        const double nhi = f < 32 ? xf : hi;
        const double nlo = f > 0 ? xl : lo;
        if (!(nhi - nlo < w) || !(nlo < nhi)) break;
        lo = nlo;
        hi = nhi;
    }
    return 0.5 * (lo + hi);
}

// Lowest Ritz value of every active problem and its convergence test.  With
// est = beta_m |s_{m-1}| (residual norm of the Ritz pair) and gap = second
// minus lowest Ritz value (or gap_in from an earlier phase), a problem has
// converged when
//   e_tol > 0:   est^2 / gap <= e_tol |theta| and |theta - theta_prev| <= e_tol |theta|
//   res_tol > 0: est <= res_tol |theta|
//   stall > 0:   |theta - theta_prev| <= stall |theta| since the last check
// or when its Krylov space ends.  Sectors with an unconverged set stay active.
// One warp per problem: the tridiagonal is staged in shared memory
// (kCheckArrays arrays of stride m + 2 per warp) and the eigenvalues are
// found by 33-section over the lanes.
constexpr int kCheckArrays = 6;
__global__ void k_bcheck(BatchArgs a, BLz lz, int nsets, double stall, double res_tol, double e_tol,
                         const double* __restrict__ gap_in, double* __restrict__ gap_out,
                         double* __restrict__ theta, double* __restrict__ theta_prev,
                         int* __restrict__ msteps, int* __restrict__ conv, int* __restrict__ active_next,
                         int* __restrict__ open_cnt) {
    extern __shared__ __align__(16) unsigned char s_chk[];
    const int m = *lz.iter;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int stride = m + 2;
    double* sa = reinterpret_cast<double*>(s_chk) + (size_t)wib * kCheckArrays * stride;
    double* sb = sa + stride;    // beta_i
    double* sb2 = sb + stride;   // beta_i^2
    double* sL = sb2 + stride;
    double* sD = sL + stride;
    double* sx = sD + stride;
    const int np = lz.n_prob;
    const int wpb = blockDim.x >> 5;
    for (int p = blockIdx.x * wpb + wib; p < np; p += gridDim.x * wpb) {
        const int s = p / a.nsp, set = p % a.nsp;
        if (!a.active[s] || conv[p]) continue;
        for (int i = lane; i <= m; i += 32) {
            if (i < m) sa[i] = lz.alpha[(int64_t)i * np + p];
            const double bb = lz.beta[(int64_t)i * np + p];
            sb[i] = bb;
            sb2[i] = bb * bb;
        }
        __syncwarp();
        // a (near) zero beta ends this problem's Krylov space: truncate there
        const int i0 = max(msteps[p], 1);
        int me = m;
        for (int base = i0; base <= m; base += 32) {
            const int i = base + lane;
            const bool small = i <= m && !(sb[i] > 1e-13 * (fabs(sa[i - 1]) + 1e-300));
            const unsigned bal = __ballot_sync(0xffffffffu, small);
            if (bal) {
                me = base + __ffs(bal) - 1;
                break;
            }
        }
        const bool brk = me < m || (me == m && !(sb[m] > 1e-13 * (fabs(sa[m - 1]) + 1e-300)));
        const bool first = msteps[p] == 0;
        // Gershgorin bracket of T_me
        double glo = 1e300, ghi = -1e300;
        for (int i = lane; i < me; i += 32) {
            const double r = (i > 0 ? fabs(sb[i]) : 0.0) + (i < me - 1 ? fabs(sb[i + 1]) : 0.0);
            glo = fmin(glo, sa[i] - r);
            ghi = fmax(ghi, sa[i] + r);
        }
        for (int o = 16; o; o >>= 1) {
            glo = fmin(glo, __shfl_xor_sync(0xffffffffu, glo, o));
            ghi = fmax(ghi, __shfl_xor_sync(0xffffffffu, ghi, o));
        }
        const double span = fmax(fabs(glo), fabs(ghi));
        glo -= 1e-12 * span + 1e-300;
        ghi += 1e-12 * span + 1e-300;
        // theta can only decrease as the Krylov space grows: try a narrow
        // bracket below the previous value first
        const double prev = theta_prev[p];
        double lo = glo, hi = ghi;
        if (!first) {
            const double w = 1e-3 * fmax(fabs(prev), 1e-300);
            const double x = lane == 0 ? prev - w : prev + 8.0 * 2.2e-16 * fabs(prev) + 1e-300;
            const int c = lane < 2 ? sturm_count_poly(sa, sb2, me, x) : 0;
            const int c0 = __shfl_sync(0xffffffffu, c, 0), c1 = __shfl_sync(0xffffffffu, c, 1);
            const double x0 = __shfl_sync(0xffffffffu, x, 0), x1 = __shfl_sync(0xffffffffu, x, 1);
            if (c0 == 0 && x0 > lo) lo = x0;
            if (c1 >= 1 && x1 < hi) hi = x1;
        }
        const double th = warp_kth_eig(sa, sb2, me, 0, lo, hi, 4.5e-16, 0.0);
        const double sc = fmax(fabs(th), 1e-300);
        bool done = brk;
        double own_gap = -1.0;
        if (!done) {
            double est = 0.0;
            if (lane == 0) {
                // last component of the unit eigenvector of T_me for th:
                // inverse iteration with LDL^T of T - th I (tiny pivots replaced)
                double scale = 0.0;
                for (int i = 0; i < me; ++i) scale = fmax(scale, fabs(sa[i] - th));
                const double tiny = 1e-15 * fmax(scale, 1e-300);
                double d = sa[0] - th;
                for (int i = 0; i < me; ++i) {
                    if (i > 0) {
                        const double l = sb[i] / sD[i - 1];
                        sL[i - 1] = l;
                        d = sa[i] - th - l * sb[i];
                    }
                    if (fabs(d) < tiny) d = d < 0 ? -tiny : tiny;
                    sD[i] = d;
                }
                for (int i = 0; i < me; ++i) sx[i] = 1.0;
                double last = 0.0;
                for (int it = 0; it < 2; ++it) {
                    for (int i = 1; i < me; ++i) sx[i] -= sL[i - 1] * sx[i - 1];
                    for (int i = 0; i < me; ++i) sx[i] /= sD[i];
                    for (int i = me - 2; i >= 0; --i) sx[i] -= sL[i] * sx[i + 1];
                    double nrm = 0.0;
                    for (int i = 0; i < me; ++i) nrm += sx[i] * sx[i];
                    nrm = sqrt(nrm);
                    for (int i = 0; i < me; ++i) sx[i] /= nrm;
                    last = sx[me - 1];
                }
                est = sb[me] * fabs(last);
            }
            est = __shfl_sync(0xffffffffu, est, 0);
            if (res_tol > 0 && est <= res_tol * sc) done = true;
            // the gap (to the next Ritz value that is not a ghost copy of theta)
            // only matters once the residual is small
            if (!done && est <= 1e-3 * sc && (e_tol > 0 || gap_out)) {
                own_gap = 1e-10 * sc;
                const double xg = th + 1e-10 * sc;
                const int cg = sturm_count_poly(sa, sb2, me, xg);  // same on every lane
                if (cg < min(me, 5)) {
                    const double tk = warp_kth_eig(sa, sb2, me, cg, xg, ghi, 0.0, 1e-7 * (ghi - th));
                    if (tk - th > 1e-10 * sc) own_gap = tk - th;
                }
                const double gap = gap_in ? fmin(fmin(fmax(gap_in[p], 1e-10 * sc), lz.gap_cap * sc), own_gap)
                                          : own_gap;
                // energy bound plus a settled theta (a close level not yet
                // resolved keeps theta moving while the gap estimate is too large)
                if (e_tol > 0 && !first && est * est / gap <= e_tol * sc && fabs(th - prev) <= e_tol * sc)
                    done = true;
            }
            // FP32 floor: theta no longer moves and the residual is moderate
            if (stall > 0 && !first && fabs(th - prev) <= stall * sc && est <= 1e-3 * sc) done = true;
        }
        if (lane == 0) {
            msteps[p] = me;
            theta[p] = th;
            if (gap_out && own_gap > 0) gap_out[p] = own_gap;
            conv[p] = done ? 1 : 0;
            theta_prev[p] = th;
            if (!done && set < nsets) {
                atomicOr(active_next + s, 1);
                if (open_cnt) atomicAdd(open_cnt + s, 1);
            }
        }
        __syncwarp();
    }
}

// Loop control of the device-side Lanczos loop (one block), after the test of
// one block of `check` steps:
//  - products += check * sum_s active[s] * weight[s]  (problems stepped),
//  - active <- active_next, then active_next and open_cnt are cleared,
//  - the loop continues while a sector is active, another block of steps fits
//    under `cap`, the compacted continuation would not pay (its cost
//    sum_s rows_s * 32 * ceil(open_s / 32) above compact_ratio times the
//    current sum_s active_s * rows_s * nsp) and fewer than max_loops blocks ran.
struct LoopCtl {
    int loops;
    int reason;   // 1 converged, 2 step cap, 3 compaction, 4 loop bound
    double products;
};
__global__ void k_bloop_ctl(cudaGraphConditionalHandle h, int in_graph, int n_sectors, int* __restrict__ active,
                            int* __restrict__ active_next, int* __restrict__ open_cnt,
                            const int64_t* __restrict__ nrows, const int* __restrict__ weight, int nsp,
                            int check, int cap, const int* __restrict__ iter, int max_loops,
                            double compact_ratio, const int* __restrict__ group, int n_groups,
                            LoopCtl* __restrict__ ctl) {
    __shared__ double red[32];
    double prev_w = 0.0, any = 0.0, cost_now = 0.0, cost_c = 0.0;
    for (int s = threadIdx.x; s < n_sectors; s += blockDim.x) {
        const int an = active_next[s];
        prev_w += (double)active[s] * weight[s];
        any += an;
        if (an) {
            cost_now += (double)nrows[s] * nsp;
            if (!group) cost_c += (double)nrows[s] * 32.0 * (double)((open_cnt[s] + 31) / 32);
        }
    }
    if (group) {
        // a compacted sub-batch: the open problems of all its virtual sectors
        // over one base sector (group) would share the packed sectors
        for (int g = threadIdx.x; g < n_groups; g += blockDim.x) {
            int open = 0;
            int64_t rows = 0;
            for (int s = 0; s < n_sectors; ++s)
                if (group[s] == g && active_next[s]) {
                    open += open_cnt[s];
                    rows = nrows[s];
                }
            cost_c += (double)rows * 32.0 * (double)((open + 31) / 32);
        }
    }
    prev_w = block_sum(prev_w, red);
    any = block_sum(any, red);
    cost_now = block_sum(cost_now, red);
    cost_c = block_sum(cost_c, red);
    __syncthreads();
    for (int s = threadIdx.x; s < n_sectors; s += blockDim.x) {
        active[s] = active_next[s];
        active_next[s] = 0;
        open_cnt[s] = 0;
    }
    if (threadIdx.x == 0) {
        ctl->products += (double)check * prev_w;
        ctl->loops += 1;
        int go = 1, reason = 0;
        if (any == 0.0) { go = 0; reason = 1; }
        else if (*iter + check > cap) { go = 0; reason = 2; }
        else if (compact_ratio > 0.0 && cost_c <= compact_ratio * cost_now) { go = 0; reason = 3; }
        else if (ctl->loops >= max_loops) { go = 0; reason = 4; }
        ctl->reason = reason;
        if (in_graph) cudaGraphSetConditional(h, go);
    }
}

// Inverse iteration on T_m - th I (LDL^T without pivoting, tiny pivots
// replaced) for problem p; adds the unit eigenvector to out[i][p].
__device__ void add_ritz_vector(const BLz& lz, int p, int m, double th, double* L, double* D,
                                double* x, double* out) {
    const int np = lz.n_prob;
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(lz.alpha[(int64_t)i * np + p] - th));
    double tiny = 1e-15 * fmax(scale, 1e-300);
    double d = lz.alpha[p] - th;
    for (int i = 0; i < m; ++i) {
        if (i > 0) {
            double e = lz.beta[(int64_t)i * np + p];
            double l = e / D[(int64_t)(i - 1) * np + p];
            L[(int64_t)(i - 1) * np + p] = l;
            d = lz.alpha[(int64_t)i * np + p] - th - l * e;
        }
        if (fabs(d) < tiny) d = d < 0 ? -tiny : tiny;
        D[(int64_t)i * np + p] = d;
    }
    for (int i = 0; i < m; ++i) x[(int64_t)i * np + p] = 1.0;
    for (int it = 0; it < 2; ++it) {
        for (int i = 1; i < m; ++i)
            x[(int64_t)i * np + p] -= L[(int64_t)(i - 1) * np + p] * x[(int64_t)(i - 1) * np + p];
        for (int i = 0; i < m; ++i) x[(int64_t)i * np + p] /= D[(int64_t)i * np + p];
        for (int i = m - 2; i >= 0; --i)
            x[(int64_t)i * np + p] -= L[(int64_t)i * np + p] * x[(int64_t)(i + 1) * np + p];
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += x[(int64_t)i * np + p] * x[(int64_t)i * np + p];
        nrm = sqrt(nrm);
        double sg = x[p] < 0 ? -1.0 : 1.0;
        for (int i = 0; i < m; ++i) x[(int64_t)i * np + p] *= sg / nrm;
    }
    for (int i = 0; i < m; ++i) out[(int64_t)i * np + p] += x[(int64_t)i * np + p];
}

// Ritz coefficients of every problem: the lowest Ritz vector plus the Ritz
// vectors of up to three further Ritz values within 1e-4 |theta| of it
// (ghost copies, within 1e-10, excluded).  A partner level that close may
// swap order with the ground state under FP32 rounding; starting the FP64
// restart from the sum keeps both in its Krylov space.  Scratch arrays [i][p].
__global__ void k_britz(BLz lz, const int* __restrict__ msteps, const double* __restrict__ theta,
                        double* __restrict__ L, double* __restrict__ D, double* __restrict__ x,
                        double* __restrict__ ritz, double* __restrict__ gap_out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < lz.n_prob; p += gridDim.x * blockDim.x) {
        const int np = lz.n_prob;
        const int m = msteps[p];
        const double th = theta[p];
        const double sc = fmax(fabs(th), 1e-300);
        for (int i = 0; i < m; ++i) ritz[(int64_t)i * np + p] = 0.0;
        add_ritz_vector(lz, p, m, th, L, D, x, ritz);
        // Ritz values 1..4, each found by bisection at most once
        double tks[5];
        int known = 1;
        auto kth_value = [&](int kth) {
            while (known <= kth) {
                tks[known] = bis_kth(lz.alpha, lz.beta, np, p, m, known);
                ++known;
            }
            return tks[kth];
        };
        if (gap_out) {  // gap to the next Ritz value that is not a ghost copy
            double g = 1e-10 * sc;
            for (int kth = 1; kth < min(m, 5); ++kth) {
                double tk = kth_value(kth);
                if (tk - th > 1e-10 * sc) { g = tk - th; break; }
            }
            gap_out[p] = g;
        }
        for (int kth = 1; kth < min(m, 4); ++kth) {
            const double tk = kth_value(kth);
            if (tk - th > 1e-4 * sc) break;
            if (tk - th > 1e-10 * sc) add_ritz_vector(lz, p, m, tk, L, D, x, ritz);
        }
    }
}

// ------------------------------------------------------ compacted sub-batch
// The unconverged problems of a phase continue their Lanczos recurrences in a
// packed layout: virtual sector v holds up to nsp_c problems of base sector
// vs_base[v], slot q being base set vs_set[v * nsp_c + q] (slots past the
// real ones repeat the last real problem and start converged).

// dst[v][r][q] = src[vs_base[v]][r][vs_set[v][q]], one block per tile of 32 rows.
template <class V>
__global__ void k_bgather_vec(BatchArgs ac, const int* __restrict__ slot_src, const int64_t* __restrict__ sec_elem_s,
                              int nsp_s, const V* __restrict__ src, V* __restrict__ dst) {
    const int tile = blockIdx.x;
    const int v = ac.tile_sector[tile];
    const int nsp_c = ac.nsp;
    const int q = threadIdx.x % nsp_c;
    const int sp = slot_src[v * nsp_c + q];  // source problem: source sector * nsp_s + set
    const int64_t eb = sec_elem_s[sp / nsp_s] + sp % nsp_s, ec = ac.sec_elem[v];
    const int64_t r_end = min(ac.sec_nrows[v], (int64_t)ac.tile_row0[tile] + kBTile);
    for (int64_t r = ac.tile_row0[tile] + threadIdx.x / nsp_c; r < r_end; r += blockDim.x / nsp_c)
        dst[ec + r * nsp_c + q] = src[eb + r * nsp_s];
}

// alpha_i (i < j), beta_i (i <= j) and the convergence-test state of the
// migrated problems; slot_src maps a slot to its source problem.
__global__ void k_bgather_state(int n_prob_c, int n_prob_s, int j, const int* __restrict__ slot_src,
                                const int* __restrict__ real_c, const double* __restrict__ alpha_s,
                                const double* __restrict__ beta_s, const double* __restrict__ thp_s,
                                const int* __restrict__ ms_s, const double* __restrict__ gap_s,
                                double* __restrict__ alpha_c, double* __restrict__ beta_c,
                                double* __restrict__ thp_c, int* __restrict__ ms_c, double* __restrict__ gap_c,
                                int* __restrict__ conv_c) {
    for (int pc = blockIdx.x * blockDim.x + threadIdx.x; pc < n_prob_c; pc += gridDim.x * blockDim.x) {
        const int p = slot_src[pc];
        for (int i = 0; i < j; ++i) alpha_c[(int64_t)i * n_prob_c + pc] = alpha_s[(int64_t)i * n_prob_s + p];
        for (int i = 0; i <= j; ++i) beta_c[(int64_t)i * n_prob_c + pc] = beta_s[(int64_t)i * n_prob_s + p];
        thp_c[pc] = thp_s[p];
        ms_c[pc] = ms_s[p];
        if (gap_s) gap_c[pc] = gap_s[p];
        conv_c[pc] = real_c[pc] ? 0 : 1;
    }
}

// Results of the real slots back into the source problem arrays.
__global__ void k_bscatter_state(int n_prob_c, const int* __restrict__ slot_src, const int* __restrict__ real_c,
                                 const double* __restrict__ th_c, const int* __restrict__ ms_c,
                                 const int* __restrict__ conv_c, double* __restrict__ th_s,
                                 int* __restrict__ ms_s, int* __restrict__ conv_s) {
    for (int pc = blockIdx.x * blockDim.x + threadIdx.x; pc < n_prob_c; pc += gridDim.x * blockDim.x) {
        if (!real_c[pc]) continue;
        const int p = slot_src[pc];
        th_s[p] = th_c[pc];
        ms_s[p] = ms_c[pc];
        conv_s[p] = conv_c[pc];
    }
}

// psi = sum_{i < m_p} ritz[i][p] v_i over the stored basis (FP64 result).
template <class V>
__global__ void k_bpsi(BatchArgs a, int64_t tot, const V* __restrict__ vring, int maxm,
                       const int* __restrict__ msteps, const double* __restrict__ ritz, int n_prob,
                       void* psi) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot;
         e += (int64_t)gridDim.x * blockDim.x) {
        int s = 0;
        while (a.sec_elem[s + 1] <= e) ++s;
        int set = (int)((e - a.sec_elem[s]) % a.nsp);
        int p = s * a.nsp + set;
        int m = min(msteps[p], maxm);
        double2 acc = make_double2(0.0, 0.0);
        for (int i = 0; i < m; ++i) {
            double c = ritz[(int64_t)i * n_prob + p];
            double2 v = Sc<V>::to2(vring[(int64_t)i * tot + e]);
            acc.x += c * v.x;
            acc.y += c * v.y;
        }
        if constexpr (Sc<V>::cplx) reinterpret_cast<double2*>(psi)[e] = acc;
        else reinterpret_cast<double*>(psi)[e] = acc.x;
    }
}

// ------------------------------------------------- batch assembly (device)
// A SELL slice holds 32 rows; padding entries repeat the row index with a
// zero value and are dropped (a zero entry contributes nothing).
__device__ __forceinline__ bool sell_pad(uint32_t c, int64_t r, double v) { return c == (uint32_t)r && v == 0.0; }
__device__ __forceinline__ bool sell_pad(uint32_t c, int64_t r, double2 v) {
    return c == (uint32_t)r && v.x == 0.0 && v.y == 0.0;
}
__device__ __forceinline__ double2 widen2(double v) { return make_double2(v, 0.0); }
__device__ __forceinline__ double2 widen2(double2 v) { return v; }

// cnt[r] = entries of row r that are not padding (r < n); cnt[n] = 0.
template <class VI>
__global__ void k_sell_row_count(int64_t n, const int64_t* __restrict__ off, const int* __restrict__ w,
                                 const uint32_t* __restrict__ col, const VI* __restrict__ val,
                                 int64_t* __restrict__ cnt) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= n; r += (int64_t)gridDim.x * blockDim.x) {
        if (r == n) { cnt[n] = 0; continue; }
        const int64_t sl = r >> 5, lane = r & 31;
        int64_t c = 0;
        for (int jj = 0; jj < w[sl]; ++jj) {
            const int64_t pos = off[sl] + (int64_t)jj * 32 + lane;
            c += sell_pad(col[pos], r, val[pos]) ? 0 : 1;
        }
        cnt[r] = c;
    }
}

// Row r's entries at rp[r].. in slice order (the order of the single-sector table).
template <class VI>
__global__ void k_sell_to_csr(int64_t n, const int64_t* __restrict__ off, const int* __restrict__ w,
                              const uint32_t* __restrict__ col, const VI* __restrict__ val,
                              const int64_t* __restrict__ rp, uint32_t* __restrict__ ocol,
                              double2* __restrict__ oval) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sl = r >> 5, lane = r & 31;
        int64_t o = rp[r];
        for (int jj = 0; jj < w[sl]; ++jj) {
            const int64_t pos = off[sl] + (int64_t)jj * 32 + lane;
            const uint32_t c = col[pos];
            const VI v = val[pos];
            if (sell_pad(c, r, v)) continue;
            ocol[o] = c;
            oval[o] = widen2(v);
            ++o;
        }
    }
}

template <class VI>
__global__ void k_widen(int64_t n, const VI* __restrict__ in, double2* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = widen2(in[i]);
}

__device__ __forceinline__ void narrow(double2 v, double& d, float& f) { d = v.x; f = (float)v.x; }
__device__ __forceinline__ void narrow(double2 v, double2& d, float2& f) {
    d = v;
    f = make_float2((float)v.x, (float)v.y);
}

// One sector's CSR part and diagonals placed into its kind's arrays: row
// pointers offset by the sector's first entry, values in FP64 and FP32.
struct PlaceArgs {
    int64_t n, nnz, ent0;
    const int64_t* rp;
    const uint32_t* col;
    const double2 *val, *dxy, *dz;
    int64_t* row_ptr;   // at the sector's row base
    uint32_t* ocol;     // at the sector's first entry
};
template <class V64, class V32>
__global__ void k_place_sector(PlaceArgs a, V64* __restrict__ val64, V32* __restrict__ val32,
                               V64* __restrict__ dxy64, V32* __restrict__ dxy32, V64* __restrict__ dz64,
                               V32* __restrict__ dz32) {
    const int64_t m = a.n + 1 > a.nnz ? a.n + 1 : a.nnz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (i <= a.n) a.row_ptr[i] = a.ent0 + a.rp[i];
        if (i < a.nnz) {
            a.ocol[i] = a.col[i];
            narrow(a.val[i], val64[i], val32[i]);
        }
        if (i < a.n) {
            narrow(a.dxy[i], dxy64[i], dxy32[i]);
            narrow(a.dz[i], dz64[i], dz32[i]);
        }
    }
}

}  // namespace qmb

using namespace qmb;

// One kind (real or complex) of sectors.
struct BKind {
    int n_sectors = 0;
    std::vector<int> sec_index;        // positions in the caller's sector list
    std::vector<int64_t> nrows;        // per sector
    std::vector<int64_t> sec_elem;     // [n+1]
    std::vector<int> tile_sector, tile_row0, sec_tile0, sec_ntiles;
    DevBuf<int> d_tile_sector, d_tile_row0, d_sec_tile0, d_sec_ntiles, d_tiles, d_active;
    DevBuf<unsigned> d_ctr;      // work queue head + retired blocks
    DevBuf<unsigned> d_sec_ctr;  // per-sector finished tiles
    int variant[2] = {-1, -1};    // tuned k_bhv variant per precision (FP32, FP64)
    int ring_hint = 0;            // Krylov ring slots the phases on this handle needed
    DevBuf<unsigned char> ws_ring, ws_w;  // Lanczos workspace kept between solves
    std::unique_ptr<BKind> compact;        // descriptor of the last compacted sub-batch
    float tune_ms[2][8] = {};  // tuner timings per precision and variant
    DevBuf<int64_t> d_sec_elem, d_nrows, d_row_ptr, d_row_base, d_row0;
    std::vector<int64_t> h_row_base, h_row0;  // per sector, as on the device
    DevBuf<uint32_t> d_col;
    DevBuf<unsigned char> val64, val32, dxy64, dxy32, dz64, dz32;
    int64_t nnz = 0, rows = 0;
    int n_tiles = 0;
    int max_tile_entries = 1;
};

struct qmb_batch_s {
    int device = 0;
    int n_sectors = 0, n_sets = 0, nsp = 0, spl = 8, n_groups = 1;
    BKind kind[2];  // 0 real, 1 complex
    qmb::WsPool ws;  // temporaries of the solves, reused from one solve to the next
    std::vector<int> sector_kind, sector_pos;
    DevBuf<double> cxy, cz;
};

namespace qmb {

static BatchArgs make_args(const qmb_batch_s* b, const BKind& k) {
    BatchArgs a;
    a.n_sectors = k.n_sectors;
    a.nsp = b->nsp;
    a.n_groups = b->n_groups;
    a.tile_sector = k.d_tile_sector.p;
    a.tile_row0 = k.d_tile_row0.p;
    a.sec_elem = k.d_sec_elem.p;
    a.sec_nrows = k.d_nrows.p;
    a.row_ptr = k.d_row_ptr.p;
    a.row_base = k.d_row_base.p;
    a.row0 = k.d_row0.p;
    a.col = k.d_col.p;
    a.val = nullptr;
    a.dxy = nullptr;
    a.dz = nullptr;
    a.cxy = b->cxy.p;
    a.cz = b->cz.p;
    a.active = k.d_active.p;
    a.max_tile_entries = k.max_tile_entries;
    a.c_stride = 0;
    return a;
}

// Kernel variants the tuner chooses from: gathers in flight per thread
// (UNR), the register budget (MINB resident blocks per SM), whether a row's
// own x[r] and v_{j-1}[r] loads are hoisted ahead of its gathers, and the
// slices per thread: one 16-byte slice of each gathered row (variants 0-2),
// two (3-5) or four (6-7).  Wider slices mean fewer threads per row, so more
// rows of a tile are in flight per block, and an entry's index and value
// reads and address arithmetic serve more sets.
constexpr int kBVariants = 8;
constexpr int kBSlices[kBVariants] = {1, 1, 1, 2, 2, 2, 4, 4};

template <class V, int SPL, int UNR, int MINB, bool HOIST>
static void launch_bhv_v(const BatchArgs& a, BKind& k, const V* x, V* y, V* vring, int K, BLz lz,
                         const double* ritz, void* psi, int lanczos, cudaStream_t st) {
    auto kern = k_bhv<V, SPL, UNR, MINB, HOIST>;
    const size_t smem = (size_t)a.max_tile_entries * (sizeof(V) + sizeof(uint32_t));
    static int grid[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    int& g = grid[dev & 63];
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (g == 0) {
        int per_sm = 0, sms = 148;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBThreads, smem);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g = std::max(1, per_sm) * sms;
    }
    g_kernels += 1;
    kern<<<std::min(g, k.n_tiles), kBThreads, smem, st>>>(a, k.n_tiles, k.d_ctr.p, x, y, vring, K, lz, ritz,
                                                          psi, lanczos);
}

// Whether variant v can run this batch: a row needs at least 32 threads.
template <class V>
static bool bhv_variant_ok(int v, int nsp, int spl) {
    const int w = kBSlices[v] * spl;
    return w * (int)sizeof(V) <= 64 && nsp / w >= 32;
}

template <class V, int SPL>
static void launch_bhv(int variant, const BatchArgs& a, BKind& k, const V* x, V* y, V* vring, int K,
                       BLz lz, const double* ritz, void* psi, int lanczos, cudaStream_t st) {
    if (k.n_tiles == 0) return;
    QMB_REQUIRE(variant >= 0 && variant < kBVariants && bhv_variant_ok<V>(variant, a.nsp, SPL),
                QMB_ERR_UNSUPPORTED, "k_bhv variant does not fit this batch's set count");
    switch (variant) {
        case 0: launch_bhv_v<V, SPL, 4, 4, false>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st); break;
        case 1: launch_bhv_v<V, SPL, 4, 4, true>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st); break;
        case 2: launch_bhv_v<V, SPL, 8, 2, false>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st); break;
        default:
            if constexpr (2 * SPL * sizeof(V) <= 64) {
                if (variant == 3) launch_bhv_v<V, 2 * SPL, 4, 2, true>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
                else if (variant == 4) launch_bhv_v<V, 2 * SPL, 2, 3, true>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
                else if (variant == 5) launch_bhv_v<V, 2 * SPL, 2, 4, true>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
                else if constexpr (4 * SPL * sizeof(V) <= 64) {
                    if (variant == 6) launch_bhv_v<V, 4 * SPL, 2, 2, true>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
                    else launch_bhv_v<V, 4 * SPL, 1, 2, true>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
                }
            }
            break;
    }
}

// sets per thread: one 16-byte access, at most nsp/32
template <class V>
static int spl_for(int nsp) {
    int spl = (int)(16 / sizeof(V));
    while (spl > 1 && nsp / spl < 32) spl /= 2;
    return spl;
}

template <class V>
static void bhv_variant(int variant, const BatchArgs& a, BKind& k, const V* x, V* y, V* vring, int K,
                        BLz lz, const double* ritz, void* psi, int lanczos, cudaStream_t st) {
    const int spl = spl_for<V>(a.nsp);
    if constexpr (sizeof(V) <= 4)
        if (spl == 4) return launch_bhv<V, 4>(variant, a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
    if constexpr (sizeof(V) <= 8)
        if (spl == 2) return launch_bhv<V, 2>(variant, a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
    launch_bhv<V, 1>(variant, a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
}

// Autotuner: times every variant on this batch's own matrices (plain H*v on
// scratch vectors, best of 3) and keeps the fastest for the precision.
// Tuner choices by batch shape (device, scalar size, padded sets, sectors,
// tiles, largest tile, rows, entries), shared by the handles of a process.
struct TuneKey {
    int dev, vsize, nsp, n_sectors, n_tiles, max_tile;
    int64_t rows, nnz;
    bool operator<(const TuneKey& o) const {
        return std::tie(dev, vsize, nsp, n_sectors, n_tiles, max_tile, rows, nnz) <
               std::tie(o.dev, o.vsize, o.nsp, o.n_sectors, o.n_tiles, o.max_tile, o.rows, o.nnz);
    }
};
struct TuneEntry {
    int variant = 0;
    float ms[kBVariants] = {};
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneEntry> g_tune_cache;

template <class V>
static void bupdate_any(const BatchArgs& a, const BKind& k, V* w, const V* vring, int K, BLz lz, cudaStream_t st);
template <class V>
static void bnorm0_any(const BatchArgs& a, const BKind& k, const V* w, BLz lz, cudaStream_t st);

// The variants are timed in the form the solve runs, K1 of a Lanczos step
// (the product with the epilogue that reads v_{j-1}, writes v_j and y and
// sums alpha), at step 1 of a seeded start on scratch vectors; the plain
// product (qmb_batch_hv) uses the same choice.
template <class V>
static int tuned_variant(const BatchArgs& a, BKind& k, bool f64, cudaStream_t st) {
    int& v = k.variant[f64 ? 1 : 0];
    if (v >= 0) return v;
    // QMB_BHV_VARIANT=0..7 fixes the variant.  The variants may round the
    // epilogue's products and sums differently (the compiler fuses them per
    // instantiation), so fixing it makes results reproducible across machines.
    if (const char* fe = std::getenv("QMB_BHV_VARIANT")) {
        const int fv = std::atoi(fe);
        if (fe[0] >= '0' && fe[0] <= '9' && fv >= 0 && fv < kBVariants &&
            bhv_variant_ok<V>(fv, a.nsp, spl_for<V>(a.nsp))) {
            v = fv;
            return v;
        }
    }
    // a batch of the same shape tuned before in this process reuses the choice
    int dev = 0;
    QMB_CUDA_TRY(cudaGetDevice(&dev));
    const TuneKey key{dev, (int)sizeof(V), a.nsp, k.n_sectors, k.n_tiles, k.max_tile_entries, k.rows, k.nnz};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            for (int c = 0; c < kBVariants; ++c) k.tune_ms[f64 ? 1 : 0][c] = it->second.ms[c];
            v = it->second.variant;
            return v;
        }
    }
    const int64_t tot = k.sec_elem[k.n_sectors];
    const int n_prob = k.n_sectors * a.nsp;
    DevBuf<V> w(2 * (size_t)tot), ring(2 * (size_t)tot);
    DevBuf<double> alpha(4 * (size_t)n_prob), beta(5 * (size_t)n_prob),
        partials((size_t)std::max(1, k.n_tiles) * a.nsp);
    DevBuf<int> iter(1), act(k.n_sectors);
    iter.zero(st);
    std::vector<int> ones(k.n_sectors, 1);
    act.upload(ones.data(), k.n_sectors, st);
    BatchArgs at = a;
    at.active = act.p;  // every sector, whatever the caller's phase has active
    BLz lz{alpha.p, beta.p, partials.p, iter.p, n_prob, k.d_sec_ctr.p, k.d_sec_tile0.p, k.d_sec_ntiles.p};
    k_bstart<V><<<grid_for(tot, 256), 256, 0, st>>>(at, tot, 0, 2212456ull, nullptr, w.p);
    bnorm0_any<V>(at, k, w.p, lz, st);
    k_bbeta0<<<(n_prob + 255) / 256, 256, 0, st>>>(at, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz);
    // one step, so that the timed launches run at step 1 (v_0 read, v_1 written)
    bhv_variant<V>(0, at, k, w.p, w.p, ring.p, 2, lz, nullptr, nullptr, 1, st);
    bupdate_any<V>(at, k, w.p, ring.p, 2, lz, st);
    k_badvance<<<1, 32, 0, st>>>(lz);
    cudaEvent_t e0, e1;
    QMB_CUDA_TRY(cudaEventCreate(&e0));
    QMB_CUDA_TRY(cudaEventCreate(&e1));
    // variants timed round-robin (five rounds, minimum per variant), so that
    // clock ramp-up or a one-off delay does not decide the choice
    // variants that cannot run this batch are skipped
    bool fits[kBVariants];
    float tmin[kBVariants];
    for (int c = 0; c < kBVariants; ++c) {
        tmin[c] = 1e30f;
        fits[c] = bhv_variant_ok<V>(c, a.nsp, spl_for<V>(a.nsp));
        if (fits[c]) bhv_variant<V>(c, at, k, w.p, w.p, ring.p, 2, lz, nullptr, nullptr, 1, st);  // warm
    }
    for (int r = 0; r < 5; ++r)
        for (int c = 0; c < kBVariants; ++c) {
            if (!fits[c]) continue;
            cudaEventRecord(e0, st);
            bhv_variant<V>(c, at, k, w.p, w.p, ring.p, 2, lz, nullptr, nullptr, 1, st);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            tmin[c] = std::min(tmin[c], ms);
        }
    float best = 1e30f;
    int arg = 0;
    for (int c = 0; c < kBVariants; ++c) {
        k.tune_ms[f64 ? 1 : 0][c] = tmin[c];
        if (tmin[c] < best) {
            best = tmin[c];
            arg = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_launch("k_bhv tuning");
    v = arg;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        if (g_tune_cache.size() >= 512) g_tune_cache.clear();
        TuneEntry& e = g_tune_cache[key];
        e.variant = arg;
        for (int c = 0; c < kBVariants; ++c) e.ms[c] = tmin[c];
    }
    return v;
}

template <class V>
static void bhv_any(const BatchArgs& a, BKind& k, const V* x, V* y, V* vring, int K, BLz lz,
                    const double* ritz, void* psi, int lanczos, cudaStream_t st) {
    const bool f64 = std::is_same<typename Sc<V>::real, double>::value;
    const int v = k.variant[f64 ? 1 : 0] >= 0 ? k.variant[f64 ? 1 : 0] : 0;
    bhv_variant<V>(v, a, k, x, y, vring, K, lz, ritz, psi, lanczos, st);
}

template <class V>
static void bupdate_any(const BatchArgs& a, const BKind& k, V* w, const V* vring, int K, BLz lz,
                        cudaStream_t st) {
    if (k.n_tiles == 0) return;
    g_kernels += 1;
    k_bupdate<V><<<k.n_tiles, a.nsp, 0, st>>>(a, k.n_tiles, w, vring, K, lz);
}

template <class V>
static void bnorm0_any(const BatchArgs& a, const BKind& k, const V* w, BLz lz, cudaStream_t st) {
    if (k.n_tiles == 0) return;
    g_kernels += 1;
    k_bnorm0<V><<<k.n_tiles, a.nsp, 0, st>>>(a, k.n_tiles, w, lz);
}

constexpr int kRingStart = 128;  // first Krylov ring size of a handle, in vectors
// real sectors with fewer rows than this fraction of the complex ones are
// solved in the complex kind
constexpr double kMergeRealFrac = 0.25;

// QMB_RING_START=n (n >= 3) sets the first ring size instead (memory-tight runs).
static int ring_start() {
    const char* e = std::getenv("QMB_RING_START");
    const int v = e ? std::atoi(e) : 0;
    return v >= 3 ? v : kRingStart;
}

// Krylov vectors of vec_bytes each that fit in about half of the free
// device memory (at most want); 0 when fewer than 16 fit.
static int krylov_slots(size_t vec_bytes, int want, size_t cached = 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 0;
    fr += cached;
    size_t n = (size_t)(0.5 * (double)fr) / std::max<size_t>(vec_bytes, 1);
    if (n < 16) return 0;
    return (int)std::min<size_t>(n, (size_t)want);
}

// QMB_TRACE=1 prints per-phase steps and times of batched solves to stderr.
// Compaction threshold: the unconverged problems move to a packed layout
// once it costs at most this fraction of the current one (QMB_COMPACT_RATIO).
static double compact_ratio() {
    const char* e = std::getenv("QMB_COMPACT_RATIO");
    const double v = e ? std::atof(e) : 0.4;
    return v > 0.0 && v < 1.0 ? v : 0.4;
}

// The threshold inside a compacted sub-batch (QMB_SUB_COMPACT_RATIO, off by
// default): its virtual sectors over one base sector merge into fewer.  On
// the L=20 batch (34 virtual sectors over 20 base sectors after the first
// compaction) further levels (34 -> 24 -> 19 sectors at thresholds up to
// 0.85) cost as much in host round trips and gathers as their smaller tail
// saved: 110-116 ms against 110 ms per mixed solve.
static double sub_compact_ratio() {
    const char* e = std::getenv("QMB_SUB_COMPACT_RATIO");
    const double v = e ? std::atof(e) : 0.0;
    return v > 0.0 && v < 1.0 ? v : 0.0;
}

// QMB_HOST_LOOP=1: device loops launched block by block from the host
static bool host_loop() {
    const char* e = std::getenv("QMB_HOST_LOOP");
    return e && e[0] == '1';
}

static bool trace_on() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("QMB_TRACE");
        v = (e && *e && *e != '0') ? 1 : 0;
    }
    return v == 1;
}

struct BPhase {
    std::vector<double> theta;   // [n_prob]
    std::vector<int> msteps, conv;
    int steps = 0;
    double products = 0;  // sector H*v products computed (active sectors x sets x steps)
};

// Convergence test of every problem after m steps: one warp per problem,
// shared memory for the staged tridiagonals.
static void launch_check(const BatchArgs& a, const BLz& lz, int nsets, double stall, double res_tol,
                         double e_tol, const double* gap_in, double* gap_out, double* theta,
                         double* theta_prev, int* msteps, int* conv, int* active_next, int m,
                         cudaStream_t st, int* open_cnt = nullptr) {
    const size_t per_warp = sizeof(double) * kCheckArrays * (size_t)(m + 2);
    const int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (96u << 10) / per_warp));
    const size_t smem = per_warp * wpb;
    if (smem > (48u << 10))
        cudaFuncSetAttribute(k_bcheck, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int nblk = (lz.n_prob + wpb - 1) / wpb;
    g_kernels += 1;
    k_bcheck<<<nblk, 32 * wpb, smem, st>>>(a, lz, nsets, stall, res_tol, e_tol, gap_in, gap_out, theta,
                                           theta_prev, msteps, conv, active_next, open_cnt);
}

// Runs blocks of `check` Lanczos steps followed by the convergence test as a
// device-side loop (a CUDA graph with a conditional WHILE node), from step j0
// until k_bloop_ctl stops it: no host round trip per block.  `step` enqueues
// one Lanczos step on a stream.  active holds the sectors stepped in the
// first block.  Returns the step count reached, the stop reason and the
// problems stepped.
struct LoopOut {
    int done;
    int reason;
    double products;
};
template <class StepFn>
static LoopOut device_loop(StepFn&& step, const BatchArgs& a, const BLz& lz, int nsets, double stall,
                           double res_tol, double e_tol, const double* gap_in, double* gap_out, double* theta,
                           double* theta_prev, int* msteps, int* conv, int* active, int* active_next,
                           const int64_t* d_nrows, const int* d_weight, int n_sectors, int check, int j0,
                           int cap, double compact_ratio, cudaStream_t st, const int* d_group = nullptr,
                           int n_groups = 0) {
    LoopOut out{j0, 2, 0.0};
    if (j0 + check > cap) return out;
    Buf<LoopCtl> ctl = ws_take<LoopCtl>(1);
    Buf<int> open_cnt = ws_take<int>(n_sectors);
    ctl.zero(st);
    open_cnt.zero(st);
    QMB_CUDA_TRY(cudaMemsetAsync(active_next, 0, sizeof(int) * n_sectors, st));
    const int max_loops = (cap - j0) / check + 1;
    if (host_loop()) {
        // the same blocks launched from the host, with the loop control read
        // back after each (QMB_HOST_LOOP=1: every kernel visible to a profiler)
        LoopCtl hc{};
        for (;;) {
            for (int t = 0; t < check; ++t) step(st);
            launch_check(a, lz, nsets, stall, res_tol, e_tol, gap_in, gap_out, theta, theta_prev, msteps, conv,
                         active_next, cap, st, open_cnt.p);
            g_kernels += 1;
            k_bloop_ctl<<<1, 256, 0, st>>>(cudaGraphConditionalHandle{}, 0, n_sectors, active, active_next,
                                           open_cnt.p, d_nrows, d_weight, a.nsp, check, cap, lz.iter, max_loops,
                                           compact_ratio, d_group, n_groups, ctl.p);
            check_launch("host loop block");
            QMB_CUDA_TRY(cudaMemcpyAsync(&hc, ctl.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
            QMB_CUDA_TRY(cudaStreamSynchronize(st));
            if (hc.reason != 0) break;
        }
        int it = 0;
        QMB_CUDA_TRY(cudaMemcpyAsync(&it, lz.iter, sizeof(int), cudaMemcpyDeviceToHost, st));
        QMB_CUDA_TRY(cudaStreamSynchronize(st));
        out.done = it;
        out.reason = hc.reason;
        out.products = hc.products;
        return out;
    }
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    struct GG {
        cudaGraph_t& g;
        cudaGraphExec_t& e;
        ~GG() {
            if (e) cudaGraphExecDestroy(e);
            if (g) cudaGraphDestroy(g);
        }
    } gg{g, ex};
    QMB_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    QMB_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    // zero-initialised parameter block (the struct has no default constructor)
    alignas(cudaGraphNodeParams) unsigned char np_raw[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(np_raw);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    QMB_CUDA_TRY(cudaGraphAddNode(&node, g, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    QMB_CUDA_TRY(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const double kernels_before = g_kernels;  // capture records kernels; they run once per loop
    for (int t = 0; t < check; ++t) step(st);
    launch_check(a, lz, nsets, stall, res_tol, e_tol, gap_in, gap_out, theta, theta_prev, msteps, conv,
                 active_next, cap, st, open_cnt.p);
    g_kernels += 1;
    k_bloop_ctl<<<1, 256, 0, st>>>(h, 1, n_sectors, active, active_next, open_cnt.p, d_nrows, d_weight, a.nsp,
                                   check, cap, lz.iter, max_loops, compact_ratio, d_group, n_groups, ctl.p);
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &captured);
    QMB_CUDA_TRY(ce);
    const double body_kernels = g_kernels - kernels_before;
    g_kernels = kernels_before;
    QMB_CUDA_TRY(cudaGraphInstantiate(&ex, g, 0));
    QMB_CUDA_TRY(cudaGraphLaunch(ex, st));
    LoopCtl hc;
    int it = 0;
    QMB_CUDA_TRY(cudaMemcpyAsync(&hc, ctl.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
    QMB_CUDA_TRY(cudaMemcpyAsync(&it, lz.iter, sizeof(int), cudaMemcpyDeviceToHost, st));
    QMB_CUDA_TRY(cudaStreamSynchronize(st));
    out.done = it;
    out.reason = hc.reason;
    out.products = hc.products;
    g_kernels += body_kernels * hc.loops;
    return out;
}

// A layout the compaction reads the unconverged problems from: the base kind
// (nsp sets a sector) or an earlier compacted sub-batch (32 slots a virtual
// sector).  Source sector s lies over base sector base_of[s]; its vectors
// start at d_sec_elem[s]; problem p = s * nsp + set.
struct CSrc {
    int n_sectors = 0, nsp = 0;
    std::vector<int> base_of;        // [n_sectors]
    const int64_t* d_sec_elem = nullptr;
    std::vector<double> cx, cz;      // couplings per source problem
    std::vector<int> real;           // 1 for a real problem (not padding)
    const double* alpha = nullptr;   // [j][n_prob] as in BLz
    const double* beta = nullptr;
    double* theta = nullptr;
    double* theta_prev = nullptr;
    const double* gap = nullptr;     // phase-1 gap per problem, or null
    int* msteps = nullptr;
    int* conv = nullptr;
    int n_prob() const { return n_sectors * nsp; }
};

// Continues the Lanczos recurrences of the unconverged problems of a phase
// (K = 2 ring, no Ritz vector wanted) in a compacted sub-batch of 32 slots
// per virtual sector, from step j up to step cap.  src describes the layout
// they come from (w_j and v_{j-1} at w_src and v_src) and conv_h its
// convergence flags after step j.  When the unconverged problems of the
// sub-batch again fill few enough slots, they move on into a smaller one (up
// to kCompactDepth levels).  Results (theta, steps, flags) go back into the
// source arrays; returns the step count reached.
constexpr int kCompactDepth = 3;
template <class V>
static int run_compacted(qmb_batch_s* b, BKind& k, std::unique_ptr<BKind>& holder, bool f64, const BatchArgs& a_base,
                         const CSrc& src, const V* w_src, const V* v_src, int j, int cap, double stall,
                         double res_tol, double e_tol, int check, const std::vector<int>& conv_h, int depth,
                         double& products, int& n_hv, cudaStream_t st) {
    constexpr int NC = 32;
    // virtual sectors: the open problems of each base sector, 32 a sector
    std::vector<std::vector<int>> open_of(k.n_sectors);
    for (int p = 0; p < src.n_prob(); ++p)
        if (src.real[p] && !conv_h[p]) open_of[src.base_of[p / src.nsp]].push_back(p);
    std::vector<int> vs_base, slot_src, real;
    std::vector<int> n_real;
    for (int s = 0; s < k.n_sectors; ++s) {
        const std::vector<int>& open = open_of[s];
        for (size_t c = 0; c < open.size(); c += NC) {
            vs_base.push_back(s);
            const int nr = (int)std::min<size_t>(NC, open.size() - c);
            n_real.push_back(nr);
            for (int q = 0; q < NC; ++q) {
                slot_src.push_back(open[c + std::min(q, nr - 1)]);
                real.push_back(q < nr ? 1 : 0);
            }
        }
    }
    const int nv = (int)vs_base.size();
    if (nv == 0) return j;
    // the compacted layout's descriptor is kept on the kind and refilled
    if (!holder) holder = std::make_unique<BKind>();
    BKind& ck = *holder;
    ck.nrows.clear();
    ck.sec_tile0.clear();
    ck.sec_ntiles.clear();
    ck.tile_sector.clear();
    ck.tile_row0.clear();
    ck.n_sectors = nv;
    // the compacted layout has NC slots a row: a multi-slice variant that
    // needs more sets a row gives way to the fastest one-slice variant
    for (int f = 0; f < 2; ++f) {
        int v = k.variant[f];
        if (v >= 0 && kBSlices[v] > 1) {
            int best = 0;
            for (int c = 1; c < kBVariants; ++c)
                if (kBSlices[c] == 1 && k.tune_ms[f][c] > 0.f &&
                    (k.tune_ms[f][best] <= 0.f || k.tune_ms[f][c] < k.tune_ms[f][best]))
                    best = c;
            v = best;
        }
        ck.variant[f] = v;
        for (int c = 0; c < kBVariants; ++c) ck.tune_ms[f][c] = k.tune_ms[f][c];
    }
    ck.max_tile_entries = k.max_tile_entries;
    std::vector<int64_t> rb(nv), r0(nv);
    ck.sec_elem.assign(1, 0);
    for (int v = 0; v < nv; ++v) {
        const int s = vs_base[v];
        ck.nrows.push_back(k.nrows[s]);
        ck.sec_elem.push_back(ck.sec_elem.back() + k.nrows[s] * NC);
        rb[v] = k.h_row_base[s];
        r0[v] = k.h_row0[s];
        ck.sec_tile0.push_back((int)ck.tile_sector.size());
        ck.sec_ntiles.push_back(k.sec_ntiles[s]);
        for (int t = 0; t < k.sec_ntiles[s]; ++t) {
            ck.tile_sector.push_back(v);
            ck.tile_row0.push_back(t * kBTile);
        }
    }
    ck.n_tiles = (int)ck.tile_sector.size();
    const int64_t tot_c = ck.sec_elem[nv];
    const int n_prob_c = nv * NC;
    auto up_i = [&](DevBuf<int>& d, const std::vector<int>& h) {
        if (d.n < h.size()) d.alloc(h.size());
        d.upload(h.data(), h.size(), st);
    };
    auto up_l = [&](DevBuf<int64_t>& d, const std::vector<int64_t>& h) {
        if (d.n < h.size()) d.alloc(h.size());
        d.upload(h.data(), h.size(), st);
    };
    up_i(ck.d_tile_sector, ck.tile_sector);
    up_i(ck.d_tile_row0, ck.tile_row0);
    up_i(ck.d_sec_tile0, ck.sec_tile0);
    up_i(ck.d_sec_ntiles, ck.sec_ntiles);
    up_l(ck.d_sec_elem, ck.sec_elem);
    up_l(ck.d_nrows, ck.nrows);
    up_l(ck.d_row_base, rb);
    up_l(ck.d_row0, r0);
    std::vector<int> ones(nv, 1);
    up_i(ck.d_active, ones);
    if (ck.d_ctr.n < 2) ck.d_ctr.alloc(2);
    ck.d_ctr.zero(st);
    if (ck.d_sec_ctr.n < (size_t)nv) ck.d_sec_ctr.alloc(nv);
    ck.d_sec_ctr.zero(st);
    Buf<int> d_slot_src = ws_take<int>(slot_src.size()), d_real = ws_take<int>(real.size());
    d_slot_src.upload(slot_src.data(), slot_src.size(), st);
    d_real.upload(real.data(), real.size(), st);
    // couplings of each slot
    std::vector<double> cx(n_prob_c), cz(n_prob_c);
    for (int pc = 0; pc < n_prob_c; ++pc) {
        cx[pc] = src.cx[slot_src[pc]];
        cz[pc] = src.cz[slot_src[pc]];
    }
    Buf<double> d_cx = ws_take<double>(n_prob_c), d_cz = ws_take<double>(n_prob_c);
    d_cx.upload(cx.data(), n_prob_c, st);
    d_cz.upload(cz.data(), n_prob_c, st);
    BatchArgs ac = a_base;  // matrix arrays of the base kind
    ac.n_sectors = nv;
    ac.nsp = NC;
    ac.tile_sector = ck.d_tile_sector.p;
    ac.tile_row0 = ck.d_tile_row0.p;
    ac.sec_elem = ck.d_sec_elem.p;
    ac.sec_nrows = ck.d_nrows.p;
    ac.row_base = ck.d_row_base.p;
    ac.row0 = ck.d_row0.p;
    ac.cxy = d_cx.p;
    ac.cz = d_cz.p;
    ac.c_stride = NC;
    ac.active = ck.d_active.p;
    // recurrence state: w_j, v_{j-1}, alpha/beta history, test state
    Buf<V> wc = ws_take<V>(2 * (size_t)tot_c), vc = ws_take<V>(2 * (size_t)tot_c);
    g_kernels += 1;
    k_bgather_vec<V><<<ck.n_tiles, 256, 0, st>>>(ac, d_slot_src.p, src.d_sec_elem, src.nsp, w_src,
                                                 wc.p + (int64_t)(j & 1) * tot_c);
    g_kernels += 1;
    k_bgather_vec<V><<<ck.n_tiles, 256, 0, st>>>(ac, d_slot_src.p, src.d_sec_elem, src.nsp, v_src,
                                                 vc.p + (int64_t)((j + 1) & 1) * tot_c);
    Buf<double> alpha = ws_take<double>((size_t)(cap + 1) * n_prob_c),
        beta = ws_take<double>((size_t)(cap + 2) * n_prob_c),
        partials = ws_take<double>((size_t)ck.n_tiles * NC),
        theta = ws_take<double>(n_prob_c),
        theta_prev = ws_take<double>(n_prob_c),
        gap = ws_take<double>(n_prob_c);
    Buf<int> iter = ws_take<int>(1),
        msteps = ws_take<int>(n_prob_c),
        conv = ws_take<int>(n_prob_c),
        active_next = ws_take<int>(nv);
    g_kernels += 1;
    k_bgather_state<<<(n_prob_c + 255) / 256, 256, 0, st>>>(
        n_prob_c, src.n_prob(), j, d_slot_src.p, d_real.p, src.alpha, src.beta, src.theta_prev, src.msteps,
        src.gap, alpha.p, beta.p, theta_prev.p, msteps.p, gap.p, conv.p);
    iter.upload(&j, 1, st);
    check_launch("compaction");
    BLz lz{alpha.p, beta.p, partials.p, iter.p, n_prob_c, ck.d_sec_ctr.p, ck.d_sec_tile0.p, ck.d_sec_ntiles.p};
    lz.gap_cap = restart_gap_cap();
    auto step = [&](cudaStream_t ss) {
        bhv_any<V>(ac, ck, wc.p, wc.p, vc.p, 2, lz, nullptr, nullptr, 1, ss);
        bupdate_any<V>(ac, ck, wc.p, vc.p, 2, lz, ss);
        g_kernels += 1;
        k_badvance<<<1, 32, 0, ss>>>(lz);
    };
    const double* gap_c = src.gap ? gap.p : nullptr;
    int done = j;
    {
        Buf<int> d_w = ws_take<int>(nv);
        d_w.upload(n_real.data(), nv, st);
        const double ratio = depth + 1 < kCompactDepth ? sub_compact_ratio() : 0.0;
        Buf<int> d_group = ws_take<int>(nv);
        d_group.upload(vs_base.data(), nv, st);
        LoopOut lo = device_loop(step, ac, lz, NC, stall, res_tol, e_tol, gap_c, nullptr, theta.p, theta_prev.p,
                                 msteps.p, conv.p, ck.d_active.p, active_next.p, ck.d_nrows.p, d_w.p, nv,
                                 std::max(1, check), j, cap, ratio, st, d_group.p, k.n_sectors);
        done = lo.done;
        products += lo.products;
        n_hv += done - j;
        if (trace_on())
            std::fprintf(stderr, "[qmb batch] compacted %s loop (level %d): %d virtual sectors, steps %d..%d, stop reason %d\n",
                         f64 ? "fp64" : "fp32", depth + 1, nv, j, done, lo.reason);
        if (lo.reason == 3) {
            // the unconverged problems of this sub-batch move into a smaller one
            CSrc me;
            me.n_sectors = nv;
            me.nsp = NC;
            me.base_of = vs_base;
            me.d_sec_elem = ck.d_sec_elem.p;
            me.cx = cx;
            me.cz = cz;
            me.real = real;
            me.alpha = alpha.p;
            me.beta = beta.p;
            me.theta = theta.p;
            me.theta_prev = theta_prev.p;
            me.gap = gap_c;
            me.msteps = msteps.p;
            me.conv = conv.p;
            std::vector<int> hc(n_prob_c);
            conv.download(hc.data(), n_prob_c, st);
            QMB_CUDA_TRY(cudaStreamSynchronize(st));
            done = run_compacted<V>(b, k, ck.compact, f64, a_base, me, wc.p + (int64_t)(done & 1) * tot_c,
                                    vc.p + (int64_t)((done + 1) & 1) * tot_c, done, cap, stall, res_tol, e_tol,
                                    check, hc, depth + 1, products, n_hv, st);
        } else if (lo.reason != 1 && done < cap) {
            std::vector<int> act(nv);
            ck.d_active.download(act.data(), nv, st);
            QMB_CUDA_TRY(cudaStreamSynchronize(st));
            double w = 0;
            for (int v = 0; v < nv; ++v) w += (double)act[v] * n_real[v];
            const int rem = cap - done;
            for (int t = 0; t < rem; ++t) step(st);
            products += rem * w;
            done += rem;
            n_hv += rem;
            QMB_CUDA_TRY(cudaMemsetAsync(active_next.p, 0, sizeof(int) * nv, st));
            launch_check(ac, lz, NC, stall, res_tol, e_tol, gap_c, nullptr, theta.p, theta_prev.p, msteps.p,
                         conv.p, active_next.p, done, st);
            check_launch("compacted last steps");
        }
    }
    g_kernels += 1;
    k_bscatter_state<<<(n_prob_c + 255) / 256, 256, 0, st>>>(n_prob_c, d_slot_src.p, d_real.p, theta.p, msteps.p,
                                                            conv.p, src.theta, src.msteps, src.conv);
    check_launch("compaction results");
    QMB_CUDA_TRY(cudaStreamSynchronize(st));
    return done;
}

// Batched Lanczos phase over one kind with vectors V (and matrix values of
// the same precision).  start: 0 splitmix (seed), 2 copy of psi_in (FP64).
template <class V>
static BPhase run_bphase(qmb_batch_s* b, BKind& k, bool f64, int max_iter, double stall, double res_tol,
                         double e_tol, const double* gap_in, double* gap_out, int check, int start,
                         uint64_t seed, const void* psi_in, void* psi_out, int store_slots, int& n_hv,
                         cudaStream_t st, const int* init_active = nullptr) {
    BPhase out;
    const auto t_begin = std::chrono::steady_clock::now();
    const int64_t tot = k.sec_elem[k.n_sectors];
    const int n_prob = k.n_sectors * b->nsp;
    int64_t minrows = INT64_MAX;
    for (auto r : k.nrows) minrows = std::min(minrows, r);
    const int cap = std::max(1, max_iter);
    (void)minrows;
    // Krylov basis kept on the device (ring of K vectors); when the phase
    // runs longer than the ring, the Ritz vector is regenerated instead.
    // K_full slots would hold the whole phase; the ring starts at what the
    // earlier phases on this handle needed (at least kRingStart slots) and
    // doubles when a phase reaches its end.
    const size_t vec_bytes = std::max<size_t>((size_t)tot * sizeof(V), 1);
    int K_full = store_slots > 2 ? std::min(store_slots, cap + 1) : 2;
    int K = K_full > 2 ? std::min(K_full, std::max(ring_start(), k.ring_hint)) : 2;
    if (K_full > 2) K = std::max(K, std::min(K_full, (int)(k.ws_ring.n / vec_bytes)));
    // workspace cached on the handle (grown on demand, reused by later solves)
    auto grow = [&](DevBuf<unsigned char>& buf, size_t bytes) {
        if (buf.n < bytes) {
            buf.release();
            buf.alloc(bytes);
        }
    };
    grow(k.ws_w, 2 * (size_t)tot * sizeof(V));
    grow(k.ws_ring, (size_t)K * vec_bytes);
    struct View { V* p; } wbuf{reinterpret_cast<V*>(k.ws_w.p)}, vring{reinterpret_cast<V*>(k.ws_ring.p)};
    Buf<double> alpha = ws_take<double>((size_t)(cap + 1) * n_prob),
        beta = ws_take<double>((size_t)(cap + 2) * n_prob),
        partials = ws_take<double>((size_t)std::max(1, k.n_tiles) * b->nsp),
        theta = ws_take<double>(n_prob),
        theta_prev = ws_take<double>(n_prob),
        ritz = ws_take<double>((size_t)(cap + 1) * n_prob),
        Ls = ws_take<double>((size_t)(cap + 1) * n_prob),
        Ds = ws_take<double>((size_t)(cap + 1) * n_prob);
    Buf<int> iter = ws_take<int>(1),
        msteps = ws_take<int>(n_prob),
        conv = ws_take<int>(n_prob),
        active_next = ws_take<int>(k.n_sectors);
    QMB_CUDA_TRY(cudaMemsetAsync(theta_prev.p, 0, sizeof(double) * n_prob, st));
    QMB_CUDA_TRY(cudaMemsetAsync(conv.p, 0, sizeof(int) * n_prob, st));
    QMB_CUDA_TRY(cudaMemsetAsync(msteps.p, 0, sizeof(int) * n_prob, st));
    QMB_CUDA_TRY(cudaMemsetAsync(ritz.p, 0, ritz.n * sizeof(double), st));
    QMB_CUDA_TRY(cudaMemsetAsync(alpha.p, 0, alpha.n * sizeof(double), st));
    QMB_CUDA_TRY(cudaMemsetAsync(beta.p, 0, beta.n * sizeof(double), st));
    if (init_active) {
        QMB_CUDA_TRY(cudaMemcpyAsync(k.d_active.p, init_active, sizeof(int) * k.n_sectors,
                                     cudaMemcpyDeviceToDevice, st));
    } else {
        std::vector<int> ones(k.n_sectors, 1);
        k.d_active.upload(ones.data(), k.n_sectors, st);
    }
    BatchArgs a = make_args(b, k);
    a.val = f64 ? k.val64.p : k.val32.p;
    a.dxy = f64 ? k.dxy64.p : k.dxy32.p;
    a.dz = f64 ? k.dz64.p : k.dz32.p;
    BLz lz{alpha.p, beta.p, partials.p, iter.p, n_prob, k.d_sec_ctr.p, k.d_sec_tile0.p, k.d_sec_ntiles.p};
    lz.gap_cap = restart_gap_cap();
    const int rb = 256, rg = (n_prob + rb - 1) / rb;
    tuned_variant<V>(a, k, f64, st);
    g_kernels += 1;
    k_bstart<V><<<grid_for(tot, 256), 256, 0, st>>>(a, tot, start, seed, psi_in, wbuf.p);
    bnorm0_any<V>(a, k, wbuf.p, lz, st);
    g_kernels += 1;
    k_bbeta0<<<rg, rb, 0, st>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz);
    check_launch("batch start");
    auto step = [&](cudaStream_t ss) {
        bhv_any<V>(a, k, wbuf.p, wbuf.p, vring.p, K, lz, nullptr, nullptr, 1, ss);
        bupdate_any<V>(a, k, wbuf.p, vring.p, K, lz, ss);
        g_kernels += 1;
        k_badvance<<<1, 32, 0, ss>>>(lz);
    };
    int done = 0;
    if (trace_on()) {
        QMB_CUDA_TRY(cudaStreamSynchronize(st));
        std::fprintf(stderr, "[qmb batch] %s setup: %.2f ms\n", f64 ? "fp64" : "fp32",
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count());
    }
    {
        std::vector<int> wts(k.n_sectors, b->n_sets);
        Buf<int> d_w = ws_take<int>(k.n_sectors);
        d_w.upload(wts.data(), k.n_sectors, st);
        const bool can_compact = !psi_out && K == 2;
        LoopOut lo{0, 2, 0.0};
        for (int j0 = 0;;) {
            const int cap_run = K < K_full ? std::min(cap, K - 1) : cap;
            lo = device_loop(step, a, lz, b->n_sets, stall, res_tol, e_tol, gap_in, gap_out, theta.p,
                             theta_prev.p, msteps.p, conv.p, k.d_active.p, active_next.p, k.d_nrows.p, d_w.p,
                             k.n_sectors, std::max(1, check), j0, cap_run, can_compact ? compact_ratio() : 0.0, st);
            out.products += lo.products;
            n_hv += lo.done - j0;
            j0 = lo.done;
            if (lo.reason != 2 || cap_run >= cap) break;
            // the ring is full: continue in one twice as large, the filled
            // slots copied over (slot i holds v_i while no slot was reused);
            // without the memory the ring stays and wraps from here on
            const int K2 = std::min(K_full, 2 * K);
            void* np = nullptr;
            if (cudaMalloc(&np, (size_t)K2 * vec_bytes) != cudaSuccess) {
                (void)cudaGetLastError();
                K_full = K;
                continue;
            }
            QMB_CUDA_TRY(cudaMemcpyAsync(np, vring.p, (size_t)j0 * vec_bytes, cudaMemcpyDeviceToDevice, st));
            QMB_CUDA_TRY(cudaStreamSynchronize(st));
            k.ws_ring.release();
            k.ws_ring.p = reinterpret_cast<unsigned char*>(np);
            k.ws_ring.n = (size_t)K2 * vec_bytes;
            vring.p = reinterpret_cast<V*>(np);
            K = K2;
            if (trace_on()) std::fprintf(stderr, "[qmb batch] ring grown to %d slots at step %d\n", K, j0);
        }
        done = lo.done;
        if (K > 2) k.ring_hint = std::max(k.ring_hint, done + 1 + std::max(1, check));
        if (trace_on())
            std::fprintf(stderr, "[qmb batch] %s loop: %d steps, stop reason %d, %.2f ms to here\n",
                         f64 ? "fp64" : "fp32", done, lo.reason,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count());
        if (lo.reason == 3) {
            std::vector<int> hc(n_prob);
            conv.download(hc.data(), n_prob, st);
            QMB_CUDA_TRY(cudaStreamSynchronize(st));
            CSrc base;
            base.n_sectors = k.n_sectors;
            base.nsp = b->nsp;
            base.base_of.resize(k.n_sectors);
            for (int s = 0; s < k.n_sectors; ++s) base.base_of[s] = s;
            base.d_sec_elem = k.d_sec_elem.p;
            std::vector<double> hx(b->nsp), hz(b->nsp);
            b->cxy.download(hx.data(), b->nsp, st);
            b->cz.download(hz.data(), b->nsp, st);
            QMB_CUDA_TRY(cudaStreamSynchronize(st));
            base.cx.resize(n_prob);
            base.cz.resize(n_prob);
            base.real.resize(n_prob);
            for (int p = 0; p < n_prob; ++p) {
                base.cx[p] = hx[p % b->nsp];
                base.cz[p] = hz[p % b->nsp];
                base.real[p] = p % b->nsp < b->n_sets ? 1 : 0;
            }
            base.alpha = lz.alpha;
            base.beta = lz.beta;
            base.theta = theta.p;
            base.theta_prev = theta_prev.p;
            base.gap = gap_in;
            base.msteps = msteps.p;
            base.conv = conv.p;
            done = run_compacted<V>(b, k, k.compact, f64, a, base, wbuf.p + (int64_t)(done & 1) * tot,
                                    vring.p + (int64_t)((done + 1) & 1) * tot, done, cap, stall, res_tol, e_tol,
                                    check, hc, 0, out.products, n_hv, st);
        } else if (lo.reason != 1 && done < cap) {
            // the last steps (fewer than a block) with one test at the end
            std::vector<int> act(k.n_sectors);
            k.d_active.download(act.data(), k.n_sectors, st);
            QMB_CUDA_TRY(cudaStreamSynchronize(st));
            int na = 0;
            for (int v : act) na += v;
            const int rem = cap - done;
            for (int t = 0; t < rem; ++t) step(st);
            out.products += (double)rem * na * b->n_sets;
            done += rem;
            n_hv += rem;
            QMB_CUDA_TRY(cudaMemsetAsync(active_next.p, 0, sizeof(int) * k.n_sectors, st));
            launch_check(a, lz, b->n_sets, stall, res_tol, e_tol, gap_in, gap_out, theta.p, theta_prev.p,
                         msteps.p, conv.p, active_next.p, done, st);
            QMB_CUDA_TRY(cudaMemcpyAsync(k.d_active.p, active_next.p, sizeof(int) * k.n_sectors,
                                         cudaMemcpyDeviceToDevice, st));
            check_launch("batch last steps");
        }
    }
    out.steps = done;
    if (trace_on()) {
        QMB_CUDA_TRY(cudaStreamSynchronize(st));
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();
        std::fprintf(stderr, "[qmb batch] phase %s: %d steps, ring %d, start %d, %.2f ms to here\n",
                     f64 ? "fp64" : "fp32", done, K, start, ms);
    }
    // Ritz vectors (FP64) for the next phase or the caller
    if (psi_out) {
        Buf<double> xs = ws_take<double>((size_t)(cap + 1) * n_prob);
        cudaEvent_t te[3] = {nullptr, nullptr, nullptr};
        if (trace_on())
            for (auto& e : te) {
                QMB_CUDA_TRY(cudaEventCreate(&e));
            }
        if (te[0]) QMB_CUDA_TRY(cudaEventRecord(te[0], st));
        g_kernels += 1;
        // one thread per problem, long serial loops: 32-thread blocks spread
        // the problems over every SM (5,120 problems are 20 blocks of 256)
        k_britz<<<(n_prob + 31) / 32, 32, 0, st>>>(lz, msteps.p, theta.p, Ls.p, Ds.p, xs.p, ritz.p, gap_out);
        if (te[1]) QMB_CUDA_TRY(cudaEventRecord(te[1], st));
        if (K > 2 && done < K) {
            g_kernels += 1;
            k_bpsi<V><<<grid_for(tot, 256), 256, 0, st>>>(a, tot, vring.p, K, msteps.p, ritz.p, n_prob,
                                                          psi_out);
            if (te[2]) {
                QMB_CUDA_TRY(cudaEventRecord(te[2], st));
                QMB_CUDA_TRY(cudaEventSynchronize(te[2]));
                float a_ms = 0, b_ms = 0;
                cudaEventElapsedTime(&a_ms, te[0], te[1]);
                cudaEventElapsedTime(&b_ms, te[1], te[2]);
                std::fprintf(stderr, "[qmb batch] ritz: k_britz %.2f ms, k_bpsi %.2f ms (device), %.2f ms to here\n",
                             a_ms, b_ms,
                             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count());
            }
        } else {
            QMB_CUDA_TRY(cudaMemsetAsync(psi_out, 0, (Sc<V>::cplx ? 16 : 8) * tot, st));
            std::vector<int> all(k.n_sectors, 1);
            k.d_active.upload(all.data(), k.n_sectors, st);
            g_kernels += 1;
            k_bstart<V><<<grid_for(tot, 256), 256, 0, st>>>(a, tot, start, seed, psi_in, wbuf.p);
            bnorm0_any<V>(a, k, wbuf.p, lz, st);
            g_kernels += 1;
            k_bbeta0<<<rg, rb, 0, st>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz);
            // regeneration runs every problem to the longest m; coefficients
            // beyond a problem's own m are zero (k_britz wrote m entries)
            for (int j = 0; j < done; ++j) {
                bhv_any<V>(a, k, wbuf.p, wbuf.p, vring.p, K, lz, ritz.p, psi_out, 1, st);
                bupdate_any<V>(a, k, wbuf.p, vring.p, K, lz, st);
                g_kernels += 1;
                k_badvance<<<1, 32, 0, st>>>(lz);
                ++n_hv;
                out.products += (double)k.n_sectors * b->n_sets;
            }
        }
        check_launch("batch ritz");
        for (auto& e : te)
            if (e) cudaEventDestroy(e);
    }
    out.theta.resize(n_prob);
    out.msteps.resize(n_prob);
    out.conv.resize(n_prob);
    theta.download(out.theta.data(), n_prob, st);
    msteps.download(out.msteps.data(), n_prob, st);
    conv.download(out.conv.data(), n_prob, st);
    QMB_CUDA_TRY(cudaStreamSynchronize(st));
    return out;
}

}  // namespace qmb

// ------------------------------------------------------------------ C ABI
extern "C" qmb_status qmb_batch_create(const qmb_batch_desc* d, qmb_batch* out) {
    return guarded([&] {
        QMB_REQUIRE(d && out && d->sectors && d->terms_xy && d->terms_z, QMB_ERR_INVALID, "null argument");
        *out = nullptr;
        QMB_REQUIRE(d->n_sectors >= 1 && d->n_sectors <= 4096, QMB_ERR_INVALID, "n_sectors must be in 1..4096");
        QMB_REQUIRE(d->n_sets >= 1 && d->n_sets <= 256, QMB_ERR_INVALID, "n_sets must be in 1..256");
        DeviceGuard dg(d->device);
        auto b = std::make_unique<qmb_batch_s>();
        b->device = d->device;
        b->n_sectors = d->n_sectors;
        b->n_sets = d->n_sets;
        int nsp = 32;
        while (nsp < d->n_sets) nsp *= 2;
        b->nsp = nsp;
        b->n_groups = 1;
        b->spl = spl_for<float2>(nsp);
        b->sector_kind.resize(d->n_sectors);
        b->sector_pos.resize(d->n_sectors);
        // per-sector matrices through the single-sector builder, turned into
        // CSR on the device (the sector's SELL table never leaves HBM)
        struct Part {
            std::vector<int64_t> row_ptr;      // host copy, for the tile tables
            DevBuf<int64_t> rp;                // [n+1] entry offsets within the sector
            DevBuf<uint32_t> col;              // [nnz]
            DevBuf<double2> val, dxy, dz;      // [nnz], [n], [n]
        };
        std::vector<Part> parts(d->n_sectors);
        const auto t_create = std::chrono::steady_clock::now();
        double ms_build = 0.0, ms_csr = 0.0;
        auto ms_since = [](std::chrono::steady_clock::time_point t) {
            return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
        };
        DevBuf<unsigned char> scan_tmp;
        DevBuf<int64_t> row_cnt;
        for (int s = 0; s < d->n_sectors; ++s) {
            auto t_part = std::chrono::steady_clock::now();
            qmb_sector sec = d->sectors[s];
            QMB_REQUIRE(sec && sec->has_irrep, QMB_ERR_INVALID, "every sector needs a selected irrep");
            QMB_REQUIRE(sec->device == d->device, QMB_ERR_INVALID, "sectors must live on the batch device");
            qmb_ham hx = nullptr, hz = nullptr;
            qmb_status st = qmb_ham_create(sec, d->terms_xy, QMB_PREC_FP64, &hx);
            if (st != QMB_OK) throw Error{st, std::string("terms_xy: ") + qmb_last_error()};
            std::unique_ptr<qmb_ham_s> ox(hx);
            st = qmb_ham_create(sec, d->terms_z, QMB_PREC_FP64, &hz);
            if (st != QMB_OK) throw Error{st, std::string("terms_z: ") + qmb_last_error()};
            std::unique_ptr<qmb_ham_s> oz(hz);
            QMB_REQUIRE(hz->nnz == 0, QMB_ERR_INVALID, "terms_z must be diagonal");
            ms_build += ms_since(t_part);
            t_part = std::chrono::steady_clock::now();
            const int64_t n = hx->n;
            b->sector_kind[s] = (hx->cplx || hz->cplx) ? 1 : 0;
            Part& P = parts[s];
            P.rp.alloc(n + 1);
            P.row_ptr.assign(n + 1, 0);
            if (n == 0) P.rp.zero();
            if (n > 0) {
                const int gb = grid_for(n, 256);
                if (row_cnt.n < (size_t)(n + 1)) row_cnt.alloc(n + 1);
                if (hx->cplx)
                    k_sell_row_count<double2><<<gb, 256>>>(n, hx->slice_off.p, hx->slice_w.p, hx->col.p,
                                                           reinterpret_cast<const double2*>(hx->val64.p), row_cnt.p);
                else
                    k_sell_row_count<double><<<gb, 256>>>(n, hx->slice_off.p, hx->slice_w.p, hx->col.p,
                                                          reinterpret_cast<const double*>(hx->val64.p), row_cnt.p);
                check_launch("batch row counts");
                size_t tb = 0;
                QMB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, row_cnt.p, P.rp.p, n + 1));
                if (scan_tmp.n < tb) scan_tmp.alloc(tb);
                QMB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp.p, tb, row_cnt.p, P.rp.p, n + 1));
                P.rp.download(P.row_ptr.data(), n + 1);
                QMB_CUDA_TRY(cudaStreamSynchronize(0));
            }
            const int64_t nnz = P.row_ptr[n];
            P.col.alloc(std::max<int64_t>(nnz, 1));
            P.val.alloc(std::max<int64_t>(nnz, 1));
            P.dxy.alloc(std::max<int64_t>(n, 1));
            P.dz.alloc(std::max<int64_t>(n, 1));
            if (n > 0) {
                const int gb = grid_for(n, 256);
                if (hx->cplx) {
                    k_sell_to_csr<double2><<<gb, 256>>>(n, hx->slice_off.p, hx->slice_w.p, hx->col.p,
                                                        reinterpret_cast<const double2*>(hx->val64.p), P.rp.p,
                                                        P.col.p, P.val.p);
                    k_widen<double2><<<gb, 256>>>(n, reinterpret_cast<const double2*>(hx->diag64.p), P.dxy.p);
                } else {
                    k_sell_to_csr<double><<<gb, 256>>>(n, hx->slice_off.p, hx->slice_w.p, hx->col.p,
                                                       reinterpret_cast<const double*>(hx->val64.p), P.rp.p,
                                                       P.col.p, P.val.p);
                    k_widen<double><<<gb, 256>>>(n, reinterpret_cast<const double*>(hx->diag64.p), P.dxy.p);
                }
                if (hz->cplx) k_widen<double2><<<gb, 256>>>(n, reinterpret_cast<const double2*>(hz->diag64.p), P.dz.p);
                else k_widen<double><<<gb, 256>>>(n, reinterpret_cast<const double*>(hz->diag64.p), P.dz.p);
                check_launch("batch CSR");
            }
            // the builder's tables are freed with ox/oz: finish reading them first
            QMB_CUDA_TRY(cudaStreamSynchronize(0));
            ms_csr += ms_since(t_part);
        }
        // Real sectors that are a small part of a batch with complex ones join
        // the complex kind (zero imaginary parts): on their own, their
        // phases would be launch- and latency-bound steps run one after the
        // other with the complex kind's.
        {
            int64_t rows_kind[2] = {0, 0};
            for (int s = 0; s < d->n_sectors; ++s)
                rows_kind[b->sector_kind[s]] += (int64_t)parts[s].row_ptr.size() - 1;
            const char* me = std::getenv("QMB_MERGE_REAL");
            const bool merge = !(me && me[0] == '0');
            if (merge && rows_kind[0] > 0 && rows_kind[1] > 0 &&
                (double)rows_kind[0] < kMergeRealFrac * (double)rows_kind[1])
                for (int s = 0; s < d->n_sectors; ++s) b->sector_kind[s] = 1;
        }
        const auto t_assemble = std::chrono::steady_clock::now();
        // assemble the two kinds: host tile tables, device placement of the parts
        for (int kd = 0; kd < 2; ++kd) {
            BKind& K = b->kind[kd];
            std::vector<int64_t> row_base, row0, ent0;
            int64_t n_rp = 0, n_ent = 0, n_rows = 0;
            K.sec_elem.assign(1, 0);
            for (int s = 0; s < d->n_sectors; ++s) {
                if (b->sector_kind[s] != kd) continue;
                Part& P = parts[s];
                int ks = K.n_sectors++;
                b->sector_pos[s] = ks;
                K.sec_index.push_back(s);
                int64_t n = (int64_t)P.row_ptr.size() - 1;
                K.nrows.push_back(n);
                K.rows += n;
                K.sec_elem.push_back(K.sec_elem.back() + n * b->nsp);
                row_base.push_back(n_rp);
                row0.push_back(n_rows);
                ent0.push_back(n_ent);
                n_rp += n + 1;
                n_rows += n;
                n_ent += P.row_ptr[n];
                K.sec_tile0.push_back((int)K.tile_sector.size());
                int nt = (int)((n + kBTile - 1) / kBTile);
                K.sec_ntiles.push_back(nt);
                for (int t = 0; t < nt; ++t) {
                    K.tile_sector.push_back(ks);
                    K.tile_row0.push_back(t * kBTile);
                    int64_t re = std::min<int64_t>(n, (int64_t)(t + 1) * kBTile);
                    K.max_tile_entries = std::max<int>(K.max_tile_entries,
                                                       (int)(P.row_ptr[re] - P.row_ptr[(int64_t)t * kBTile]));
                }
            }
            if (!K.n_sectors) continue;
            K.nnz = n_ent;
            K.n_tiles = (int)K.tile_sector.size();
            std::vector<int> tiles(K.n_tiles);
            for (int t = 0; t < K.n_tiles; ++t) tiles[t] = t;
            auto up_i = [](DevBuf<int>& dbuf, const std::vector<int>& v) { dbuf.alloc(std::max<size_t>(1, v.size())); if (!v.empty()) dbuf.upload(v.data(), v.size()); };
            auto up_l = [](DevBuf<int64_t>& dbuf, const std::vector<int64_t>& v) { dbuf.alloc(std::max<size_t>(1, v.size())); if (!v.empty()) dbuf.upload(v.data(), v.size()); };
            up_i(K.d_tile_sector, K.tile_sector);
            up_i(K.d_tile_row0, K.tile_row0);
            up_i(K.d_sec_tile0, K.sec_tile0);
            up_i(K.d_sec_ntiles, K.sec_ntiles);
            up_i(K.d_tiles, tiles);
            K.d_active.alloc(K.n_sectors);
            K.d_ctr.alloc(2);
            K.d_ctr.zero();
            K.d_sec_ctr.alloc(K.n_sectors);
            K.d_sec_ctr.zero();
            up_l(K.d_sec_elem, K.sec_elem);
            up_l(K.d_nrows, K.nrows);
            up_l(K.d_row_base, row_base);
            up_l(K.d_row0, row0);
            K.h_row_base = row_base;
            K.h_row0 = row0;
            K.d_row_ptr.alloc(std::max<int64_t>(1, n_rp));
            K.d_col.alloc(std::max<int64_t>(1, n_ent));
            // values in the sector kind's scalar types
            const size_t sv = kd ? sizeof(double2) : sizeof(double), sf = kd ? sizeof(float2) : sizeof(float);
            K.val64.alloc(std::max<int64_t>(1, n_ent) * sv);
            K.val32.alloc(std::max<int64_t>(1, n_ent) * sf);
            K.dxy64.alloc(std::max<int64_t>(1, n_rows) * sv);
            K.dxy32.alloc(std::max<int64_t>(1, n_rows) * sf);
            K.dz64.alloc(std::max<int64_t>(1, n_rows) * sv);
            K.dz32.alloc(std::max<int64_t>(1, n_rows) * sf);
            for (int ks = 0; ks < K.n_sectors; ++ks) {
                Part& P = parts[K.sec_index[ks]];
                const int64_t n = K.nrows[ks], ne = P.row_ptr[n];
                const int gb = grid_for(std::max<int64_t>(n + 1, ne), 256);
                PlaceArgs pa{n, ne, ent0[ks], P.rp.p, P.col.p, P.val.p, P.dxy.p, P.dz.p,
                             K.d_row_ptr.p + row_base[ks], K.d_col.p + ent0[ks]};
                if (kd)
                    k_place_sector<double2, float2><<<gb, 256>>>(
                        pa, reinterpret_cast<double2*>(K.val64.p) + ent0[ks], reinterpret_cast<float2*>(K.val32.p) + ent0[ks],
                        reinterpret_cast<double2*>(K.dxy64.p) + row0[ks], reinterpret_cast<float2*>(K.dxy32.p) + row0[ks],
                        reinterpret_cast<double2*>(K.dz64.p) + row0[ks], reinterpret_cast<float2*>(K.dz32.p) + row0[ks]);
                else
                    k_place_sector<double, float><<<gb, 256>>>(
                        pa, reinterpret_cast<double*>(K.val64.p) + ent0[ks], reinterpret_cast<float*>(K.val32.p) + ent0[ks],
                        reinterpret_cast<double*>(K.dxy64.p) + row0[ks], reinterpret_cast<float*>(K.dxy32.p) + row0[ks],
                        reinterpret_cast<double*>(K.dz64.p) + row0[ks], reinterpret_cast<float*>(K.dz32.p) + row0[ks]);
                check_launch("batch placement");
            }
        }
        b->cxy.alloc(b->nsp);
        b->cz.alloc(b->nsp);
        b->cxy.zero();
        b->cz.zero();
        QMB_CUDA_TRY(cudaDeviceSynchronize());
        if (trace_on())
            std::fprintf(stderr, "[qmb batch] create: sector matrices %.1f ms, device CSR %.1f ms, "
                         "assembly %.1f ms, total %.1f ms\n", ms_build, ms_csr,
                         ms_since(t_assemble), ms_since(t_create));
        *out = b.release();
    });
}

extern "C" qmb_status qmb_batch_destroy(qmb_batch b) {
    return guarded([&] {
        if (!b) return;
        DeviceGuard dg(b->device);
        delete b;
    });
}

static double batch_bytes(const qmb_batch_s* b, bool f64) {
    double tot = 0;
    for (int kd = 0; kd < 2; ++kd) {
        const BKind& k = b->kind[kd];
        double vs = (f64 ? 8.0 : 4.0) * (kd ? 2 : 1);
        // x read once + y written once per (row, set); shared tables once
        tot += (double)k.rows * b->n_sets * 2 * vs + (double)k.nnz * (4 + vs) + (double)k.rows * 2 * vs;
    }
    return tot;
}

extern "C" qmb_status qmb_batch_get_info(qmb_batch b, qmb_batch_info* info) {
    return guarded([&] {
        QMB_REQUIRE(b && info, QMB_ERR_INVALID, "null argument");
        info->rows_total = b->kind[0].rows + b->kind[1].rows;
        info->elems_total = info->rows_total * b->n_sets;
        info->bytes_hv_fp64 = batch_bytes(b, true);
        info->bytes_hv_fp32 = batch_bytes(b, false);
        info->rows_per_block = kBTile;
        info->sets_per_thread = b->spl;
        info->set_stride = b->nsp;
        const BKind& kc = b->kind[1].n_sectors ? b->kind[1] : b->kind[0];
        info->variant_fp32 = kc.variant[0];
        info->variant_fp64 = kc.variant[1];
        for (int c = 0; c < kBVariants; ++c) {
            info->tune_ms_fp32[c] = kc.tune_ms[0][c];
            info->tune_ms_fp64[c] = kc.tune_ms[1][c];
        }
        info->nnz_total = b->kind[0].nnz + b->kind[1].nnz;
        for (int kd = 0; kd < 2; ++kd) {
            const BKind& k = b->kind[kd];
            const size_t vb = (size_t)k.sec_elem.back() * (kd ? sizeof(float2) : sizeof(float));
            info->ring_slots[kd] = (k.n_sectors && vb) ? (int)(k.ws_ring.n / vb) : 0;
        }
    });
}

extern "C" qmb_status qmb_batch_layout(qmb_batch b, int64_t* offsets, int* is_complex) {
    return guarded([&] {
        QMB_REQUIRE(b && offsets, QMB_ERR_INVALID, "null argument");
        // real sectors first, then complex ones; each [row][set] with set
        // stride info.set_stride; offsets count scalars (complex = 2)
        const int64_t r_elems = b->kind[0].n_sectors ? b->kind[0].sec_elem[b->kind[0].n_sectors] : 0;
        int64_t end = r_elems;
        for (int s = 0; s < b->n_sectors; ++s) {
            int kd = b->sector_kind[s];
            const BKind& k = b->kind[kd];
            int ks = b->sector_pos[s];
            offsets[s] = kd ? r_elems + 2 * k.sec_elem[ks] : k.sec_elem[ks];
            if (is_complex) is_complex[s] = kd;
        }
        if (b->kind[1].n_sectors) end = r_elems + 2 * b->kind[1].sec_elem[b->kind[1].n_sectors];
        offsets[b->n_sectors] = end;
    });
}

// Device-side batched H*v in the internal padded layout of one kind.
namespace qmb {
template <class V>
static void batch_hv_kind(qmb_batch_s* b, BKind& k, bool f64, const V* x, V* y, cudaStream_t st) {
    if (!k.n_sectors) return;
    BatchArgs a = make_args(b, k);
    a.val = f64 ? k.val64.p : k.val32.p;
    a.dxy = f64 ? k.dxy64.p : k.dxy32.p;
    a.dz = f64 ? k.dz64.p : k.dz32.p;
    BLz lz{nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, nullptr};
    int v = tuned_variant<V>(a, k, f64, st);
    // the multi-slice variants read 32- or 64-byte runs: caller vectors that
    // are only 16-byte aligned take a one-slice variant
    if ((((uintptr_t)x | (uintptr_t)y) & 63) && kBSlices[v] > 1) v = 0;
    bhv_variant<V>(v, a, k, x, y, nullptr, 1, lz, nullptr, nullptr, 0, st);
    check_launch("k_bhv");
}
}  // namespace qmb

extern "C" qmb_status qmb_batch_hv(qmb_batch b, int prec, const void* x_dev, void* y_dev, void* stream) {
    return guarded([&] {
        QMB_REQUIRE(b && x_dev && y_dev, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(prec == QMB_PREC_FP64 || prec == QMB_PREC_FP32, QMB_ERR_INVALID, "bad prec");
        QMB_REQUIRE((((uintptr_t)x_dev | (uintptr_t)y_dev) & 15) == 0, QMB_ERR_INVALID,
                    "x_dev and y_dev must be 16-byte aligned");
        DeviceGuard dg(b->device);
        cudaStream_t st = (cudaStream_t)stream;
        bool f64 = prec == QMB_PREC_FP64;
        // internal layout: real kind block first, then complex kind block,
        // both padded to nsp sets (see qmb_batch_internal_elems)
        const int64_t r_elems = b->kind[0].n_sectors ? b->kind[0].sec_elem[b->kind[0].n_sectors] : 0;
        const char* xc = (const char*)x_dev;
        char* yc = (char*)y_dev;
        size_t rs = f64 ? 8 : 4;
        if (f64) {
            batch_hv_kind<double>(b, b->kind[0], true, (const double*)xc, (double*)yc, st);
            batch_hv_kind<double2>(b, b->kind[1], true, (const double2*)(xc + r_elems * rs), (double2*)(yc + r_elems * rs), st);
        } else {
            batch_hv_kind<float>(b, b->kind[0], false, (const float*)xc, (float*)yc, st);
            batch_hv_kind<float2>(b, b->kind[1], false, (const float2*)(xc + r_elems * rs), (float2*)(yc + r_elems * rs), st);
        }
    });
}

namespace qmb {
// K1 of `reps` Lanczos steps of one kind from a seeded start, each launch
// bracketed by events; the steps' K2 and advance run between them untimed.
template <class V>
static double k1_kind_ms(qmb_batch_s* b, BKind& k, bool f64, int reps, cudaStream_t st) {
    if (!k.n_sectors || !k.n_tiles) return 0.0;
    const int64_t tot = k.sec_elem[k.n_sectors];
    const int n_prob = k.n_sectors * b->nsp;
    const int cap = reps + 2;
    DevBuf<V> w(2 * (size_t)tot), ring(2 * (size_t)tot);
    DevBuf<double> alpha((size_t)(cap + 1) * n_prob), beta((size_t)(cap + 2) * n_prob),
        partials((size_t)k.n_tiles * b->nsp);
    DevBuf<int> iter(1);
    iter.zero(st);
    std::vector<int> ones(k.n_sectors, 1);
    k.d_active.upload(ones.data(), k.n_sectors, st);
    BatchArgs a = make_args(b, k);
    a.val = f64 ? k.val64.p : k.val32.p;
    a.dxy = f64 ? k.dxy64.p : k.dxy32.p;
    a.dz = f64 ? k.dz64.p : k.dz32.p;
    BLz lz{alpha.p, beta.p, partials.p, iter.p, n_prob, k.d_sec_ctr.p, k.d_sec_tile0.p, k.d_sec_ntiles.p};
    const int rb = 256, rg = (n_prob + rb - 1) / rb;
    tuned_variant<V>(a, k, f64, st);
    k_bstart<V><<<grid_for(tot, 256), 256, 0, st>>>(a, tot, 0, 2212456ull, nullptr, w.p);
    bnorm0_any<V>(a, k, w.p, lz, st);
    k_bbeta0<<<rg, rb, 0, st>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz);
    std::vector<cudaEvent_t> ev(2 * (size_t)(reps + 1));
    for (auto& e : ev) QMB_CUDA_TRY(cudaEventCreate(&e));
    struct EvG {
        std::vector<cudaEvent_t>& v;
        ~EvG() { for (auto e : v) cudaEventDestroy(e); }
    } evg{ev};
    for (int j = 0; j <= reps; ++j) {  // step 0 warms up
        QMB_CUDA_TRY(cudaEventRecord(ev[2 * j], st));
        bhv_any<V>(a, k, w.p, w.p, ring.p, 2, lz, nullptr, nullptr, 1, st);
        QMB_CUDA_TRY(cudaEventRecord(ev[2 * j + 1], st));
        bupdate_any<V>(a, k, w.p, ring.p, 2, lz, st);
        k_badvance<<<1, 32, 0, st>>>(lz);
    }
    check_launch("k1 timing");
    QMB_CUDA_TRY(cudaStreamSynchronize(st));
    double ms = 0.0;
    for (int j = 1; j <= reps; ++j) {
        float t = 0.0f;
        QMB_CUDA_TRY(cudaEventElapsedTime(&t, ev[2 * j], ev[2 * j + 1]));
        ms += t;
    }
    return ms / reps;
}
}  // namespace qmb

extern "C" qmb_status qmb_batch_k1_time(qmb_batch b, int prec, int reps, double* ms, double* bytes) {
    return guarded([&] {
        QMB_REQUIRE(b && ms && bytes, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(prec == QMB_PREC_FP64 || prec == QMB_PREC_FP32, QMB_ERR_INVALID, "bad prec");
        QMB_REQUIRE(reps >= 1 && reps <= 1000, QMB_ERR_INVALID, "reps must be in 1..1000");
        DeviceGuard dg(b->device);
        const bool f64 = prec == QMB_PREC_FP64;
        cudaStream_t st;
        QMB_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct SG { cudaStream_t s; ~SG() { cudaStreamDestroy(s); } } sg{st};
        double t = 0.0;
        if (f64) {
            t += k1_kind_ms<double>(b, b->kind[0], true, reps, st);
            t += k1_kind_ms<double2>(b, b->kind[1], true, reps, st);
        } else {
            t += k1_kind_ms<float>(b, b->kind[0], false, reps, st);
            t += k1_kind_ms<float2>(b, b->kind[1], false, reps, st);
        }
        // the product's bytes, plus v_{j-1} read and v_j written per (row, set)
        double extra = 0.0;
        for (int kd = 0; kd < 2; ++kd)
            extra += 2.0 * (double)b->kind[kd].rows * b->n_sets * (f64 ? 8.0 : 4.0) * (kd ? 2 : 1);
        *ms = t;
        *bytes = batch_bytes(b, f64) + extra;
    });
}

extern "C" qmb_status qmb_batch_solve(qmb_batch b, const double* c_xy, const double* c_z,
                                      const qmb_lanczos_opts* opts, double* E0,
                                      qmb_lanczos_result* summary) {
    return guarded([&] {
        QMB_REQUIRE(b && c_xy && c_z && opts && E0, QMB_ERR_INVALID, "null argument");
        const qmb_lanczos_opts& o = *opts;
        QMB_REQUIRE(o.mode >= 0 && o.mode <= 2, QMB_ERR_INVALID, "unknown mode");
        QMB_REQUIRE(o.max_iter >= 1 && o.max_iter <= 1024, QMB_ERR_INVALID, "max_iter must be in 1..1024");
        QMB_REQUIRE(o.reorth == 0, QMB_ERR_UNSUPPORTED, "batched solves run without reorthogonalisation");
        DeviceGuard dg(b->device);
        cudaStream_t st;
        QMB_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct SG { cudaStream_t s; ~SG() { cudaStreamDestroy(s); } } sg{st};
        cudaEvent_t e0, e1;
        QMB_CUDA_TRY(cudaEventCreate(&e0));
        QMB_CUDA_TRY(cudaEventCreate(&e1));
        struct EG { cudaEvent_t a, c; ~EG() { cudaEventDestroy(a); cudaEventDestroy(c); } } eg{e0, e1};
        QMB_CUDA_TRY(cudaEventRecord(e0, st));
        // couplings (padded sets repeat the last set)
        std::vector<double> hx(b->nsp), hz(b->nsp);
        for (int i = 0; i < b->nsp; ++i) {
            int src = std::min(i, b->n_sets - 1);
            hx[i] = c_xy[src];
            hz[i] = c_z[src];
            QMB_REQUIRE(std::isfinite(hx[i]) && std::isfinite(hz[i]), QMB_ERR_INVALID, "non-finite coupling");
        }
        b->cxy.upload(hx.data(), b->nsp, st);
        b->cz.upload(hz.data(), b->nsp, st);
        const int check = o.check_every > 0 ? o.check_every : 10;
        const double tol64 = o.tol > 0 ? o.tol : 1e-12;
        g_kernels = 0;
        b->ws.next = 0;
        g_ws = &b->ws;
        struct WsGuard {
            ~WsGuard() { g_ws = nullptr; }
        } ws_guard;
        int n_hv = 0, it_low = 0, it_tot = 0;
        double products = 0;
        bool all_conv = true;
        std::vector<double> result(b->n_sectors * (size_t)b->n_sets, 0.0), low(result.size(), 0.0);
        const auto t_solve = std::chrono::steady_clock::now();
        auto solve_ms = [&]() {
            return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_solve).count();
        };
        for (int kd = 0; kd < 2; ++kd) {
            BKind& k = b->kind[kd];
            if (!k.n_sectors) continue;
            if (trace_on()) std::fprintf(stderr, "[qmb batch] kind %d starts at %.2f ms\n", kd, solve_ms());
            const int64_t tot = k.sec_elem[k.n_sectors];
            const int n_prob = k.n_sectors * b->nsp;
            int64_t minrows = INT64_MAX;
            for (auto r : k.nrows) minrows = std::min(minrows, r);
            BPhase ph;
            if (o.mode == QMB_MODE_FP64) {
                ph = kd ? run_bphase<double2>(b, k, true, o.max_iter, 0.0, 0.0, tol64, nullptr, nullptr, check, 0, o.seed, nullptr, nullptr, 0, n_hv, st)
                        : run_bphase<double>(b, k, true, o.max_iter, 0.0, 0.0, tol64, nullptr, nullptr, check, 0, o.seed, nullptr, nullptr, 0, n_hv, st);
                it_tot = std::max(it_tot, ph.steps);
                it_low = it_tot;
                products += ph.products;
            } else {
                Buf<unsigned char> psi = ws_take<unsigned char>(tot * (kd ? 16 : 8));
                const int slots = o.mode == QMB_MODE_MIXED ? krylov_slots((size_t)tot * (kd ? 8 : 4), o.max_iter + 1, k.ws_ring.n) : 0;
                Buf<double> gapb = ws_take<double>((size_t)k.n_sectors * b->nsp);
                gapb.zero(st);
                void* psi_out = o.mode == QMB_MODE_MIXED ? (void*)psi.p : nullptr;
                // FP32 phase: Ritz pair accurate enough that the FP64 restart
                // needs few steps (residual or energy bound)
                BPhase p1 = kd ? run_bphase<float2>(b, k, false, o.max_iter, 0.0, 1e-6, 1e-9, nullptr, gapb.p, check, 0, o.seed, nullptr, psi_out, slots, n_hv, st)
                               : run_bphase<float>(b, k, false, o.max_iter, 0.0, 1e-6, 1e-9, nullptr, gapb.p, check, 0, o.seed, nullptr, psi_out, slots, n_hv, st);
                it_low = std::max(it_low, p1.steps);
                products += p1.products;
                for (int s = 0; s < k.n_sectors; ++s)
                    for (int set = 0; set < b->n_sets; ++set)
                        low[(size_t)set * b->n_sectors + k.sec_index[s]] = p1.theta[(size_t)s * b->nsp + set];
                ph = p1;
                it_tot = std::max(it_tot, p1.steps);
                if (o.mode == QMB_MODE_MIXED) {
                    if (trace_on()) {
                        std::fprintf(stderr, "[qmb batch] fp32 phase returned at %.2f ms\n", solve_ms());
                        // steps each problem needed, and the last step of each sector
                        int hist[8] = {0};
                        std::string smax;
                        for (int s = 0; s < k.n_sectors; ++s) {
                            int mx = 0;
                            for (int set = 0; set < b->n_sets; ++set) {
                                const int m = p1.msteps[(size_t)s * b->nsp + set];
                                mx = std::max(mx, m);
                                hist[std::min(7, m / 20)]++;
                            }
                            smax += " " + std::to_string(mx);
                        }
                        std::fprintf(stderr, "[qmb batch] fp32 steps per problem 0-19..140+: %d %d %d %d %d %d %d %d; "
                                     "per sector max:%s\n", hist[0], hist[1], hist[2], hist[3], hist[4], hist[5],
                                     hist[6], hist[7], smax.c_str());
                    }
                    // zero-step check: FP64 Rayleigh quotient and residual of the
                    // FP32 Ritz vectors; accepted problems need no FP64 steps
                    const int n_prob = k.n_sectors * b->nsp;
                    std::vector<double> e_rq(n_prob);
                    std::vector<int> act(k.n_sectors, 0);
                    Buf<int> act_d = ws_take<int>(k.n_sectors),
                        ok = ws_take<int>(n_prob);
                    {
                        BatchArgs a = make_args(b, k);
                        a.val = k.val64.p;
                        a.dxy = k.dxy64.p;
                        a.dz = k.dz64.p;
                        Buf<unsigned char> hy = ws_take<unsigned char>(tot * (kd ? 16 : 8));
                        Buf<double> part = ws_take<double>(2 * (size_t)k.n_tiles * b->nsp),
                            sums = ws_take<double>(2 * (size_t)n_prob),
                            Eq = ws_take<double>(n_prob),
                            r2 = ws_take<double>(2 * (size_t)n_prob);
                        BLz lz0{nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, nullptr};
                        std::vector<int> ones(k.n_sectors, 1);
                        k.d_active.upload(ones.data(), k.n_sectors, st);
                        const int rb2 = 256, rg2 = (n_prob + 255) / 256;
                        if (kd) {
                            tuned_variant<double2>(a, k, true, st);
                            bhv_any<double2>(a, k, (const double2*)psi.p, (double2*)hy.p, nullptr, 1, lz0, nullptr, nullptr, 0, st);
                            g_kernels += 1;
                            k_bdot<double2><<<k.n_tiles, b->nsp, 0, st>>>(a, k.n_tiles, (const double2*)psi.p, (const double2*)hy.p, nullptr, part.p);
                        } else {
                            tuned_variant<double>(a, k, true, st);
                            bhv_any<double>(a, k, (const double*)psi.p, (double*)hy.p, nullptr, 1, lz0, nullptr, nullptr, 0, st);
                            g_kernels += 1;
                            k_bdot<double><<<k.n_tiles, b->nsp, 0, st>>>(a, k.n_tiles, (const double*)psi.p, (const double*)hy.p, nullptr, part.p);
                        }
                        g_kernels += 1;
                        k_bsum<<<rg2, rb2, 0, st>>>(a, k.n_tiles, k.d_sec_tile0.p, k.d_sec_ntiles.p, part.p, 2, n_prob, sums.p);
                        g_kernels += 1;
                        k_brq_energy<<<rg2, rb2, 0, st>>>(n_prob, sums.p, Eq.p);
                        g_kernels += 1;
                        if (kd) k_bdot<double2><<<k.n_tiles, b->nsp, 0, st>>>(a, k.n_tiles, (const double2*)psi.p, (const double2*)hy.p, Eq.p, part.p);
                        else k_bdot<double><<<k.n_tiles, b->nsp, 0, st>>>(a, k.n_tiles, (const double*)psi.p, (const double*)hy.p, Eq.p, part.p);
                        g_kernels += 1;
                        k_bsum<<<rg2, rb2, 0, st>>>(a, k.n_tiles, k.d_sec_tile0.p, k.d_sec_ntiles.p, part.p, 1, n_prob, r2.p);
                        act_d.zero(st);
                        g_kernels += 1;
                        k_brq_accept<<<rg2, rb2, 0, st>>>(a, n_prob, b->n_sets, Eq.p, r2.p, sums.p + n_prob, gapb.p, tol64,
                                                          restart_gap_cap(), ok.p, act_d.p);
                        check_launch("rq check");
                        if (trace_on()) {
                            QMB_CUDA_TRY(cudaStreamSynchronize(st));
                            std::fprintf(stderr, "[qmb batch] rq kernels done at %.2f ms\n", solve_ms());
                        }
                        Eq.download(e_rq.data(), n_prob, st);
                        act_d.download(act.data(), k.n_sectors, st);
                        QMB_CUDA_TRY(cudaStreamSynchronize(st));
                        if (trace_on()) {
                            std::vector<double> hr2(n_prob), hs(2 * (size_t)n_prob), hg(n_prob);
                            std::vector<int> hok(n_prob);
                            r2.download(hr2.data(), n_prob, st);
                            sums.download(hs.data(), 2 * (size_t)n_prob, st);
                            gapb.download(hg.data(), n_prob, st);
                            ok.download(hok.data(), n_prob, st);
                            QMB_CUDA_TRY(cudaStreamSynchronize(st));
                            int hist[8] = {0}, nacc = 0, nact = 0;
                            double worst = 0;
                            for (int p = 0; p < n_prob; ++p) {
                                if (p % b->nsp >= b->n_sets) continue;
                                double sc = std::max(std::fabs(e_rq[p]), 1e-300);
                                double r = std::sqrt(hr2[p] / std::max(hs[n_prob + p], 1e-300)) / sc;
                                int bin = r <= 0 ? 0 : std::min(7, std::max(0, (int)std::floor(-std::log10(r)) - 3));
                                hist[bin]++;
                                nacc += hok[p];
                                worst = std::max(worst, r * r * sc / std::max(hg[p], 1e-300));
                            }
                            for (int v : act) nact += v;
                            std::fprintf(stderr, "[qmb batch] rq check: accepted %d, sectors left %d/%d, worst r^2/gap/|E| %.2e, "
                                         "r/|E| decades 1e-3..1e-10: %d %d %d %d %d %d %d %d\n",
                                         nacc, nact, k.n_sectors, worst, hist[0], hist[1], hist[2], hist[3], hist[4],
                                         hist[5], hist[6], hist[7]);
                        }
                        ++n_hv;
                    }
                    if (trace_on()) std::fprintf(stderr, "[qmb batch] rq check done at %.2f ms\n", solve_ms());
                    int m2 = o.refine_max_iter > 0 ? o.refine_max_iter : 300;
                    bool any = false;
                    for (int v : act) any |= v != 0;
                    BPhase p2;
                    if (any) {
                        p2 = kd ? run_bphase<double2>(b, k, true, m2, 0.0, 0.0, tol64, gapb.p, nullptr, 4, 2, 0, psi.p, nullptr, 0, n_hv, st, act_d.p)
                                : run_bphase<double>(b, k, true, m2, 0.0, 0.0, tol64, gapb.p, nullptr, 4, 2, 0, psi.p, nullptr, 0, n_hv, st, act_d.p);
                    } else {
                        p2.theta.assign(n_prob, 0.0);
                        p2.conv.assign(n_prob, 1);
                        p2.msteps.assign(n_prob, 0);
                    }
                    if (trace_on() && any) {
                        int hist[8] = {0};
                        for (int s = 0; s < k.n_sectors; ++s)
                            for (int set = 0; set < b->n_sets; ++set)
                                hist[std::min(7, p2.msteps[(size_t)s * b->nsp + set] / 8)]++;
                        std::fprintf(stderr, "[qmb batch] restart steps per problem 0-7..56+: %d %d %d %d %d %d %d %d\n",
                                     hist[0], hist[1], hist[2], hist[3], hist[4], hist[5], hist[6], hist[7]);
                    }
                    // sectors that skipped the restart keep the Rayleigh quotient
                    for (int s = 0; s < k.n_sectors; ++s)
                        if (!act[s])
                            for (int set = 0; set < b->nsp; ++set) {
                                p2.theta[(size_t)s * b->nsp + set] = e_rq[(size_t)s * b->nsp + set];
                                p2.conv[(size_t)s * b->nsp + set] = 1;
                            }
                    it_tot = std::max(it_tot, p1.steps + p2.steps);
                    products += p2.products;
                    ph = p2;
                }
            }
            for (int s = 0; s < k.n_sectors; ++s)
                for (int set = 0; set < b->n_sets; ++set) {
                    size_t p = (size_t)s * b->nsp + set;
                    result[(size_t)set * b->n_sectors + k.sec_index[s]] = ph.theta[p];
                    if (!ph.conv[p]) all_conv = false;
                }
            (void)n_prob;
        }
        QMB_CUDA_TRY(cudaEventRecord(e1, st));
        QMB_CUDA_TRY(cudaEventSynchronize(e1));
        std::memcpy(E0, result.data(), sizeof(double) * result.size());
        if (summary) {
            std::memset(summary, 0, sizeof(*summary));
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            summary->ms_total = ms;
            summary->ms_hv = -1;
            summary->iters = it_tot;
            summary->iters_low = it_low;
            summary->n_hv = n_hv;
            summary->n_products = products;
            summary->n_launches = g_kernels;
            summary->converged = all_conv ? 1 : 0;
            summary->E0 = *std::min_element(result.begin(), result.end());
            summary->E0_low = o.mode == QMB_MODE_FP64 ? summary->E0 : *std::min_element(low.begin(), low.end());
            summary->residual = -1;
            summary->residual_ref = -1;
        }
    });
}
