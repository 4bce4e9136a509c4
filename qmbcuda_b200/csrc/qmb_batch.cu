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
#include <memory>

#include "qmb_ham.cuh"
#include "qmb_lanczos.cuh"

namespace qmb {

constexpr int kBWarps = 8;          // warps per block
constexpr int kBRowsPerWarp = 8;    // rows per warp per tile
constexpr int kBTile = kBWarps * kBRowsPerWarp;

struct BatchArgs {
    int n_sectors;
    int nsp;                     // padded sets (multiple of 32*SPL)
    int n_groups;                // set groups of 32*SPL
    const int* tile_sector;      // [n_tiles]
    const int* tile_row0;        // [n_tiles]
    const int64_t* sec_elem;     // [n_sectors+1] element offset (rows*nsp)
    const int64_t* sec_nrows;    // [n_sectors]
    const int64_t* row_ptr;      // concatenated CSR row pointers (global entry index)
    const int64_t* row_base;     // [n_sectors] index of the sector's first row in row_ptr
    const uint32_t* col;
    const void* val;             // double/double2/float/float2 per sector kind
    const void* dxy;             // diagonal of A  [rows]
    const void* dz;              // diagonal of D  [rows]
    const double* cxy;           // [nsp]
    const double* cz;            // [nsp]
    const int* active;           // [n_sectors]
};

// Per sector, real and complex storage live in separate arrays; a kernel
// launch covers sectors of one kind (kind 0 real, 1 complex).
template <class V>
struct VecN {
    V v[8];
};

template <class V, class M, int SPL>
__device__ __forceinline__ void load_sets(const V* __restrict__ p, V (&o)[SPL]) {
#pragma unroll
    for (int q = 0; q < SPL; ++q) o[q] = p[q];
}

// K1 (batched): y = H w_j / beta_j - beta_j v_{j-1}; v_j = w_j / beta_j;
// alpha partials per (tile, set).  Also plain y = H x when lz == nullptr.
struct BLz {
    double* alpha;      // [cap][n_prob]
    double* beta;       // [cap+1][n_prob]
    double* partials;   // [n_tiles][nsp]
    int* iter;
    int n_prob;
};

template <class V, int SPL>
__global__ void __launch_bounds__(kBWarps * 32) k_bhv(BatchArgs a, const int* __restrict__ tiles,
                                                      int n_tiles, const V* __restrict__ X0,
                                                      V* __restrict__ Y0, V* __restrict__ vring,
                                                      int K, BLz lz, const double* __restrict__ ritz,
                                                      void* psi_v, int lanczos) {
    using M = V;
    __shared__ double red[kBWarps][32 * SPL];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ti = blockIdx.x / a.n_groups;
    const int grp = blockIdx.x % a.n_groups;
    if (ti >= n_tiles) return;
    const int tile = tiles[ti];
    const int s = a.tile_sector[tile];
    if (lanczos && !a.active[s]) return;
    const int64_t nrows = a.sec_nrows[s];
    const int nsp = a.nsp;
    const int set0 = grp * 32 * SPL + lane * SPL;
    const int j = lanczos ? *lz.iter : 0;
    const int64_t eo = a.sec_elem[s];
    const V* X = X0 + (lanczos ? (int64_t)(j & 1) * a.sec_elem[a.n_sectors] : 0) + eo;
    V* Y = Y0 + (lanczos ? (int64_t)((j + 1) & 1) * a.sec_elem[a.n_sectors] : 0) + eo;
    const int64_t tot = a.sec_elem[a.n_sectors];
    V* Vc = lanczos ? vring + (int64_t)(j % K) * tot + eo : nullptr;
    const V* Vp = lanczos ? vring + (int64_t)((j + K - 1) % K) * tot + eo : nullptr;
    const M* val = reinterpret_cast<const M*>(a.val);
    const M* dxy = reinterpret_cast<const M*>(a.dxy);
    const M* dz = reinterpret_cast<const M*>(a.dz);
    double cx[SPL], cz[SPL], bj[SPL], inv[SPL], cr[SPL], apar[SPL];
    const int prob0 = s * nsp + set0;
#pragma unroll
    for (int q = 0; q < SPL; ++q) {
        cx[q] = a.cxy[set0 + q];
        cz[q] = a.cz[set0 + q];
        bj[q] = lanczos ? lz.beta[(int64_t)j * lz.n_prob + prob0 + q] : 1.0;
        inv[q] = 1.0 / bj[q];
        cr[q] = ritz ? ritz[(int64_t)j * lz.n_prob + prob0 + q] : 0.0;
        apar[q] = 0.0;
    }
    const int64_t rb = a.row_base[s];
    const int r_begin = a.tile_row0[tile] + warp * kBRowsPerWarp;
    for (int rr = 0; rr < kBRowsPerWarp; ++rr) {
        const int64_t r = r_begin + rr;
        if (r >= nrows) break;
        V acc[SPL];
#pragma unroll
        for (int q = 0; q < SPL; ++q) acc[q] = Sc<V>::zero();
        const int64_t p0 = a.row_ptr[rb + r], p1 = a.row_ptr[rb + r + 1];
        for (int64_t pc = p0; pc < p1; pc += 32) {
            int cnt = (int)min((int64_t)32, p1 - pc);
            uint32_t mc = 0;
            M mv = Sc<M>::zero();
            if (lane < cnt) {
                mc = a.col[pc + lane];
                mv = val[pc + lane];
            }
            for (int k = 0; k < cnt; ++k) {
                uint32_t c = __shfl_sync(0xffffffffu, mc, k);
                M v;
                if constexpr (Sc<M>::cplx) {
                    v.x = __shfl_sync(0xffffffffu, mv.x, k);
                    v.y = __shfl_sync(0xffffffffu, mv.y, k);
                } else {
                    v = __shfl_sync(0xffffffffu, mv, k);
                }
                const V* xp = X + (int64_t)c * nsp + set0;
                V xv[SPL];
                load_sets<V, M, SPL>(xp, xv);
#pragma unroll
                for (int q = 0; q < SPL; ++q) acc[q] = Sc<V>::fma(v, xv[q], acc[q]);
            }
        }
        V xr[SPL];
        load_sets<V, M, SPL>(X + r * nsp + set0, xr);
        const M dx = dxy[rb + r], dzz = dz[rb + r];
        V vp[SPL];
        if (lanczos && j > 0) load_sets<V, M, SPL>(Vp + r * nsp + set0, vp);
#pragma unroll
        for (int q = 0; q < SPL; ++q) {
            V hx = Sc<V>::add(Sc<V>::scale(Sc<V>::fma(dx, xr[q], acc[q]), cx[q]),
                              Sc<V>::scale(Sc<V>::mul(dzz, xr[q]), cz[q]));
            if (!lanczos) {
                Y[r * nsp + set0 + q] = hx;
                continue;
            }
            V vj = Sc<V>::scale(xr[q], inv[q]);
            V y = Sc<V>::scale(hx, inv[q]);
            if (j > 0) y = Sc<V>::sub(y, Sc<V>::scale(vp[q], bj[q]));
            Vc[r * nsp + set0 + q] = vj;
            Y[r * nsp + set0 + q] = y;
            apar[q] += Sc<V>::re_conj_mul(vj, y);
            if (psi_v && cr[q] != 0.0) {
                double* ps = reinterpret_cast<double*>(psi_v);
                if constexpr (Sc<V>::cplx) {
                    double2* p2 = reinterpret_cast<double2*>(psi_v) + eo + r * nsp + set0 + q;
                    double2 t = cvt<double2>(vj);
                    p2->x += cr[q] * t.x;
                    p2->y += cr[q] * t.y;
                } else {
                    ps[eo + r * nsp + set0 + q] += cr[q] * (double)vj;
                }
            }
        }
    }
    if (!lanczos) return;
#pragma unroll
    for (int q = 0; q < SPL; ++q) red[warp][lane * SPL + q] = apar[q];
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * SPL; i += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < kBWarps; ++w) t += red[w][i];
        lz.partials[(int64_t)tile * nsp + grp * 32 * SPL + i] = t;
    }
}

// K2 (batched): w_{j+1} = y - alpha_j v_j; ||w_{j+1}||^2 partials.
template <class V, int SPL>
__global__ void __launch_bounds__(kBWarps * 32) k_bupdate(BatchArgs a, const int* __restrict__ tiles,
                                                          int n_tiles, V* __restrict__ W0,
                                                          const V* __restrict__ vring, int K, BLz lz) {
    __shared__ double red[kBWarps][32 * SPL];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ti = blockIdx.x / a.n_groups;
    const int grp = blockIdx.x % a.n_groups;
    if (ti >= n_tiles) return;
    const int tile = tiles[ti];
    const int s = a.tile_sector[tile];
    if (!a.active[s]) return;
    const int64_t nrows = a.sec_nrows[s];
    const int nsp = a.nsp;
    const int set0 = grp * 32 * SPL + lane * SPL;
    const int j = *lz.iter;
    const int64_t tot = a.sec_elem[a.n_sectors];
    const int64_t eo = a.sec_elem[s];
    V* Y = W0 + (int64_t)((j + 1) & 1) * tot + eo;
    const V* Vc = vring + (int64_t)(j % K) * tot + eo;
    double al[SPL], acc[SPL];
#pragma unroll
    for (int q = 0; q < SPL; ++q) {
        al[q] = lz.alpha[(int64_t)j * lz.n_prob + s * nsp + set0 + q];
        acc[q] = 0.0;
    }
    const int r_begin = a.tile_row0[tile] + warp * kBRowsPerWarp;
    for (int rr = 0; rr < kBRowsPerWarp; ++rr) {
        const int64_t r = r_begin + rr;
        if (r >= nrows) break;
#pragma unroll
        for (int q = 0; q < SPL; ++q) {
            int64_t e = r * nsp + set0 + q;
            V y = Sc<V>::sub(Y[e], Sc<V>::scale(Vc[e], al[q]));
            Y[e] = y;
            acc[q] += Sc<V>::abs2(y);
        }
    }
#pragma unroll
    for (int q = 0; q < SPL; ++q) red[warp][lane * SPL + q] = acc[q];
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * SPL; i += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < kBWarps; ++w) t += red[w][i];
        lz.partials[(int64_t)tile * nsp + grp * 32 * SPL + i] = t;
    }
}

// Sums the tile partials of every problem in tile order.  what 0: alpha[j],
// 1: beta[j+1] = sqrt(sum) and the step advances (thread 0).
__global__ void k_breduce(BatchArgs a, const int* __restrict__ sec_tile0,
                          const int* __restrict__ sec_ntiles, BLz lz, int what) {
    const int j = *lz.iter;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < lz.n_prob; p += gridDim.x * blockDim.x) {
        int s = p / a.nsp, set = p % a.nsp;
        if (!a.active[s]) continue;
        double t = 0.0;
        int t0 = sec_tile0[s], nt = sec_ntiles[s];
        for (int k = 0; k < nt; ++k) t += lz.partials[(int64_t)(t0 + k) * a.nsp + set];
        if (what == 0) lz.alpha[(int64_t)j * lz.n_prob + p] = t;
        else lz.beta[(int64_t)(j + 1) * lz.n_prob + p] = sqrt(t);
    }
}

__global__ void k_badvance(BLz lz) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *lz.iter += 1;
}

// Start vectors (splitmix uniform(-1,1) or a copy) and beta_0 per problem.
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

// ||w0||^2 partials per (tile, set), reusing the update kernel's layout.
template <class V, int SPL>
__global__ void __launch_bounds__(kBWarps * 32) k_bnorm0(BatchArgs a, const int* __restrict__ tiles,
                                                         int n_tiles, const V* __restrict__ W0, BLz lz) {
    __shared__ double red[kBWarps][32 * SPL];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ti = blockIdx.x / a.n_groups;
    const int grp = blockIdx.x % a.n_groups;
    if (ti >= n_tiles) return;
    const int tile = tiles[ti];
    const int s = a.tile_sector[tile];
    const int64_t nrows = a.sec_nrows[s];
    const int nsp = a.nsp;
    const int set0 = grp * 32 * SPL + lane * SPL;
    const V* X = W0 + a.sec_elem[s];
    double acc[SPL];
#pragma unroll
    for (int q = 0; q < SPL; ++q) acc[q] = 0.0;
    const int r_begin = a.tile_row0[tile] + warp * kBRowsPerWarp;
    for (int rr = 0; rr < kBRowsPerWarp; ++rr) {
        const int64_t r = r_begin + rr;
        if (r >= nrows) break;
#pragma unroll
        for (int q = 0; q < SPL; ++q) acc[q] += Sc<V>::abs2(X[r * nsp + set0 + q]);
    }
#pragma unroll
    for (int q = 0; q < SPL; ++q) red[warp][lane * SPL + q] = acc[q];
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * SPL; i += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < kBWarps; ++w) t += red[w][i];
        lz.partials[(int64_t)tile * nsp + grp * 32 * SPL + i] = t;
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
__device__ double bis_min(const double* al, const double* be, int n_prob, int p, int m) {
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
        if (cnt >= 1) hi = x;
        else lo = x;
        if (hi - lo <= 4.5e-16 * fmax(fabs(lo), fabs(hi))) break;
    }
    return 0.5 * (lo + hi);
}

__global__ void k_bcheck(BatchArgs a, BLz lz, int nsets, double stall, double tol,
                         double* __restrict__ theta, double* __restrict__ theta_prev,
                         int* __restrict__ msteps, int* __restrict__ conv, int* __restrict__ active_next) {
    const int m = *lz.iter;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < lz.n_prob; p += gridDim.x * blockDim.x) {
        int s = p / a.nsp, set = p % a.nsp;
        if (!a.active[s] || conv[p]) continue;
        msteps[p] = m;
        double th = bis_min(lz.alpha, lz.beta, lz.n_prob, p, m);
        double prev = theta_prev[p];
        theta[p] = th;
        double sc = fmax(fabs(th), 1e-300);
        double bm = lz.beta[(int64_t)m * lz.n_prob + p];
        bool done = (fabs(th - prev) <= stall * sc) || (bm <= 1e-13 * sc);
        (void)tol;
        conv[p] = done ? 1 : 0;
        theta_prev[p] = th;
        if (!done && set < nsets) atomicOr(active_next + s, 1);
    }
}

// Ritz coefficients of every problem: inverse iteration on T_m - theta I
// (LDL^T without pivoting, tiny pivots replaced).  Scratch arrays [i][p].
__global__ void k_britz(BLz lz, const int* __restrict__ msteps, const double* __restrict__ theta,
                        double* __restrict__ L, double* __restrict__ D, double* __restrict__ ritz) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < lz.n_prob; p += gridDim.x * blockDim.x) {
        const int np = lz.n_prob;
        const int m = msteps[p];
        const double th = theta[p];
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
        for (int i = 0; i < m; ++i) ritz[(int64_t)i * np + p] = 1.0;
        for (int it = 0; it < 2; ++it) {
            // forward: y_{i+1} = b_{i+1} - l_i y_i
            for (int i = 1; i < m; ++i)
                ritz[(int64_t)i * np + p] -= L[(int64_t)(i - 1) * np + p] * ritz[(int64_t)(i - 1) * np + p];
            for (int i = 0; i < m; ++i) ritz[(int64_t)i * np + p] /= D[(int64_t)i * np + p];
            for (int i = m - 2; i >= 0; --i)
                ritz[(int64_t)i * np + p] -= L[(int64_t)i * np + p] * ritz[(int64_t)(i + 1) * np + p];
            double nrm = 0.0;
            for (int i = 0; i < m; ++i) nrm += ritz[(int64_t)i * np + p] * ritz[(int64_t)i * np + p];
            nrm = sqrt(nrm);
            double sg = ritz[p] < 0 ? -1.0 : 1.0;
            for (int i = 0; i < m; ++i) ritz[(int64_t)i * np + p] *= sg / nrm;
        }
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
    DevBuf<int64_t> d_sec_elem, d_nrows, d_row_ptr, d_row_base;
    DevBuf<uint32_t> d_col;
    DevBuf<unsigned char> val64, val32, dxy64, dxy32, dz64, dz32;
    int64_t nnz = 0, rows = 0;
    int n_tiles = 0;
};

struct qmb_batch_s {
    int device = 0;
    int n_sectors = 0, n_sets = 0, nsp = 0, spl = 8, n_groups = 1;
    BKind kind[2];  // 0 real, 1 complex
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
    a.col = k.d_col.p;
    a.val = nullptr;
    a.dxy = nullptr;
    a.dz = nullptr;
    a.cxy = b->cxy.p;
    a.cz = b->cz.p;
    a.active = k.d_active.p;
    return a;
}

template <class V, int SPL>
static void launch_bhv(const BatchArgs& a, const BKind& k, const V* x, V* y, V* vring, int K,
                       BLz lz, const double* ritz, void* psi, int lanczos, cudaStream_t st) {
    int blocks = k.n_tiles * a.n_groups;
    if (blocks == 0) return;
    k_bhv<V, SPL><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, x, y, vring, K, lz,
                                                    ritz, psi, lanczos);
}

template <class V>
static void bhv_any(int spl, const BatchArgs& a, const BKind& k, const V* x, V* y, V* vring, int K,
                    BLz lz, const double* ritz, void* psi, int lanczos, cudaStream_t st) {
    switch (spl) {
        case 1: launch_bhv<V, 1>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st); break;
        case 2: launch_bhv<V, 2>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st); break;
        case 4: launch_bhv<V, 4>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st); break;
        default: launch_bhv<V, 8>(a, k, x, y, vring, K, lz, ritz, psi, lanczos, st); break;
    }
}

template <class V>
static void bupdate_any(int spl, const BatchArgs& a, const BKind& k, V* w, const V* vring, int K,
                        BLz lz, cudaStream_t st) {
    int blocks = k.n_tiles * a.n_groups;
    if (blocks == 0) return;
    switch (spl) {
        case 1: k_bupdate<V, 1><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, vring, K, lz); break;
        case 2: k_bupdate<V, 2><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, vring, K, lz); break;
        case 4: k_bupdate<V, 4><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, vring, K, lz); break;
        default: k_bupdate<V, 8><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, vring, K, lz); break;
    }
}

template <class V>
static void bnorm0_any(int spl, const BatchArgs& a, const BKind& k, const V* w, BLz lz, cudaStream_t st) {
    int blocks = k.n_tiles * a.n_groups;
    if (blocks == 0) return;
    switch (spl) {
        case 1: k_bnorm0<V, 1><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, lz); break;
        case 2: k_bnorm0<V, 2><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, lz); break;
        case 4: k_bnorm0<V, 4><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, lz); break;
        default: k_bnorm0<V, 8><<<blocks, kBWarps * 32, 0, st>>>(a, k.d_tiles.p, k.n_tiles, w, lz); break;
    }
}

struct BPhase {
    std::vector<double> theta;   // [n_prob]
    std::vector<int> msteps, conv;
    int steps = 0;
};

// Batched Lanczos phase over one kind with vectors V (and matrix values of
// the same precision).  start: 0 splitmix (seed), 2 copy of psi_in (FP64).
template <class V>
static BPhase run_bphase(qmb_batch_s* b, BKind& k, bool f64, int max_iter, double stall, int check,
                         int start, uint64_t seed, const void* psi_in, void* psi_out, bool store,
                         int& n_hv, cudaStream_t st) {
    BPhase out;
    const int64_t tot = k.sec_elem[k.n_sectors];
    const int n_prob = k.n_sectors * b->nsp;
    int64_t minrows = INT64_MAX;
    for (auto r : k.nrows) minrows = std::min(minrows, r);
    const int cap = std::max(1, (int)std::min<int64_t>(max_iter, minrows));
    const int K = store ? cap + 1 : 2;
    DevBuf<V> wbuf(2 * (size_t)tot), vring((size_t)K * tot);
    DevBuf<double> alpha((size_t)(cap + 1) * n_prob), beta((size_t)(cap + 2) * n_prob),
        partials((size_t)std::max(1, k.n_tiles) * b->nsp), theta(n_prob), theta_prev(n_prob),
        ritz((size_t)(cap + 1) * n_prob), Ls((size_t)(cap + 1) * n_prob), Ds((size_t)(cap + 1) * n_prob);
    DevBuf<int> iter(1), msteps(n_prob), conv(n_prob), active_next(k.n_sectors);
    QMB_CUDA_TRY(cudaMemsetAsync(theta_prev.p, 0, sizeof(double) * n_prob, st));
    QMB_CUDA_TRY(cudaMemsetAsync(conv.p, 0, sizeof(int) * n_prob, st));
    QMB_CUDA_TRY(cudaMemsetAsync(ritz.p, 0, ritz.n * sizeof(double), st));
    QMB_CUDA_TRY(cudaMemsetAsync(alpha.p, 0, alpha.n * sizeof(double), st));
    QMB_CUDA_TRY(cudaMemsetAsync(beta.p, 0, beta.n * sizeof(double), st));
    std::vector<int> ones(k.n_sectors, 1);
    k.d_active.upload(ones.data(), k.n_sectors, st);
    BatchArgs a = make_args(b, k);
    a.val = f64 ? k.val64.p : k.val32.p;
    a.dxy = f64 ? k.dxy64.p : k.dxy32.p;
    a.dz = f64 ? k.dz64.p : k.dz32.p;
    BLz lz{alpha.p, beta.p, partials.p, iter.p, n_prob};
    const int rb = 256, rg = (n_prob + rb - 1) / rb;
    k_bstart<V><<<grid_for(tot, 256), 256, 0, st>>>(a, tot, start, seed, psi_in, wbuf.p);
    bnorm0_any<V>(b->spl, a, k, wbuf.p, lz, st);
    k_bbeta0<<<rg, rb, 0, st>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz);
    check_launch("batch start");
    auto step = [&](cudaStream_t ss) {
        bhv_any<V>(b->spl, a, k, wbuf.p, wbuf.p, vring.p, K, lz, nullptr, nullptr, 1, ss);
        k_breduce<<<rg, rb, 0, ss>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz, 0);
        bupdate_any<V>(b->spl, a, k, wbuf.p, vring.p, K, lz, ss);
        k_breduce<<<rg, rb, 0, ss>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz, 1);
        k_badvance<<<1, 32, 0, ss>>>(lz);
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    QMB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    step(st);
    if (cudaStreamEndCapture(st, &graph) == cudaSuccess) {
        if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) exec = nullptr;
    }
    cudaGetLastError();
    int done = 0;
    std::vector<int> act(k.n_sectors);
    while (done < cap) {
        int todo = std::min(std::max(1, check), cap - done);
        for (int t = 0; t < todo; ++t) {
            if (exec) QMB_CUDA_TRY(cudaGraphLaunch(exec, st));
            else step(st);
        }
        check_launch("batch step");
        done += todo;
        n_hv += todo;
        QMB_CUDA_TRY(cudaMemsetAsync(active_next.p, 0, sizeof(int) * k.n_sectors, st));
        k_bcheck<<<rg, rb, 0, st>>>(a, lz, b->n_sets, stall, 0.0, theta.p, theta_prev.p, msteps.p,
                                    conv.p, active_next.p);
        QMB_CUDA_TRY(cudaMemcpyAsync(k.d_active.p, active_next.p, sizeof(int) * k.n_sectors,
                                     cudaMemcpyDeviceToDevice, st));
        active_next.download(act.data(), k.n_sectors, st);
        QMB_CUDA_TRY(cudaStreamSynchronize(st));
        bool any = false;
        for (int v : act) any |= v != 0;
        if (!any) break;
    }
    out.steps = done;
    // Ritz vectors (FP64) for the next phase or the caller
    if (psi_out) {
        k_britz<<<rg, rb, 0, st>>>(lz, msteps.p, theta.p, Ls.p, Ds.p, ritz.p);
        if (store) {
            k_bpsi<V><<<grid_for(tot, 256), 256, 0, st>>>(a, tot, vring.p, K, msteps.p, ritz.p, n_prob,
                                                          psi_out);
        } else {
            QMB_CUDA_TRY(cudaMemsetAsync(psi_out, 0, (Sc<V>::cplx ? 16 : 8) * tot, st));
            std::vector<int> all(k.n_sectors, 1);
            k.d_active.upload(all.data(), k.n_sectors, st);
            k_bstart<V><<<grid_for(tot, 256), 256, 0, st>>>(a, tot, start, seed, psi_in, wbuf.p);
            bnorm0_any<V>(b->spl, a, k, wbuf.p, lz, st);
            k_bbeta0<<<rg, rb, 0, st>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz);
            // regeneration runs every problem to the longest m; coefficients
            // beyond a problem's own m are zero (k_britz wrote m entries)
            for (int j = 0; j < done; ++j) {
                bhv_any<V>(b->spl, a, k, wbuf.p, wbuf.p, vring.p, K, lz, ritz.p, psi_out, 1, st);
                k_breduce<<<rg, rb, 0, st>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz, 0);
                bupdate_any<V>(b->spl, a, k, wbuf.p, vring.p, K, lz, st);
                k_breduce<<<rg, rb, 0, st>>>(a, k.d_sec_tile0.p, k.d_sec_ntiles.p, lz, 1);
                k_badvance<<<1, 32, 0, st>>>(lz);
                ++n_hv;
            }
        }
        check_launch("batch ritz");
    }
    out.theta.resize(n_prob);
    out.msteps.resize(n_prob);
    out.conv.resize(n_prob);
    theta.download(out.theta.data(), n_prob, st);
    msteps.download(out.msteps.data(), n_prob, st);
    conv.download(out.conv.data(), n_prob, st);
    QMB_CUDA_TRY(cudaStreamSynchronize(st));
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
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
        int spl = 1;
        while (32 * spl < d->n_sets && spl < 8) spl *= 2;
        b->spl = spl;
        b->n_groups = (d->n_sets + 32 * spl - 1) / (32 * spl);
        b->nsp = b->n_groups * 32 * spl;
        b->sector_kind.resize(d->n_sectors);
        b->sector_pos.resize(d->n_sectors);
        // per-sector matrices through the single-sector builder
        struct Part {
            std::vector<int64_t> row_ptr;
            std::vector<uint32_t> col;
            std::vector<double2> val;
            std::vector<double2> dxy, dz;
        };
        std::vector<Part> parts(d->n_sectors);
        for (int s = 0; s < d->n_sectors; ++s) {
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
            const int64_t n = hx->n;
            bool cplx = hx->cplx || hz->cplx;
            b->sector_kind[s] = cplx ? 1 : 0;
            // SELL -> CSR on the host (the shared tables are small)
            std::vector<int64_t> off(hx->n_slices + 1);
            std::vector<int> w(hx->n_slices);
            hx->slice_off.download(off.data(), hx->n_slices + 1);
            hx->slice_w.download(w.data(), hx->n_slices);
            std::vector<uint32_t> col(std::max<int64_t>(hx->padded, 1));
            std::vector<double2> val(std::max<int64_t>(hx->padded, 1));
            std::vector<double2> dx(n), dz(n);
            hx->col.download(col.data(), col.size());
            if (hx->cplx) {
                hx->val64.download(reinterpret_cast<unsigned char*>(val.data()), sizeof(double2) * val.size());
                hx->diag64.download(reinterpret_cast<unsigned char*>(dx.data()), sizeof(double2) * n);
            } else {
                std::vector<double> tv(val.size()), td(n);
                hx->val64.download(reinterpret_cast<unsigned char*>(tv.data()), sizeof(double) * tv.size());
                hx->diag64.download(reinterpret_cast<unsigned char*>(td.data()), sizeof(double) * n);
                for (size_t i = 0; i < tv.size(); ++i) val[i] = make_double2(tv[i], 0.0);
                for (int64_t i = 0; i < n; ++i) dx[i] = make_double2(td[i], 0.0);
            }
            if (hz->cplx) {
                hz->diag64.download(reinterpret_cast<unsigned char*>(dz.data()), sizeof(double2) * n);
            } else {
                std::vector<double> td(n);
                hz->diag64.download(reinterpret_cast<unsigned char*>(td.data()), sizeof(double) * n);
                for (int64_t i = 0; i < n; ++i) dz[i] = make_double2(td[i], 0.0);
            }
            QMB_CUDA_TRY(cudaDeviceSynchronize());
            Part& P = parts[s];
            P.row_ptr.assign(1, 0);
            for (int64_t r = 0; r < n; ++r) {
                int64_t sl = r >> 5, lane = r & 31;
                for (int jj = 0; jj < w[sl]; ++jj) {
                    int64_t pos = off[sl] + (int64_t)jj * 32 + lane;
                    double2 v = val[pos];
                    if (col[pos] == (uint32_t)r && v.x == 0.0 && v.y == 0.0) continue;  // padding
                    P.col.push_back(col[pos]);
                    P.val.push_back(v);
                }
                P.row_ptr.push_back((int64_t)P.col.size());
            }
            P.dxy = std::move(dx);
            P.dz = std::move(dz);
        }
        // assemble the two kinds
        for (int kd = 0; kd < 2; ++kd) {
            BKind& K = b->kind[kd];
            std::vector<int64_t> row_ptr, row_base;
            std::vector<uint32_t> col;
            std::vector<double2> val, dxy, dz;
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
                row_base.push_back((int64_t)row_ptr.size());
                int64_t eb = (int64_t)col.size();
                for (int64_t r = 0; r <= n; ++r) row_ptr.push_back(eb + P.row_ptr[r]);
                col.insert(col.end(), P.col.begin(), P.col.end());
                val.insert(val.end(), P.val.begin(), P.val.end());
                dxy.insert(dxy.end(), P.dxy.begin(), P.dxy.end());
                dz.insert(dz.end(), P.dz.begin(), P.dz.end());
                K.sec_tile0.push_back((int)K.tile_sector.size());
                int nt = (int)((n + kBTile - 1) / kBTile);
                K.sec_ntiles.push_back(nt);
                for (int t = 0; t < nt; ++t) {
                    K.tile_sector.push_back(ks);
                    K.tile_row0.push_back(t * kBTile);
                }
            }
            if (!K.n_sectors) continue;
            K.nnz = (int64_t)col.size();
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
            up_l(K.d_sec_elem, K.sec_elem);
            up_l(K.d_nrows, K.nrows);
            up_l(K.d_row_ptr, row_ptr);
            up_l(K.d_row_base, row_base);
            K.d_col.alloc(std::max<size_t>(1, col.size()));
            if (!col.empty()) K.d_col.upload(col.data(), col.size());
            // values in the sector kind's scalar types
            auto store = [&](DevBuf<unsigned char>& d64, DevBuf<unsigned char>& d32, const std::vector<double2>& v) {
                size_t n = std::max<size_t>(1, v.size());
                if (kd == 1) {
                    std::vector<float2> f(n);
                    for (size_t i = 0; i < v.size(); ++i) f[i] = make_float2((float)v[i].x, (float)v[i].y);
                    d64.alloc(n * sizeof(double2));
                    d32.alloc(n * sizeof(float2));
                    if (!v.empty()) d64.upload(reinterpret_cast<const unsigned char*>(v.data()), v.size() * sizeof(double2));
                    d32.upload(reinterpret_cast<const unsigned char*>(f.data()), n * sizeof(float2));
                } else {
                    std::vector<double> r(n, 0.0);
                    std::vector<float> f(n, 0.0f);
                    for (size_t i = 0; i < v.size(); ++i) { r[i] = v[i].x; f[i] = (float)v[i].x; }
                    d64.alloc(n * sizeof(double));
                    d32.alloc(n * sizeof(float));
                    d64.upload(reinterpret_cast<const unsigned char*>(r.data()), n * sizeof(double));
                    d32.upload(reinterpret_cast<const unsigned char*>(f.data()), n * sizeof(float));
                }
            };
            store(K.val64, K.val32, val);
            store(K.dxy64, K.dxy32, dxy);
            store(K.dz64, K.dz32, dz);
        }
        b->cxy.alloc(b->nsp);
        b->cz.alloc(b->nsp);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
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
    BLz lz{nullptr, nullptr, nullptr, nullptr, 0};
    bhv_any<V>(b->spl, a, k, x, y, nullptr, 1, lz, nullptr, nullptr, 0, st);
    check_launch("k_bhv");
}
}  // namespace qmb

extern "C" qmb_status qmb_batch_hv(qmb_batch b, int prec, const void* x_dev, void* y_dev, void* stream) {
    return guarded([&] {
        QMB_REQUIRE(b && x_dev && y_dev, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(prec == QMB_PREC_FP64 || prec == QMB_PREC_FP32, QMB_ERR_INVALID, "bad prec");
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
        const double stall64 = o.tol > 0 ? o.tol : 1e-12;
        int n_hv = 0, it_low = 0, it_tot = 0;
        bool all_conv = true;
        std::vector<double> result(b->n_sectors * (size_t)b->n_sets, 0.0), low(result.size(), 0.0);
        for (int kd = 0; kd < 2; ++kd) {
            BKind& k = b->kind[kd];
            if (!k.n_sectors) continue;
            const int64_t tot = k.sec_elem[k.n_sectors];
            const int n_prob = k.n_sectors * b->nsp;
            int64_t minrows = INT64_MAX;
            for (auto r : k.nrows) minrows = std::min(minrows, r);
            BPhase ph;
            if (o.mode == QMB_MODE_FP64) {
                int cap = (int)std::min<int64_t>(o.max_iter, minrows);
                bool store = fits_device((size_t)(cap + 4) * tot * (kd ? 16 : 8));
                ph = kd ? run_bphase<double2>(b, k, true, o.max_iter, stall64, check, 0, o.seed, nullptr, nullptr, store, n_hv, st)
                        : run_bphase<double>(b, k, true, o.max_iter, stall64, check, 0, o.seed, nullptr, nullptr, store, n_hv, st);
                it_tot = std::max(it_tot, ph.steps);
                it_low = it_tot;
            } else {
                int cap = (int)std::min<int64_t>(o.max_iter, minrows);
                bool store = fits_device((size_t)(cap + 4) * tot * (kd ? 8 : 4));
                DevBuf<unsigned char> psi(tot * (kd ? 16 : 8));
                double stall32 = 2e-7;
                BPhase p1 = kd ? run_bphase<float2>(b, k, false, o.max_iter, stall32, check, 0, o.seed, nullptr, o.mode == QMB_MODE_MIXED ? psi.p : nullptr, store, n_hv, st)
                               : run_bphase<float>(b, k, false, o.max_iter, stall32, check, 0, o.seed, nullptr, o.mode == QMB_MODE_MIXED ? psi.p : nullptr, store, n_hv, st);
                it_low = std::max(it_low, p1.steps);
                for (int s = 0; s < k.n_sectors; ++s)
                    for (int set = 0; set < b->n_sets; ++set)
                        low[(size_t)set * b->n_sectors + k.sec_index[s]] = p1.theta[(size_t)s * b->nsp + set];
                ph = p1;
                it_tot = std::max(it_tot, p1.steps);
                if (o.mode == QMB_MODE_MIXED) {
                    int m2 = o.refine_max_iter > 0 ? o.refine_max_iter : 60;
                    int cap2 = (int)std::min<int64_t>(m2, minrows);
                    bool store2 = fits_device((size_t)(cap2 + 4) * tot * (kd ? 16 : 8));
                    BPhase p2 = kd ? run_bphase<double2>(b, k, true, m2, stall64, std::min(check, 5), 2, 0, psi.p, nullptr, store2, n_hv, st)
                                   : run_bphase<double>(b, k, true, m2, stall64, std::min(check, 5), 2, 0, psi.p, nullptr, store2, n_hv, st);
                    it_tot = std::max(it_tot, p1.steps + p2.steps);
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
            summary->converged = all_conv ? 1 : 0;
            summary->E0 = *std::min_element(result.begin(), result.end());
            summary->E0_low = o.mode == QMB_MODE_FP64 ? summary->E0 : *std::min_element(low.begin(), low.end());
            summary->residual = -1;
            summary->residual_ref = -1;
        }
    });
}
