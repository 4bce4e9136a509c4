// qmb_sector.cu -- symmetry-adapted basis of a fixed-Sz sector on the GPU.
//
// Replaces BuildBasisStates + BuildSRStates of the reference
// (exact_diagonalization/HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:276-400;
// kernels SetUpSRS / SolveSRS_min / SetUpSRS_from_indices / ComputeSRSNorms /
// ComputeOrbitIndices, exact_diagonalization/utils.cu:39-80,716-805).
// Instead of materialising the C(L,k) x G orbit table, each thread walks 64
// consecutive strings of the sector (unrank once, then Gosper steps), tests
// "no element maps s below s" and sets a bit; an order-preserving compaction
// of the set bits yields the ascending representative table directly.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "qmb_sector.cuh"

namespace qmb {

// C(n, k) for n, k <= 64 in constant memory (65*65 uint64 = 33.8 KB); used
// by unrank(), where all lanes of a warp walk the same positions.
__constant__ uint64_t c_binom[65 * 65];

__device__ __forceinline__ uint64_t dbinom(int n, int k) { return c_binom[n * 65 + k]; }

// Inverse of the ascending-order rank (combinatorial number system).
__device__ __forceinline__ uint64_t unrank(uint64_t r, int L, int k) {
    uint64_t s = 0;
    for (int p = L - 1; p >= 0 && k > 0; --p) {
        uint64_t c = dbinom(p, k);
        if (r >= c) {
            s |= 1ull << p;
            r -= c;
            --k;
        }
    }
    return s;
}

namespace {
struct BinomTable {
    uint64_t tab[65][65];
    BinomTable() {
        for (int a = 0; a <= 64; ++a) {
            tab[a][0] = 1;
            for (int b = 1; b <= 64; ++b) tab[a][b] = a == 0 ? 0 : tab[a - 1][b - 1] + tab[a - 1][b];
        }
    }
};
}  // namespace

uint64_t host_binom(int n, int k) {
    static const BinomTable t;  // built once; thread-safe initialisation of a local static
    if (n < 0 || k < 0 || n > 64 || k > 64) return 0;
    return t.tab[n][k];
}

/* Copies the binomial table into this device's constant memory, once per
 * device and process.  Several host threads may create sectors at once: the
 * first one for a device uploads while the others wait on the same flag; an
 * upload that throws leaves the flag unset, so the next call retries. */
static void upload_binomials() {
    int dev = 0;
    QMB_CUDA_TRY(cudaGetDevice(&dev));
    static std::once_flag done[64];
    auto upload = [] {
        std::vector<uint64_t> t(65 * 65);
        for (int n = 0; n <= 64; ++n)
            for (int k = 0; k <= 64; ++k) t[n * 65 + k] = host_binom(n, k);
        QMB_CUDA_TRY(cudaMemcpyToSymbol(c_binom, t.data(), sizeof(uint64_t) * t.size()));
    };
    if (dev >= 0 && dev < 64)
        std::call_once(done[dev], upload);
    else
        upload();
}

// ------------------------------------------------------------------ kernels
__global__ void k_rep_words(GroupArgs g, int k, uint64_t n_states, uint64_t n_words,
                            uint64_t* __restrict__ words, uint32_t* __restrict__ counts) {
    extern __shared__ __align__(16) unsigned char smem[];
    GroupSmem sm = load_group(g, smem);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words;
         w += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r0 = w * 64;
        uint64_t s = unrank(r0, g.L, k);
        uint64_t bits = 0;
        int n = (int)min((uint64_t)64, n_states - r0);
        for (int i = 0; i < n; ++i) {
            if (is_rep(g, sm, s)) bits |= 1ull << i;
            if (s) s = next_comb(s);
        }
        words[w] = bits;
        counts[w] = (uint32_t)__popcll(bits);
    }
}

__global__ void k_rep_write(int L, int k, uint64_t n_words, const uint64_t* __restrict__ words,
                            const uint64_t* __restrict__ offsets, uint64_t* __restrict__ reps) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words;
         w += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t bits = words[w];
        if (!bits) continue;
        uint64_t o = offsets[w];
        uint64_t s = unrank(w * 64, L, k);
        for (int i = 0; bits; ++i) {
            if (bits & 1ull) reps[o++] = s;
            bits >>= 1;
            if (s) s = next_comb(s);
        }
    }
}

__global__ void k_bucket(const uint64_t* __restrict__ reps, int64_t R, int shift, uint64_t n_b,
                         uint32_t* __restrict__ bucket) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b <= n_b;
         b += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t key = (b == n_b) ? ~0ull : (b << shift);
        int64_t lo = 0, hi = R;
        if (b == n_b) { bucket[b] = (uint32_t)R; continue; }
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (reps[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        bucket[b] = (uint32_t)lo;
    }
}

// norm = sqrt(n_ext * |Re sum_{h in Stab(r)} chi(h)|) / n_ext and the active flag.
__global__ void k_norms(GroupArgs g, const uint64_t* __restrict__ reps, int64_t R, double tol,
                        double* __restrict__ norms, int* __restrict__ active) {
    extern __shared__ __align__(16) unsigned char smem[];
    GroupSmem sm = load_group(g, smem);
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < R;
         o += (int64_t)gridDim.x * blockDim.x) {
        uint64_t r = reps[o];
        double sr = 0.0;
        for (int e = 0; e < g.n_ext; ++e)
            if (apply_elem(g, sm, e, r) == r) sr += g.chars[e].x;
        double nv = sqrt(fabs(sr * g.n_ext)) / (double)g.n_ext;
        norms[o] = nv;
        active[o] = nv >= tol ? 1 : 0;
    }
}

__global__ void k_active_maps(int64_t R, const int* __restrict__ active,
                              const int64_t* __restrict__ pos, int64_t* __restrict__ row_of_orbit,
                              int64_t* __restrict__ orbit_of_row) {
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < R;
         o += (int64_t)gridDim.x * blockDim.x) {
        if (active[o]) {
            row_of_orbit[o] = pos[o];
            orbit_of_row[pos[o]] = o;
        } else {
            row_of_orbit[o] = -1;
        }
    }
}

// Reference-layout orbit map: rank -> (orbit, largest element reaching it).
__global__ void k_orbit_map(GroupArgs g, RepTable t, int k, uint64_t n_states,
                            uint32_t* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    GroupSmem sm = load_group(g, smem);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_states;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = unrank(i, g.L, k);
        int e0;
        uint64_t r = orbit_min(g, sm, s, &e0);
        int64_t o = find_rep(t, r);
        int best = -1;
        for (int e = g.n_ext - 1; e >= 0; --e)
            if (apply_elem(g, sm, e, r) == s) { best = e; break; }
        out[2 * i] = (uint32_t)o;
        out[2 * i + 1] = (uint32_t)best;
    }
}

__global__ void k_lookup(GroupArgs g, RepTable t, int k, const uint64_t* __restrict__ in,
                         int64_t n, int64_t* __restrict__ orbit, int32_t* __restrict__ elem) {
    extern __shared__ __align__(16) unsigned char smem[];
    GroupSmem sm = load_group(g, smem);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t s = in[i];
        if ((s & ~g.mask) || __popcll(s) != k) {
            orbit[i] = -1;
            elem[i] = -1;
            continue;
        }
        int e;
        uint64_t r = orbit_min(g, sm, s, &e);
        orbit[i] = find_rep(t, r);
        elem[i] = e;
    }
}

int grid_for(int64_t n, int block) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t g = (n + block - 1) / block;
    int64_t cap = (int64_t)sms * 32;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

void set_group_smem_attr(const void* kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        QMB_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)bytes));
}

// Detects whether every site map is a torus translation with rows of W bits.
static bool detect_rotations(const std::vector<uint32_t>& perm, int L, int G, int W,
                             std::vector<ElemRot>& out) {
    if (L % W) return false;
    int rows = L / W;
    out.resize(G);
    uint64_t mask = (L == 64) ? ~0ull : ((1ull << L) - 1);
    for (int g = 0; g < G; ++g) {
        const uint32_t* p = perm.data() + (size_t)g * L;
        int a = (int)p[0] / W, c = (int)p[0] % W;
        for (int q = 0; q < L; ++q) {
            int i = q / W, j = q % W;
            int want = ((i + a) % rows) * W + (j + c) % W;
            if ((int)p[q] != want) return false;
        }
        uint64_t lo = 0;
        for (int q = 0; q < L; ++q)
            if (q % W < W - c) lo |= 1ull << q;
        out[g].lo = lo & mask;
        out[g].rr = (uint32_t)(a * W);
        out[g].ri = (uint32_t)c;
    }
    return true;
}

}  // namespace qmb

using namespace qmb;

namespace qmb {

void sector_check_desc(const qmb_sector_desc* d) {
    QMB_REQUIRE(d->L >= 1 && d->L <= 64, QMB_ERR_INVALID, "L must be in 1..64");
    QMB_REQUIRE(d->n_up >= 0 && d->n_up <= d->L, QMB_ERR_INVALID, "n_up must be in 0..L");
    QMB_REQUIRE(d->n_perm >= 1 && d->n_perm <= kMaxPerm, QMB_ERR_INVALID,
                "n_perm must be in 1..512");
    QMB_REQUIRE(d->perm, QMB_ERR_INVALID, "perm is null");
    QMB_REQUIRE(!d->spin_flip || 2 * d->n_up == d->L, QMB_ERR_INVALID,
                "spin inversion needs 2*n_up == L");
    const int L = d->L, G = d->n_perm;
    for (int g = 0; g < G; ++g) {
        std::vector<int> seen(L, 0);
        for (int q = 0; q < L; ++q) {
            uint32_t v = d->perm[(size_t)g * L + q];
            QMB_REQUIRE(v < (uint32_t)L && !seen[v], QMB_ERR_INVALID,
                        "perm row " + std::to_string(g) + " is not a permutation of 0..L-1");
            seen[v] = 1;
        }
    }
}

// Fields and group tables of a sector (everything but the representatives).
void sector_setup(qmb_sector_s* s, const qmb_sector_desc* d) {
    const int L = d->L, G = d->n_perm;
    s->device = d->device;
    s->L = L;
    s->n_up = d->n_up;
    s->G = G;
    s->flip = d->spin_flip ? 1 : 0;
    s->n_ext = G * (1 + s->flip);
    s->perm.assign(d->perm, d->perm + (size_t)G * L);
    s->n_states = (int64_t)host_binom(L, d->n_up);
    QMB_REQUIRE(s->n_states > 0, QMB_ERR_INVALID, "empty sector");

    // group: word rotations when possible, else nibble tables
    std::vector<ElemRot> rots;
    bool structured = false;
    for (int W = L; W >= 1 && !structured; --W)
        if (L % W == 0 && detect_rotations(s->perm, L, G, W, rots)) {
            structured = true;
            s->W = W;
        }
    s->structured = structured ? 1 : 0;
    s->n_chunks = (L + 3) / 4;
    // all L rotations of a chain of at most 32 sites, element 0 the identity
    s->full_rot = 0;
    if (structured && s->W == L && G == L && L <= 32 && rots[0].ri == 0) {
        std::vector<int> seen(L, 0);
        bool distinct = true;
        for (int g = 0; g < G; ++g) distinct = distinct && !seen[rots[g].ri]++;
        s->full_rot = distinct ? 1 : 0;
    }
    // all R x W translations of a torus of W <= 8 site rows (R <= 32), element 0 the identity
    s->full_torus = 0;
    if (structured && s->W < L && s->W <= 8 && L / s->W <= 32 && G == L && rots[0].ri == 0 && rots[0].rr == 0) {
        std::vector<int> seen(L, 0);
        bool distinct = true;
        for (int g = 0; g < G; ++g) {
            const int idx = (int)(rots[g].rr / s->W) * s->W + (int)rots[g].ri;
            distinct = distinct && idx < L && !seen[idx]++;
        }
        s->full_torus = distinct ? 1 : 0;
    }
    if (structured) {
        s->rot.alloc(G);
        s->rot.upload(rots.data(), G);
    }
    std::vector<uint64_t> tab((size_t)G * s->n_chunks * 16, 0);
    for (int g = 0; g < G; ++g)
        for (int c = 0; c < s->n_chunks; ++c)
            for (int v = 0; v < 16; ++v) {
                uint64_t y = 0;
                for (int b = 0; b < 4; ++b) {
                    int q = 4 * c + b;
                    if (q < L && (v >> b & 1)) y |= 1ull << s->perm[(size_t)g * L + q];
                }
                tab[((size_t)g * s->n_chunks + c) * 16 + v] = y;
            }
    s->tables.alloc(tab.size());
    s->tables.upload(tab.data(), tab.size());
}

// Counts stored representatives that are not the minimum of their orbit.
__global__ void k_check_reps(GroupArgs g, const uint64_t* __restrict__ reps, int64_t R,
                             unsigned long long* __restrict__ bad) {
    extern __shared__ __align__(16) unsigned char smem[];
    GroupSmem gs = load_group(g, smem);
    unsigned long long nb = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x) {
        int e;
        if (orbit_min(g, gs, reps[i], &e) != reps[i]) ++nb;
    }
    if (nb) atomicAdd(bad, nb);
}

qmb_sector_s* sector_from_reps(const qmb_sector_desc* d, const uint64_t* reps, int64_t R) {
    sector_check_desc(d);
    DeviceGuard dg(d->device);
    upload_binomials();
    auto s = std::make_unique<qmb_sector_s>();
    sector_setup(s.get(), d);
    QMB_REQUIRE(R > 0 && R < (1ll << 32) && R <= s->n_states, QMB_ERR_INVALID,
                "stored representative count out of range");
    const uint64_t mask = d->L == 64 ? ~0ull : ((1ull << d->L) - 1);
    for (int64_t i = 0; i < R; ++i) {
        QMB_REQUIRE((reps[i] & ~mask) == 0 && __builtin_popcountll(reps[i]) == d->n_up, QMB_ERR_INVALID,
                    "a stored representative is not in the sector");
        QMB_REQUIRE(i == 0 || reps[i] > reps[i - 1], QMB_ERR_INVALID,
                    "stored representatives are not strictly ascending");
    }
    s->R = R;
    s->reps.alloc(R);
    s->reps.upload(reps, R);
    GroupArgs ga = s->group_args();
    size_t gsm = group_smem_bytes(ga);
    DevBuf<unsigned long long> bad(1);
    bad.zero();
    set_group_smem_attr((const void*)k_check_reps, gsm);
    k_check_reps<<<grid_for(R, 256), 256, gsm>>>(ga, s->reps.p, R, bad.p);
    check_launch("k_check_reps");
    unsigned long long nb = 0;
    QMB_CUDA_TRY(cudaMemcpy(&nb, bad.p, sizeof(nb), cudaMemcpyDeviceToHost));
    QMB_REQUIRE(nb == 0, QMB_ERR_INVALID, "stored representatives are not orbit minima of this group");
    sector_buckets(s.get());
    return s.release();
}

// Lookup buckets on the top T bits of the rank space over s->reps.  (Fewer
// bits, about four representatives a bucket, shrink the table from 64 MB to
// 8 MB at L=32 but made the matrix-free product slower: 21.2 -> 25.5 ms, the
// extra probes cost more than the smaller table saves.)
void sector_buckets(qmb_sector_s* s) {
    const int L = s->L;
    s->T = std::min(L, 24);
    uint64_t n_b = 1ull << s->T;
    s->bucket.alloc(n_b + 1);
    k_bucket<<<grid_for((int64_t)n_b + 1, 256), 256>>>(s->reps.p, s->R, L - s->T, n_b, s->bucket.p);
    check_launch("k_bucket");
    QMB_CUDA_TRY(cudaDeviceSynchronize());
}

}  // namespace qmb

extern "C" qmb_status qmb_sector_create(const qmb_sector_desc* d, qmb_sector* out) {
    return guarded([&] {
        QMB_REQUIRE(d && out, QMB_ERR_INVALID, "null argument");
        *out = nullptr;
        sector_check_desc(d);
        DeviceGuard dg(d->device);
        upload_binomials();
        auto s = new qmb_sector_s();
        std::unique_ptr<qmb_sector_s> own(s);
        sector_setup(s, d);
        const int L = s->L;
        GroupArgs ga = s->group_args();
        size_t gsm = group_smem_bytes(ga);

        // representative bit words
        uint64_t n_words = ((uint64_t)s->n_states + 63) / 64;
        DevBuf<uint64_t> words(n_words);
        DevBuf<uint32_t> counts(n_words + 1);
        DevBuf<uint64_t> offsets(n_words + 1);
        set_group_smem_attr((const void*)k_rep_words, gsm);
        k_rep_words<<<grid_for((int64_t)n_words, 256), 256, gsm>>>(ga, s->n_up, s->n_states,
                                                                   n_words, words.p, counts.p);
        check_launch("k_rep_words");
        QMB_CUDA_TRY(cudaMemsetAsync(counts.p + n_words, 0, sizeof(uint32_t)));
        size_t tmp_bytes = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts.p, offsets.p, n_words + 1);
        DevBuf<unsigned char> tmp(tmp_bytes);
        cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, counts.p, offsets.p, n_words + 1);
        uint64_t R = 0;
        QMB_CUDA_TRY(cudaMemcpy(&R, offsets.p + n_words, sizeof(uint64_t), cudaMemcpyDeviceToHost));
        QMB_REQUIRE(R > 0 && R < (1ull << 32), QMB_ERR_UNSUPPORTED,
                    "orbit count must be in 1..2^32-1");
        s->R = (int64_t)R;
        s->reps.alloc(R);
        k_rep_write<<<grid_for((int64_t)n_words, 256), 256>>>(L, s->n_up, n_words, words.p,
                                                              offsets.p, s->reps.p);
        check_launch("k_rep_write");
        sector_buckets(s);
        *out = own.release();
    });
}

extern "C" qmb_status qmb_sector_destroy(qmb_sector s) {
    return guarded([&] {
        if (!s) return;
        DeviceGuard dg(s->device);
        delete s;
    });
}

extern "C" qmb_status qmb_sector_get_info(qmb_sector s, qmb_sector_info* info) {
    return guarded([&] {
        QMB_REQUIRE(s && info, QMB_ERR_INVALID, "null argument");
        info->n_states = s->n_states;
        info->n_orbits = s->R;
        info->n_active = s->has_irrep ? s->n_active : 0;
        info->n_ext = s->n_ext;
        info->structured = s->structured;
        info->is_real = s->is_real ? 1 : 0;
    });
}

namespace qmb {
// Irrep selection: characters, norms and the active-row maps.
void sector_select_irrep(qmb_sector_s* s, const double* chars, double tol_norm) {
    s->chars.resize(s->n_ext);
    s->is_real = true;
    std::vector<double2> ch(s->n_ext);
    for (int e = 0; e < s->n_ext; ++e) {
        s->chars[e] = {chars[2 * e], chars[2 * e + 1]};
        ch[e] = make_double2(chars[2 * e], chars[2 * e + 1]);
        QMB_REQUIRE(std::isfinite(chars[2 * e]) && std::isfinite(chars[2 * e + 1]),
                    QMB_ERR_INVALID, "non-finite character");
        if (std::fabs(chars[2 * e + 1]) > 1e-12) s->is_real = false;
    }
    s->tol_norm = tol_norm;
    s->chars_dev.alloc(s->n_ext);
    s->chars_dev.upload(ch.data(), s->n_ext);
    GroupArgs ga = s->group_args();
    size_t gsm = group_smem_bytes(ga);
    s->norms.alloc(s->R);
    DevBuf<int> active(s->R + 1);
    DevBuf<int64_t> pos(s->R + 1);
    set_group_smem_attr((const void*)k_norms, gsm);
    k_norms<<<grid_for(s->R, 256), 256, gsm>>>(ga, s->reps.p, s->R, tol_norm, s->norms.p,
                                               active.p);
    check_launch("k_norms");
    QMB_CUDA_TRY(cudaMemsetAsync(active.p + s->R, 0, sizeof(int)));
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, active.p, pos.p, s->R + 1);
    DevBuf<unsigned char> tmp(tmp_bytes);
    cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, active.p, pos.p, s->R + 1);
    int64_t na = 0;
    QMB_CUDA_TRY(cudaMemcpy(&na, pos.p + s->R, sizeof(int64_t), cudaMemcpyDeviceToHost));
    s->n_active = na;
    s->row_of_orbit.alloc(s->R);
    s->orbit_of_row.alloc(na > 0 ? na : 1);
    k_active_maps<<<grid_for(s->R, 256), 256>>>(s->R, active.p, pos.p, s->row_of_orbit.p,
                                                s->orbit_of_row.p);
    check_launch("k_active_maps");
    QMB_CUDA_TRY(cudaDeviceSynchronize());
    s->has_irrep = true;
    ++s->irrep_gen;
}
}  // namespace qmb

extern "C" qmb_status qmb_sector_set_irrep(qmb_sector s, const double* chars, double tol_norm) {
    return guarded([&] {
        QMB_REQUIRE(s && chars, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(tol_norm >= 0, QMB_ERR_INVALID, "tol_norm must be >= 0");
        DeviceGuard dg(s->device);
        sector_select_irrep(s, chars, tol_norm);
    });
}

extern "C" qmb_status qmb_sector_reps(qmb_sector s, uint64_t* reps, int64_t cap) {
    return guarded([&] {
        QMB_REQUIRE(s && reps, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(cap >= s->R, QMB_ERR_INVALID, "capacity below the orbit count");
        DeviceGuard dg(s->device);
        s->reps.download(reps, s->R);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
    });
}

extern "C" qmb_status qmb_sector_norms(qmb_sector s, double* norms, int64_t cap) {
    return guarded([&] {
        QMB_REQUIRE(s && norms, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(s->has_irrep, QMB_ERR_INVALID, "no irrep selected");
        QMB_REQUIRE(cap >= s->R, QMB_ERR_INVALID, "capacity below the orbit count");
        DeviceGuard dg(s->device);
        s->norms.download(norms, s->R);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
    });
}

extern "C" qmb_status qmb_sector_active(qmb_sector s, int64_t* orbit_of_row, int64_t cap) {
    return guarded([&] {
        QMB_REQUIRE(s && orbit_of_row, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(s->has_irrep, QMB_ERR_INVALID, "no irrep selected");
        QMB_REQUIRE(cap >= s->n_active, QMB_ERR_INVALID, "capacity below the active count");
        DeviceGuard dg(s->device);
        if (s->n_active) s->orbit_of_row.download(orbit_of_row, s->n_active);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
    });
}

extern "C" qmb_status qmb_sector_orbit_map(qmb_sector s, uint32_t* orbit_indices, int64_t cap) {
    return guarded([&] {
        QMB_REQUIRE(s && orbit_indices, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(cap >= 2 * s->n_states, QMB_ERR_INVALID, "capacity below 2*n_states");
        DeviceGuard dg(s->device);
        GroupArgs ga = s->group_args();
        size_t gsm = group_smem_bytes(ga);
        DevBuf<uint32_t> out(2 * s->n_states);
        set_group_smem_attr((const void*)k_orbit_map, gsm);
        k_orbit_map<<<grid_for(s->n_states, 256), 256, gsm>>>(ga, s->rep_table(), s->n_up,
                                                              s->n_states, out.p);
        check_launch("k_orbit_map");
        out.download(orbit_indices, 2 * s->n_states);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
    });
}

extern "C" qmb_status qmb_sector_lookup(qmb_sector s, const uint64_t* t, int64_t n, int64_t* orbit,
                                        int32_t* element) {
    return guarded([&] {
        QMB_REQUIRE(s && t && orbit && element, QMB_ERR_INVALID, "null argument");
        if (n <= 0) return;
        DeviceGuard dg(s->device);
        GroupArgs ga = s->group_args();
        size_t gsm = group_smem_bytes(ga);
        DevBuf<uint64_t> in(n);
        DevBuf<int64_t> o(n);
        DevBuf<int32_t> e(n);
        in.upload(t, n);
        set_group_smem_attr((const void*)k_lookup, gsm);
        k_lookup<<<grid_for(n, 256), 256, gsm>>>(ga, s->rep_table(), s->n_up, in.p, n, o.p, e.p);
        check_launch("k_lookup");
        o.download(orbit, n);
        e.download(element, n);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
    });
}
