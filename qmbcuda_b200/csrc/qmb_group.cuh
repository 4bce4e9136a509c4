// qmb_group.cuh -- group-element application on device.
#pragma once
#include "qmb_common.cuh"

namespace qmb {

// One site map as word operations (structured groups).
struct ElemRot {
    uint64_t lo;  // bits moved up by the in-row rotation
    uint32_t rr;  // whole-word rotation (bits)
    uint32_t ri;  // in-row rotation (bits)
};

constexpr int kMaxPerm = 512;        // site maps per group
constexpr int kTableSmemMax = 96 * 1024;

// Group description handed to kernels by value.
struct GroupArgs {
    int L, G, n_ext, structured, W, n_chunks;
    int full_rot;             // a chain group of all L rotations, element 0 the identity
    int full_torus;           // all R x W translations of a torus of W-site rows (W <= 8), element 0 the identity
    uint64_t mask;
    const ElemRot* rot;       // [G] device
    const uint64_t* tables;   // [G][n_chunks][16] device
    const double2* chars;     // [n_ext] device (selected irrep), may be null
};

// Shared-memory copy of the group, loaded by every thread block.
struct GroupSmem {
    const ElemRot* rot;
    const uint64_t* tab;
    const int* gofr;          // full_rot / full_torus: element of translation (a rows, c sites) at a * W + c
    const uint8_t* minrot;    // full_torus: smallest rotation of each W-bit row value
    const uint8_t* rotmask;   // full_torus: the rotations reaching it (bit c)
};

// Bytes of dynamic shared memory a kernel needs for the group.
__host__ __device__ inline size_t group_smem_bytes(const GroupArgs& g) {
    if (g.structured) return sizeof(ElemRot) * (size_t)g.G + sizeof(int) * 64 + 2 * 256;
    size_t t = sizeof(uint64_t) * (size_t)g.G * g.n_chunks * 16;
    return t <= (size_t)kTableSmemMax ? t : 0;
}

// Cooperative load of the group into dynamic shared memory `sm`.
__device__ __forceinline__ GroupSmem load_group(const GroupArgs& g, unsigned char* sm) {
    GroupSmem out;
    out.gofr = nullptr;
    out.minrot = out.rotmask = nullptr;
    if (g.structured) {
        ElemRot* r = reinterpret_cast<ElemRot*>(sm);
        int* gofr = reinterpret_cast<int*>(r + g.G);
        uint8_t* minrot = reinterpret_cast<uint8_t*>(gofr + 64);
        uint8_t* rotmask = minrot + 256;
        for (int i = threadIdx.x; i < g.G; i += blockDim.x) {
            r[i] = g.rot[i];
            if (g.full_rot || g.full_torus) gofr[(int)(g.rot[i].rr / g.W) * g.W + (int)g.rot[i].ri] = i;
        }
        if (g.full_torus)
            for (int v = threadIdx.x; v < (1 << g.W); v += blockDim.x) {
                int best = 1 << g.W, m = 0;
                for (int c = 0; c < g.W; ++c) {
                    const int y = c ? (((v << c) | (v >> (g.W - c))) & ((1 << g.W) - 1)) : v;
                    if (y < best) {
                        best = y;
                        m = 1 << c;
                    } else if (y == best) {
                        m |= 1 << c;
                    }
                }
                minrot[v] = (uint8_t)best;
                rotmask[v] = (uint8_t)m;
            }
        out.rot = r;
        out.tab = g.tables;
        out.gofr = gofr;
        out.minrot = minrot;
        out.rotmask = rotmask;
    } else {
        size_t n = (size_t)g.G * g.n_chunks * 16;
        if (n * sizeof(uint64_t) <= (size_t)kTableSmemMax) {
            uint64_t* t = reinterpret_cast<uint64_t*>(sm);
            for (size_t i = threadIdx.x; i < n; i += blockDim.x) t[i] = g.tables[i];
            out.tab = t;
        } else {
            out.tab = g.tables;
        }
        out.rot = g.rot;
    }
    __syncthreads();
    return out;
}

// Image of s under site map g (no inversion).
__device__ __forceinline__ uint64_t apply_site_map(const GroupArgs& g, const GroupSmem& sm, int gi,
                                                   uint64_t s) {
    if (g.structured) {
        ElemRot e = sm.rot[gi];
        uint64_t y = rotl_bits(s, (int)e.rr, g.L, g.mask);
        return rot_rows(y, (int)e.ri, g.W, e.lo);
    }
    const uint64_t* t = sm.tab + (size_t)gi * g.n_chunks * 16;
    uint64_t y = 0;
#pragma unroll 4
    for (int c = 0; c < g.n_chunks; ++c) y |= t[c * 16 + (int)((s >> (4 * c)) & 15ull)];
    return y;
}

// Image under extended element e = z*G + g.
__device__ __forceinline__ uint64_t apply_elem(const GroupArgs& g, const GroupSmem& sm, int e,
                                               uint64_t s) {
    int z = e >= g.G;
    int gi = z ? e - g.G : e;
    uint64_t y = apply_site_map(g, sm, gi, s);
    return z ? (y ^ g.mask) : y;
}

// Structured groups on at most 32 sites: the same site maps in 32-bit
// arithmetic (a 64-bit shift, mask or compare costs several 32-bit ALU
// instructions, and the orbit search is ALU-bound).  Same loop order and
// comparisons as the 64-bit forms, so the same element is chosen.
__device__ __forceinline__ uint32_t rot32_bits(uint32_t x, int r, int L, uint32_t mask) {
    if (r == 0) return x;
    return ((x << r) | (x >> (L - r))) & mask;
}

__device__ __forceinline__ uint32_t rot32_rows(uint32_t x, int c, int W, uint32_t lo) {
    if (c == 0) return x;
    return ((x & lo) << c) | ((x & ~lo) >> (W - c));
}

__device__ __forceinline__ uint32_t apply_site_map32(const GroupArgs& g, const GroupSmem& sm, int gi, uint32_t s) {
    const ElemRot e = sm.rot[gi];
    return rot32_rows(rot32_bits(s, (int)e.rr, g.L, (uint32_t)g.mask), (int)e.ri, g.W, (uint32_t)e.lo);
}

__device__ __forceinline__ uint32_t chain_orbit_min(const GroupArgs& g, const GroupSmem& sm, uint32_t x,
                                                    int* elem);
__device__ __forceinline__ uint64_t torus_orbit_min(const GroupArgs& g, const GroupSmem& sm, uint64_t t,
                                                    int* elem);

// True iff no element maps s below s (s is its orbit's minimum).
__device__ __forceinline__ bool is_rep(const GroupArgs& g, const GroupSmem& sm, uint64_t s) {
    if (g.full_rot) {
        int e;
        return chain_orbit_min(g, sm, (uint32_t)s, &e) == (uint32_t)s;
    }
    if (g.full_torus) {
        int e;
        return torus_orbit_min(g, sm, s, &e) == s;
    }
    if (g.structured && g.L <= 32) {
        const uint32_t x = (uint32_t)s, m = (uint32_t)g.mask;
        const bool flip = g.n_ext > g.G;
        // one row (a chain): every element is a rotation, read off the doubled word
        const bool chain = g.W == g.L;
        const uint64_t xx = ((uint64_t)x << g.L) | x;
        for (int gi = 0; gi < g.G; ++gi) {
            // a 32-site chain rotates by a funnel shift; shorter ones read the doubled word
            const uint32_t y = chain ? (g.L == 32 ? __funnelshift_l(x, x, (int)sm.rot[gi].ri)
                                                  : (uint32_t)(xx >> (g.L - (int)sm.rot[gi].ri)) & m)
                                     : apply_site_map32(g, sm, gi, x);
            if (y < x) return false;
            if (flip && (y ^ m) < x) return false;
        }
        return true;
    }
    for (int gi = 0; gi < g.G; ++gi) {
        uint64_t y = apply_site_map(g, sm, gi, s);
        if (y < s) return false;
        if (g.n_ext > g.G && (y ^ g.mask) < s) return false;
    }
    return true;
}

// The orbit minimum of x under all L rotations of a chain (and, with flip,
// their complements), and the first element reaching it in the (element,
// inversion) order of orbit_min's loop.  A rotation's leading zeros are a run
// of zeros of the string, so the minimum brings the top of a longest run of
// zeros (bit p zero, bit p+1 one, cyclically) to bit L-1, and every rotation
// reaching it does.  The tops are filtered down to those of the longest runs
// (one AND a step, as many steps as the longest run is long), and only those
// rotations are compared: usually one or two instead of L, or 2L with flip.
__device__ __forceinline__ uint32_t rotl_chain(uint32_t v, int r, int L, uint32_t m) {
    return L == 32 ? __funnelshift_l(v, v, r) : (r ? (((v << r) | (v >> (L - r))) & m) : v);
}

__device__ __forceinline__ uint32_t chain_orbit_min(const GroupArgs& g, const GroupSmem& sm, uint32_t x,
                                                    int* elem) {
    const int L = g.L;
    const uint32_t m = (uint32_t)g.mask;
    const int nz = g.n_ext > g.G ? 2 : 1;
    uint32_t tops[2] = {0u, 0u};
    int run[2] = {-1, -1};
#pragma unroll
    for (int z = 0; z < 2; ++z) {
        if (z >= nz) break;
        const uint32_t v = z ? (~x & m) : x;
        const uint32_t zeros = ~v & m;
        uint32_t c = zeros & rotl_chain(v, L - 1, L, m);  // bit p zero, bit p+1 one
        if (!c) {  // constant string
            run[z] = v ? 0 : L;
            continue;
        }
        int k = 1;
        uint32_t below = zeros;
        for (;;) {
            below = rotl_chain(below, 1, L, m);  // bit p: zero k bits below p
            const uint32_t nx = c & below;
            if (!nx) break;
            c = nx;
            ++k;
        }
        tops[z] = c;
        run[z] = k;
    }
    const int longest = max(run[0], run[1]);
    uint32_t best = x;  // element 0, the identity
    int bg = 0, bz = 0;
#pragma unroll
    for (int z = 0; z < 2; ++z) {
        if (z >= nz || run[z] != longest) continue;
        const uint32_t v = z ? (~x & m) : x;
        uint32_t c = tops[z];
        if (!c && v < best) {  // constant: every rotation gives v, element 0 first
            best = v;
            bg = 0;
            bz = z;
        }
        while (c) {
            const int p = __ffs(c) - 1;
            c &= c - 1;
            const int r = L - 1 - p;
            const uint32_t y = rotl_chain(v, r, L, m);
            const int gi = sm.gofr[r];
            if (y < best || (y == best && (gi < bg || (gi == bg && z < bz)))) {
                best = y;
                bg = gi;
                bz = z;
            }
        }
    }
    *elem = bz ? bg + g.G : bg;
    return best;
}

// The orbit minimum of t under all R x W translations of a torus of W-site
// rows (and, with flip, their complements), and the first element reaching
// it in the (element, inversion) order of orbit_min's loop.  The image of
// translation (a rows, c sites) has as its top row (the most significant W
// bits) row R-1-a of the string rotated by c, so the minimum's top row is the
// smallest rotation of any row: only the translations that bring such a row,
// rotated to that value, to the top are tried (usually a few of the R W, or
// 2 R W with flip).
__device__ __forceinline__ uint64_t torus_orbit_min(const GroupArgs& g, const GroupSmem& sm, uint64_t t,
                                                    int* elem) {
    const int W = g.W, R = g.L / g.W;
    const uint64_t wmask = (1ull << W) - 1;
    const int nz = g.n_ext > g.G ? 2 : 1;
    int top[2] = {1 << 30, 1 << 30};
    unsigned rows[2] = {0u, 0u};
    for (int z = 0; z < nz; ++z) {
        const uint64_t v = z ? (~t & g.mask) : t;
        for (int i = 0; i < R; ++i) {
            const int m = sm.minrot[(v >> (i * W)) & wmask];
            if (m < top[z]) {
                top[z] = m;
                rows[z] = 1u << i;
            } else if (m == top[z]) {
                rows[z] |= 1u << i;
            }
        }
    }
    const int best_top = min(top[0], top[1]);
    uint64_t best = t;  // element 0, the identity
    int bg = 0, bz = 0;
    for (int z = 0; z < nz; ++z) {
        if (top[z] != best_top) continue;
        const uint64_t v = z ? (~t & g.mask) : t;
        unsigned rw = rows[z];
        while (rw) {
            const int i = __ffs(rw) - 1;
            rw &= rw - 1;
            const int a = R - 1 - i;  // row i moves to the top
            unsigned cm = sm.rotmask[(v >> (i * W)) & wmask];
            while (cm) {
                const int c = __ffs(cm) - 1;
                cm &= cm - 1;
                const int gi = sm.gofr[a * W + c];
                const uint64_t y = apply_site_map(g, sm, gi, v);
                if (y < best || (y == best && (gi < bg || (gi == bg && z < bz)))) {
                    best = y;
                    bg = gi;
                    bz = z;
                }
            }
        }
    }
    *elem = bz ? bg + g.G : bg;
    return best;
}

// Minimum of the orbit of t and the first element reaching it.
__device__ __forceinline__ uint64_t orbit_min(const GroupArgs& g, const GroupSmem& sm, uint64_t t,
                                              int* elem) {
    if (g.full_rot) return chain_orbit_min(g, sm, (uint32_t)t, elem);
    if (g.full_torus) return torus_orbit_min(g, sm, t, elem);
    if (g.structured && g.L <= 32) {
        const uint32_t x = (uint32_t)t, m = (uint32_t)g.mask;
        const bool flip = g.n_ext > g.G;
        uint32_t best = x;
        int be = 0;
        // one row (a chain): every element is a rotation, read off the doubled word
        const bool chain = g.W == g.L;
        const uint64_t xx = ((uint64_t)x << g.L) | x;
        for (int gi = 0; gi < g.G; ++gi) {
            // a 32-site chain rotates by a funnel shift; shorter ones read the doubled word
            const uint32_t y = chain ? (g.L == 32 ? __funnelshift_l(x, x, (int)sm.rot[gi].ri)
                                                  : (uint32_t)(xx >> (g.L - (int)sm.rot[gi].ri)) & m)
                                     : apply_site_map32(g, sm, gi, x);
            if (y < best) { best = y; be = gi; }
            if (flip) {
                const uint32_t yz = y ^ m;
                if (yz < best) { best = yz; be = gi + g.G; }
            }
        }
        if (be == 0 && best == x && apply_site_map32(g, sm, 0, x) != x) {
            for (int e = 1; e < g.n_ext; ++e)
                if (apply_elem(g, sm, e, t) == t) { be = e; break; }
        }
        *elem = be;
        return best;
    }
    uint64_t best = t;
    int be = 0;
    bool flip = g.n_ext > g.G;
    for (int gi = 0; gi < g.G; ++gi) {
        uint64_t y = apply_site_map(g, sm, gi, t);
        if (y < best) { best = y; be = gi; }
        if (flip) {
            uint64_t yz = y ^ g.mask;
            if (yz < best) { best = yz; be = gi + g.G; }
        }
    }
    // element 0 is checked first above; if t itself is minimal and element 0
    // is not the identity, find an element that fixes t.
    if (be == 0 && best == t && apply_site_map(g, sm, 0, t) != t) {
        for (int e = 1; e < g.n_ext; ++e)
            if (apply_elem(g, sm, e, t) == t) { be = e; break; }
    }
    *elem = be;
    return best;
}

// Orbit index of representative r in the sorted table, or -1.  bucket[b]
// holds the first table position whose string has top bits >= b.
struct RepTable {
    const uint64_t* reps;
    const uint32_t* bucket;  // [2^T + 1]
    int64_t R;
    int shift;               // L - T
};

__device__ __forceinline__ int64_t find_rep(const RepTable& t, uint64_t r) {
    uint64_t b = r >> t.shift;
    int64_t lo = t.bucket[b], hi = t.bucket[b + 1];
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        uint64_t v = __ldg(t.reps + mid);
        if (v < r) lo = mid + 1;
        else hi = mid;
    }
    return (lo < t.R && t.reps[lo] == r) ? lo : -1;
}

}  // namespace qmb
