// qmb_ham.cuh -- Hamiltonian storage and the row operators used by H*v.
#pragma once
#include <cstdlib>

#include "qmb_scalar.cuh"
#include "qmb_sector.cuh"

namespace qmb {

constexpr int kMaxTerms = 4096;

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }
constexpr int kMaxCol = 8;

// Operator tables on device: op = code << 8 | site.
struct TermsArgs {
    int n_terms, n_col;
    const int* n_ops;
    const uint16_t* ops;
    const double2* scalar;
};

struct TermsSmem {
    int n_terms, n_col;
    const int* n_ops;
    const uint16_t* ops;
    const double2* scalar;
};

__host__ __device__ inline size_t terms_smem_bytes(const TermsArgs& t) {
    size_t b = sizeof(double2) * t.n_terms;        // scalars first (16-byte aligned)
    b += sizeof(int) * t.n_terms;
    b += sizeof(uint16_t) * (size_t)t.n_terms * t.n_col;
    return (b + 15) & ~(size_t)15;
}

__device__ __forceinline__ TermsSmem load_terms(const TermsArgs& t, unsigned char* sm) {
    double2* sc = reinterpret_cast<double2*>(sm);
    int* no = reinterpret_cast<int*>(sc + t.n_terms);
    uint16_t* op = reinterpret_cast<uint16_t*>(no + t.n_terms);
    for (int i = threadIdx.x; i < t.n_terms; i += blockDim.x) {
        sc[i] = t.scalar[i];
        no[i] = t.n_ops[i];
    }
    for (int i = threadIdx.x; i < t.n_terms * t.n_col; i += blockDim.x) op[i] = t.ops[i];
    __syncthreads();
    TermsSmem s;
    s.n_terms = t.n_terms;
    s.n_col = t.n_col;
    s.n_ops = no;
    s.ops = op;
    s.scalar = sc;
    return s;
}

// Everything a row generator needs.
struct RowGen {
    GroupArgs g;
    RepTable rt;
    TermsArgs terms;
    const double* norms;          // [R]
    const int64_t* row_of_orbit;  // [R]
    const int64_t* orbit_of_row;  // [n_active]
    double tol;
    int n_up;
    int* err;                     // set to 1 when a term leaves the sector
};


// Term hi applied to the basis string src: false when an operator
// annihilates it, else the image *t and the coefficient *coef.  Ops act from
// the first column on; codes other than SZ, SP and SM act as the identity.
__device__ __forceinline__ bool apply_term(const TermsSmem& ts, int hi, uint64_t src, uint64_t* t_out,
                                           double2* coef_out) {
    uint64_t t = src;
    double2 coef = ts.scalar[hi];
    const uint16_t* op = ts.ops + hi * ts.n_col;
    for (int h2 = 0; h2 < ts.n_ops[hi]; ++h2) {
        const int code = op[h2] >> 8, site = op[h2] & 0xff;
        const int spin = (int)((t >> site) & 1ull);
        if (code == QMB_OP_SM) {
            if (!spin) return false;
            t &= ~(1ull << site);
        } else if (code == QMB_OP_SP) {
            if (spin) return false;
            t |= 1ull << site;
        } else if (code == QMB_OP_SZ) {
            const double f = spin ? 0.5 : -0.5;
            coef.x *= f;
            coef.y *= f;
        }
    }
    *t_out = t;
    *coef_out = coef;
    return true;
}

// The diagonal element of the row of src: the terms that map src to itself.
__device__ __forceinline__ double2 row_diagonal(const TermsSmem& ts, uint64_t src) {
    double2 d = make_double2(0.0, 0.0);
    for (int hi = 0; hi < ts.n_terms; ++hi) {
        uint64_t t;
        double2 coef;
        if (apply_term(ts, hi, src, &t, &coef) && t == src) {
            d.x += coef.x;
            d.y += coef.y;
        }
    }
    return d;
}

// Where gen_row_look finds a generated representative r: the sector's orbit
// table, each entry scaled by n(target) / n(source).  find() returns 1 with
// the orbit and the factor, 0 for a null orbit (the entry is dropped), -1
// when r is not in the sector.
struct OrbitLookup {
    double ns;
    __device__ __forceinline__ int find(const RowGen& rg, uint64_t r, int64_t* idx, double* f) const {
        const int64_t o = find_rep(rg.rt, r);
        if (o < 0) return -1;
        const double nt = rg.norms[o];
        if (nt < rg.tol) return 0;
        *idx = o;
        *f = nt / ns;
        return 1;
    }
};

// Enumerates the entries of the row whose source string is src generated by
// terms h0 .. h1-1: emit(index, value) for every off-diagonal entry, with the
// index and the norm factor from look.find(); the diagonal is returned.
// Rule of BuildHamiltonianXXZForAbelianGroup (exact_diagonalization/utils.cu:83-184).
template <class Look, class Emit>
__device__ __forceinline__ double2 gen_row_look(const RowGen& rg, const GroupSmem& gs,
                                                const TermsSmem& ts, int h0, int h1, uint64_t src,
                                                const Look& look, Emit&& emit) {
    double2 diag = make_double2(0.0, 0.0);
    for (int hi = h0; hi < h1; ++hi) {
        uint64_t t;
        double2 coef;
        if (!apply_term(ts, hi, src, &t, &coef)) continue;
        if (t == src) {
            diag.x += coef.x;
            diag.y += coef.y;
            continue;
        }
        if (__popcll(t) != rg.n_up) {
            *rg.err = 1;
            continue;
        }
        int e;
        const uint64_t r = orbit_min(rg.g, gs, t, &e);
        int64_t o;
        double f;
        const int found = look.find(rg, r, &o, &f);
        if (found < 0) {
            *rg.err = 2;
            continue;
        }
        if (!found) continue;
        // t = g_e^{-1}(rep): chi(g_t) = conj(chi(e)) for a unitary 1-D irrep
        double2 ch = rg.g.chars[e];
        double2 v = make_double2((coef.x * ch.x + coef.y * ch.y) * f,
                                 (coef.y * ch.x - coef.x * ch.y) * f);
        emit(o, v);
    }
    return diag;
}

// gen_row_look over the sector's orbit table: emit(orbit, value), the source
// orbit's norm ns.
template <class Emit>
__device__ __forceinline__ double2 gen_row_range(const RowGen& rg, const GroupSmem& gs,
                                                 const TermsSmem& ts, int h0, int h1, uint64_t src,
                                                 double ns, Emit&& emit) {
    return gen_row_look(rg, gs, ts, h0, h1, src, OrbitLookup{ns}, static_cast<Emit&&>(emit));
}

// All terms of the table.
template <class Emit>
__device__ __forceinline__ double2 gen_row(const RowGen& rg, const GroupSmem& gs,
                                           const TermsSmem& ts, uint64_t src, double ns,
                                           Emit&& emit) {
    return gen_row_range(rg, gs, ts, 0, ts.n_terms, src, ns, static_cast<Emit&&>(emit));
}

// --------------------------------------------------------- stored operator
// Sliced ELL: 32-row slices, slot j of row r at off[r/32] + j*32 + r%32.
template <class M>
struct SellOp {
    int64_t n;
    const int64_t* off;   // [n_slices]
    const int* width;     // [n_slices]
    const uint32_t* col;
    const M* val;
    const M* diag;
    static constexpr size_t smem_bytes() { return 0; }
    __device__ void init(unsigned char*) {}
    template <class V>
    void pre(const V*, const int*, cudaStream_t) const {}
    // (H x)_r * scale; x_r is returned through xr.
    template <class V>
    __device__ __forceinline__ V row(int64_t r, const V* __restrict__ x, V& xr) const {
        int64_t s = r >> 5;
        int lane = (int)(r & 31);
        const uint32_t* c = col + off[s] + lane;
        const M* v = val + off[s] + lane;
        int w = width[s];
        V acc = Sc<V>::zero();
        xr = x[r];
        acc = Sc<V>::mul(cvt<V>(diag[r]), xr);
        int j = 0;
        for (; j + 4 <= w; j += 4) {
            uint32_t c0 = __ldg(c + 0 * 32), c1 = __ldg(c + 1 * 32), c2 = __ldg(c + 2 * 32),
                     c3 = __ldg(c + 3 * 32);
            M v0 = __ldg(v + 0 * 32), v1 = __ldg(v + 1 * 32), v2 = __ldg(v + 2 * 32),
              v3 = __ldg(v + 3 * 32);
            V x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
            acc = Sc<V>::fma(cvt<V>(v0), x0, acc);
            acc = Sc<V>::fma(cvt<V>(v1), x1, acc);
            acc = Sc<V>::fma(cvt<V>(v2), x2, acc);
            acc = Sc<V>::fma(cvt<V>(v3), x3, acc);
            c += 4 * 32;
            v += 4 * 32;
        }
        for (; j < w; ++j) {
            uint32_t c0 = __ldg(c);
            M v0 = __ldg(v);
            acc = Sc<V>::fma(cvt<V>(v0), __ldg(x + c0), acc);
            c += 32;
            v += 32;
        }
        return acc;
    }
};

// Column-blocked coded sliced ELL: the columns are split into nb blocks of
// 2^shift rows and every block has its own sliced ELL (32-row slices,
// column-major inside a slice) whose 32-bit entries pack an 8-bit value code
// (into a dictionary of at most 255 values; code 0 is the padding, value 0)
// above the 24-bit column inside the block.  For sectors whose vector is
// larger than L2 (FP32 values) a product makes one pass per block in block
// order, so the part of x a pass gathers from (one block, at most 64 MB)
// stays in L2 while the matrix streams from HBM once: passes 0 .. nb-2
// (pre(), k_cb_pass) leave partial row sums in ytmp, and the last pass is
// row(), which adds its block and hands the row to the calling kernel.  A
// single block (nb = 1) serves matrices whose vector fits L2 but whose entry
// stream is large (FP32, and real FP64 values): 4 bytes an entry instead of
// 8 or 12.
template <class M>  // float, float2 or double
struct CbSellOp {
    int64_t n;
    int nb;                 // column blocks
    int shift;              // block of a column = col >> shift
    int64_t n_slices;
    const int64_t* off;     // [nb * n_slices] first slot of slice s in block b
    const int* width;       // [nb * n_slices]
    const uint32_t* packed;
    const M* dict;          // [256] in global memory, staged in shared memory
    const M* diag;
    void* ytmp;             // [n] partial sums in the product's vector type
    M* sdict;
    static constexpr size_t smem_bytes() { return 256 * sizeof(M); }
    __device__ void init(unsigned char* sm) {
        sdict = reinterpret_cast<M*>(sm);
        for (int i = threadIdx.x; i < 256; i += blockDim.x) sdict[i] = dict[i];
        __syncthreads();
    }
    // acc + the entries of row r in column block b
    template <class V>
    __device__ __forceinline__ V block_sum(int b, int64_t r, const V* __restrict__ x, V acc) const {
        const int64_t s = r >> 5;
        const int lane = (int)(r & 31);
        const uint32_t* p = packed + off[(int64_t)b * n_slices + s] + lane;
        const int w = width[(int64_t)b * n_slices + s];
        const V* xb = x + ((int64_t)b << shift);
        int j = 0;
        for (; j + 4 <= w; j += 4) {
            uint32_t p0 = __ldcs(p + 0 * 32), p1 = __ldcs(p + 1 * 32), p2 = __ldcs(p + 2 * 32),
                     p3 = __ldcs(p + 3 * 32);
            V x0 = __ldg(xb + (p0 & 0xffffffu)), x1 = __ldg(xb + (p1 & 0xffffffu)),
              x2 = __ldg(xb + (p2 & 0xffffffu)), x3 = __ldg(xb + (p3 & 0xffffffu));
            acc = Sc<V>::fma(cvt<V>(sdict[p0 >> 24]), x0, acc);
            acc = Sc<V>::fma(cvt<V>(sdict[p1 >> 24]), x1, acc);
            acc = Sc<V>::fma(cvt<V>(sdict[p2 >> 24]), x2, acc);
            acc = Sc<V>::fma(cvt<V>(sdict[p3 >> 24]), x3, acc);
            p += 4 * 32;
        }
        for (; j < w; ++j) {
            uint32_t p0 = __ldcs(p);
            acc = Sc<V>::fma(cvt<V>(sdict[p0 >> 24]), __ldg(xb + (p0 & 0xffffffu)), acc);
            p += 32;
        }
        return acc;
    }
    // the last pass: (H x)_r from the partial sums of the earlier passes
    template <class V>
    __device__ __forceinline__ V row(int64_t r, const V* __restrict__ x, V& xr) const {
        xr = x[r];
        const V acc = nb > 1 ? reinterpret_cast<const V*>(ytmp)[r] : Sc<V>::mul(cvt<V>(diag[r]), xr);
        return block_sum(nb - 1, r, x, acc);
    }
    template <class V>
    void pre(const V* x0, const int* iter, cudaStream_t s) const;
};

// One pass of a column-blocked product: ytmp = (b == 0 ? D x : ytmp) + A_b x,
// where x = x0, or with iter the half of the Lanczos work buffer x0 that step
// *iter reads (as k_lz_hv does).
template <class M, class V>
__global__ void __launch_bounds__(256) k_cb_pass(CbSellOp<M> op, int b, const V* __restrict__ x0,
                                                 const int* __restrict__ iter) {
    extern __shared__ __align__(16) unsigned char smem_cb[];
    op.init(smem_cb);
    const V* x = x0 + (iter ? (int64_t)((*iter) & 1) * op.n : 0);
    V* yt = reinterpret_cast<V*>(op.ytmp);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < op.n;
         r += (int64_t)gridDim.x * blockDim.x) {
        const V acc = b == 0 ? Sc<V>::mul(cvt<V>(op.diag[r]), x[r]) : yt[r];
        yt[r] = op.block_sum(b, r, x, acc);
    }
}

int grid_for(int64_t n, int block);

template <class M>
template <class V>
void CbSellOp<M>::pre(const V* x0, const int* iter, cudaStream_t s) const {
    for (int b = 0; b + 1 < nb; ++b)
        k_cb_pass<M, V><<<grid_for(n, 256), 256, smem_bytes(), s>>>(*this, b, x0, iter);
}

// Reference row-major ELL (caller-owned, LanczosEigVals_CUDA layout).
template <class M>
struct RefEllOp {
    int64_t n;
    int W;
    const uint32_t* ind;
    const M* val;
    const int16_t* track;
    static constexpr size_t smem_bytes() { return 0; }
    __device__ void init(unsigned char*) {}
    template <class V>
    void pre(const V*, const int*, cudaStream_t) const {}
    template <class V>
    __device__ __forceinline__ V row(int64_t r, const V* __restrict__ x, V& xr) const {
        xr = x[r];
        V acc = Sc<V>::zero();
        int nt = track[r];
        for (int i = 0; i < nt; ++i)
            acc = Sc<V>::fma(cvt<V>(val[r * W + i]), x[ind[r * W + i]], acc);
        return acc;
    }
};

// The matrix-free operator's lookup: the representatives of the active
// orbits in row order (ascending), 32-bit when L <= 32, with a bucket table on
// their top bits, so a generated representative maps straight to its row.
// The norm factor is left out (f = 1): the operator gathers n(c) x_c and
// divides the row by its own norm.
// Slot of a representative in the matrix-free hash table: the splitmix64
// finaliser (Steele, Lea and Flood 2014) of the representative.
__host__ __device__ __forceinline__ uint64_t mf_hash_slot(uint64_t r, uint64_t mask) {
    r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
    r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
    return (r ^ (r >> 31)) & mask;
}
constexpr uint64_t kMfHashEmpty = ~0ull;

struct ActiveLookup {
    const uint32_t* reps32;  // [n] or null
    const uint64_t* reps64;  // [n] when reps32 is null
    const uint32_t* bucket;  // [n_b + 1]: rows of bucket b (top bits r >> shift == b)
    int shift;               // the largest representative's bit length - 24, at least 0
    uint64_t n_b;
    int64_t n;
    int all_active;          // every orbit is a row: a miss is outside the sector
    // Open-addressing table (linear probing, at most half full) of the rows
    // of a sector whose representative table is larger than L2: one 64-bit
    // word per row, (representative << hidx) | row, kMfHashEmpty when free.
    // A lookup then reads one word (usually one 32-byte sector) instead of a
    // bucket entry and a binary search over 8-byte representatives.
    const uint64_t* hash;    // [hmask + 1] or null
    uint64_t hmask;
    int hidx;                // bits of the row index in a word
    __device__ __forceinline__ int find(const RowGen& rg, uint64_t r, int64_t* idx, double* f) const {
        if (hash) {
            uint64_t slot = mf_hash_slot(r, hmask);
            for (uint64_t it = 0; it <= hmask; ++it) {
                const uint64_t w = __ldg(hash + slot);
                if (w == kMfHashEmpty) break;
                if ((w >> hidx) == r) {
                    *idx = (int64_t)(w & ((1ull << hidx) - 1));
                    *f = 1.0;
                    return 1;
                }
                slot = (slot + 1) & hmask;
            }
            if (all_active) return -1;
            return find_rep(rg.rt, r) < 0 ? -1 : 0;  // a null orbit, or outside the sector
        }
        const uint64_t b = r >> shift;
        int64_t lo = 0, hi = 0;
        if (b < n_b) {
            lo = bucket[b];
            hi = bucket[b + 1];
        }
        bool hit;
        if (reps32) {
            const uint32_t k = (uint32_t)r;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (__ldg(reps32 + mid) < k) lo = mid + 1;
                else hi = mid;
            }
            hit = lo < n && __ldg(reps32 + lo) == k;
        } else {
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (__ldg(reps64 + mid) < r) lo = mid + 1;
                else hi = mid;
            }
            hit = lo < n && __ldg(reps64 + lo) == r;
        }
        if (hit) {
            *idx = lo;
            *f = 1.0;
            return 1;
        }
        if (all_active) return -1;
        return find_rep(rg.rt, r) < 0 ? -1 : 0;  // a null orbit, or outside the sector
    }
    // Warp-cooperative form of find() over the bucket table: the 32 lanes of a
    // warp call it together (has = false for a lane without a target).  The
    // lanes' targets are taken one at a time; for each, the warp compares 32
    // consecutive representatives of its bucket range in one coalesced load
    // and a ballot gives the position (ranges longer than 32 take more
    // rounds).  A binary search makes log2(range) dependent loads per lane
    // instead, each from its own line.
    __device__ __forceinline__ int find_warp(const RowGen& rg, bool has, uint64_t r, int64_t* idx,
                                             double* f) const {
        const int lane = threadIdx.x & 31;
        int64_t lo = 0, hi = 0;
        if (has) {
            const uint64_t b = r >> shift;
            if (b < n_b) {
                lo = bucket[b];
                hi = bucket[b + 1];
            }
        }
        int64_t pos = -1;
        unsigned pend = __ballot_sync(0xffffffffu, has && lo < hi);
        while (pend) {
            const int t = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint64_t rt = __shfl_sync(0xffffffffu, r, t);
            const int64_t lt = __shfl_sync(0xffffffffu, lo, t), ht = __shfl_sync(0xffffffffu, hi, t);
            for (int64_t base = lt; base < ht; base += 32) {
                const int64_t p = base + lane;
                bool eq = false;
                if (p < ht) eq = (reps32 ? (uint64_t)__ldg(reps32 + p) : __ldg(reps64 + p)) == rt;
                const unsigned m = __ballot_sync(0xffffffffu, eq);
                if (m) {
                    if (lane == t) pos = base + __ffs(m) - 1;
                    break;
                }
            }
        }
        if (!has) return 0;
        if (pos >= 0) {
            *idx = pos;
            *f = 1.0;
            return 1;
        }
        if (all_active) return -1;
        return find_rep(rg.rt, r) < 0 ? -1 : 0;  // a null orbit, or outside the sector
    }
    // find() of two representatives at once for L <= 32 (reps32 set), in
    // 32-bit arithmetic: the two searches run in
    // lockstep, so each step has two independent loads in flight
    __device__ __forceinline__ void find32x2(const RowGen& rg, uint32_t r1, uint32_t r2, uint32_t* i1,
                                             uint32_t* i2, int* f1, int* f2) const {
        const uint32_t b1 = r1 >> shift, b2 = r2 >> shift;
        uint32_t lo1 = 0, hi1 = 0, lo2 = 0, hi2 = 0;
        if (b1 < (uint32_t)n_b) {
            lo1 = bucket[b1];
            hi1 = bucket[b1 + 1];
        }
        if (b2 < (uint32_t)n_b) {
            lo2 = bucket[b2];
            hi2 = bucket[b2 + 1];
        }
        while (lo1 < hi1 || lo2 < hi2) {
            const bool a1 = lo1 < hi1, a2 = lo2 < hi2;
            const uint32_t m1 = lo1 + ((hi1 - lo1) >> 1), m2 = lo2 + ((hi2 - lo2) >> 1);
            const uint32_t v1 = a1 ? __ldg(reps32 + m1) : 0u, v2 = a2 ? __ldg(reps32 + m2) : 0u;
            if (a1) {
                if (v1 < r1) lo1 = m1 + 1;
                else hi1 = m1;
            }
            if (a2) {
                if (v2 < r2) lo2 = m2 + 1;
                else hi2 = m2;
            }
        }
        const uint32_t nn = (uint32_t)n;
        const uint32_t w1 = lo1 < nn ? __ldg(reps32 + lo1) : ~r1, w2 = lo2 < nn ? __ldg(reps32 + lo2) : ~r2;
        *i1 = lo1;
        *i2 = lo2;
        *f1 = w1 == r1 ? 1 : (all_active ? -1 : (find_rep(rg.rt, r1) < 0 ? -1 : 0));
        *f2 = w2 == r2 ? 1 : (all_active ? -1 : (find_rep(rg.rt, r2) < 0 ? -1 : 0));
    }
};

// Two-site exchange ("hop") form of a term table, for the matrix-free
// operator: every off-diagonal term is c S+_i S-_j at two distinct sites and
// every other term is diagonal (SZ and identity operators only).  Hops on the
// same pair of sites are merged into one entry with the coefficient of each
// direction.
constexpr int kMaxHops = 512;
struct Hop {
    uint64_t pair;  // bits i < j; direction 0 raises site i (bit i zero, bit j one)
};

// A coded layout of a matrix's stored values in one precision (CbSellOp):
// per column block a sliced ELL of 32-bit entries, an 8-bit code into a
// dictionary of at most 255 values above the column inside the block.
struct CbLayout {
    int nb = 0, shift = 0, n_codes = 0;
    DevBuf<int64_t> off;
    DevBuf<int> width;
    DevBuf<uint32_t> packed;
    DevBuf<unsigned char> dict, ytmp;
};

// Matrix-free operator: regenerates every entry of the row.  pre() writes
// xs = n(c) x_c; a row then sums the unscaled entries times xs and divides by
// its own norm, so the only data a generated entry gathers are the active
// representatives it searches and one element of xs (together 8 bytes a row
// at L <= 32 in FP32: 75 MB at L = 32, inside L2).
//
// With a hop table (n_hops > 0) the diagonal comes from the stored vector
// diag and the entries of a row are the hops whose two sites differ in the
// source string: a 64-bit mask of them (per 64 hops) is formed first and its
// set bits are walked, so the threads of a warp run the orbit search and the
// lookup together instead of at the term where each finds an entry.  Up to
// 32 sites the strings, masks, representatives and row indices are 32-bit.
template <class M>
struct MfOp {
    using scalar = M;
    int64_t n;
    RowGen rg;
    ActiveLookup look;
    const double* nrow;  // [n] norm of each row's orbit
    void* xs;            // [n] scaled x in the product's vector type
    int n_hops;
    int hop_one_way;     // some hop has a zero coefficient in one direction
    const Hop* hops;     // [n_hops]
    const double2* hop_c;  // [2 n_hops]: coefficient for bit i = 0, bit j = 1; then the reverse
    const void* diag;    // [n] the diagonal (double2 for complex handles, else double)
    int cplx;
    GroupSmem gs;
    TermsSmem ts;
    const Hop* s_hops;
    const uint32_t* s_pair32;  // low words of the pairs
    const double2* s_hop_c;
    size_t gbytes;
    size_t smem_bytes() const {
        return align16(gbytes) + (n_hops ? (sizeof(Hop) + 2 * sizeof(double2) + sizeof(uint32_t)) * (size_t)n_hops
                                         : terms_smem_bytes(rg.terms));
    }
    __device__ void init(unsigned char* sm) {
        gs = load_group(rg.g, sm);
        if (n_hops) {
            double2* c = reinterpret_cast<double2*>(sm + align16(gbytes));
            Hop* hp = reinterpret_cast<Hop*>(c + 2 * n_hops);
            uint32_t* p32 = reinterpret_cast<uint32_t*>(hp + n_hops);
            for (int i = threadIdx.x; i < n_hops; i += blockDim.x) {
                hp[i] = hops[i];
                p32[i] = (uint32_t)hops[i].pair;
                c[2 * i] = hop_c[2 * i];
                c[2 * i + 1] = hop_c[2 * i + 1];
            }
            s_hops = hp;
            s_pair32 = p32;
            s_hop_c = c;
            __syncthreads();
        } else {
            ts = load_terms(rg.terms, sm + align16(gbytes));
        }
    }
    template <class V>
    void pre(const V* x0, const int* iter, cudaStream_t s) const;
    // sum over the hop entries of the row of src (strings beyond 32 sites)
    template <class V>
    __device__ __forceinline__ V hop_sum64(uint64_t src, const V* __restrict__ xsv) const {
        V acc = Sc<V>::zero();
        for (int base = 0; base < n_hops; base += 64) {
            const int nb = min(64, n_hops - base);
            uint64_t live = 0;
            for (int b = 0; b < nb; ++b) live |= (uint64_t)(__popcll(src & s_hops[base + b].pair) & 1) << b;
            while (live) {
                const int b = base + __ffsll((long long)live) - 1;
                live &= live - 1;
                const uint64_t pair = s_hops[b].pair;
                const double2 cf = s_hop_c[2 * b + ((src & pair & (0ull - pair)) ? 1 : 0)];
                if (hop_one_way && cf.x == 0.0 && cf.y == 0.0) continue;  // no term in this direction
                int e;
                const uint64_t rr = orbit_min(rg.g, gs, src ^ pair, &e);
                int64_t c;
                double f;
                const int found = look.find(rg, rr, &c, &f);
                if (found <= 0) {
                    if (found < 0) *rg.err = 2;
                    continue;
                }
                const double2 ch = rg.g.chars[e];
                const double2 v = make_double2(cf.x * ch.x + cf.y * ch.y, cf.y * ch.x - cf.x * ch.y);
                acc = Sc<V>::fma(Sc<V>::from(v), __ldg(xsv + c), acc);
            }
        }
        return acc;
    }
    // the same up to 32 sites (reps32 set) in 32-bit arithmetic, taking the
    // row's entries two at a time: both orbit minima, then both lookups in
    // lockstep, then both gathers
    template <class V>
    __device__ __forceinline__ V hop_sum32x2(uint32_t src, const V* __restrict__ xsv) const {
        V acc = Sc<V>::zero();
        for (int base = 0; base < n_hops; base += 64) {
            const int nb = min(64, n_hops - base);
            uint64_t live = 0;
            for (int b = 0; b < nb; ++b) live |= (uint64_t)(__popc(src & s_pair32[base + b]) & 1) << b;
            while (live) {
                const int b1 = base + __ffsll((long long)live) - 1;
                live &= live - 1;
                const bool two = live != 0;
                const int b2 = two ? base + __ffsll((long long)live) - 1 : b1;
                live &= live - (two ? 1 : 0);
                const uint32_t p1 = s_pair32[b1], p2 = s_pair32[b2];
                const double2 cf1 = s_hop_c[2 * b1 + ((src & p1 & (0u - p1)) ? 1 : 0)];
                const double2 cf2 = s_hop_c[2 * b2 + ((src & p2 & (0u - p2)) ? 1 : 0)];
                int e1, e2;
                const uint32_t t1 = src ^ p1, t2 = src ^ p2;
                const uint32_t r1 = rg.g.full_rot ? chain_orbit_min(rg.g, gs, t1, &e1)
                                                  : (uint32_t)orbit_min(rg.g, gs, t1, &e1);
                const uint32_t r2 = rg.g.full_rot ? chain_orbit_min(rg.g, gs, t2, &e2)
                                                  : (uint32_t)orbit_min(rg.g, gs, t2, &e2);
                uint32_t c1, c2;
                int f1, f2;
                look.find32x2(rg, r1, r2, &c1, &c2, &f1, &f2);
                // a direction without a term (one-way hops) contributes nothing
                const bool z1 = hop_one_way && cf1.x == 0.0 && cf1.y == 0.0;
                const bool z2 = !two || (hop_one_way && cf2.x == 0.0 && cf2.y == 0.0);
                if (!z1 && f1 < 0) *rg.err = 2;
                if (!z2 && f2 < 0) *rg.err = 2;
                const bool u1 = !z1 && f1 > 0, u2 = !z2 && f2 > 0;
                const V x1 = u1 ? __ldg(xsv + c1) : Sc<V>::zero();
                const V x2 = u2 ? __ldg(xsv + c2) : Sc<V>::zero();
                if (u1) {
                    const double2 ch = rg.g.chars[e1];
                    acc = Sc<V>::fma(Sc<V>::from(make_double2(cf1.x * ch.x + cf1.y * ch.y, cf1.y * ch.x - cf1.x * ch.y)),
                                     x1, acc);
                }
                if (u2) {
                    const double2 ch = rg.g.chars[e2];
                    acc = Sc<V>::fma(Sc<V>::from(make_double2(cf2.x * ch.x + cf2.y * ch.y, cf2.y * ch.x - cf2.x * ch.y)),
                                     x2, acc);
                }
            }
        }
        return acc;
    }
    // The hop sum with the warp-cooperative lookup: the 32 lanes (rows) of a
    // warp step through their live hops together, one hop a lane a round,
    // until every lane's hops are done (act = false: a lane without a row).
    template <class V>
    __device__ __forceinline__ V hop_sum_warp(bool act, uint64_t src, const V* __restrict__ xsv) const {
        V acc = Sc<V>::zero();
        for (int base = 0; base < n_hops; base += 64) {
            const int nb = min(64, n_hops - base);
            uint64_t live = 0;
            if (act)
                for (int b = 0; b < nb; ++b) live |= (uint64_t)(__popcll(src & s_hops[base + b].pair) & 1) << b;
            while (__any_sync(0xffffffffu, live != 0)) {
                bool has = live != 0;
                double2 cf = make_double2(0.0, 0.0);
                uint64_t rr = 0;
                int e = 0;
                if (has) {
                    const int b = base + __ffsll((long long)live) - 1;
                    live &= live - 1;
                    const uint64_t pair = s_hops[b].pair;
                    cf = s_hop_c[2 * b + ((src & pair & (0ull - pair)) ? 1 : 0)];
                    if (hop_one_way && cf.x == 0.0 && cf.y == 0.0) has = false;  // no term in this direction
                    else rr = orbit_min(rg.g, gs, src ^ pair, &e);
                }
                int64_t c = 0;
                double f;
                const int found = look.find_warp(rg, has, rr, &c, &f);
                if (has && found < 0) *rg.err = 2;
                if (has && found > 0) {
                    const double2 ch = rg.g.chars[e];
                    const double2 v = make_double2(cf.x * ch.x + cf.y * ch.y, cf.y * ch.x - cf.x * ch.y);
                    acc = Sc<V>::fma(Sc<V>::from(v), __ldg(xsv + c), acc);
                }
            }
        }
        return acc;
    }
    // row() with the warp-cooperative lookup (hop form only); every lane of
    // the warp calls it, act = false where the lane has no row (r is then any
    // valid row and the result is not used)
    template <class V>
    __device__ __forceinline__ V row_warp(bool act, int64_t r, const V* __restrict__ x, V& xr) const {
        const uint64_t rep = look.reps32 ? (uint64_t)look.reps32[r] : look.reps64[r];
        const uint64_t src = apply_elem(rg.g, gs, 0, rep);
        xr = x[r];
        V acc = hop_sum_warp<V>(act, src, reinterpret_cast<const V*>(xs));
        const double2 d = cplx ? reinterpret_cast<const double2*>(diag)[r]
                               : make_double2(reinterpret_cast<const double*>(diag)[r], 0.0);
        acc = Sc<V>::scale(acc, 1.0 / nrow[r]);
        return Sc<V>::fma(Sc<V>::from(d), xr, acc);
    }
    template <class V>
    __device__ __forceinline__ V row(int64_t r, const V* __restrict__ x, V& xr) const {
        const uint64_t rep = look.reps32 ? (uint64_t)look.reps32[r] : look.reps64[r];
        const uint64_t src = apply_elem(rg.g, gs, 0, rep);
        const V* __restrict__ xsv = reinterpret_cast<const V*>(xs);
        xr = x[r];
        V acc;
        double2 d;
        if (n_hops) {
            acc = look.reps32 ? hop_sum32x2<V>((uint32_t)src, xsv) : hop_sum64<V>(src, xsv);
            d = cplx ? reinterpret_cast<const double2*>(diag)[r]
                     : make_double2(reinterpret_cast<const double*>(diag)[r], 0.0);
        } else {
            acc = Sc<V>::zero();
            d = gen_row_look(rg, gs, ts, 0, ts.n_terms, src, look, [&](int64_t c, double2 v) {
                acc = Sc<V>::fma(Sc<V>::from(v), __ldg(xsv + c), acc);
            });
        }
        acc = Sc<V>::scale(acc, 1.0 / nrow[r]);
        acc = Sc<V>::fma(Sc<V>::from(d), xr, acc);
        return acc;
    }
};

// Minimum resident blocks of 256 threads a product kernel over Op is compiled
// for: the matrix-free operator is issue- and latency-bound and runs best at
// five (at most 48 registers a thread).
template <class Op> struct OpMinBlocks { static constexpr int value = 1; };
template <class M> struct OpMinBlocks<MfOp<M>> { static constexpr int value = 5; };

// xs = n(c) x_c for the matrix-free operator, where x = x0, or with iter the
// half of the Lanczos work buffer x0 that step *iter reads.
template <class V>
__global__ void __launch_bounds__(256) k_mf_scale(int64_t n, const double* __restrict__ nrow,
                                                  const V* __restrict__ x0, const int* __restrict__ iter,
                                                  V* __restrict__ xs) {
    const V* x = x0 + (iter ? (int64_t)((*iter) & 1) * n : 0);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        xs[r] = Sc<V>::scale(x[r], nrow[r]);
}

template <class M>
template <class V>
void MfOp<M>::pre(const V* x0, const int* iter, cudaStream_t s) const {
    k_mf_scale<V><<<grid_for(n, 256), 256, 0, s>>>(n, nrow, x0, iter, reinterpret_cast<V*>(xs));
}

}  // namespace qmb

// Hamiltonian handle.
struct qmb_ham_s {
    qmb_sector sector = nullptr;
    int irrep_gen = 0;  // the sector irrep the handle was built for
    int device = 0;
    int64_t n = 0;
    bool cplx = false;
    int prec = 0;
    int64_t n_slices = 0, padded = 0, nnz = 0;
    int max_row = 0;
    qmb::DevBuf<int64_t> slice_off;
    qmb::DevBuf<int> slice_w;
    qmb::DevBuf<uint32_t> col;        // plain columns
    qmb::DevBuf<unsigned char> val64, val32, diag64, diag32;
    // coded layouts of the stored values (CbSellOp): FP32 (column-blocked for
    // vectors larger than L2, else one block) and real FP64 (one block)
    qmb::CbLayout cb32, cb64;
    bool cb64_shared = false;  // cb64 reads cb32's packed entries (its own dictionary and partial sums)
    // terms kept for the matrix-free operator
    int n_terms = 0, n_col = 0;
    qmb::DevBuf<int> t_nops;
    qmb::DevBuf<uint16_t> t_ops;
    qmb::DevBuf<double2> t_scalar;
    qmb::DevBuf<int> err;
    // hop form of the terms (n_hops > 0), for the matrix-free operator
    int n_hops = 0;
    int hop_one_way = 0;
    qmb::DevBuf<qmb::Hop> hops;
    qmb::DevBuf<double2> hop_c;
    // matrix-free lookup over the active orbits (mf_tables(), on first use)
    bool mf_ready = false;
    int mf_shift = 0;
    uint64_t mf_nb = 0;
    qmb::DevBuf<uint32_t> mf_reps32;   // [n] active representatives, L <= 32
    qmb::DevBuf<uint64_t> mf_reps64;   // [n] L > 32 with null orbits (else the sector's table)
    qmb::DevBuf<uint32_t> mf_bucket;   // [mf_nb + 1]
    qmb::DevBuf<uint64_t> mf_hash;     // rows by representative, beyond 32 sites when the table exceeds L2
    uint64_t mf_hmask = 0;
    int mf_hidx = 0;
    qmb::DevBuf<double> mf_norm;       // [n] norm of each row's orbit
    qmb::DevBuf<unsigned char> mf_diag;  // [n] diagonal with a hop table (double2 if complex)
    qmb::DevBuf<unsigned char> mf_xs;  // [n] n(c) x_c in the product's vector type
    // Lanczos buffers kept between qmb_lanczos calls (one call at a time on
    // a handle): the stored basis ring, the two work vectors, and the ring
    // slots the last solve used
    qmb::DevBuf<unsigned char> lz_ring, lz_wbuf;
    int lz_ring_hint = 0;
    // ground state kept by qmb_lanczos
    qmb::DevBuf<unsigned char> psi;
    int64_t psi_n = 0;

    qmb::TermsArgs terms_args() const {
        qmb::TermsArgs t;
        t.n_terms = n_terms;
        t.n_col = n_col;
        t.n_ops = t_nops.p;
        t.ops = t_ops.p;
        t.scalar = t_scalar.p;
        return t;
    }
    qmb::RowGen row_gen() const {
        qmb::RowGen r;
        r.g = sector->group_args();
        r.rt = sector->rep_table();
        r.terms = terms_args();
        r.norms = sector->norms.p;
        r.row_of_orbit = sector->row_of_orbit.p;
        r.orbit_of_row = sector->orbit_of_row.p;
        r.tol = sector->tol_norm;
        r.n_up = sector->n_up;
        r.err = err.p;
        return r;
    }
    template <class M> qmb::SellOp<M> sell(bool fp64) const {
        qmb::SellOp<M> op;
        op.n = n;
        op.off = slice_off.p;
        op.width = slice_w.p;
        op.col = col.p;
        op.val = reinterpret_cast<const M*>(fp64 ? val64.p : val32.p);
        op.diag = reinterpret_cast<const M*>(fp64 ? diag64.p : diag32.p);
        return op;
    }
    template <class M> qmb::CbSellOp<M> cb() const {
        constexpr bool f64 = sizeof(typename qmb::Sc<M>::real) == 8;
        const qmb::CbLayout& L = f64 ? cb64 : cb32;
        const qmb::CbLayout& E = (f64 && cb64_shared) ? cb32 : L;  // where the entries live
        qmb::CbSellOp<M> op;
        op.n = n;
        op.nb = L.nb;
        op.shift = L.shift;
        op.n_slices = n_slices;
        op.off = E.off.p;
        op.width = E.width.p;
        op.packed = E.packed.p;
        op.dict = reinterpret_cast<const M*>(L.dict.p);
        op.diag = reinterpret_cast<const M*>(f64 ? diag64.p : diag32.p);
        op.ytmp = L.ytmp.p;
        op.sdict = nullptr;
        return op;
    }
    // the matrix-free operator (mf_tables() must have run)
    template <class M> qmb::MfOp<M> mf() const {
        qmb::MfOp<M> op;
        op.n = n;
        op.rg = row_gen();
        op.look.reps32 = mf_reps32.p;
        op.look.reps64 = mf_reps32.p ? nullptr : (mf_reps64.p ? mf_reps64.p : sector->reps.p);
        op.look.bucket = mf_bucket.p;
        op.look.shift = mf_shift;
        op.look.n_b = mf_nb;
        op.look.n = n;
        op.look.all_active = sector->n_active == sector->R ? 1 : 0;
        // QMB_MF_HASH=0 searches the bucket table even where the hash table exists
        const char* he = std::getenv("QMB_MF_HASH");
        op.look.hash = (mf_hash.p && !(he && he[0] == '0')) ? mf_hash.p : nullptr;
        op.look.hmask = mf_hmask;
        op.look.hidx = mf_hidx;
        op.nrow = mf_norm.p;
        op.xs = mf_xs.p;
        op.n_hops = n_hops;
        op.hop_one_way = hop_one_way;
        op.hops = hops.p;
        op.hop_c = hop_c.p;
        op.diag = mf_diag.p;
        op.cplx = cplx ? 1 : 0;
        op.s_hops = nullptr;
        op.s_pair32 = nullptr;
        op.s_hop_c = nullptr;
        op.gbytes = qmb::group_smem_bytes(op.rg.g);
        return op;
    }
};

namespace qmb {
// Builds the matrix-free operator's tables on the handle (once).
void mf_tables(qmb_ham_s* h);
// The hop form of a validated term table (for the matrix-free operator).
void hop_form(qmb_ham_s* h, const qmb_terms* t);
// The coded FP32 layout of a built matrix, when it pays (CbSellOp).
void build_cb(qmb_ham_s* h);
// Upload operator tables (validated) into the handle's term buffers.
void upload_terms(qmb_ham_s* h, const qmb_terms* t, int L);
int grid_for(int64_t n, int block);
void set_group_smem_attr(const void* kernel, size_t bytes);
bool fits_device(size_t bytes);
}  // namespace qmb
