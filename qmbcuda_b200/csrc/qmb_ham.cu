// qmb_ham.cu -- symmetric-basis XXZ matrix on the GPU.
//
// Builds the matrix of the active rows of a sector's irrep from operator
// tables with the rule of BuildHamiltonianXXZForAbelianGroup
// (exact_diagonalization/utils.cu:83-184), into a sliced ELL layout: rows in
// 32-row slices, slot j of the slice stored contiguously for its 32 rows, so
// a warp's loads of one slot are one coalesced 128-byte (FP32) / 256-byte
// (FP64) transaction.  Slice width = longest row of the slice.  The diagonal
// is a separate dense vector.  Two passes: count entries per row, then fill.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "qmb_ham.cuh"

namespace qmb {

// The hop form of a validated term table (MfOp): every term either diagonal
// (SZ and identity operators) or one SP and one SM at two distinct sites with
// nothing else; otherwise n_hops = 0 and the operator runs the general term
// loop.  Hops on the same two sites merge, per direction.
void hop_form(qmb_ham_s* h, const qmb_terms* t) {
    h->n_hops = 0;
    std::vector<Hop> hp;
    std::vector<double2> cf;
    for (int i = 0; i < t->n_terms; ++i) {
        int sp = -1, sm = -1, n_sz = 0, n_other = 0;
        for (int j = 0; j < t->n_ops[i]; ++j) {
            const int c = t->op_code[i * t->n_col + j], st = t->op_site[i * t->n_col + j];
            if (c == QMB_OP_SP) {
                if (sp >= 0) ++n_other;
                sp = st;
            } else if (c == QMB_OP_SM) {
                if (sm >= 0) ++n_other;
                sm = st;
            } else if (c == QMB_OP_SZ) {
                ++n_sz;
            }
        }
        if (sp < 0 && sm < 0) continue;  // diagonal
        if (sp < 0 || sm < 0 || sp == sm || n_sz || n_other) return;
        const int a = std::min(sp, sm), b = std::max(sp, sm);
        const uint64_t pair = (1ull << a) | (1ull << b);
        size_t k = 0;
        while (k < hp.size() && hp[k].pair != pair) ++k;
        if (k == hp.size()) {
            if ((int)hp.size() == kMaxHops) return;
            hp.push_back(Hop{pair});
            cf.push_back(make_double2(0.0, 0.0));
            cf.push_back(make_double2(0.0, 0.0));
        }
        // raising the lower site a (bit a zero, bit b one) is direction 0
        double2& c = cf[2 * k + (sp == a ? 0 : 1)];
        c.x += t->scalar[2 * i];
        c.y += t->scalar[2 * i + 1];
    }
    if (hp.empty()) return;
    h->hop_one_way = 0;
    for (const double2& c : cf)
        if (c.x == 0.0 && c.y == 0.0) h->hop_one_way = 1;
    h->hops.alloc(hp.size());
    h->hops.upload(hp.data(), hp.size());
    h->hop_c.alloc(cf.size());
    h->hop_c.upload(cf.data(), cf.size());
    h->n_hops = (int)hp.size();
}

void upload_terms(qmb_ham_s* h, const qmb_terms* t, int L) {
    QMB_REQUIRE(t && t->n_ops && t->op_code && t->op_site && t->scalar, QMB_ERR_INVALID,
                "terms: null table");
    QMB_REQUIRE(t->n_terms >= 0 && t->n_terms <= kMaxTerms, QMB_ERR_INVALID,
                "terms: n_terms must be in 0..4096");
    QMB_REQUIRE(t->n_col >= 1 && t->n_col <= kMaxCol, QMB_ERR_INVALID,
                "terms: n_col must be in 1..8");
    std::vector<int> nops(t->n_terms);
    std::vector<uint16_t> ops((size_t)t->n_terms * t->n_col, 0);
    std::vector<double2> sc(t->n_terms);
    for (int i = 0; i < t->n_terms; ++i) {
        QMB_REQUIRE(t->n_ops[i] >= 0 && t->n_ops[i] <= t->n_col, QMB_ERR_INVALID,
                    "terms: n_ops out of range");
        nops[i] = t->n_ops[i];
        for (int j = 0; j < t->n_ops[i]; ++j) {
            int c = t->op_code[i * t->n_col + j], s = t->op_site[i * t->n_col + j];
            QMB_REQUIRE(c >= 0 && c <= 255, QMB_ERR_INVALID, "terms: op code out of range");
            QMB_REQUIRE(s >= 0 && s < L, QMB_ERR_INVALID, "terms: site out of range");
            ops[(size_t)i * t->n_col + j] = (uint16_t)(c << 8 | s);
        }
        sc[i] = make_double2(t->scalar[2 * i], t->scalar[2 * i + 1]);
        QMB_REQUIRE(std::isfinite(sc[i].x) && std::isfinite(sc[i].y), QMB_ERR_INVALID,
                    "terms: non-finite scalar");
    }
    hop_form(h, t);
    h->n_terms = t->n_terms;
    h->n_col = t->n_col;
    h->t_nops.alloc(std::max(1, t->n_terms));
    h->t_ops.alloc(std::max<size_t>(1, ops.size()));
    h->t_scalar.alloc(std::max(1, t->n_terms));
    if (t->n_terms) {
        h->t_nops.upload(nops.data(), nops.size());
        h->t_ops.upload(ops.data(), ops.size());
        h->t_scalar.upload(sc.data(), sc.size());
    }
}

static size_t gen_smem(const RowGen& rg) {
    return align16(group_smem_bytes(rg.g)) + terms_smem_bytes(rg.terms);
}

#define QMB_LOAD_GEN(rg)                                             \
    extern __shared__ __align__(16) unsigned char smem[];            \
    GroupSmem gs = load_group((rg).g, smem);                         \
    TermsSmem ts = load_terms((rg).terms, smem + align16(group_smem_bytes((rg).g)))

// -------------------------------------------------------------- kernels
__global__ void k_ell_count(RowGen rg, int64_t n, int* __restrict__ cnt) {
    QMB_LOAD_GEN(rg);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = rg.orbit_of_row[r];
        uint64_t src = apply_elem(rg.g, gs, 0, rg.rt.reps[o]);
        int c = 0;
        gen_row(rg, gs, ts, src, rg.norms[o], [&](int64_t, double2) { ++c; });
        cnt[r] = c;
    }
}

__global__ void k_slice_width(const int* __restrict__ cnt, int64_t n, int64_t n_slices,
                              int* __restrict__ width, int64_t* __restrict__ slots) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n_slices;
         s += (int64_t)gridDim.x * blockDim.x) {
        int w = 0;
        for (int i = 0; i < 32; ++i) {
            int64_t r = s * 32 + i;
            if (r < n) w = max(w, cnt[r]);
        }
        width[s] = w;
        slots[s] = (int64_t)w * 32;
    }
}

template <class M>
__global__ void k_ell_fill(RowGen rg, int64_t n, const int64_t* __restrict__ off,
                           const int* __restrict__ width, uint32_t* __restrict__ col,
                           M* __restrict__ val, M* __restrict__ diag) {
    QMB_LOAD_GEN(rg);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = rg.orbit_of_row[r];
        uint64_t src = apply_elem(rg.g, gs, 0, rg.rt.reps[o]);
        int64_t s = r >> 5;
        int64_t base = off[s] + (r & 31);
        int w = width[s];
        int j = 0;
        double2 d = gen_row(rg, gs, ts, src, rg.norms[o], [&](int64_t ot, double2 v) {
            if (j < w) {
                col[base + (int64_t)j * 32] = (uint32_t)rg.row_of_orbit[ot];
                val[base + (int64_t)j * 32] = Sc<M>::from(v);
            }
            ++j;
        });
        for (; j < w; ++j) {
            col[base + (int64_t)j * 32] = (uint32_t)r;
            val[base + (int64_t)j * 32] = Sc<M>::zero();
        }
        diag[r] = Sc<M>::from(d);
    }
}

// Reference row-major layout over all orbits (null rows: track 0, ind[row*W] = row).
__global__ void k_ell_ref(RowGen rg, int64_t R, int W, uint32_t* __restrict__ ind,
                          double2* __restrict__ val, int16_t* __restrict__ track,
                          int* __restrict__ overflow) {
    QMB_LOAD_GEN(rg);
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < R;
         id += (int64_t)gridDim.x * blockDim.x) {
        ind[id * W] = (uint32_t)id;
        double ns = rg.norms[id];
        if (ns < rg.tol) continue;
        uint64_t src = apply_elem(rg.g, gs, 0, rg.rt.reps[id]);
        int t = 1;
        double2 d = gen_row(rg, gs, ts, src, ns, [&](int64_t ot, double2 v) {
            if (t < W) {
                ind[id * W + t] = (uint32_t)ot;
                val[id * W + t] = v;
            } else {
                *overflow = 1;
            }
            ++t;
        });
        val[id * W] = d;
        track[id] = (int16_t)min(t, 32767);
    }
}

template <class Op, class V>
__global__ void __launch_bounds__(256, OpMinBlocks<Op>::value) k_hv(Op op, const V* __restrict__ x, V* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem_hv[];
    op.init(smem_hv);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < op.n;
         r += (int64_t)gridDim.x * blockDim.x) {
        V xr;
        y[r] = op.row(r, x, xr);
    }
}

// The matrix-free product with the warp-cooperative lookup (hop form): the
// rows run a warp at a time, so that every lane takes part in the warp's
// lookups, including lanes past the last row.
template <class M, class V>
__global__ void __launch_bounds__(256, 5) k_hv_mfw(MfOp<M> op, const V* __restrict__ x, V* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem_hv[];
    op.init(smem_hv);
    const int lane = threadIdx.x & 31;
    for (int64_t r0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x - lane; r0 < op.n;
         r0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = r0 + lane;
        const bool act = r < op.n;
        V xr;
        const V v = op.template row_warp<V>(act, act ? r : r0, x, xr);
        if (act) y[r] = v;
    }
}

template <class M32, class M64>
__global__ void k_narrow(const M64* __restrict__ a, M32* __restrict__ b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        b[i] = cvt<M32>(a[i]);
}

// ------------------------------------------------------------- helpers
template <class Op, class V>
void launch_hv(const Op& op, const V* x, V* y, cudaStream_t st, size_t smem) {
    const void* fn = (const void*)k_hv<Op, V>;
    set_group_smem_attr(fn, smem);
    op.pre(x, (const int*)nullptr, st);  // column-block passes or the matrix-free scaling, if any
    k_hv<Op, V><<<grid_for(op.n, 256), 256, smem, st>>>(op, x, y);
    check_launch("k_hv");
}

void build_sell(qmb_ham_s* h) {
    RowGen rg = h->row_gen();
    size_t sm = gen_smem(rg);
    int64_t n = h->n;
    DevBuf<int> cnt(n);
    set_group_smem_attr((const void*)k_ell_count, sm);
    k_ell_count<<<grid_for(n, 128), 128, sm>>>(rg, n, cnt.p);
    check_launch("k_ell_count");
    h->n_slices = (n + 31) / 32;
    h->slice_w.alloc(h->n_slices);
    DevBuf<int64_t> slots(h->n_slices + 1);
    QMB_CUDA_TRY(cudaMemset(slots.p + h->n_slices, 0, sizeof(int64_t)));
    k_slice_width<<<grid_for(h->n_slices, 256), 256>>>(cnt.p, n, h->n_slices, h->slice_w.p,
                                                       slots.p);
    check_launch("k_slice_width");
    h->slice_off.alloc(h->n_slices + 1);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, slots.p, h->slice_off.p, h->n_slices + 1);
    DevBuf<unsigned char> tmp(tb);
    cub::DeviceScan::ExclusiveSum(tmp.p, tb, slots.p, h->slice_off.p, h->n_slices + 1);
    QMB_CUDA_TRY(cudaMemcpy(&h->padded, h->slice_off.p + h->n_slices, sizeof(int64_t),
                            cudaMemcpyDeviceToHost));
    // statistics
    std::vector<int> hc(n);
    cnt.download(hc.data(), n);
    QMB_CUDA_TRY(cudaDeviceSynchronize());
    h->nnz = 0;
    h->max_row = 0;
    for (int64_t i = 0; i < n; ++i) {
        h->nnz += hc[i];
        h->max_row = std::max(h->max_row, hc[i]);
    }
    int err = 0;
    QMB_CUDA_TRY(cudaMemcpy(&err, h->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    QMB_REQUIRE(err == 0, QMB_ERR_INVALID,
                err == 1 ? "a term changes the number of up spins (not an XXZ-type term)"
                         : "a target string has no representative (inconsistent group)");

    size_t es = h->cplx ? sizeof(double2) : sizeof(double);
    h->col.alloc(std::max<int64_t>(h->padded, 1));
    h->val64.alloc(std::max<int64_t>(h->padded, 1) * es);
    h->diag64.alloc(n * es);
    QMB_CUDA_TRY(cudaMemset(h->col.p, 0, sizeof(uint32_t) * h->col.n));
    QMB_CUDA_TRY(cudaMemset(h->val64.p, 0, h->val64.n));
    if (h->cplx) {
        set_group_smem_attr((const void*)k_ell_fill<double2>, sm);
        k_ell_fill<double2><<<grid_for(n, 128), 128, sm>>>(
            rg, n, h->slice_off.p, h->slice_w.p, h->col.p, (double2*)h->val64.p,
            (double2*)h->diag64.p);
    } else {
        set_group_smem_attr((const void*)k_ell_fill<double>, sm);
        k_ell_fill<double><<<grid_for(n, 128), 128, sm>>>(rg, n, h->slice_off.p, h->slice_w.p,
                                                           h->col.p, (double*)h->val64.p,
                                                           (double*)h->diag64.p);
    }
    check_launch("k_ell_fill");
    if (h->prec & QMB_PREC_FP32) {
        size_t e32 = h->cplx ? sizeof(float2) : sizeof(float);
        h->val32.alloc(std::max<int64_t>(h->padded, 1) * e32);
        h->diag32.alloc(n * e32);
        if (h->cplx) {
            k_narrow<float2, double2><<<grid_for(h->padded, 256), 256>>>(
                (double2*)h->val64.p, (float2*)h->val32.p, h->padded);
            k_narrow<float2, double2><<<grid_for(n, 256), 256>>>((double2*)h->diag64.p,
                                                                (float2*)h->diag32.p, n);
        } else {
            k_narrow<float, double><<<grid_for(h->padded, 256), 256>>>(
                (double*)h->val64.p, (float*)h->val32.p, h->padded);
            k_narrow<float, double><<<grid_for(n, 256), 256>>>((double*)h->diag64.p,
                                                              (float*)h->diag32.p, n);
        }
        check_launch("k_narrow");
    }
    QMB_CUDA_TRY(cudaDeviceSynchronize());
}

// ------------------------------------------ column-blocked coded layout
constexpr int kCbMaxBlocks = 32;                     // column blocks at most
constexpr size_t kCbBlockBytes = (size_t)64 << 20;   // x bytes of one column block
constexpr double kCbMinVecBytes = 256.0 * (1 << 20); // vectors from this size on (2x L2)
constexpr double kCbMinStreamBytes = 256.0 * (1 << 20);  // single block: plain entries (8 B) from this size on
constexpr double kCbMaxSingleVecBytes = 96.0 * (1 << 20);  // single FP64 block: x bytes up to this (L2 126 MB)
constexpr int kCbMissCap = 1024;                     // values outside the dictionary kept per pass

// Bit pattern of a matrix value (the dictionary key).
__device__ __forceinline__ uint64_t val_key(float v) { return __float_as_uint(v); }
__device__ __forceinline__ uint64_t val_key(float2 v) {
    return ((uint64_t)__float_as_uint(v.y) << 32) | __float_as_uint(v.x);
}
__device__ __forceinline__ uint64_t val_key(double v) { return (uint64_t)__double_as_longlong(v); }
__device__ __forceinline__ bool val_zero(float v) { return v == 0.0f; }
__device__ __forceinline__ bool val_zero(double v) { return v == 0.0; }
__device__ __forceinline__ bool val_zero(float2 v) { return v.x == 0.0f && v.y == 0.0f; }
__device__ __forceinline__ bool val_zero(double2 v) { return v.x == 0.0 && v.y == 0.0; }

// Every stride-th slot of the sliced ELL's FP32 values (dictionary sample).
template <class M>
__global__ void k_cb_sample(const M* __restrict__ val, int64_t padded, int64_t stride, int64_t n_out,
                            uint64_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_out;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i * stride;
        out[i] = k < padded ? val_key(val[k]) : 0ull;
    }
}

// Entries of row r (nonzero values) per column block: cnt[b * n + r].
template <class M>
__global__ void k_cb_count(SellOp<M> a, int shift, int nb, uint8_t* __restrict__ cnt) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.n;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = r >> 5;
        const int lane = (int)(r & 31);
        const int w = a.width[s];
        int c[kCbMaxBlocks];
        for (int b = 0; b < nb; ++b) c[b] = 0;
        for (int j = 0; j < w; ++j) {
            const int64_t k = a.off[s] + (int64_t)j * 32 + lane;
            if (val_zero(a.val[k])) continue;
            c[a.col[k] >> shift] += 1;
        }
        for (int b = 0; b < nb; ++b) cnt[(int64_t)b * a.n + r] = (uint8_t)c[b];
    }
}

// Width of every (block, slice) and its slot count, slots[b * n_slices + s].
__global__ void k_cb_width(const uint8_t* __restrict__ cnt, int64_t n, int64_t n_slices, int nb,
                           int* __restrict__ width, int64_t* __restrict__ slots) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)nb * n_slices;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / n_slices);
        const int64_t s = i % n_slices;
        int w = 0;
        for (int l = 0; l < 32; ++l) {
            const int64_t r = s * 32 + l;
            if (r < n) w = max(w, (int)cnt[(int64_t)b * n + r]);
        }
        width[i] = w;
        slots[i] = (int64_t)w * 32;
    }
}

// Packs every nonzero entry as code << 24 | column inside its block into its
// block's slice.  A value outside the dictionary goes into the open-addressed
// set miss_keys [kCbMissCap] (empty slots hold ~0); miss[0] counts the
// distinct values inserted, miss[1] the ones that found no free slot.
template <class M>
__global__ void k_cb_fill(SellOp<M> a, int shift, int nb, const int64_t* __restrict__ off,
                          const uint64_t* __restrict__ keys, int n_keys, uint32_t* __restrict__ packed,
                          int* __restrict__ miss, unsigned long long* __restrict__ miss_keys) {
    __shared__ uint64_t sk[256];
    for (int i = threadIdx.x; i < n_keys; i += blockDim.x) sk[i] = keys[i];
    __syncthreads();
    const int64_t n_slices = (a.n + 31) / 32;
    const uint32_t lmask = (1u << shift) - 1u;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.n;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = r >> 5;
        const int lane = (int)(r & 31);
        const int w = a.width[s];
        int pos[kCbMaxBlocks];
        for (int b = 0; b < nb; ++b) pos[b] = 0;
        for (int j = 0; j < w; ++j) {
            const int64_t k = a.off[s] + (int64_t)j * 32 + lane;
            const M v = a.val[k];
            if (val_zero(v)) continue;
            const uint64_t key = val_key(v);
            int lo = 0, hi = n_keys;  // first key >= key
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (sk[mid] < key) lo = mid + 1;
                else hi = mid;
            }
            if (lo == n_keys || sk[lo] != key) {
                uint32_t hsh = (uint32_t)(key ^ (key >> 29)) * 0x9e3779b1u;
                int probe = 0;
                for (; probe < kCbMissCap; ++probe) {
                    const int at = (int)((hsh + (uint32_t)probe) & (uint32_t)(kCbMissCap - 1));
                    const unsigned long long prev = atomicCAS(miss_keys + at, ~0ull, (unsigned long long)key);
                    if (prev == ~0ull) atomicAdd(miss, 1);
                    if (prev == ~0ull || prev == key) break;
                }
                if (probe == kCbMissCap) atomicAdd(miss + 1, 1);
                continue;
            }
            const uint32_t c = a.col[k];
            const int b = (int)(c >> shift);
            packed[off[(int64_t)b * n_slices + s] + (int64_t)pos[b] * 32 + lane] =
                ((uint32_t)(lo + 1) << 24) | (c & lmask);
            pos[b] += 1;
        }
    }
}

// The column-blocked coded FP32 layout of a built matrix (CbSellOp), when its
// vector is larger than L2 (at least kCbMinVecBytes), every row has fewer
// than 256 entries, the FP32 off-diagonal values take at most 255 distinct
// values and the layout fits in free memory.  Otherwise the handle keeps the
// plain sliced ELL only.  QMB_COLUMN_BLOCKS=0 turns the layout off.
// QMB_TRACE=1 says why a matrix gets no column-blocked layout.
static void cb_skip(const char* why) {
    const char* e = std::getenv("QMB_TRACE");
    if (e && *e && *e != '0') std::fprintf(stderr, "[qmb ham] no column-blocked layout: %s\n", why);
}

template <class M>
static void build_cb_t(qmb_ham_s* h, int forced_shift, bool single, CbLayout& L) {
    constexpr bool f64 = sizeof(typename Sc<M>::real) == 8;
    const int64_t n = h->n;
    const size_t es = sizeof(M);
    int shift = 24;
    if (!single)
        while (shift > 10 && ((size_t)1 << shift) * es > kCbBlockBytes) --shift;
    if (forced_shift) shift = forced_shift;
    const int nb = (int)((n + ((int64_t)1 << shift) - 1) >> shift);
    if (nb < (single ? 1 : 2) || nb > (single ? 1 : kCbMaxBlocks) || h->max_row > 255) {
        cb_skip("block count or row length out of range");
        return;
    }
    SellOp<M> a = h->sell<M>(f64);
    // dictionary from a strided sample of the values
    const int64_t n_samp = std::min<int64_t>(h->padded, (int64_t)1 << 20);
    const int64_t stride = std::max<int64_t>(1, h->padded / n_samp);
    std::vector<uint64_t> keys;
    {
        DevBuf<uint64_t> smp(n_samp);
        k_cb_sample<M><<<grid_for(n_samp, 256), 256>>>(a.val, h->padded, stride, n_samp, smp.p);
        check_launch("k_cb_sample");
        std::vector<uint64_t> hs(n_samp);
        smp.download(hs.data(), n_samp);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
        std::sort(hs.begin(), hs.end());
        hs.erase(std::unique(hs.begin(), hs.end()), hs.end());
        for (uint64_t k : hs) {
            // +-0 in every component
            const bool zero = f64 ? (k << 1) == 0
                                  : es == 4 ? ((uint32_t)k << 1) == 0
                                            : (((uint32_t)k << 1) == 0 && ((uint32_t)(k >> 32) << 1) == 0);
            if (!zero) keys.push_back(k);
        }
    }
    if (keys.empty() || keys.size() > 255) {
        cb_skip("no values, or more than 255 distinct values in the sample");
        return;
    }
    // per-block widths and offsets
    const int64_t ns = h->n_slices;
    size_t fr = 0, tot = 0;
    QMB_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    if ((size_t)nb * n + 2 * n * 16 > fr / 2) {
        cb_skip("not enough free memory for the counts");
        return;
    }
    DevBuf<uint8_t> cnt((size_t)nb * n);
    k_cb_count<M><<<grid_for(n, 256), 256>>>(a, shift, nb, cnt.p);
    check_launch("k_cb_count");
    DevBuf<int> width((size_t)nb * ns);
    DevBuf<int64_t> slots((size_t)nb * ns + 1), off((size_t)nb * ns + 1);
    QMB_CUDA_TRY(cudaMemset(slots.p + (size_t)nb * ns, 0, sizeof(int64_t)));
    k_cb_width<<<grid_for((int64_t)nb * ns, 256), 256>>>(cnt.p, n, ns, nb, width.p, slots.p);
    check_launch("k_cb_width");
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, slots.p, off.p, (int64_t)nb * ns + 1);
    DevBuf<unsigned char> tmp(tb);
    cub::DeviceScan::ExclusiveSum(tmp.p, tb, slots.p, off.p, (int64_t)nb * ns + 1);
    int64_t total = 0;
    QMB_CUDA_TRY(cudaMemcpy(&total, off.p + (size_t)nb * ns, sizeof(int64_t), cudaMemcpyDeviceToHost));
    cnt.release();
    QMB_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    const size_t need = (size_t)total * 4 + (size_t)n * (h->cplx ? 16 : 8);
    if (need > fr / 10 * 9) {
        cb_skip("not enough free memory for the packed entries");
        return;
    }
    DevBuf<uint32_t> packed(std::max<int64_t>(total, 1));
    QMB_CUDA_TRY(cudaMemset(packed.p, 0, sizeof(uint32_t) * packed.n));
    DevBuf<int> miss(2);
    DevBuf<unsigned long long> mkeys(kCbMissCap);
    // values the sample missed join the dictionary and the pass repeats (it
    // rewrites every entry in place)
    for (int round = 0;; ++round) {
        DevBuf<uint64_t> dkeys(keys.size());
        dkeys.upload(keys.data(), keys.size());
        miss.zero();
        QMB_CUDA_TRY(cudaMemset(mkeys.p, 0xff, sizeof(unsigned long long) * kCbMissCap));
        k_cb_fill<M><<<grid_for(n, 256), 256>>>(a, shift, nb, off.p, dkeys.p, (int)keys.size(), packed.p,
                                                miss.p, mkeys.p);
        check_launch("k_cb_fill");
        int hm[2] = {0, 0};
        QMB_CUDA_TRY(cudaMemcpy(hm, miss.p, sizeof(hm), cudaMemcpyDeviceToHost));
        if (hm[0] == 0 && hm[1] == 0) break;
        if (hm[1] > 0 || round == 2) {
            cb_skip("more distinct values than the dictionary holds");
            return;
        }
        std::vector<unsigned long long> extra(kCbMissCap);
        QMB_CUDA_TRY(cudaMemcpy(extra.data(), mkeys.p, sizeof(unsigned long long) * kCbMissCap,
                                cudaMemcpyDeviceToHost));
        for (unsigned long long k : extra)
            if (k != ~0ull) keys.push_back(k);
        std::sort(keys.begin(), keys.end());
        keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
        if (keys.size() > 255) {
            cb_skip("more than 255 distinct values");
            return;
        }
    }
    // dictionary: code 0 is the padding (value 0), code c the key c-1
    std::vector<M> dict(256);
    std::memset(dict.data(), 0, sizeof(M) * 256);
    for (size_t i = 0; i < keys.size(); ++i) std::memcpy(&dict[i + 1], &keys[i], sizeof(M));
    L.dict.alloc(256 * sizeof(M));
    QMB_CUDA_TRY(cudaMemcpy(L.dict.p, dict.data(), 256 * sizeof(M), cudaMemcpyHostToDevice));
    if (nb > 1) L.ytmp.alloc((size_t)n * (h->cplx ? 16 : 8));
    L.off = std::move(off);
    L.width = std::move(width);
    L.packed = std::move(packed);
    L.nb = nb;
    L.shift = shift;
    L.n_codes = (int)keys.size();
    QMB_CUDA_TRY(cudaDeviceSynchronize());
}

// The FP64 values of a matrix whose FP32 values are coded: when every FP32
// code stands for one FP64 value (and no FP64 value rounds to an FP32 zero),
// the FP64 products read the same packed entries through an FP64 dictionary
// of their own, so the FP64 coded layout costs no entry memory.
constexpr unsigned long long kDictEmpty = 0x7ff4dead0000beefull;  // a NaN pattern
template <class M32, class M64>
__global__ void k_cb_dict64(SellOp<M32> a, const M64* __restrict__ val64, const uint64_t* __restrict__ keys,
                            int n_keys, unsigned long long* __restrict__ dict_bits, int* __restrict__ bad) {
    __shared__ uint64_t sk[256];
    for (int i = threadIdx.x; i < n_keys; i += blockDim.x) sk[i] = keys[i];
    __syncthreads();
    constexpr int W = (int)(sizeof(M64) / 8);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.n;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = r >> 5;
        const int lane = (int)(r & 31);
        const int w = a.width[s];
        for (int j = 0; j < w; ++j) {
            const int64_t k = a.off[s] + (int64_t)j * 32 + lane;
            const M32 v = a.val[k];
            const M64 v64 = val64[k];
            if (val_zero(v)) {
                if (!val_zero(v64)) atomicExch(bad, 1);
                continue;
            }
            const uint64_t key = val_key(v);
            int lo = 0, hi = n_keys;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (sk[mid] < key) lo = mid + 1;
                else hi = mid;
            }
            if (lo == n_keys || sk[lo] != key) {
                atomicExch(bad, 1);
                continue;
            }
            const unsigned long long* vb = reinterpret_cast<const unsigned long long*>(&v64);
#pragma unroll
            for (int q = 0; q < W; ++q) {
                const unsigned long long prev = atomicCAS(dict_bits + (lo + 1) * W + q, kDictEmpty, vb[q]);
                if (prev != kDictEmpty && prev != vb[q]) atomicExch(bad, 1);
            }
        }
    }
}

template <class M32, class M64>
static void share_cb64_t(qmb_ham_s* h) {
    const CbLayout& L32 = h->cb32;
    const int n_keys = L32.n_codes;
    std::vector<M32> d32(256);
    QMB_CUDA_TRY(cudaMemcpy(d32.data(), L32.dict.p, 256 * sizeof(M32), cudaMemcpyDeviceToHost));
    std::vector<uint64_t> keys(n_keys);
    for (int i = 0; i < n_keys; ++i) {
        uint64_t k = 0;
        std::memcpy(&k, &d32[i + 1], sizeof(M32));  // the bits val_key() reads: x low, y high
        keys[i] = k;
    }
    constexpr int W = (int)(sizeof(M64) / 8);
    DevBuf<uint64_t> dkeys(std::max(1, n_keys));
    dkeys.upload(keys.data(), n_keys);
    std::vector<unsigned long long> hb(256 * W, kDictEmpty);
    DevBuf<unsigned long long> bits(256 * W);
    bits.upload(hb.data(), hb.size());
    DevBuf<int> bad(1);
    bad.zero();
    SellOp<M32> a = h->sell<M32>(false);
    k_cb_dict64<M32, M64><<<grid_for(h->n, 256), 256>>>(a, reinterpret_cast<const M64*>(h->val64.p), dkeys.p,
                                                         n_keys, bits.p, bad.p);
    check_launch("k_cb_dict64");
    int hbad = 0;
    QMB_CUDA_TRY(cudaMemcpy(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (hbad) {
        cb_skip("FP64 values do not map one to one onto the FP32 codes");
        return;
    }
    bits.download(hb.data(), hb.size());
    QMB_CUDA_TRY(cudaDeviceSynchronize());
    std::vector<M64> dict(256);
    std::memset(dict.data(), 0, sizeof(M64) * 256);
    for (int c = 1; c <= n_keys; ++c)
        if (hb[(size_t)c * W] != kDictEmpty) std::memcpy(&dict[c], &hb[(size_t)c * W], sizeof(M64));
    if (L32.nb > 1) {
        size_t fr = 0, tot = 0;
        QMB_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        if ((size_t)h->n * sizeof(M64) > fr / 4) {
            cb_skip("not enough free memory for the FP64 partial sums");
            return;
        }
        h->cb64.ytmp.alloc((size_t)h->n * sizeof(M64));
    }
    h->cb64.dict.alloc(256 * sizeof(M64));
    QMB_CUDA_TRY(cudaMemcpy(h->cb64.dict.p, dict.data(), 256 * sizeof(M64), cudaMemcpyHostToDevice));
    h->cb64.nb = L32.nb;
    h->cb64.shift = L32.shift;
    h->cb64.n_codes = n_keys;
    h->cb64_shared = true;
}

//
// The same layout with one block (every column in the 24-bit field) serves a
// matrix whose vectors fit L2 but whose entry stream is large (the plain FP32
// entries, 8 or 12 bytes, at least kCbMinStreamBytes): its 32-bit coded entries
// halve (real) or third (complex) the bytes a product streams.
//
// QMB_CB_SHIFT=s (10..24) builds the layout with blocks of 2^s rows for any
// matrix with at least two blocks, whatever its size (small cases exercise
// the layout in tests).
void build_cb(qmb_ham_s* h) {
    if (const char* e = std::getenv("QMB_COLUMN_BLOCKS"))
        if (e[0] == '0') return;
    int forced = 0;
    if (const char* e = std::getenv("QMB_CB_SHIFT")) {
        const int v = std::atoi(e);
        if (v >= 10 && v <= 24) forced = v;
    }
    const bool blocked = (double)h->n * (h->cplx ? 8 : 4) >= kCbMinVecBytes;
    const bool single = !blocked && h->n <= ((int64_t)1 << 24) &&
                        (double)h->padded * (h->cplx ? 12 : 8) >= kCbMinStreamBytes;
    if ((h->prec & QMB_PREC_FP32) && h->val32.p && (forced || blocked || single)) {
        if (h->cplx) build_cb_t<float2>(h, forced, single && !forced, h->cb32);
        else build_cb_t<float>(h, forced, single && !forced, h->cb32);
    }
    // real FP64 values: one block when x (8 bytes a row) stays well inside L2
    // and the plain entries (12 bytes) stream at least kCbMinStreamBytes
    if ((h->prec & QMB_PREC_FP64) && h->val64.p && !h->cplx && (double)h->n * 8 <= kCbMaxSingleVecBytes &&
        (double)h->padded * 12 >= kCbMinStreamBytes)
        build_cb_t<double>(h, 0, true, h->cb64);
    // otherwise FP64 values share the FP32 layout's entries where they can
    const char* se = std::getenv("QMB_CB_SHARE64");
    if (h->cb64.nb == 0 && h->cb32.nb > 0 && h->val64.p && h->val32.p && !(se && se[0] == '0')) {
        if (h->cplx) share_cb64_t<float2, double2>(h);
        else share_cb64_t<float, double>(h);
    }
}

// Row-order copies for the matrix-free lookup: each row's representative
// (32-bit, 64-bit or neither) and its orbit's norm.
__global__ void k_mf_rows(int64_t n, const int64_t* __restrict__ orbit_of_row, const uint64_t* __restrict__ reps,
                          const double* __restrict__ norms, uint32_t* __restrict__ reps32,
                          uint64_t* __restrict__ reps64, double* __restrict__ nrow) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = orbit_of_row[r];
        nrow[r] = norms[o];
        if (reps32) reps32[r] = (uint32_t)reps[o];
        if (reps64) reps64[r] = reps[o];
    }
}

// bucket[b] = first row whose representative's top bits are >= b.
template <class K>
__global__ void k_mf_bucket(const K* __restrict__ reps, int64_t n, int shift, uint64_t n_b,
                            uint32_t* __restrict__ bucket) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b <= n_b;
         b += (uint64_t)gridDim.x * blockDim.x) {
        if (b == n_b) {
            bucket[b] = (uint32_t)n;
            continue;
        }
        const uint64_t key = b << shift;
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((uint64_t)reps[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        bucket[b] = (uint32_t)lo;
    }
}

// Fills the matrix-free hash table: row i under its representative.
__global__ void k_mf_hash(const uint64_t* __restrict__ reps, int64_t n, uint64_t* __restrict__ tab, uint64_t mask,
                          int hidx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t r = reps[i];
        const uint64_t w = (r << hidx) | (uint64_t)i;
        uint64_t slot = mf_hash_slot(r, mask);
        for (uint64_t it = 0; it <= mask; ++it) {  // the table is at most half full
            const unsigned long long prev =
                atomicCAS(reinterpret_cast<unsigned long long*>(tab + slot), kMfHashEmpty, (unsigned long long)w);
            if (prev == kMfHashEmpty) break;
            slot = (slot + 1) & mask;
        }
    }
}

// Representative tables at least this large (beyond 32 sites) also get the
// hash table: four times what stays comfortably in the 126 MB L2.
constexpr double kMfHashMinBytes = 512.0 * 1024 * 1024;

// The stored diagonal of the hop form.
template <class D>
__global__ void k_mf_diag(RowGen rg, int64_t n, D* __restrict__ diag) {
    QMB_LOAD_GEN(rg);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t src = apply_elem(rg.g, gs, 0, rg.rt.reps[rg.orbit_of_row[r]]);
        const double2 d = row_diagonal(ts, src);
        if constexpr (sizeof(D) == sizeof(double2)) diag[r] = d;
        else diag[r] = d.x;
    }
}

// The matrix-free operator's tables.  The rows' representatives in row
// order (32-bit up to 32 sites; beyond, the sector's table when every orbit
// is active), the bucket table over them on the top 24 bits of the largest
// one, the rows' norms, the diagonal of the hop form and the xs buffer.
void mf_tables(qmb_ham_s* h) {
    if (h->mf_ready) return;
    qmb_sector_s* s = h->sector;
    const int64_t n = h->n;
    const bool all = s->n_active == s->R;
    const bool r32 = s->L <= 32;
    h->mf_norm.alloc(n);
    if (r32) h->mf_reps32.alloc(n);
    else if (!all) h->mf_reps64.alloc(n);
    k_mf_rows<<<grid_for(n, 256), 256>>>(n, s->orbit_of_row.p, s->reps.p, s->norms.p, h->mf_reps32.p,
                                         h->mf_reps64.p, h->mf_norm.p);
    check_launch("k_mf_rows");
    int64_t o_last = 0;  // rows ascend with their representatives: the last is the largest
    uint64_t top = 0;
    QMB_CUDA_TRY(cudaMemcpy(&o_last, s->orbit_of_row.p + (n - 1), sizeof(int64_t), cudaMemcpyDeviceToHost));
    QMB_CUDA_TRY(cudaMemcpy(&top, s->reps.p + o_last, sizeof(uint64_t), cudaMemcpyDeviceToHost));
    int bits = 0;
    while (bits < 64 && (top >> bits)) ++bits;
    h->mf_shift = std::max(0, bits - 24);
    h->mf_nb = (top >> h->mf_shift) + 1;
    h->mf_bucket.alloc(h->mf_nb + 1);
    const int g = grid_for((int64_t)h->mf_nb + 1, 256);
    if (r32) k_mf_bucket<uint32_t><<<g, 256>>>(h->mf_reps32.p, n, h->mf_shift, h->mf_nb, h->mf_bucket.p);
    else k_mf_bucket<uint64_t><<<g, 256>>>(all ? s->reps.p : h->mf_reps64.p, n, h->mf_shift, h->mf_nb,
                                              h->mf_bucket.p);
    check_launch("k_mf_bucket");
    // beyond 32 sites with a representative table well beyond L2: the hash
    // table, when a representative and a row index fit one word (top bit 0);
    // QMB_MF_HASH=1 builds it at any size (tests)
    int ibits = 1;
    while (ibits < 63 && ((n - 1) >> ibits)) ++ibits;
    const char* he = std::getenv("QMB_MF_HASH");
    const bool force_hash = he && he[0] == '1';
    uint64_t slots = 1;
    while (slots < 2 * (uint64_t)n) slots <<= 1;
    size_t fr = 0, tot = 0;
    QMB_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    // the table is an accelerator: without room for it (a quarter of the
    // free memory) the bucket search serves alone
    if (!r32 && (force_hash || (double)n * 8 >= kMfHashMinBytes) && bits + ibits <= 63 &&
        slots * sizeof(uint64_t) <= fr / 4) {
        h->mf_hash.alloc(slots);
        QMB_CUDA_TRY(cudaMemset(h->mf_hash.p, 0xff, slots * sizeof(uint64_t)));
        h->mf_hmask = slots - 1;
        h->mf_hidx = ibits;
        k_mf_hash<<<grid_for(n, 256), 256>>>(all ? s->reps.p : h->mf_reps64.p, n, h->mf_hash.p, h->mf_hmask,
                                             ibits);
        check_launch("k_mf_hash");
    }
    if (h->n_hops) {
        const RowGen rg = h->row_gen();
        const size_t sm = gen_smem(rg);
        h->mf_diag.alloc((size_t)n * (h->cplx ? 16 : 8));
        if (h->cplx) {
            set_group_smem_attr((const void*)k_mf_diag<double2>, sm);
            k_mf_diag<double2><<<grid_for(n, 128), 128, sm>>>(rg, n, reinterpret_cast<double2*>(h->mf_diag.p));
        } else {
            set_group_smem_attr((const void*)k_mf_diag<double>, sm);
            k_mf_diag<double><<<grid_for(n, 128), 128, sm>>>(rg, n, reinterpret_cast<double*>(h->mf_diag.p));
        }
        check_launch("k_mf_diag");
    }
    h->mf_xs.alloc((size_t)n * (h->cplx ? 16 : 8));
    QMB_CUDA_TRY(cudaDeviceSynchronize());
    h->mf_ready = true;
}

}  // namespace qmb

using namespace qmb;

static bool terms_complex(const qmb_terms* t) {
    for (int i = 0; i < t->n_terms; ++i)
        if (std::fabs(t->scalar[2 * i + 1]) > 0.0) return true;
    return false;
}

extern "C" qmb_status qmb_ham_create(qmb_sector s, const qmb_terms* terms, int prec,
                                     qmb_ham* out) {
    return guarded([&] {
        QMB_REQUIRE(s && terms && out, QMB_ERR_INVALID, "null argument");
        *out = nullptr;
        QMB_REQUIRE(s->has_irrep, QMB_ERR_INVALID, "select an irrep before building H");
        QMB_REQUIRE((prec & (QMB_PREC_FP64 | QMB_PREC_FP32)) != 0, QMB_ERR_INVALID,
                    "prec must include QMB_PREC_FP64 and/or QMB_PREC_FP32");
        QMB_REQUIRE(s->n_active > 0, QMB_ERR_INVALID, "the selected irrep has no active orbit");
        QMB_REQUIRE(s->n_active < (1ll << 32), QMB_ERR_UNSUPPORTED, "more than 2^32 rows");
        DeviceGuard dg(s->device);
        auto h = std::make_unique<qmb_ham_s>();
        h->sector = s;
        h->device = s->device;
        h->n = s->n_active;
        h->irrep_gen = s->irrep_gen;
        h->prec = prec | QMB_PREC_FP64;  // FP64 values are always built first
        h->cplx = !s->is_real || terms_complex(terms);
        upload_terms(h.get(), terms, s->L);
        h->err.alloc(1);
        h->err.zero();
        build_sell(h.get());
        build_cb(h.get());
        if (!(prec & QMB_PREC_FP64)) {
            // keep FP64 values only when asked for; the matrix-free path needs none
            h->val64.release();
            h->prec = prec;
        }
        *out = h.release();
    });
}

extern "C" qmb_status qmb_ham_destroy(qmb_ham h) {
    return guarded([&] {
        if (!h) return;
        DeviceGuard dg(h->device);
        delete h;
    });
}

extern "C" qmb_status qmb_ham_get_info(qmb_ham h, qmb_ham_info* info) {
    return guarded([&] {
        QMB_REQUIRE(h && info, QMB_ERR_INVALID, "null argument");
        info->n_rows = h->n;
        info->nnz_offdiag = h->nnz;
        info->padded = h->padded;
        info->max_row = h->max_row;
        info->is_complex = h->cplx ? 1 : 0;
        info->n_codes = h->cb32.n_codes;
        info->coded = h->cb32.nb > 0 ? 1 : 0;
        info->coded_fp64 = h->cb64.nb > 0 ? 1 : 0;
        double vs64 = h->cplx ? 16 : 8, vs32 = h->cplx ? 8 : 4;
        // compulsory traffic: index + value per off-diagonal, diagonal value,
        // x read once, y written once
        info->bytes_fp64 = (double)h->nnz * (4 + vs64) + (double)h->n * (vs64 + 2 * vs64);
        info->bytes_fp32 = (double)h->nnz * (4 + vs32) + (double)h->n * (vs32 + 2 * vs32);
    });
}

extern "C" qmb_status qmb_ham_export_ref(qmb_sector s, const qmb_terms* terms, int W,
                                         uint32_t* ind, double* val, int16_t* track) {
    return guarded([&] {
        QMB_REQUIRE(s && terms && ind && val && track, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(s->has_irrep, QMB_ERR_INVALID, "select an irrep first");
        QMB_REQUIRE(W >= 1, QMB_ERR_INVALID, "W must be >= 1");
        DeviceGuard dg(s->device);
        qmb_ham_s tmp;
        tmp.sector = s;
        tmp.device = s->device;
        upload_terms(&tmp, terms, s->L);
        tmp.err.alloc(1);
        tmp.err.zero();
        RowGen rg = tmp.row_gen();
        size_t sm = gen_smem(rg);
        int64_t R = s->R;
        DevBuf<uint32_t> di((size_t)R * W);
        DevBuf<double2> dv((size_t)R * W);
        DevBuf<int16_t> dt(R);
        DevBuf<int> ov(1);
        di.zero();
        dv.zero();
        dt.zero();
        ov.zero();
        set_group_smem_attr((const void*)k_ell_ref, sm);
        k_ell_ref<<<grid_for(R, 128), 128, sm>>>(rg, R, W, di.p, dv.p, dt.p, ov.p);
        check_launch("k_ell_ref");
        int overflow = 0, err = 0;
        QMB_CUDA_TRY(cudaMemcpy(&overflow, ov.p, sizeof(int), cudaMemcpyDeviceToHost));
        QMB_CUDA_TRY(cudaMemcpy(&err, tmp.err.p, sizeof(int), cudaMemcpyDeviceToHost));
        QMB_REQUIRE(err == 0, QMB_ERR_INVALID, "a term changes the number of up spins");
        QMB_REQUIRE(!overflow, QMB_ERR_ELL_OVERFLOW, "a row needs more than W slots");
        di.download(ind, (size_t)R * W);
        dv.download(reinterpret_cast<double2*>(val), (size_t)R * W);
        dt.download(track, R);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
    });
}

extern "C" qmb_status qmb_ham_export_nosym(int L, int n_up, const qmb_terms* terms, int W,
                                           uint32_t* ind, double* val, int16_t* track,
                                           int device) {
    qmb_sector s = nullptr;
    std::vector<uint32_t> id(L > 0 && L <= 64 ? L : 1);
    for (int q = 0; q < (int)id.size(); ++q) id[q] = q;
    qmb_sector_desc d{L, n_up, 1, id.data(), 0, device};
    qmb_status st = qmb_sector_create(&d, &s);
    if (st != QMB_OK) return st;
    double one[2] = {1.0, 0.0};
    st = qmb_sector_set_irrep(s, one, 0.5);
    if (st == QMB_OK) st = qmb_ham_export_ref(s, terms, W, ind, val, track);
    qmb_status st2 = qmb_sector_destroy(s);
    return st != QMB_OK ? st : st2;
}

namespace qmb {
// y = H x dispatch over storage and precision.
void hv_dispatch(const qmb_ham_s* h, int prec, const void* x, void* y, cudaStream_t st,
                 bool matrix_free) {
    bool f64 = (prec == QMB_PREC_FP64);
    QMB_REQUIRE(prec == QMB_PREC_FP64 || prec == QMB_PREC_FP32, QMB_ERR_INVALID,
                "prec must be QMB_PREC_FP64 or QMB_PREC_FP32");
    if (matrix_free) {
        // QMB_MF_LOOKUP=warp: the warp-cooperative lookup over the bucket table
        const char* le = std::getenv("QMB_MF_LOOKUP");
        if (le && std::strcmp(le, "warp") == 0 && h->n_hops) {
            auto run = [&](auto op, auto* xv, auto* yv) {
                using V = std::remove_const_t<std::remove_pointer_t<decltype(xv)>>;
                using MT = typename decltype(op)::scalar;
                op.look.hash = nullptr;
                const size_t sm = op.smem_bytes();
                set_group_smem_attr((const void*)k_hv_mfw<MT, V>, sm);
                op.pre(xv, (const int*)nullptr, st);
                k_hv_mfw<MT, V><<<grid_for(op.n, 256), 256, sm, st>>>(op, xv, yv);
                check_launch("k_hv_mfw");
            };
            if (h->cplx) {
                if (f64) run(h->mf<double2>(), (const double2*)x, (double2*)y);
                else run(h->mf<float2>(), (const float2*)x, (float2*)y);
            } else {
                if (f64) run(h->mf<double>(), (const double*)x, (double*)y);
                else run(h->mf<float>(), (const float*)x, (float*)y);
            }
            return;
        }
        if (h->cplx) {
            if (f64) { auto op = h->mf<double2>(); launch_hv(op, (const double2*)x, (double2*)y, st, op.smem_bytes()); }
            else { auto op = h->mf<float2>(); launch_hv(op, (const float2*)x, (float2*)y, st, op.smem_bytes()); }
        } else {
            if (f64) { auto op = h->mf<double>(); launch_hv(op, (const double*)x, (double*)y, st, op.smem_bytes()); }
            else { auto op = h->mf<float>(); launch_hv(op, (const float*)x, (float*)y, st, op.smem_bytes()); }
        }
        return;
    }
    QMB_REQUIRE(f64 ? h->val64.p != nullptr : h->val32.p != nullptr, QMB_ERR_INVALID,
                "the handle does not hold values of the requested precision");
    if (h->cplx) {
        if (f64 && h->cb64.nb > 0) launch_hv(h->cb<double2>(), (const double2*)x, (double2*)y, st, CbSellOp<double2>::smem_bytes());
        else if (f64) launch_hv(h->sell<double2>(true), (const double2*)x, (double2*)y, st, 0);
        else if (h->cb32.nb > 0) launch_hv(h->cb<float2>(), (const float2*)x, (float2*)y, st, CbSellOp<float2>::smem_bytes());
        else launch_hv(h->sell<float2>(false), (const float2*)x, (float2*)y, st, 0);
    } else {
        if (f64 && h->cb64.nb > 0) launch_hv(h->cb<double>(), (const double*)x, (double*)y, st, CbSellOp<double>::smem_bytes());
        else if (f64) launch_hv(h->sell<double>(true), (const double*)x, (double*)y, st, 0);
        else if (h->cb32.nb > 0) launch_hv(h->cb<float>(), (const float*)x, (float*)y, st, CbSellOp<float>::smem_bytes());
        else launch_hv(h->sell<float>(false), (const float*)x, (float*)y, st, 0);
    }
}
}  // namespace qmb

extern "C" qmb_status qmb_hv(qmb_ham h, int prec, const void* x_dev, void* y_dev, void* stream) {
    return guarded([&] {
        QMB_REQUIRE(h && x_dev && y_dev, QMB_ERR_INVALID, "null argument");
        DeviceGuard dg(h->device);
        hv_dispatch(h, prec, x_dev, y_dev, (cudaStream_t)stream, false);
    });
}

extern "C" qmb_status qmb_hv_matrix_free(qmb_ham h, int prec, const void* x_dev, void* y_dev,
                                         void* stream) {
    return guarded([&] {
        QMB_REQUIRE(h && x_dev && y_dev, QMB_ERR_INVALID, "null argument");
        DeviceGuard dg(h->device);
        mf_tables(h);
        hv_dispatch(h, prec, x_dev, y_dev, (cudaStream_t)stream, true);
    });
}

extern "C" qmb_status qmb_hv_host(qmb_ham h, int prec, const void* x, void* y) {
    return guarded([&] {
        QMB_REQUIRE(h && x && y, QMB_ERR_INVALID, "null argument");
        DeviceGuard dg(h->device);
        size_t es = (prec == QMB_PREC_FP64 ? 8 : 4) * (h->cplx ? 2 : 1);
        DevBuf<unsigned char> dx(h->n * es), dy(h->n * es);
        QMB_CUDA_TRY(cudaMemcpy(dx.p, x, h->n * es, cudaMemcpyHostToDevice));
        hv_dispatch(h, prec, dx.p, dy.p, 0, false);
        QMB_CUDA_TRY(cudaMemcpy(y, dy.p, h->n * es, cudaMemcpyDeviceToHost));
    });
}
