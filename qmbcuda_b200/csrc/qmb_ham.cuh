// qmb_ham.cuh -- Hamiltonian storage and the row operators used by H*v.
#pragma once
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


// Enumerates the entries of the row whose source string is src (norm ns)
// generated by terms h0 .. h1-1: emit(orbit, value) for every off-diagonal
// entry, the diagonal is returned.
// Rule of BuildHamiltonianXXZForAbelianGroup (exact_diagonalization/utils.cu:83-184).
template <class Emit>
__device__ __forceinline__ double2 gen_row_range(const RowGen& rg, const GroupSmem& gs,
                                                 const TermsSmem& ts, int h0, int h1, uint64_t src,
                                                 double ns, Emit&& emit) {
    double2 diag = make_double2(0.0, 0.0);
    for (int hi = h0; hi < h1; ++hi) {
        uint64_t t = src;
        double2 coef = ts.scalar[hi];
        bool bad = false;
        const uint16_t* op = ts.ops + hi * ts.n_col;
        for (int h2 = 0; h2 < ts.n_ops[hi]; ++h2) {
            int code = op[h2] >> 8, site = op[h2] & 0xff;
            int spin = (int)((t >> site) & 1ull);
            if (code == QMB_OP_SM) {
                if (!spin) { bad = true; break; }
                t &= ~(1ull << site);
            } else if (code == QMB_OP_SP) {
                if (spin) { bad = true; break; }
                t |= 1ull << site;
            } else if (code == QMB_OP_SZ) {
                double f = spin ? 0.5 : -0.5;
                coef.x *= f;
                coef.y *= f;
            }
        }
        if (bad) continue;
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
        uint64_t r = orbit_min(rg.g, gs, t, &e);
        int64_t o = find_rep(rg.rt, r);
        if (o < 0) {
            *rg.err = 2;
            continue;
        }
        double nt = rg.norms[o];
        if (nt < rg.tol) continue;
        // t = g_e^{-1}(rep): chi(g_t) = conj(chi(e)) for a unitary 1-D irrep
        double2 ch = rg.g.chars[e];
        double f = nt / ns;
        double2 v = make_double2((coef.x * ch.x + coef.y * ch.y) * f,
                                 (coef.y * ch.x - coef.x * ch.y) * f);
        emit(o, v);
    }
    return diag;
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

// Column-blocked coded sliced ELL (FP32 values), for sectors whose vector
// is larger than L2: the columns are split into nb blocks of 2^shift rows and
// every block has its own sliced ELL (32-row slices, column-major inside a
// slice) whose 32-bit entries pack an 8-bit value code (into a dictionary of
// at most 255 FP32 values; code 0 is the padding, value 0) above the 24-bit
// column inside the block.  A product makes one pass per block in block
// order, so the part of x a pass gathers from (one block, at most 64 MB)
// stays in L2 while the matrix streams from HBM once: passes 0 .. nb-2
// (pre(), k_cb_pass) leave partial row sums in ytmp, and the last pass is
// row(), which adds its block and hands the row to the calling kernel.
template <class M>  // float or float2
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

// Matrix-free operator: regenerates every entry of the row.
template <class M>
struct MfOp {
    int64_t n;
    RowGen rg;
    GroupSmem gs;
    TermsSmem ts;
    size_t gbytes;
    size_t smem_bytes() const { return align16(gbytes) + terms_smem_bytes(rg.terms); }
    __device__ void init(unsigned char* sm) {
        gs = load_group(rg.g, sm);
        ts = load_terms(rg.terms, sm + align16(gbytes));
    }
    template <class V>
    void pre(const V*, const int*, cudaStream_t) const {}
    template <class V>
    __device__ __forceinline__ V row(int64_t r, const V* __restrict__ x, V& xr) const {
        int64_t o = rg.orbit_of_row[r];
        uint64_t src = apply_elem(rg.g, gs, 0, rg.rt.reps[o]);
        double ns = rg.norms[o];
        xr = x[r];
        V acc = Sc<V>::zero();
        double2 d = gen_row(rg, gs, ts, src, ns, [&](int64_t ot, double2 v) {
            int64_t c = rg.row_of_orbit[ot];
            acc = Sc<V>::fma(Sc<V>::from(v), __ldg(x + c), acc);
        });
        acc = Sc<V>::fma(Sc<V>::from(d), xr, acc);
        return acc;
    }
};

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
    // column-blocked coded FP32 layout (CbSellOp), built for vectors larger than L2
    int cb_nb = 0, cb_shift = 0, n_codes = 0;
    qmb::DevBuf<int64_t> cb_off;
    qmb::DevBuf<int> cb_width;
    qmb::DevBuf<uint32_t> cb_packed;
    qmb::DevBuf<unsigned char> cb_dict, cb_ytmp;
    // terms kept for the matrix-free operator
    int n_terms = 0, n_col = 0;
    qmb::DevBuf<int> t_nops;
    qmb::DevBuf<uint16_t> t_ops;
    qmb::DevBuf<double2> t_scalar;
    qmb::DevBuf<int> err;
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
        qmb::CbSellOp<M> op;
        op.n = n;
        op.nb = cb_nb;
        op.shift = cb_shift;
        op.n_slices = n_slices;
        op.off = cb_off.p;
        op.width = cb_width.p;
        op.packed = cb_packed.p;
        op.dict = reinterpret_cast<const M*>(cb_dict.p);
        op.diag = reinterpret_cast<const M*>(diag32.p);
        op.ytmp = cb_ytmp.p;
        op.sdict = nullptr;
        return op;
    }
    template <class M> qmb::MfOp<M> mf() const {
        qmb::MfOp<M> op;
        op.n = n;
        op.rg = row_gen();
        op.gbytes = qmb::group_smem_bytes(op.rg.g);
        return op;
    }
};

namespace qmb {
// Upload operator tables (validated) into the handle's term buffers.
void upload_terms(qmb_ham_s* h, const qmb_terms* t, int L);
int grid_for(int64_t n, int block);
void set_group_smem_attr(const void* kernel, size_t bytes);
bool fits_device(size_t bytes);
}  // namespace qmb
