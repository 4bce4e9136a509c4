// qmb_expval.cu -- zero-temperature expectation values <psi|A|psi> in a
// symmetry-adapted sector, for operators that are sums of products of Sz, S+
// and S-.  This is the computation of ComputeStaticExpValZeroT
// (exact_diagonalization/HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:421-601,
// exact_diagonalization/HeisenbergHamAbelianSymms_CUDA.cu:448-617) and of its
// kernel ExpecValArbOperatorAbelianIrrepProjHeisenbergZeroT
// (exact_diagonalization/utils.cu:442-550) with its thrust reduction.
//
// Method.  psi lies in a one-dimensional irrep of the sector's group, so
// <psi|A|psi> = <psi|U_e^-1 A U_e|psi> for every element e, and A can be
// replaced by its group average Abar = (1/n_ext) sum_e U_e^-1 A U_e (site
// maps, and Sz -> -Sz, S+ <-> S- for the spin-inversion elements).  Abar
// commutes with the group, so its matrix on the symmetric basis follows from
// its action on the representatives alone: the rule of the Hamiltonian
// (gen_row_range).  One pass over the rows then gives
//     s = sum_r conj(psi_r) (Abar psi)_r,
// and with operator tables in the Hamiltonian's convention (each term the
// daggered operator sequence with a conjugated scalar, as BuildOperatorVecs
// writes it) the expectation value is conj(s) / <psi|psi>.
//
// The reference applies the operator to every member of every orbit (|G|
// applications per term and row) and finds the target orbit through a table
// over the whole Sz sector.  Here the group average is formed once on the
// host, identical terms are merged, terms that change Sz are dropped (they
// have zero expectation in a fixed-Sz sector), and each row applies the
// averaged terms to its representative only.  Many operators share one
// launch: their terms sit back to back in shared memory, one segment per
// operator (or per part of an operator when it does not fit), and every
// segment reduces separately.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "qmb_ham.cuh"
#include "qmb_b200.h"

namespace qmb {
namespace {

constexpr int kEvBlock = 256;
constexpr size_t kEvSmemCap = 200 * 1024;  // dynamic shared memory per block

// Group average of one operator table: the distinct terms (op words
// code << 8 | site, in application order) with their summed scalars, in
// order of first appearance.
struct AvgTerms {
    std::vector<std::vector<uint16_t>> keys;
    std::vector<std::complex<double>> sc;
};

// Open-addressing table over terms packed into 128 bits (up to 8 factors of
// 16 bits) plus the factor count.
class TermTable {
public:
    explicit TermTable(size_t n_insert) {
        size_t cap = 16;
        while (cap < 2 * n_insert) cap <<= 1;
        slots_.assign(cap, Slot{});
        mask_ = cap - 1;
    }
    void add(const uint16_t* w, int n, std::complex<double> v) {
        uint64_t a = 0, b = 0;
        for (int i = 0; i < n && i < 4; ++i) a |= (uint64_t)w[i] << (16 * i);
        for (int i = 4; i < n; ++i) b |= (uint64_t)w[i] << (16 * (i - 4));
        uint64_t h = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull + (uint64_t)n) * 0xC2B2AE3D27D4EB4Full;
        h ^= h >> 29;
        for (size_t i = h & mask_;; i = (i + 1) & mask_) {
            Slot& s = slots_[i];
            if (!s.used) {
                s = Slot{a, b, n, true, v};
                order_.push_back(i);
                return;
            }
            if (s.a == a && s.b == b && s.n == n) {
                s.v += v;
                return;
            }
        }
    }
    void emit(AvgTerms& out) const {
        for (size_t i : order_) {
            const Slot& s = slots_[i];
            if (s.v == 0.0) continue;
            std::vector<uint16_t> k(s.n);
            for (int j = 0; j < s.n; ++j) k[j] = (uint16_t)((j < 4 ? s.a >> (16 * j) : s.b >> (16 * (j - 4))) & 0xffff);
            out.keys.push_back(std::move(k));
            out.sc.push_back(s.v);
        }
    }

private:
    struct Slot {
        uint64_t a = 0, b = 0;
        int n = 0;
        bool used = false;
        std::complex<double> v = 0.0;
    };
    std::vector<Slot> slots_;
    std::vector<size_t> order_;
    size_t mask_ = 0;
};

void average_terms(const qmb_sector_s* s, const qmb_terms& A, AvgTerms& out) {
    QMB_REQUIRE(A.n_terms >= 0, QMB_ERR_INVALID, "expval: n_terms must be >= 0");
    if (A.n_terms == 0) return;
    QMB_REQUIRE(A.n_ops && A.op_code && A.op_site && A.scalar, QMB_ERR_INVALID,
                "expval: null table");
    QMB_REQUIRE(A.n_col >= 1 && A.n_col <= kMaxCol, QMB_ERR_INVALID, "expval: n_col must be in 1..8");
    const int L = s->L, G = s->G, ne = s->n_ext;
    TermTable tab((size_t)A.n_terms * ne);
    uint16_t base[kMaxCol], img[kMaxCol];
    for (int i = 0; i < A.n_terms; ++i) {
        QMB_REQUIRE(A.n_ops[i] >= 0 && A.n_ops[i] <= A.n_col, QMB_ERR_INVALID,
                    "expval: n_ops out of range");
        const std::complex<double> sc(A.scalar[2 * i], A.scalar[2 * i + 1]);
        QMB_REQUIRE(std::isfinite(sc.real()) && std::isfinite(sc.imag()), QMB_ERR_INVALID,
                    "expval: non-finite scalar");
        int nb = 0, n_p = 0, n_m = 0, n_z = 0;
        for (int j = 0; j < A.n_ops[i]; ++j) {
            const int c = A.op_code[i * A.n_col + j], q = A.op_site[i * A.n_col + j];
            QMB_REQUIRE(c == QMB_OP_SZ || c == QMB_OP_SP || c == QMB_OP_SM || c == QMB_OP_I,
                        QMB_ERR_INVALID, "expval: operator codes must be Sz, Sp, Sm or I");
            QMB_REQUIRE(q >= 0 && q < L, QMB_ERR_INVALID, "expval: site out of range");
            if (c == QMB_OP_I) continue;
            n_p += c == QMB_OP_SP;
            n_m += c == QMB_OP_SM;
            n_z += c == QMB_OP_SZ;
            base[nb++] = (uint16_t)(c << 8 | q);
        }
        if (n_p != n_m || sc == 0.0) continue;  // leaves the Sz sector, or zero
        for (int e = 0; e < ne; ++e) {
            const uint32_t* p = s->perm.data() + (size_t)(e % G) * L;
            const bool z = e >= G;
            for (int j = 0; j < nb; ++j) {
                int c = base[j] >> 8, q = base[j] & 0xff;
                if (z && c != QMB_OP_SZ) c = c == QMB_OP_SP ? QMB_OP_SM : QMB_OP_SP;
                img[j] = (uint16_t)(c << 8 | (int)p[q]);
            }
            // factors on distinct sites commute: order them by site
            bool distinct = true;
            for (int a = 0; a < nb && distinct; ++a)
                for (int b = a + 1; b < nb; ++b)
                    if ((img[a] & 0xff) == (img[b] & 0xff)) {
                        distinct = false;
                        break;
                    }
            if (distinct)
                std::sort(img, img + nb, [](uint16_t x, uint16_t y) { return (x & 0xff) < (y & 0xff); });
            const double sign = (z && (n_z & 1)) ? -1.0 : 1.0;
            tab.add(img, nb, sc * (sign / ne));
        }
    }
    tab.emit(out);
}

bool trace_on() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("QMB_TRACE");
        v = (e && *e && *e != '0') ? 1 : 0;
    }
    return v == 1;
}

__device__ __forceinline__ double2 block_sum2(double x, double y, double2* red) {
    for (int o = 16; o; o >>= 1) {
        x += __shfl_down_sync(0xffffffffu, x, o);
        y += __shfl_down_sync(0xffffffffu, y, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = make_double2(x, y);
    __syncthreads();
    double2 t = make_double2(0.0, 0.0);
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            t.x += red[i].x;
            t.y += red[i].y;
        }
    return t;
}

// One launch: every block strides over the rows for each segment sg and
// writes its partial sum of conj(psi_r) (Abar_sg psi)_r to part[sg][block];
// npart[block] receives the block's partial of <psi|psi>.  Segment sg =
// (d0, d1, g0, g1): diagonal terms d0..d1-1 and general terms g0..g1-1.
// A diagonal term (a product of Sz only) has the value
//     sc * (-1)^popc(mask & ~t)
// on the string t, with sc = scalar * 2^-k for k factors and mask the XOR of
// the factors' site bits (a site taken twice gives (+-1/2)^2 = 1/4, no sign).
// One block per SM fits the shared memory, so registers are not the limit.
template <class V>
__global__ void __launch_bounds__(kEvBlock, 1) k_expval(RowGen rg, int64_t n, const V* __restrict__ psi,
                                                        int n_seg, const int4* __restrict__ seg, int n_diag,
                                                        const uint64_t* __restrict__ dmask,
                                                        const double2* __restrict__ dsc,
                                                        double2* __restrict__ part, double* __restrict__ npart) {
    extern __shared__ __align__(16) unsigned char smem_ev[];
    __shared__ double2 red[kEvBlock / 32];
    const size_t gb = align16(group_smem_bytes(rg.g));
    const GroupSmem gs = load_group(rg.g, smem_ev);
    const TermsSmem ts = load_terms(rg.terms, smem_ev + gb);
    double2* s_sc = reinterpret_cast<double2*>(smem_ev + gb + terms_smem_bytes(rg.terms));
    uint64_t* s_mask = reinterpret_cast<uint64_t*>(s_sc + n_diag);
    for (int i = threadIdx.x; i < n_diag; i += blockDim.x) {
        s_sc[i] = dsc[i];
        s_mask[i] = dmask[i];
    }
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int sg = 0; sg < n_seg; ++sg) {
        const int4 sd = seg[sg];
        double ax = 0.0, ay = 0.0;
        for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += stride) {
            const int64_t o = rg.orbit_of_row[r];
            const uint64_t src = apply_elem(rg.g, gs, 0, rg.rt.reps[o]);
            const uint64_t down = ~src;
            // complex row sum even for a real psi: scalars may be complex
            const double2 pr = Sc<V>::to2(psi[r]);
            double2 y = make_double2(0.0, 0.0);
            double2 d = make_double2(0.0, 0.0);
            for (int t = sd.x; t < sd.y; ++t) {
                const double2 c = s_sc[t];
                const double f = (__popcll(s_mask[t] & down) & 1) ? -1.0 : 1.0;
                d.x = fma(f, c.x, d.x);
                d.y = fma(f, c.y, d.y);
            }
            if (sd.z < sd.w) {
                const double2 g = gen_row_range(rg, gs, ts, sd.z, sd.w, src, rg.norms[o], [&](int64_t ot, double2 v) {
                    const double2 x = Sc<V>::to2(__ldg(psi + rg.row_of_orbit[ot]));
                    y.x += v.x * x.x - v.y * x.y;
                    y.y += v.x * x.y + v.y * x.x;
                });
                d.x += g.x;
                d.y += g.y;
            }
            y.x += d.x * pr.x - d.y * pr.y;
            y.y += d.x * pr.y + d.y * pr.x;
            ax += pr.x * y.x + pr.y * y.y;  // conj(pr) * y
            ay += pr.x * y.y - pr.y * y.x;
        }
        const double2 t = block_sum2(ax, ay, red);
        if (threadIdx.x == 0) part[(size_t)sg * gridDim.x + blockIdx.x] = t;
    }
    double nn = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += stride)
        nn += Sc<V>::abs2(psi[r]);
    const double2 t = block_sum2(nn, 0.0, red);
    if (threadIdx.x == 0) npart[blockIdx.x] = t.x;
}

// Fixed-order sum of the block partials of every segment (one block each).
__global__ void __launch_bounds__(kEvBlock) k_expval_sum(const double2* __restrict__ part, int n_blocks,
                                                         double2* __restrict__ seg_out) {
    __shared__ double2 red[kEvBlock / 32];
    const double2* p = part + (size_t)blockIdx.x * n_blocks;
    double x = 0.0, y = 0.0;
    for (int i = threadIdx.x; i < n_blocks; i += blockDim.x) {
        x += p[i].x;
        y += p[i].y;
    }
    const double2 t = block_sum2(x, y, red);
    if (threadIdx.x == 0) seg_out[blockIdx.x] = t;
}

bool is_diagonal(const std::vector<uint16_t>& key) {
    for (uint16_t w : key)
        if ((w >> 8) != QMB_OP_SZ) return false;
    return true;
}

template <class V>
void run_expval(qmb_ham_s* h, const V* psi, const std::vector<AvgTerms>& ops, double* out) {
    RowGen rg = h->row_gen();
    const size_t gbytes = align16(group_smem_bytes(rg.g));
    DevBuf<int> err(1);
    err.zero();
    rg.err = err.p;

    // items of operator k back to back, its diagonal terms first
    struct Item {
        int op;
        const std::vector<uint16_t>* key;
        std::complex<double> sc;
        bool diag;
    };
    std::vector<Item> items;
    for (size_t k = 0; k < ops.size(); ++k) {
        for (size_t i = 0; i < ops[k].keys.size(); ++i)
            if (is_diagonal(ops[k].keys[i])) items.push_back({(int)k, &ops[k].keys[i], ops[k].sc[i], true});
        for (size_t i = 0; i < ops[k].keys.size(); ++i)
            if (!is_diagonal(ops[k].keys[i])) items.push_back({(int)k, &ops[k].keys[i], ops[k].sc[i], false});
    }

    const int dev = h->device;
    int sms = 148, max_smem = 0;
    QMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    QMB_CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem_cap = std::min(kEvSmemCap, (size_t)max_smem);
    QMB_REQUIRE(gbytes + 64 < smem_cap, QMB_ERR_INVALID, "expval: group tables leave no shared memory");
    auto chunk_bytes = [&](size_t n_gen, int n_col, size_t n_diag) {
        return gbytes + ((20 + 2 * (size_t)n_col) * n_gen + 15) / 16 * 16 + 24 * n_diag;
    };

    std::vector<double2> seg_sum;
    std::vector<int> seg_op;
    double norm2 = 0.0;
    bool have_norm = false;
    size_t pos = 0;
    do {
        // chunk: as many items as fit in shared memory
        struct Seg {
            int op;
            int4 r;
        };
        std::vector<Seg> segs;
        std::vector<std::vector<uint16_t>> gkeys;
        std::vector<double2> gsc, dsc;
        std::vector<uint64_t> dmask;
        int n_col = 1;
        size_t end = pos;
        for (; end < items.size(); ++end) {
            const Item& it = items[end];
            const size_t ng = gkeys.size() + (it.diag ? 0 : 1), nd = dmask.size() + (it.diag ? 1 : 0);
            const int c = it.diag ? n_col : std::max(n_col, (int)it.key->size());
            if (chunk_bytes(ng, c, nd) > smem_cap || ng > (size_t)kMaxTerms) break;
            n_col = c;
            if (segs.empty() || segs.back().op != it.op) {
                const int nd0 = (int)dmask.size(), ng0 = (int)gkeys.size();
                segs.push_back({it.op, make_int4(nd0, nd0, ng0, ng0)});
            }
            if (it.diag) {
                uint64_t m = 0;
                double f = 1.0;
                for (uint16_t w : *it.key) {
                    m ^= 1ull << (w & 0xff);
                    f *= 0.5;
                }
                dmask.push_back(m);
                dsc.push_back(make_double2(it.sc.real() * f, it.sc.imag() * f));
                segs.back().r.y += 1;
            } else {
                gkeys.push_back(*it.key);
                gsc.push_back(make_double2(it.sc.real(), it.sc.imag()));
                segs.back().r.w += 1;
            }
        }
        QMB_REQUIRE(end > pos || items.empty(), QMB_ERR_INVALID, "expval: a term does not fit");
        const int ng = (int)gkeys.size(), nd = (int)dmask.size();
        std::vector<int> nops(std::max(ng, 1), 0);
        std::vector<uint16_t> opw((size_t)std::max(ng, 1) * n_col, 0);
        for (int i = 0; i < ng; ++i) {
            nops[i] = (int)gkeys[i].size();
            std::copy(gkeys[i].begin(), gkeys[i].end(), opw.begin() + (size_t)i * n_col);
        }
        if (gsc.empty()) gsc.push_back(make_double2(0.0, 0.0));
        if (dsc.empty()) {
            dsc.push_back(make_double2(0.0, 0.0));
            dmask.push_back(0);
        }
        const int n_seg = (int)segs.size();
        std::vector<int4> seg_h(std::max(n_seg, 1), make_int4(0, 0, 0, 0));
        for (int i = 0; i < n_seg; ++i) seg_h[i] = segs[i].r;

        rg.terms.n_terms = ng;
        rg.terms.n_col = n_col;
        const size_t smem = gbytes + terms_smem_bytes(rg.terms) + 24 * (size_t)nd;
        const void* kf = (const void*)k_expval<V>;
        set_group_smem_attr(kf, smem);
        int per_sm = 0;
        QMB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_expval<V>, kEvBlock, smem));
        const int64_t want = (h->n + kEvBlock - 1) / kEvBlock;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * std::max(1, per_sm)));

        // one device block per chunk: the inputs staged and copied at once,
        // then the per-segment results with the norm partials, then the
        // block partials
        size_t off = 0;
        auto place = [&](size_t bytes) {
            const size_t o = off;
            off = align16(off + bytes);
            return o;
        };
        const size_t o_nops = place(sizeof(int) * nops.size()), o_ops = place(sizeof(uint16_t) * opw.size()),
                     o_sc = place(sizeof(double2) * gsc.size()), o_dsc = place(sizeof(double2) * dsc.size()),
                     o_mask = place(sizeof(uint64_t) * dmask.size()), o_seg = place(sizeof(int4) * seg_h.size());
        const size_t in_bytes = off;
        const size_t res_bytes = sizeof(double2) * seg_h.size() + sizeof(double) * grid;
        const size_t o_res = place(res_bytes);
        const size_t o_part = place(sizeof(double2) * seg_h.size() * grid);
        std::vector<unsigned char> stage(in_bytes);
        std::memcpy(stage.data() + o_nops, nops.data(), sizeof(int) * nops.size());
        std::memcpy(stage.data() + o_ops, opw.data(), sizeof(uint16_t) * opw.size());
        std::memcpy(stage.data() + o_sc, gsc.data(), sizeof(double2) * gsc.size());
        std::memcpy(stage.data() + o_dsc, dsc.data(), sizeof(double2) * dsc.size());
        std::memcpy(stage.data() + o_mask, dmask.data(), sizeof(uint64_t) * dmask.size());
        std::memcpy(stage.data() + o_seg, seg_h.data(), sizeof(int4) * seg_h.size());
        DevBuf<unsigned char> blk(off);
        QMB_CUDA_TRY(cudaMemcpy(blk.p, stage.data(), in_bytes, cudaMemcpyHostToDevice));
        unsigned char* b = blk.p;
        rg.terms.n_ops = reinterpret_cast<const int*>(b + o_nops);
        rg.terms.ops = reinterpret_cast<const uint16_t*>(b + o_ops);
        rg.terms.scalar = reinterpret_cast<const double2*>(b + o_sc);
        double2* seg_d = reinterpret_cast<double2*>(b + o_res);
        double* npart = reinterpret_cast<double*>(seg_d + seg_h.size());
        double2* part = reinterpret_cast<double2*>(b + o_part);
        k_expval<V><<<grid, kEvBlock, smem>>>(rg, h->n, psi, n_seg, reinterpret_cast<const int4*>(b + o_seg), nd,
                                               reinterpret_cast<const uint64_t*>(b + o_mask),
                                               reinterpret_cast<const double2*>(b + o_dsc), part, npart);
        check_launch("k_expval");
        if (n_seg) {
            k_expval_sum<<<n_seg, kEvBlock>>>(part, grid, seg_d);
            check_launch("k_expval_sum");
        }
        std::vector<unsigned char> res(res_bytes);
        QMB_CUDA_TRY(cudaMemcpy(res.data(), seg_d, res_bytes, cudaMemcpyDeviceToHost));
        const double2* hs = reinterpret_cast<const double2*>(res.data());
        const double* hn = reinterpret_cast<const double*>(hs + seg_h.size());
        for (int i = 0; i < n_seg; ++i) {
            seg_sum.push_back(hs[i]);
            seg_op.push_back(segs[i].op);
        }
        if (!have_norm) {
            for (int i = 0; i < grid; ++i) norm2 += hn[i];
            have_norm = true;
        }
        pos = end;
    } while (pos < items.size());
    int herr = 0;
    err.download(&herr, 1);
    QMB_REQUIRE(herr == 0, QMB_ERR_INVALID, "expval: a term left the sector's representative table");
    QMB_REQUIRE(norm2 > 0.0, QMB_ERR_INVALID, "expval: psi is zero");
    for (size_t k = 0; k < ops.size(); ++k) out[2 * k] = out[2 * k + 1] = 0.0;
    for (size_t i = 0; i < seg_sum.size(); ++i) {
        out[2 * seg_op[i]] += seg_sum[i].x;
        out[2 * seg_op[i] + 1] += seg_sum[i].y;
    }
    // conj(s) / <psi|psi>
    for (size_t k = 0; k < ops.size(); ++k) {
        out[2 * k] /= norm2;
        out[2 * k + 1] = -out[2 * k + 1] / norm2;
    }
}

}  // namespace
}  // namespace qmb

using namespace qmb;

extern "C" qmb_status qmb_expval(qmb_ham h, int n_ops, const qmb_terms* ops, const void* psi_dev,
                                 double* out) {
    return guarded([&] {
        QMB_REQUIRE(h && out && (ops || n_ops == 0), QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(n_ops >= 0, QMB_ERR_INVALID, "n_ops must be >= 0");
        QMB_REQUIRE(h->sector && h->sector->has_irrep, QMB_ERR_INVALID, "handle has no sector irrep");
        QMB_REQUIRE(h->irrep_gen == h->sector->irrep_gen, QMB_ERR_INVALID,
                    "the sector's irrep changed since the handle was built");
        const void* psi = psi_dev;
        if (!psi) {
            QMB_REQUIRE(h->psi.p && h->psi_n == h->n, QMB_ERR_INVALID,
                        "no ground state kept (run qmb_lanczos with want_vector, or qmb_set_ground_state)");
            psi = h->psi.p;
        }
        if (n_ops == 0) return;
        DeviceGuard dg(h->device);
        const auto t0 = std::chrono::steady_clock::now();
        // operators average independently: spread them over host threads
        std::vector<AvgTerms> avg(n_ops);
        const int nth = std::max(1, std::min<int>(n_ops, (int)std::min(16u, std::thread::hardware_concurrency())));
        std::vector<std::exception_ptr> errs(nth);
        std::atomic<int> next{0};
        auto work = [&](int tid) {
            try {
                for (int k = next++; k < n_ops; k = next++) average_terms(h->sector, ops[k], avg[k]);
            } catch (...) {
                errs[tid] = std::current_exception();
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < nth; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& th : pool) th.join();
        for (auto& e : errs)
            if (e) std::rethrow_exception(e);
        const auto t1 = std::chrono::steady_clock::now();
        if (h->cplx) run_expval<double2>(h, (const double2*)psi, avg, out);
        else run_expval<double>(h, (const double*)psi, avg, out);
        if (trace_on()) {
            size_t nt = 0;
            for (const auto& a : avg) nt += a.keys.size();
            const auto t2 = std::chrono::steady_clock::now();
            std::fprintf(stderr, "[qmb expval] %d operators, %zu averaged terms: averaging %.3f ms, kernels %.3f ms\n",
                         n_ops, nt, std::chrono::duration<double, std::milli>(t1 - t0).count(),
                         std::chrono::duration<double, std::milli>(t2 - t1).count());
        }
    });
}
