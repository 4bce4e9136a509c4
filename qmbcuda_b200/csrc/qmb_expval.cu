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
#include <complex>
#include <map>
#include <vector>

#include "qmb_ham.cuh"
#include "qmb_b200.h"

namespace qmb {
namespace {

constexpr int kEvBlock = 256;
constexpr size_t kEvSmemCap = 200 * 1024;  // dynamic shared memory per block

// Group average of one operator table: key = op words (code << 8 | site) in
// application order, value = the summed scalar.
using TermMap = std::map<std::vector<uint16_t>, std::complex<double>>;

void average_terms(const qmb_sector_s* s, const qmb_terms& A, TermMap& out) {
    QMB_REQUIRE(A.n_terms >= 0, QMB_ERR_INVALID, "expval: n_terms must be >= 0");
    if (A.n_terms == 0) return;
    QMB_REQUIRE(A.n_ops && A.op_code && A.op_site && A.scalar, QMB_ERR_INVALID,
                "expval: null table");
    QMB_REQUIRE(A.n_col >= 1 && A.n_col <= kMaxCol, QMB_ERR_INVALID, "expval: n_col must be in 1..8");
    const int L = s->L, G = s->G, ne = s->n_ext;
    std::vector<uint16_t> base, img;
    for (int i = 0; i < A.n_terms; ++i) {
        QMB_REQUIRE(A.n_ops[i] >= 0 && A.n_ops[i] <= A.n_col, QMB_ERR_INVALID,
                    "expval: n_ops out of range");
        const std::complex<double> sc(A.scalar[2 * i], A.scalar[2 * i + 1]);
        QMB_REQUIRE(std::isfinite(sc.real()) && std::isfinite(sc.imag()), QMB_ERR_INVALID,
                    "expval: non-finite scalar");
        base.clear();
        int n_p = 0, n_m = 0, n_z = 0;
        for (int j = 0; j < A.n_ops[i]; ++j) {
            const int c = A.op_code[i * A.n_col + j], q = A.op_site[i * A.n_col + j];
            QMB_REQUIRE(c == QMB_OP_SZ || c == QMB_OP_SP || c == QMB_OP_SM || c == QMB_OP_I,
                        QMB_ERR_INVALID, "expval: operator codes must be Sz, Sp, Sm or I");
            QMB_REQUIRE(q >= 0 && q < L, QMB_ERR_INVALID, "expval: site out of range");
            if (c == QMB_OP_I) continue;
            n_p += c == QMB_OP_SP;
            n_m += c == QMB_OP_SM;
            n_z += c == QMB_OP_SZ;
            base.push_back((uint16_t)(c << 8 | q));
        }
        if (n_p != n_m || sc == 0.0) continue;  // leaves the Sz sector, or zero
        for (int e = 0; e < ne; ++e) {
            const uint32_t* p = s->perm.data() + (size_t)(e % G) * L;
            const bool z = e >= G;
            img.resize(base.size());
            for (size_t j = 0; j < base.size(); ++j) {
                int c = base[j] >> 8, q = base[j] & 0xff;
                if (z && c != QMB_OP_SZ) c = c == QMB_OP_SP ? QMB_OP_SM : QMB_OP_SP;
                img[j] = (uint16_t)(c << 8 | (int)p[q]);
            }
            // factors on distinct sites commute: order them by site
            bool distinct = true;
            for (size_t a = 0; a < img.size() && distinct; ++a)
                for (size_t b = a + 1; b < img.size(); ++b)
                    if ((img[a] & 0xff) == (img[b] & 0xff)) {
                        distinct = false;
                        break;
                    }
            if (distinct)
                std::sort(img.begin(), img.end(),
                          [](uint16_t x, uint16_t y) { return (x & 0xff) < (y & 0xff); });
            const double sign = (z && (n_z & 1)) ? -1.0 : 1.0;
            out[img] += sc * (sign / ne);
        }
    }
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
// npart[block] receives the block's partial of <psi|psi>.
template <class V>
__global__ void __launch_bounds__(kEvBlock) k_expval(RowGen rg, int64_t n, const V* __restrict__ psi,
                                                     int n_seg, const int* __restrict__ seg_t,
                                                     double2* __restrict__ part,
                                                     double* __restrict__ npart) {
    extern __shared__ __align__(16) unsigned char smem_ev[];
    __shared__ double2 red[kEvBlock / 32];
    const GroupSmem gs = load_group(rg.g, smem_ev);
    const TermsSmem ts = load_terms(rg.terms, smem_ev + align16(group_smem_bytes(rg.g)));
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int sg = 0; sg < n_seg; ++sg) {
        const int t0 = seg_t[sg], t1 = seg_t[sg + 1];
        double ax = 0.0, ay = 0.0;
        for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += stride) {
            const int64_t o = rg.orbit_of_row[r];
            const uint64_t src = apply_elem(rg.g, gs, 0, rg.rt.reps[o]);
            // complex row sum even for a real psi: scalars may be complex
            const double2 pr = Sc<V>::to2(psi[r]);
            double2 y = make_double2(0.0, 0.0);
            const double2 d = gen_row_range(rg, gs, ts, t0, t1, src, rg.norms[o], [&](int64_t ot, double2 v) {
                const double2 x = Sc<V>::to2(__ldg(psi + rg.row_of_orbit[ot]));
                y.x += v.x * x.x - v.y * x.y;
                y.y += v.x * x.y + v.y * x.x;
            });
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

struct Segment {
    int op, t0, t1;  // operator, term range in the chunk
};

template <class V>
void run_expval(qmb_ham_s* h, const V* psi, const std::vector<TermMap>& ops, double* out) {
    const qmb_sector_s* s = h->sector;
    RowGen rg = h->row_gen();
    const size_t gbytes = align16(group_smem_bytes(rg.g));
    DevBuf<int> err(1);
    err.zero();
    rg.err = err.p;

    // flatten: terms of operator k back to back; chunks sized to shared memory
    struct Flat {
        int op;
        const std::vector<uint16_t>* key;
        std::complex<double> sc;
    };
    std::vector<Flat> flat;
    for (size_t k = 0; k < ops.size(); ++k)
        for (const auto& kv : ops[k]) flat.push_back({(int)k, &kv.first, kv.second});

    const int dev = h->device;
    int sms = 148, max_smem = 0;
    QMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    QMB_CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem_cap = std::min(kEvSmemCap, (size_t)max_smem);
    QMB_REQUIRE(gbytes + 64 < smem_cap, QMB_ERR_INVALID, "expval: group tables leave no shared memory");

    std::vector<double2> seg_sum;
    std::vector<int> seg_op;
    double norm2 = 0.0;
    bool have_norm = false;
    size_t pos = 0;
    do {
        // chunk [pos, end): as many terms as fit
        size_t end = pos;
        int n_col = 1;
        for (; end < flat.size(); ++end) {
            const int c = std::max(n_col, (int)flat[end].key->size());
            const size_t bytes = gbytes + ((20 + 2 * (size_t)c) * (end - pos + 1) + 15) / 16 * 16;
            if (bytes > smem_cap || end - pos + 1 > (size_t)kMaxTerms) break;
            n_col = c;
        }
        QMB_REQUIRE(end > pos || flat.empty(), QMB_ERR_INVALID, "expval: a term does not fit");
        const int nt = (int)(end - pos);
        std::vector<int> nops(std::max(nt, 1), 0);
        std::vector<uint16_t> opw((size_t)std::max(nt, 1) * n_col, 0);
        std::vector<double2> sc(std::max(nt, 1), make_double2(0.0, 0.0));
        std::vector<Segment> segs;
        for (int i = 0; i < nt; ++i) {
            const Flat& f = flat[pos + i];
            nops[i] = (int)f.key->size();
            std::copy(f.key->begin(), f.key->end(), opw.begin() + (size_t)i * n_col);
            sc[i] = make_double2(f.sc.real(), f.sc.imag());
            if (segs.empty() || segs.back().op != f.op) segs.push_back({f.op, i, i + 1});
            else segs.back().t1 = i + 1;
        }
        DevBuf<int> d_nops(nops.size());
        DevBuf<uint16_t> d_ops(opw.size());
        DevBuf<double2> d_sc(sc.size());
        d_nops.upload(nops.data(), nops.size());
        d_ops.upload(opw.data(), opw.size());
        d_sc.upload(sc.data(), sc.size());
        rg.terms.n_terms = nt;
        rg.terms.n_col = n_col;
        rg.terms.n_ops = d_nops.p;
        rg.terms.ops = d_ops.p;
        rg.terms.scalar = d_sc.p;
        const size_t smem = gbytes + terms_smem_bytes(rg.terms);
        const int n_seg = (int)segs.size();
        std::vector<int> seg_t(n_seg + 1, 0);
        for (int i = 0; i < n_seg; ++i) seg_t[i + 1] = segs[i].t1;
        DevBuf<int> d_seg(seg_t.size());
        d_seg.upload(seg_t.data(), seg_t.size());

        const void* kf = (const void*)k_expval<V>;
        set_group_smem_attr(kf, smem);
        int per_sm = 0;
        QMB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_expval<V>, kEvBlock, smem));
        const int64_t want = (h->n + kEvBlock - 1) / kEvBlock;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * std::max(1, per_sm)));
        DevBuf<double2> part((size_t)std::max(n_seg, 1) * grid), seg_d(std::max(n_seg, 1));
        DevBuf<double> npart(grid);
        k_expval<V><<<grid, kEvBlock, smem>>>(rg, h->n, psi, n_seg, d_seg.p, part.p, npart.p);
        check_launch("k_expval");
        if (n_seg) {
            k_expval_sum<<<n_seg, kEvBlock>>>(part.p, grid, seg_d.p);
            check_launch("k_expval_sum");
        }
        std::vector<double2> hs(n_seg);
        std::vector<double> hn(grid);
        if (n_seg) seg_d.download(hs.data(), n_seg);
        npart.download(hn.data(), grid);
        QMB_CUDA_TRY(cudaDeviceSynchronize());
        for (int i = 0; i < n_seg; ++i) {
            seg_sum.push_back(hs[i]);
            seg_op.push_back(segs[i].op);
        }
        if (!have_norm) {
            for (double v : hn) norm2 += v;
            have_norm = true;
        }
        pos = end;
    } while (pos < flat.size());
    int herr = 0;
    err.download(&herr, 1);
    QMB_REQUIRE(herr == 0, QMB_ERR_INVALID, "expval: a term left the sector's representative table");
    QMB_REQUIRE(norm2 > 0.0, QMB_ERR_INVALID, "expval: psi is zero");
    (void)s;
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
        std::vector<TermMap> avg(n_ops);
        for (int k = 0; k < n_ops; ++k) average_terms(h->sector, ops[k], avg[k]);
        if (h->cplx) run_expval<double2>(h, (const double2*)psi, avg, out);
        else run_expval<double>(h, (const double*)psi, avg, out);
    });
}
