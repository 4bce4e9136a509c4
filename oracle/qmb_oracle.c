/*
 * qmb_oracle.c -- CPU restatement (FP64) of the reference's XXZ exact-
 * diagonalization path.  TEST INFRASTRUCTURE ONLY: it is the checker used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.  The
 * product library (qmbcuda_b200/libqmb_b200.so) never links or calls it.
 *
 * Parity is pinned in two ways (see tests/test_oracle_pins.py):
 *   - against the reference's own kernels, compiled for the host from the
 *     unmodified sources by oracle/Makefile into oracle/_ref/ and driven by
 *     oracle/ref_harness.cpp (bit-exact tables, FP32-level values);
 *   - against committed golden fixtures under tests/golden/.
 *
 * Every function cites the reference file:line (paths relative to the
 * QMBCuda/ project directory) whose behaviour it restates.
 *
 * States are uint64 bit strings: bit q set <=> site q spin up.  Complex
 * numbers cross the boundary as interleaved (re, im) double pairs.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <complex.h>

typedef double _Complex cplx;

/* ---------------------------------------------------------------- binomials */
static uint64_t g_binom[65][65];
static int g_binom_ready = 0;

static void binom_init(void) {
    if (g_binom_ready) return;
    for (int n = 0; n <= 64; ++n) {
        g_binom[n][0] = 1;
        for (int k = 1; k <= 64; ++k)
            g_binom[n][k] = (n == 0) ? 0 : g_binom[n - 1][k - 1] + g_binom[n - 1][k];
    }
    g_binom_ready = 1;
}

uint64_t oc_binom(int n, int k) {
    binom_init();
    if (n < 0 || k < 0 || n > 64 || k > 64) return 0;
    return g_binom[n][k];
}

/* Rank of s among the strings with the same popcount, in ascending integer
 * order.  Restates GetIndexInHilbertSubspace (exactly
 * exact_diagonalization/utils.cu:9-36): scanning bits from the top, a set bit
 * at position p with r set bits at positions <= p contributes C(p, r).  The
 * reference evaluates C() with a recursive FP64 product
 * (utils/misc_funcs_gpu.cu:9-18) rounded by +0.5; here it is exact. */
uint64_t oc_rank(uint64_t s) {
    binom_init();
    uint64_t r = 0;
    int k = 0;
    for (int p = 0; p < 64; ++p) {
        if (s >> p & 1ull) {
            ++k;
            r += g_binom[p][k];
        }
    }
    return r;
}

/* Inverse of oc_rank for strings of L bits with k set bits. */
uint64_t oc_unrank(uint64_t r, int L, int k) {
    binom_init();
    uint64_t s = 0;
    for (int p = L - 1; p >= 0 && k > 0; --p) {
        uint64_t c = g_binom[p][k];
        if (r >= c) {
            s |= 1ull << p;
            r -= c;
            --k;
        }
    }
    return s;
}

/* All L-bit strings with k set bits in ascending order: what BuildBasisStates
 * produces (exact_diagonalization/HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:
 * 276-296; HeisenbergHam_CUDA.cu:41-58) by filtering 0..2^L-1 on popcount. */
int64_t oc_enumerate(int L, int k, uint64_t* out, int64_t cap) {
    binom_init();
    int64_t n = (int64_t)g_binom[L][k];
    if (n > cap) return -n;
    if (n == 0) return 0;
    uint64_t s = (k == 0) ? 0 : ((k == 64) ? ~0ull : ((1ull << k) - 1));
    for (int64_t i = 0; i < n; ++i) {
        out[i] = s;
        if (s == 0) break;
        /* next string with the same popcount (Gosper) */
        uint64_t c = s & (~s + 1);
        uint64_t rr = s + c;
        s = (((rr ^ s) >> 2) / c) | rr;
    }
    return n;
}

/* Group action.  An element is a site map perm[L] plus an optional global
 * spin inversion.  Bit q of the input moves to bit perm[q] of the output,
 * which is how SetUpSRS applies group_el (exact_diagonalization/
 * utils.cu:52-59; group_el holds the inverse site permutation,
 * symmetries/SymmetryClass.cu:58-66 + utils/misc_funcs.cu:80-90).  The
 * inversion (absent from the reference) complements all L bits. */
static inline uint64_t apply_op(uint64_t s, int L, const uint32_t* perm, int flip) {
    uint64_t out = 0;
    for (int q = 0; q < L; ++q)
        if (s >> q & 1ull) out |= 1ull << perm[q];
    if (flip) out ^= (L == 64) ? ~0ull : ((1ull << L) - 1);
    return out;
}

uint64_t oc_apply(uint64_t s, int L, const uint32_t* perm, int flip) {
    return apply_op(s, L, perm, flip);
}

/* Extended element e = z*G + g for z in {0, 1} when spin inversion is on. */
static inline uint64_t apply_ext(uint64_t s, int L, int G, const uint32_t* perm, int e) {
    int g = e % G, z = e / G;
    return apply_op(s, L, perm + (size_t)g * L, z);
}

/* Orbit representatives (minimum string of each orbit) in ascending order.
 * Restates SetUpSRS + SolveSRS_min + thrust sort/unique
 * (exact_diagonalization/utils.cu:39-64,750-762;
 * HeisenbergHamAbelianSymms_CUDA.cu:357-375).  n_ext = G (no inversion) or
 * 2G (with inversion). Returns the count, or -count if cap is too small. */
int64_t oc_reps(int L, int k, int G, const uint32_t* perm, int n_ext,
                uint64_t* reps, int64_t cap) {
    binom_init();
    int64_t n = (int64_t)g_binom[L][k];
    uint64_t s = (k == 0) ? 0 : ((1ull << k) - 1);
    int64_t R = 0;
    for (int64_t i = 0; i < n; ++i) {
        int is_rep = 1;
        for (int e = 0; e < n_ext; ++e) {
            if (apply_ext(s, L, G, perm, e) < s) { is_rep = 0; break; }
        }
        if (is_rep) {
            if (R < cap) reps[R] = s;
            ++R;
        }
        if (s == 0) break;
        uint64_t c = s & (~s + 1);
        uint64_t rr = s + c;
        s = (((rr ^ s) >> 2) / c) | rr;
    }
    return (R <= cap) ? R : -R;
}

/* Orbit norms for every irrep.  Restates ComputeSRSNorms
 * (exact_diagonalization/utils.cu:767-805):
 *   norm[o][a] = sqrt(| sum_{i,j : g_i s = g_j s} conj(chi_a(g_i)) chi_a(g_j) |) / G
 * with s = the orbit's representative and g_i running over the n_ext
 * elements (chars: [n_irr][n_ext] interleaved complex). */
void oc_norms(int L, int G, const uint32_t* perm, int n_ext, int64_t R,
              const uint64_t* reps, int n_irr, const double* chars,
              double* norms /* [R][n_irr] */) {
    uint64_t* img = (uint64_t*)malloc(sizeof(uint64_t) * n_ext);
    for (int64_t o = 0; o < R; ++o) {
        for (int e = 0; e < n_ext; ++e) img[e] = apply_ext(reps[o], L, G, perm, e);
        for (int a = 0; a < n_irr; ++a) {
            const double* ch = chars + (size_t)2 * a * n_ext;
            cplx acc = 0;
            for (int i = 0; i < n_ext; ++i)
                for (int j = 0; j < n_ext; ++j)
                    if (img[i] == img[j])
                        acc += conj(ch[2 * i] + I * ch[2 * i + 1]) * (ch[2 * j] + I * ch[2 * j + 1]);
            norms[o * n_irr + a] = sqrt(fabs(creal(acc))) / (double)n_ext;
        }
    }
    free(img);
}

/* Sector-rank -> (orbit, element) map with the reference's write order:
 * ComputeOrbitIndices (exact_diagonalization/utils.cu:66-80) lets thread
 * id = o*G + e write rank(g_e rep_o); where several elements reach the same
 * string the last sequential writer (largest e) is kept. */
void oc_orbit_map(int L, int G, const uint32_t* perm, int n_ext, int64_t R,
                  const uint64_t* reps, uint32_t* orbit_indices /* [2 * C(L,k)] */) {
    for (int64_t o = 0; o < R; ++o)
        for (int e = 0; e < n_ext; ++e) {
            uint64_t t = apply_ext(reps[o], L, G, perm, e);
            uint64_t r = oc_rank(t);
            orbit_indices[2 * r] = (uint32_t)o;
            orbit_indices[2 * r + 1] = (uint32_t)e;
        }
}

/* Shared row-writing tail of both symmetric ELL builders. */
typedef struct {
    int W, n_irr, alpha, n_ext;
    const uint32_t* oi;
    const double* norms;
    const double* chars; /* [n_irr][n_ext] complex */
    double tol;
} ell_ctx;

/* Symmetric ELL from decoded operator tables.  Restates
 * BuildHamiltonianXXZForAbelianGroup (exact_diagonalization/utils.cu:83-184)
 * with the table layout of BuildOperatorVecs
 * (HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:306-336): op codes (already
 * conjugated) 0 = Sz, 1 = Sp, 2 = Sm, others no-ops; scalars already
 * conjugated.  Rows run over all R orbits in reference row-major layout
 * (slot 0 = diagonal).  Returns the largest row count, or -1 when a row needs
 * more than W slots (the reference writes past the row in that case). */
int oc_ell_terms(int L, int G, const uint32_t* perm, int n_ext, int64_t R, const uint64_t* reps,
                 const uint32_t* orbit_indices, const double* norms, int n_irr, int alpha,
                 const double* chars, double tol_norm,
                 int n_terms, int n_col, const int* n_ops, const int* op_code, const int* op_site,
                 const double* scalar /* complex [n_terms] */,
                 int W, uint32_t* ind, double* val /* complex [R*W] */, int16_t* track) {
    (void)L;
    int max_row = 0, overflow = 0;
    for (int64_t id = 0; id < R; ++id) {
        ind[id * W] = (uint32_t)id;
        int t_ind = 1;
        double cn = norms[id * n_irr + alpha];
        if (cn < tol_norm) continue;
        uint64_t src = apply_ext(reps[id], L, G, perm, 0);
        cplx diag = 0;
        for (int hi = 0; hi < n_terms; ++hi) {
            uint64_t tgt = src;
            cplx coef = scalar[2 * hi] + I * scalar[2 * hi + 1];
            int bad = 0;
            for (int h2 = 0; h2 < n_ops[hi]; ++h2) {
                int site = op_site[hi * n_col + h2];
                int code = op_code[hi * n_col + h2];
                int spin = (int)(tgt >> site & 1ull);
                if (code == 2) { if (!spin) { bad = 1; break; } tgt &= ~(1ull << site); }
                else if (code == 1) { if (spin) { bad = 1; break; } tgt |= 1ull << site; }
                else if (code == 0) { coef *= 0.5 * (-1.0 + 2.0 * spin); }
            }
            if (bad) continue;
            if (tgt == src) { diag += coef; continue; }
            uint64_t rk = oc_rank(tgt);
            uint32_t orb = orbit_indices[2 * rk];
            uint32_t e = orbit_indices[2 * rk + 1];
            double tn = norms[(int64_t)orb * n_irr + alpha];
            if (tn < tol_norm) continue;
            if (t_ind >= W) { overflow = 1; t_ind++; continue; }
            const double* ch = chars + (size_t)2 * (alpha * n_ext + e);
            cplx v = coef * (ch[0] + I * ch[1]) * (tn / cn);
            ind[id * W + t_ind] = orb;
            val[2 * (id * W + t_ind)] = creal(v);
            val[2 * (id * W + t_ind) + 1] = cimag(v);
            t_ind++;
        }
        val[2 * (id * W)] = creal(diag);
        val[2 * (id * W) + 1] = cimag(diag);
        track[id] = (int16_t)t_ind;
        if (t_ind > max_row) max_row = t_ind;
    }
    return overflow ? -1 : max_row;
}

/* Symmetric ELL from a T_standard pair list.  Restates
 * BuildHamiltonianForAbelianGroup (exact_diagonalization/utils.cu:235-327):
 * per pair (i, j, T): diagonal += T*Jz_w/4 * sigma_i sigma_j; when bit i is
 * set and bit j clear, the string with i lowered and j raised gets
 * T*Jxy_w * chi(g) * norm_t / norm_s. */
int oc_ell_bonds(int L, int G, const uint32_t* perm, int n_ext, int64_t R, const uint64_t* reps,
                 const uint32_t* orbit_indices, const double* norms, int n_irr, int alpha,
                 const double* chars, double tol_norm,
                 int n_pairs, const int* ti, const int* tj, const double* tval /* complex */,
                 double jxy_w, double jz_w,
                 int W, uint32_t* ind, double* val, int16_t* track) {
    (void)L;
    int max_row = 0, overflow = 0;
    for (int64_t id = 0; id < R; ++id) {
        ind[id * W] = (uint32_t)id;
        int t_ind = 1;
        double cn = norms[id * n_irr + alpha];
        if (cn < tol_norm) continue;
        uint64_t src = apply_ext(reps[id], L, G, perm, 0);
        cplx diag = 0;
        for (int p = 0; p < n_pairs; ++p) {
            int i = ti[p], j = tj[p];
            cplx tv = tval[2 * p] + I * tval[2 * p + 1];
            cplx jz = tv * jz_w, jxy = tv * jxy_w;
            int si = (int)(src >> i & 1ull), sj = (int)(src >> j & 1ull);
            diag += jz * 0.25 * (-1.0 + 2.0 * si) * (-1.0 + 2.0 * sj);
            if (!si || sj) continue;
            uint64_t tgt = (src | (1ull << j)) & ~(1ull << i);
            uint64_t rk = oc_rank(tgt);
            uint32_t orb = orbit_indices[2 * rk];
            uint32_t e = orbit_indices[2 * rk + 1];
            double tn = norms[(int64_t)orb * n_irr + alpha];
            if (tn < tol_norm) continue;
            if (t_ind >= W) { overflow = 1; t_ind++; continue; }
            const double* ch = chars + (size_t)2 * (alpha * n_ext + e);
            cplx v = jxy * (ch[0] + I * ch[1]) * (tn / cn);
            ind[id * W + t_ind] = orb;
            val[2 * (id * W + t_ind)] = creal(v);
            val[2 * (id * W + t_ind) + 1] = cimag(v);
            t_ind++;
        }
        val[2 * (id * W)] = creal(diag);
        val[2 * (id * W) + 1] = cimag(diag);
        track[id] = (int16_t)t_ind;
        if (t_ind > max_row) max_row = t_ind;
    }
    return overflow ? -1 : max_row;
}

/* Full-sector ELL without symmetry.  Restates BuildHoppingHam_v2
 * (exact_diagonalization/utils.cu:381-439), including its exchange of the
 * two weights (J_z takes Jxy_w and J_xy takes Jz_w, :410-411). */
int oc_ell_nosym(int L, int k, int n_pairs, const int* ti, const int* tj, const double* tval,
                 double jxy_w, double jz_w, int W, uint32_t* ind, double* val, int16_t* track) {
    binom_init();
    int64_t n = (int64_t)g_binom[L][k];
    uint64_t s = (k == 0) ? 0 : ((1ull << k) - 1);
    int max_row = 0, overflow = 0;
    for (int64_t id = 0; id < n; ++id) {
        ind[id * W] = (uint32_t)id;
        int t_ind = 1;
        double diag = 0;
        for (int p = 0; p < n_pairs; ++p) {
            int i = ti[p], j = tj[p];
            double jz = tval[2 * p] * jxy_w, jxy = tval[2 * p] * jz_w;
            int si = (int)(s >> i & 1ull), sj = (int)(s >> j & 1ull);
            diag += jz * 0.25 * (-1.0 + 2.0 * si) * (-1.0 + 2.0 * sj);
            if (!si || sj) continue;
            uint64_t tgt = (s | (1ull << j)) & ~(1ull << i);
            if (t_ind >= W) { overflow = 1; t_ind++; continue; }
            ind[id * W + t_ind] = (uint32_t)oc_rank(tgt);
            val[2 * (id * W + t_ind)] = jxy;
            val[2 * (id * W + t_ind) + 1] = 0;
            t_ind++;
        }
        val[2 * (id * W)] = diag;
        val[2 * (id * W) + 1] = 0;
        track[id] = (int16_t)t_ind;
        if (t_ind > max_row) max_row = t_ind;
        if (s == 0) break;
        uint64_t c = s & (~s + 1);
        uint64_t rr = s + c;
        s = (((rr ^ s) >> 2) / c) | rr;
    }
    return overflow ? -1 : max_row;
}

/* y = A x for a reference-layout ELL (complex FP64).  Restates
 * SparseMatDenseVec_prod_EEL (exact_diagonalization/utils.cu:601-624). */
void oc_spmv(int64_t R, int W, const uint32_t* ind, const double* val, const int16_t* track,
             const double* x, double* y) {

    for (int64_t r = 0; r < R; ++r) {
        cplx acc = 0;
        for (int i = 0; i < track[r]; ++i) {
            int64_t q = r * W + i;
            uint32_t c = ind[q];
            acc += (val[2 * q] + I * val[2 * q + 1]) * (x[2 * (int64_t)c] + I * x[2 * (int64_t)c + 1]);
        }
        y[2 * r] = creal(acc);
        y[2 * r + 1] = cimag(acc);
    }
}

/* splitmix64 start vector, uniform(-1, 1): element i = f(seed + i). */
static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void oc_start_vector(uint64_t seed, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        uint64_t z = splitmix64(seed + (uint64_t)i);
        out[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
}

/* Zero-temperature expectation value with the rule of
 * ExpecValArbOperatorAbelianIrrepProjHeisenbergZeroT
 * (exact_diagonalization/utils.cu:442-550), then the sum over rows and the
 * division by the group size of ComputeStaticExpValZeroT
 * (HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:596-597).  Tables as that driver
 * builds them (:434-455): codes daggered (0 Sz, 1 Sp, 2 Sm, 9 I), scalars
 * conjugated.  For every orbit row and term the factors are applied to each
 * member g_e(rep) of the orbit; the target's orbit o and member index e' come
 * from the orbit map, and the row gains
 *     conj(phi_row) conj(coef * (N_o / N_row) * conj(chi(e)) * chi(e')) phi_o.
 * phi is complex [R] over all orbits.  with_break = 1 keeps the reference's
 * loop exit (a factor that annihilates one member ends the member loop of
 * that term); 0 visits every member.  Code 9 (identity) is skipped here; the
 * reference's decode map has no entry for it and applies it as Sz.
 * out = complex sum / n_ext. */
void oc_expval_ref(int L, int G, const uint32_t* perm, int n_ext, int64_t R, const uint64_t* reps,
                   const uint32_t* orbit_indices, const double* norms, int n_irr, int alpha,
                   const double* chars, double tol_norm, int n_terms, int n_col, const int* n_ops,
                   const int* op_code, const int* op_site, const double* scalar,
                   const double* phi /* complex [R] */, int with_break, double* out /* complex */) {
    cplx acc = 0;
    const double* ch = chars + (size_t)2 * alpha * n_ext;
    for (int64_t id = 0; id < R; ++id) {
        double cn = norms[id * n_irr + alpha];
        if (cn < tol_norm) continue;
        cplx pid = phi[2 * id] + I * phi[2 * id + 1];
        for (int ai = 0; ai < n_terms; ++ai) {
            for (int gi = 0; gi < n_ext; ++gi) {
                uint64_t t = apply_ext(reps[id], L, G, perm, gi);
                cplx coef = scalar[2 * ai] + I * scalar[2 * ai + 1];
                int bad = 0;
                for (int k = 0; k < n_ops[ai]; ++k) {
                    int site = op_site[ai * n_col + k], code = op_code[ai * n_col + k];
                    int spin = (int)(t >> site & 1ull);
                    if (code == 2) { if (!spin) { bad = 1; break; } t &= ~(1ull << site); }
                    else if (code == 1) { if (spin) { bad = 1; break; } t |= 1ull << site; }
                    else if (code == 0) { coef *= 0.5 * (-1.0 + 2.0 * spin); }
                }
                if (bad) {
                    if (with_break) break;
                    continue;
                }
                uint64_t rk = oc_rank(t);
                uint32_t o = orbit_indices[2 * rk];
                uint32_t e2 = orbit_indices[2 * rk + 1];
                double tn = norms[(int64_t)o * n_irr + alpha];
                if (tn < tol_norm) continue;
                cplx cg = conj(ch[2 * gi] + I * ch[2 * gi + 1]);
                cplx ce = ch[2 * e2] + I * ch[2 * e2 + 1];
                cplx val = conj(coef * (tn / cn) * cg * ce);
                acc += conj(pid) * val * (phi[2 * o] + I * phi[2 * o + 1]);
            }
        }
    }
    acc /= (double)n_ext;
    out[0] = creal(acc);
    out[1] = cimag(acc);
}
