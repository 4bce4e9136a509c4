// qmb_models.cpp -- host-side model and symmetry tables in reference layout.
//
// These produce the plain arrays that the reference's driver classes flatten
// their objects into before the GPU work starts: T_standard pair lists,
// ManyBodyOperator tables (after BuildOperatorVecs), group element arrays and
// character tables.  No GPU is touched.  Where the reference computes in
// float (coordinates, distances) the same float operations are used so range
// cut-offs fall on the same side.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "qmb_b200.h"

namespace qmb {
qmb_status fail(qmb_status s, const std::string& msg);
}

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Geom {
    int N1, N2, M;
    float a1x, a1y, a2x, a2y;
    std::vector<float> rx, ry;
};

bool load_geom(const qmb_geometry* g, Geom& o) {
    if (!g || g->N1 < 1 || g->N2 < 1 || g->n_sub < 1 || !g->rx || !g->ry) return false;
    o.N1 = g->N1;
    o.N2 = g->N2;
    o.M = g->n_sub;
    // A_mat rows: {a1x, a2x}, {a1y, a2y}
    o.a1x = (float)g->a[0];
    o.a2x = (float)g->a[1];
    o.a1y = (float)g->a[2];
    o.a2y = (float)g->a[3];
    o.rx.resize(o.M);
    o.ry.resize(o.M);
    for (int i = 0; i < o.M; ++i) {
        o.rx[i] = (float)g->rx[i];
        o.ry[i] = (float)g->ry[i];
    }
    return (long long)o.N1 * o.N2 * o.M <= 64;
}

// Site coordinates (SpinHamiltonian::CreateGeometry, lattice_models/
// ArbitrarySpinLattice.cu:43-59; T_standard.cu:20-33 builds the same list).
void sites(const Geom& g, std::vector<float>& R1, std::vector<float>& R2) {
    R1.clear();
    R2.clear();
    for (int i = 0; i < g.N1; ++i)
        for (int j = 0; j < g.N2; ++j)
            for (int a = 0; a < g.M; ++a) {
                R1.push_back((float)i * g.a1x + (float)j * g.a2x + g.rx[a]);
                R2.push_back((float)i * g.a1y + (float)j * g.a2y + g.ry[a]);
            }
}

}  // namespace

extern "C" qmb_status qmb_geometry_sites(const qmb_geometry* geom, double* R1, double* R2) {
    Geom g;
    if (!load_geom(geom, g) || !R1 || !R2)
        return qmb::fail(QMB_ERR_INVALID, "invalid geometry (N1, N2, n_sub >= 1; at most 64 sites)");
    std::vector<float> r1, r2;
    sites(g, r1, r2);
    for (size_t i = 0; i < r1.size(); ++i) {
        R1[i] = r1[i];
        R2[i] = r2[i];
    }
    return QMB_OK;
}

// T_standard<T> constructor, lattice_models/T_standard.cu:12-147.
extern "C" qmb_status qmb_tstandard_pairs(const qmb_geometry* geom, int nJ, const double* J,
                                          const double* range, int intra, int inter, int cap,
                                          int* t_ind1, int* t_ind2, double* t_val, int* n_pairs) {
    Geom g;
    if (!load_geom(geom, g) || nJ < 1 || !J || !range || !n_pairs)
        return qmb::fail(QMB_ERR_INVALID, "invalid geometry or coupling list");
    if (intra == 0 && inter == 0)
        return qmb::fail(QMB_ERR_INVALID, "both intra- and inter-cluster flags are zero");
    std::vector<float> R1, R2;
    sites(g, R1, R2);
    const int LS = (int)R1.size();
    const float a1[2] = {g.a1x * g.N1, g.a1y * g.N1};
    const float a2[2] = {g.a2x * g.N2, g.a2y * g.N2};
    const float t_hold = 0.0001f;
    struct Trip { int i1, i2; double re, im; };
    std::vector<Trip> cells[3][3];
    for (int c1 = -1; c1 < 2; ++c1)
        for (int c2 = -1; c2 < 2; ++c2) {
            float tx = (float)c1 * a1[0] + (float)c2 * a2[0];
            float ty = (float)c1 * a1[1] + (float)c2 * a2[1];
            std::vector<Trip>& out = cells[c1 + 1][c2 + 1];
            for (int i = 0; i < LS; ++i)
                for (int lsi = 0; lsi < LS; ++lsi) {
                    float dx = R1[i] - (R1[lsi] + tx);
                    float dy = R2[i] - (R2[lsi] + ty);
                    float d = (float)std::sqrt(std::pow(dx, 2) + std::pow(dy, 2));
                    if (d < t_hold) continue;
                    for (int k = 0; k < nJ; ++k) {
                        if (d > (float)range[k]) continue;
                        out.push_back({lsi, i, J[2 * k], J[2 * k + 1]});
                        break;
                    }
                }
        }
    int n = 0;
    for (int c1 = -1; c1 < 2; ++c1)
        for (int c2 = -1; c2 < 2; ++c2) {
            if (c1 == 0 && c2 == 0) {
                if (intra == 0) continue;
            } else if (inter == 0) {
                continue;
            }
            for (const Trip& t : cells[c1 + 1][c2 + 1]) {
                if (n < cap && t_ind1 && t_ind2 && t_val) {
                    t_ind1[n] = t.i1;
                    t_ind2[n] = t.i2;
                    t_val[2 * n] = t.re;
                    t_val[2 * n + 1] = t.im;
                }
                ++n;
            }
        }
    *n_pairs = n;
    if (n > cap) return qmb::fail(QMB_ERR_INVALID, "pair list longer than cap");
    return QMB_OK;
}

// CreateExtendedHeisenbergXXX, lattice_models/Heisenberg.cu:88-176.
extern "C" qmb_status qmb_extended_xxx_shells(const qmb_geometry* geom, int nJ, const double* J,
                                              int cap, int* rows, double* J_out, int* n_rows) {
    Geom g;
    if (!load_geom(geom, g) || nJ < 1 || !J || !n_rows)
        return qmb::fail(QMB_ERR_INVALID, "invalid geometry or coupling list");
    struct T4 { int v[4]; };
    std::vector<T4> terms;
    std::vector<std::pair<int, float>> dist;
    int idx = 0;
    for (int ni = -g.N1; ni < g.N1; ++ni)
        for (int nj = -g.N2; nj < g.N2; ++nj)
            for (int ai = 0; ai < g.M; ++ai)
                for (int bi = 0; bi < g.M; ++bi) {
                    terms.push_back({{ni, nj, ai, bi}});
                    float x = (float)ni * g.a1x + (float)nj * g.a2x + g.rx[ai] - g.rx[bi];
                    float y = (float)ni * g.a1y + (float)nj * g.a2y + g.ry[ai] - g.ry[bi];
                    float d = sqrtf((float)(std::pow(x, 2) + std::pow(y, 2)));
                    dist.emplace_back(idx++, d);
                }
    std::stable_sort(dist.begin(), dist.end(),
                     [](const std::pair<int, float>& a, const std::pair<int, float>& b) {
                         return a.second < b.second;
                     });
    float J_curr = (float)J[0];
    int counter = -1;
    float d_curr = dist[0].second;
    const float thold = 0.001f;
    int n = 0;
    for (size_t i = 0; i < dist.size(); ++i) {
        float d = dist[i].second;
        if (d < thold) continue;
        if (d > d_curr + thold) {
            counter += 1;
            if (counter >= nJ) break;
            J_curr = (float)J[counter];
            d_curr = d;
        }
        if (n < cap && rows && J_out) {
            std::memcpy(rows + 4 * n, terms[dist[i].first].v, sizeof(int) * 4);
            J_out[n] = J_curr;
        }
        ++n;
    }
    *n_rows = n;
    if (n > cap) return qmb::fail(QMB_ERR_INVALID, "shell list longer than cap");
    return QMB_OK;
}

// Heisenberg::CreateHamiltonian (lattice_models/Heisenberg.cu:22-79), then
// BuildOperatorVecs (HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:306-336).
extern "C" qmb_status qmb_heisenberg_terms(const qmb_geometry* geom, int n_xy, const int* xy_rows,
                                           const double* Jxy, int n_z, const int* z_rows,
                                           const double* Jz, int intra, int inter, int cap,
                                           int* n_ops, int* op_code, int* op_site, double* scalar,
                                           int* n_terms_out) {
    Geom g;
    if (!load_geom(geom, g) || n_xy < 0 || n_z < 0 || !n_terms_out || (n_xy && (!xy_rows || !Jxy)) ||
        (n_z && (!z_rows || !Jz)))
        return qmb::fail(QMB_ERR_INVALID, "invalid geometry or term rows");
    if (intra == 0 && inter == 0)
        return qmb::fail(QMB_ERR_INVALID, "both intra- and inter-cluster flags are zero");
    const int M = g.M, N1 = g.N1, N2 = g.N2, N = N1 * N2;
    int n = 0;
    auto push = [&](int c0, int s0, int c1, int s1, double re, double im) {
        if (n < cap && n_ops && op_code && op_site && scalar) {
            n_ops[n] = 2;
            op_code[2 * n] = c0;
            op_code[2 * n + 1] = c1;
            op_site[2 * n] = s0;
            op_site[2 * n + 1] = s1;
            scalar[2 * n] = re;
            scalar[2 * n + 1] = im;
        }
        ++n;
    };
    for (int uc = 0; uc < N; ++uc) {
        int j1 = uc / N2, j2 = uc % N2;
        for (int jii = 0; jii < 2; ++jii) {
            int cnt = jii == 0 ? n_xy : n_z;
            const int* rowsp = jii == 0 ? xy_rows : z_rows;
            for (int ji = 0; ji < cnt; ++ji) {
                const int* r = rowsp + 4 * ji;
                int j_site = uc * M + r[3];
                int i1 = j1 + r[0], i2 = j2 + r[1];
                if (!intra && ((i1 < 0 || i1 >= N1) || (i2 < 0 || i2 >= N2))) continue;
                // Heisenberg.cu:57 tests (i >= 0 || i < N), true for every i,
                // so inter == false skips every term; kept as written.
                if (!inter && ((i1 >= 0 || i1 < N1) || (i2 >= 0 || i2 < N2))) continue;
                i1 = ((i1 % N1) + N1) % N1;
                i2 = ((i2 % N2) + N2) % N2;
                int i_site = r[2] + M * (N2 * i1 + i2);
                if (jii == 0) {
                    // S+_i S-_j scaled by Jxy; decode row conjugated: [Sm(i), Sp(j)],
                    // scalar conjugated
                    push(QMB_OP_SM, i_site, QMB_OP_SP, j_site, Jxy[2 * ji], -Jxy[2 * ji + 1]);
                } else {
                    push(QMB_OP_SZ, i_site, QMB_OP_SZ, j_site, Jz[ji], 0.0);
                }
            }
        }
    }
    *n_terms_out = n;
    if (n > cap) return qmb::fail(QMB_ERR_INVALID, "term list longer than cap");
    return QMB_OK;
}

// SymmetryClass::GetGroupElemArr, symmetries/SymmetryClass.cu:26-71 with the
// layout transform of utils/misc_funcs.cu:80-90: if site q maps to site p,
// perm[g][p] = q.
extern "C" qmb_status qmb_group_elem_arr(int L, int G, const double* R1, const double* R2,
                                         const double* TR1, const double* TR2, uint32_t* perm) {
    if (L < 1 || L > 64 || G < 1 || !R1 || !R2 || !TR1 || !TR2 || !perm)
        return qmb::fail(QMB_ERR_INVALID, "invalid arguments");
    const double tol = 0.001;
    for (int g = 0; g < G; ++g) {
        std::vector<int> seen(L, 0);
        for (int q = 0; q < L; ++q) {
            double x = TR1[(size_t)g * L + q], y = TR2[(size_t)g * L + q];
            int p = -1;
            for (int c = 0; c < L; ++c)
                if (std::fabs(R1[c] - x) < tol && std::fabs(R2[c] - y) < tol) {
                    p = c;
                    break;
                }
            if (p < 0)
                return qmb::fail(QMB_ERR_INVALID, "element " + std::to_string(g) + ": site " +
                                                      std::to_string(q) + " has no image site");
            if (seen[p])
                return qmb::fail(QMB_ERR_INVALID, "element " + std::to_string(g) + " is not a bijection");
            seen[p] = 1;
            perm[(size_t)g * L + p] = (uint32_t)q;
        }
    }
    return QMB_OK;
}

// Tnm_group, symmetries/Groups.cu:49-113, on the lattice index grid: element
// g = nx*N2 + ny moves site (i1, i2, a) to ((i1+nx) mod N1, (i2+ny) mod N2, a).
extern "C" qmb_status qmb_group_translations(const qmb_geometry* geom, uint32_t* perm,
                                             double* chars) {
    Geom g;
    if (!load_geom(geom, g) || !perm)
        return qmb::fail(QMB_ERR_INVALID, "invalid geometry");
    const int N1 = g.N1, N2 = g.N2, M = g.M, L = N1 * N2 * M, G = N1 * N2;
    for (int nx = 0; nx < N1; ++nx)
        for (int ny = 0; ny < N2; ++ny) {
            int e = nx * N2 + ny;
            for (int i1 = 0; i1 < N1; ++i1)
                for (int i2 = 0; i2 < N2; ++i2)
                    for (int a = 0; a < M; ++a) {
                        int q = (i1 * N2 + i2) * M + a;
                        int p = (((i1 + nx) % N1) * N2 + (i2 + ny) % N2) * M + a;
                        perm[(size_t)e * L + p] = (uint32_t)q;
                    }
        }
    if (chars) {
        for (int ax = 0; ax < N1; ++ax)
            for (int ay = 0; ay < N2; ++ay)
                for (int gx = 0; gx < N1; ++gx)
                    for (int gy = 0; gy < N2; ++gy) {
                        double ph = 2.0 * kPi * ((double)ax * gx / N1 + (double)ay * gy / N2);
                        size_t k = (size_t)(ax * N2 + ay) * G + (gx * N2 + gy);
                        chars[2 * k] = std::cos(ph);
                        chars[2 * k + 1] = std::sin(ph);
                    }
    }
    return QMB_OK;
}

// Cn_group, symmetries/Groups.cu:11-43 (rotation Cn, SymmOperators.cu:6-18).
extern "C" qmb_status qmb_group_rotations(int L, const double* R1, const double* R2, int n,
                                          const double R0[2], uint32_t* perm, double* chars) {
    if (L < 1 || L > 64 || n < 1 || !R1 || !R2 || !R0 || !perm)
        return qmb::fail(QMB_ERR_INVALID, "invalid arguments");
    std::vector<double> TR1((size_t)n * L), TR2((size_t)n * L);
    for (int i = 0; i < n; ++i) {
        double th = 2.0 * kPi * i / n, c = std::cos(th), s = std::sin(th);
        for (int q = 0; q < L; ++q) {
            double x = R1[q] - R0[0], y = R2[q] - R0[1];
            TR1[(size_t)i * L + q] = c * x - s * y + R0[0];
            TR2[(size_t)i * L + q] = s * x + c * y + R0[1];
        }
    }
    qmb_status st = qmb_group_elem_arr(L, n, R1, R2, TR1.data(), TR2.data(), perm);
    if (st != QMB_OK) return st;
    if (chars)
        for (int a = 0; a < n; ++a)
            for (int i = 0; i < n; ++i) {
                double ph = 2.0 * kPi * (double)a * i / n;
                chars[2 * ((size_t)a * n + i)] = std::cos(ph);
                chars[2 * ((size_t)a * n + i) + 1] = std::sin(ph);
            }
    return QMB_OK;
}

// Pair list -> operator tables, rule of BuildHamiltonianForAbelianGroup
// (exact_diagonalization/utils.cu:278-321) and, with swap_weights, of
// BuildHoppingHam_v2 (utils.cu:406-436).
extern "C" qmb_status qmb_terms_from_pairs(int n_pairs, const int* t_ind1, const int* t_ind2,
                                           const double* t_val, double jxy_w, double jz_w,
                                           int swap_weights, int cap, int* n_ops, int* op_code,
                                           int* op_site, double* scalar, int* n_terms_out) {
    if (n_pairs < 0 || (n_pairs && (!t_ind1 || !t_ind2 || !t_val)) || !n_terms_out)
        return qmb::fail(QMB_ERR_INVALID, "invalid pair list");
    double wz = swap_weights ? jxy_w : jz_w;
    double wxy = swap_weights ? jz_w : jxy_w;
    int n = 0;
    auto push = [&](int c0, int s0, int c1, int s1, double re, double im) {
        if (n < cap && n_ops && op_code && op_site && scalar) {
            n_ops[n] = 2;
            op_code[2 * n] = c0;
            op_code[2 * n + 1] = c1;
            op_site[2 * n] = s0;
            op_site[2 * n + 1] = s1;
            scalar[2 * n] = re;
            scalar[2 * n + 1] = im;
        }
        ++n;
    };
    for (int p = 0; p < n_pairs; ++p) {
        int i = t_ind1[p], j = t_ind2[p];
        double re = t_val[2 * p], im = t_val[2 * p + 1];
        push(QMB_OP_SZ, i, QMB_OP_SZ, j, re * wz, im * wz);
        if (i != j) push(QMB_OP_SM, i, QMB_OP_SP, j, re * wxy, im * wxy);
    }
    *n_terms_out = n;
    if (n > cap) return qmb::fail(QMB_ERR_INVALID, "term list longer than cap");
    return QMB_OK;
}
