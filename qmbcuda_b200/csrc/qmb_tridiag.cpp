// qmb_tridiag.cpp -- see qmb_tridiag.h.  Written from the textbook methods
// (Sturm-sequence bisection; inverse iteration with Gaussian elimination with
// partial pivoting on a tridiagonal matrix).
#include "qmb_tridiag.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace qmb {

// Number of eigenvalues of T strictly below x (negative pivots of the LDL^T
// factorisation of T - x I).
static int sturm_count(const double* a, const double* e, int m, double x) {
    const double tiny = std::numeric_limits<double>::min() * 1e4;
    int cnt = 0;
    double d = a[0] - x;
    if (d < 0) ++cnt;
    for (int i = 1; i < m; ++i) {
        if (std::fabs(d) < tiny) d = d < 0 ? -tiny : tiny;
        d = a[i] - x - e[i - 1] * e[i - 1] / d;
        if (d < 0) ++cnt;
    }
    return cnt;
}

double tridiag_eig(const double* a, const double* e, int m, int k) {
    if (m <= 0) return 0.0;
    if (m == 1) return a[0];
    double lo = a[0], hi = a[0];
    for (int i = 0; i < m; ++i) {
        double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i < m - 1 ? std::fabs(e[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    double span = std::max(std::fabs(lo), std::fabs(hi));
    lo -= 1e-12 * span + 1e-300;
    hi += 1e-12 * span + 1e-300;
    // invariant: count(lo) <= k, count(hi) >= k + 1
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (sturm_count(a, e, m, mid) >= k + 1) hi = mid;
        else lo = mid;
        if (hi - lo <= 2.0 * std::numeric_limits<double>::epsilon() * std::max(std::fabs(lo), std::fabs(hi)))
            break;
    }
    return 0.5 * (lo + hi);
}

double tridiag_min_eig(const double* a, const double* e, int m) { return tridiag_eig(a, e, m, 0); }

// Solves (T - theta I) x = b in place of b, Gaussian elimination with
// partial pivoting (row i may swap with row i+1, creating a second
// superdiagonal).
static void tridiag_solve(const double* a, const double* e, int m, double theta, double* b) {
    std::vector<double> d(m), du(m), du2(m), dl(m);
    std::vector<int> piv(m, 0);
    const double tiny = std::numeric_limits<double>::epsilon() * 1e-3;
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = std::max(scale, std::fabs(a[i] - theta));
    for (int i = 0; i < m - 1; ++i) scale = std::max(scale, std::fabs(e[i]));
    if (scale == 0.0) scale = 1.0;
    for (int i = 0; i < m; ++i) {
        d[i] = a[i] - theta;
        du[i] = i < m - 1 ? e[i] : 0.0;
        dl[i] = i < m - 1 ? e[i] : 0.0;
        du2[i] = 0.0;
    }
    for (int i = 0; i < m - 1; ++i) {
        if (std::fabs(d[i]) >= std::fabs(dl[i])) {
            if (std::fabs(d[i]) < tiny * scale) d[i] = tiny * scale;
            double f = dl[i] / d[i];
            dl[i] = f;
            d[i + 1] -= f * du[i];
            piv[i] = 0;
        } else {
            double f = d[i] / dl[i];
            d[i] = dl[i];
            dl[i] = f;
            double t = du[i];
            du[i] = d[i + 1];
            d[i + 1] = t - f * d[i + 1];
            if (i < m - 2) {
                du2[i] = du[i + 1];
                du[i + 1] = -f * du2[i];
            }
            piv[i] = 1;
        }
    }
    if (std::fabs(d[m - 1]) < tiny * scale) d[m - 1] = tiny * scale;
    // forward: apply L^-1 with the same interchanges
    for (int i = 0; i < m - 1; ++i) {
        if (piv[i]) std::swap(b[i], b[i + 1]);
        b[i + 1] -= dl[i] * b[i];
    }
    // back substitution with U (d, du, du2)
    b[m - 1] /= d[m - 1];
    if (m > 1) b[m - 2] = (b[m - 2] - du[m - 2] * b[m - 1]) / d[m - 2];
    for (int i = m - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i];
}

void tridiag_eigvec(const double* a, const double* e, int m, double theta, double* v) {
    if (m <= 0) return;
    if (m == 1) {
        v[0] = 1.0;
        return;
    }
    for (int i = 0; i < m; ++i) v[i] = 1.0 / std::sqrt((double)m) * (1.0 + 1e-3 * ((i * 7919) % 13));
    for (int it = 0; it < 3; ++it) {
        tridiag_solve(a, e, m, theta, v);
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += v[i] * v[i];
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) {
            for (int i = 0; i < m; ++i) v[i] = i == 0 ? 1.0 : 0.0;
            return;
        }
        for (int i = 0; i < m; ++i) v[i] /= nrm;
    }
    if (v[0] < 0)
        for (int i = 0; i < m; ++i) v[i] = -v[i];
}

// Same elimination as tridiag_solve, on caller-provided arrays.
static void tridiag_solve_ws(const double* a, const double* e, int m, double theta, double* b,
                             double* d, double* du, double* du2, double* dl, int* piv) {
    const double tiny = std::numeric_limits<double>::epsilon() * 1e-3;
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = std::max(scale, std::fabs(a[i] - theta));
    for (int i = 0; i < m - 1; ++i) scale = std::max(scale, std::fabs(e[i]));
    if (scale == 0.0) scale = 1.0;
    for (int i = 0; i < m; ++i) {
        d[i] = a[i] - theta;
        du[i] = i < m - 1 ? e[i] : 0.0;
        dl[i] = i < m - 1 ? e[i] : 0.0;
        du2[i] = 0.0;
        piv[i] = 0;
    }
    for (int i = 0; i < m - 1; ++i) {
        if (std::fabs(d[i]) >= std::fabs(dl[i])) {
            if (std::fabs(d[i]) < tiny * scale) d[i] = tiny * scale;
            double f = dl[i] / d[i];
            dl[i] = f;
            d[i + 1] -= f * du[i];
        } else {
            double f = d[i] / dl[i];
            d[i] = dl[i];
            dl[i] = f;
            double t = du[i];
            du[i] = d[i + 1];
            d[i + 1] = t - f * d[i + 1];
            if (i < m - 2) {
                du2[i] = du[i + 1];
                du[i + 1] = -f * du2[i];
            }
            piv[i] = 1;
        }
    }
    if (std::fabs(d[m - 1]) < tiny * scale) d[m - 1] = tiny * scale;
    for (int i = 0; i < m - 1; ++i) {
        if (piv[i]) std::swap(b[i], b[i + 1]);
        b[i + 1] -= dl[i] * b[i];
    }
    b[m - 1] /= d[m - 1];
    if (m > 1) b[m - 2] = (b[m - 2] - du[m - 2] * b[m - 1]) / d[m - 2];
    for (int i = m - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i];
}

void tridiag_eigvec_ws(const double* a, const double* e, int m, double theta, double* v,
                       double* work, int* iwork) {
    if (m <= 0) return;
    if (m == 1) {
        v[0] = 1.0;
        return;
    }
    double *d = work, *du = work + m, *du2 = work + 2 * m, *dl = work + 3 * m;
    for (int i = 0; i < m; ++i) v[i] = 1.0 / std::sqrt((double)m) * (1.0 + 1e-3 * ((i * 7919) % 13));
    for (int it = 0; it < 3; ++it) {
        tridiag_solve_ws(a, e, m, theta, v, d, du, du2, dl, iwork);
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += v[i] * v[i];
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) {
            for (int i = 0; i < m; ++i) v[i] = i == 0 ? 1.0 : 0.0;
            return;
        }
        for (int i = 0; i < m; ++i) v[i] /= nrm;
    }
    if (v[0] < 0)
        for (int i = 0; i < m; ++i) v[i] = -v[i];
}

}  // namespace qmb
