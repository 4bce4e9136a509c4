// qmb_sector.cuh -- internal sector object shared by the modules.
#pragma once
#include <complex>
#include <vector>

#include "qmb_group.cuh"

struct qmb_sector_s {
    int device = 0;
    int L = 0, n_up = 0, G = 0, n_ext = 0, flip = 0;
    int64_t n_states = 0, R = 0, n_active = 0;
    std::vector<uint32_t> perm;  // host copy [G][L]

    // group on device
    int structured = 0, W = 0, n_chunks = 0;
    int full_rot = 0;  // a chain group of all L <= 32 rotations, element 0 the identity
    int full_torus = 0;  // all translations of a torus of W <= 8 site rows, element 0 the identity
    qmb::DevBuf<qmb::ElemRot> rot;
    qmb::DevBuf<uint64_t> tables;

    // orbit table
    qmb::DevBuf<uint64_t> reps;     // [R] ascending
    qmb::DevBuf<uint32_t> bucket;   // [2^T + 1]
    int T = 0;

    // selected irrep
    bool has_irrep = false;
    int irrep_gen = 0;  // counts qmb_sector_set_irrep calls
    uint64_t reps_sum = 0;  // checksum of reps for table files (0: not computed yet)
    bool is_real = true;
    double tol_norm = 1e-5;
    std::vector<std::complex<double>> chars;  // [n_ext]
    qmb::DevBuf<double2> chars_dev;           // [n_ext]
    qmb::DevBuf<double> norms;                // [R]
    qmb::DevBuf<int64_t> row_of_orbit;        // [R], -1 for null orbits
    qmb::DevBuf<int64_t> orbit_of_row;        // [n_active]

    qmb::GroupArgs group_args() const {
        qmb::GroupArgs g;
        g.L = L;
        g.G = G;
        g.n_ext = n_ext;
        g.structured = structured;
        g.W = W;
        g.n_chunks = n_chunks;
        g.full_rot = full_rot;
        g.full_torus = full_torus;
        g.mask = (L == 64) ? ~0ull : ((1ull << L) - 1);
        g.rot = rot.p;
        g.tables = tables.p;
        g.chars = chars_dev.p;
        return g;
    }
    qmb::RepTable rep_table() const {
        qmb::RepTable t;
        t.reps = reps.p;
        t.bucket = bucket.p;
        t.R = R;
        t.shift = L - T;
        return t;
    }
};

#include "qmb_b200.h"

namespace qmb {
// Pieces of qmb_sector_create / qmb_sector_set_irrep shared with the
// table-file loader (qmb_store.cu).
void sector_check_desc(const qmb_sector_desc* d);
void sector_setup(qmb_sector_s* s, const qmb_sector_desc* d);
void sector_buckets(qmb_sector_s* s);
void sector_select_irrep(qmb_sector_s* s, const double* chars, double tol_norm);
// A sector from stored representatives instead of an enumeration.  The
// representatives are checked: ascending, in the sector, and each the
// minimum of its orbit under the group.
qmb_sector_s* sector_from_reps(const qmb_sector_desc* d, const uint64_t* reps, int64_t R);
}  // namespace qmb
