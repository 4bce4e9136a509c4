/*
 * qmb_b200.h -- C ABI of the B200-native XXZ/Heisenberg exact-diagonalization
 * engine (libqmb_b200.so).
 *
 * The reference (jeohjee/QMBCuda) crosses into its GPU layer inside C++
 * driver constructors, after flattening its model and symmetry objects into
 * plain arrays.  Each entry point below takes those arrays and replaces one
 * reference interface; the citation beside it names the reference file:line
 * (paths relative to the reference's QMBCuda/ directory).
 *
 * Conventions
 *  - Every call returns qmb_status; QMB_OK == 0.  No C++ exception crosses
 *    the boundary.  qmb_last_error() gives a message for the calling thread.
 *  - States are uint64 bit strings, bit q set <=> site q spin up (L <= 64).
 *  - Group elements use the reference layout: perm[g*L + q] is the site the
 *    spin at site q moves to (the inverse site permutation that
 *    SymmetryClass::GetGroupElemArr produces).  Element 0 is applied to each
 *    orbit representative to obtain a row's source string (as the reference
 *    does); groups built here put the identity first.
 *  - Complex numbers are interleaved (re, im) doubles.
 *  - Handles own their device memory.  A handle may be used by one host
 *    thread at a time; distinct handles are independent.
 *  - "_dev" pointers are device pointers; everything else is host memory.
 */
#ifndef QMB_B200_H
#define QMB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QMB_ABI_VERSION 1

#if defined(__GNUC__)
#define QMB_API __attribute__((visibility("default")))
#else
#define QMB_API
#endif

typedef int qmb_status;
#define QMB_OK 0
#define QMB_ERR_INVALID 1       /* bad argument or inconsistent tables            */
#define QMB_ERR_CUDA 2          /* CUDA runtime error (message has the details)   */
#define QMB_ERR_NOMEM 3         /* device or host allocation failed               */
#define QMB_ERR_ELL_OVERFLOW 4  /* a row needs more slots than the given width    */
#define QMB_ERR_NOT_CONVERGED 5 /* Lanczos stopped at max_iter above tolerance    */
#define QMB_ERR_TIMEOUT 6       /* reserved: no entry point of this version spins on
                                 * the device, so none returns it                 */
#define QMB_ERR_UNSUPPORTED 7   /* valid request outside what this build handles  */
#define QMB_ERR_NO_DEVICE 8     /* no CUDA device is visible                      */
#define QMB_ERR_IO 9            /* a table file could not be opened, read or written */
#define QMB_ERR_CORRUPT 10      /* a table file fails its checksums or layout checks */

/* Operator codes: the values of OperatorType
 * (quantum_operators/SingleParticleOperators.h:4). */
#define QMB_OP_SZ 0
#define QMB_OP_SP 1
#define QMB_OP_SM 2
#define QMB_OP_I 9

QMB_API int qmb_abi_version(void);
QMB_API const char* qmb_last_error(void);
QMB_API const char* qmb_status_string(qmb_status s);
/* Number of visible CUDA devices (0 on a host without a GPU). */
QMB_API int qmb_device_count(void);

/* Measurement entry point, no counterpart in the reference: the current
 * device's bandwidth (GB/s) for gathering whole rows of row_bytes bytes at
 * scattered rows of a buffer of `rows` rows that stays in L2, the access
 * pattern of the batched product's x gathers, with nothing else in the
 * kernel (about `gathers` rows, kernel time in *ms, best of five launches).
 * row_bytes is 16 times a power of two, at most 4096. */
QMB_API qmb_status qmb_l2_gather_probe(int64_t rows, int row_bytes, int64_t gathers, double* gbs, double* ms);

/* ======================================================= host-side helpers
 * Pure host code (no GPU): model and symmetry tables in reference layout. */

/* LatticeGeometryInfo (geometry/base.h:5-11).  a[0..3] = A_mat row-major:
 * a1 = (a[0], a[2]), a2 = (a[1], a[3]). */
typedef struct {
    int N1, N2, n_sub;
    double a[4];
    const double* rx; /* [n_sub] */
    const double* ry; /* [n_sub] */
} qmb_geometry;

/* Site coordinates in reference order, site = (i*N2 + j)*n_sub + alpha
 * (SpinHamiltonian::CreateGeometry, lattice_models/ArbitrarySpinLattice.cu:43-59). */
QMB_API qmb_status qmb_geometry_sites(const qmb_geometry* geom, double* R1, double* R2);

/* T_standard<T> pair list (lattice_models/T_standard.cu:12-147): ordered
 * (T_ind1, T_ind2, value) triples over the 3x3 image cells.  *n_pairs gets
 * the count; QMB_ERR_INVALID if it exceeds cap (nothing written past cap). */
QMB_API qmb_status qmb_tstandard_pairs(const qmb_geometry* geom, int nJ, const double* J /* complex */,
                               const double* range, int intra, int inter, int cap, int* t_ind1,
                               int* t_ind2, double* t_val /* complex */, int* n_pairs);

/* Coupling shells of CreateExtendedHeisenbergXXX (lattice_models/
 * Heisenberg.cu:88-176): rows (di, dj, a, b) with their J, sorted by
 * distance, J_vec[n] assigned to the n-th distance shell.  Jxy and Jz rows
 * are identical in the reference; one list is returned. */
QMB_API qmb_status qmb_extended_xxx_shells(const qmb_geometry* geom, int nJ, const double* J, int cap,
                                   int* rows /* [cap][4] */, double* J_out, int* n_rows);

/* Heisenberg::CreateHamiltonian (lattice_models/Heisenberg.cu:22-79) followed
 * by BuildOperatorVecs (exact_diagonalization/
 * HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:306-336): operator tables with
 * op codes and scalars already conjugated, two operators per term.
 * Term order: unit cell, then the Jxy rows (S+_i S-_j with Jxy), then the Jz
 * rows (Sz_i Sz_j with Jz), as the reference builds them.  n_terms_out gets
 * the count; QMB_ERR_INVALID if it exceeds cap. */
QMB_API qmb_status qmb_heisenberg_terms(const qmb_geometry* geom, int n_xy, const int* xy_rows /* [n][4] */,
                                const double* Jxy /* complex [n_xy] */, int n_z,
                                const int* z_rows /* [n][4] */, const double* Jz, int intra,
                                int inter, int cap, int* n_ops /* [cap] */,
                                int* op_code /* [cap][2] */, int* op_site /* [cap][2] */,
                                double* scalar /* complex [cap] */, int* n_terms_out);

/* Group element arrays from transformed coordinates, as
 * SymmetryClass::GetGroupElemArr (symmetries/SymmetryClass.cu:26-71 with
 * utils/misc_funcs.cu:80-90): TR1/TR2 [G][L] are the images of the sites
 * (R1, R2); coordinates match within 1e-3.  QMB_ERR_INVALID if a site has no
 * image. */
QMB_API qmb_status qmb_group_elem_arr(int L, int G, const double* R1, const double* R2, const double* TR1,
                              const double* TR2, uint32_t* perm /* [G][L] */);

/* Tnm_group (symmetries/Groups.cu:49-113): all N1*N2 lattice translations,
 * element g = nx*N2 + ny, as reference-layout arrays, plus the character
 * table chi[a][g] = exp(2 pi i (ax*nx/N1 + ay*ny/N2)), a = ax*N2 + ay. */
QMB_API qmb_status qmb_group_translations(const qmb_geometry* geom, uint32_t* perm /* [G][L] */,
                                  double* chars /* complex [G][G] */);

/* Cn_group (symmetries/Groups.cu:11-43) on the given sites: element i is the
 * rotation by 2 pi i / n about R0; chars[a][i] = exp(2 pi i a*i / n). */
QMB_API qmb_status qmb_group_rotations(int L, const double* R1, const double* R2, int n,
                               const double R0[2], uint32_t* perm /* [n][L] */,
                               double* chars /* complex [n][n] */);

/* T_standard pair list -> operator tables with the rule of
 * BuildHamiltonianForAbelianGroup (exact_diagonalization/utils.cu:235-327):
 * each pair (i, j, T) gives a diagonal term Sz_i Sz_j with T*Jz_w and, for
 * i != j, a hopping term that lowers i and raises j with T*Jxy_w.  Entries
 * keep the pair order.  swap_weights exchanges the two weights, as
 * BuildHoppingHam_v2 does (utils.cu:410-411). */
QMB_API qmb_status qmb_terms_from_pairs(int n_pairs, const int* t_ind1, const int* t_ind2,
                                const double* t_val /* complex */, double jxy_w, double jz_w,
                                int swap_weights, int cap, int* n_ops, int* op_code, int* op_site,
                                double* scalar, int* n_terms_out);

/* ================================================================ sectors
 * The fixed-Sz sector of L sites with n_up up spins, reduced by an Abelian
 * group of site permutations and, optionally, global spin inversion (an
 * extension: the reference has none).  With spin inversion the element set
 * is e = z*G + g (z = 0, 1), and a character row supplies n_ext = 2G values.
 * Replaces BuildBasisStates + BuildSRStates
 * (exact_diagonalization/HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:276-400). */
typedef struct qmb_sector_s* qmb_sector;

typedef struct {
    int L;
    int n_up;
    int n_perm;            /* G >= 1 */
    const uint32_t* perm;  /* [G][L], reference layout */
    int spin_flip;         /* 1: include global spin inversion (needs 2*n_up == L) */
    int device;            /* CUDA device ordinal */
} qmb_sector_desc;

typedef struct {
    int64_t n_states;  /* C(L, n_up) */
    int64_t n_orbits;  /* representatives (all orbits) */
    int64_t n_active;  /* non-null orbits of the selected irrep (0 before one is set) */
    int n_ext;         /* G or 2G */
    int structured;    /* 1 if every element runs as word rotations */
    int is_real;       /* selected irrep's characters are real */
} qmb_sector_info;

QMB_API qmb_status qmb_sector_create(const qmb_sector_desc* desc, qmb_sector* out);
QMB_API qmb_status qmb_sector_destroy(qmb_sector s);
QMB_API qmb_status qmb_sector_get_info(qmb_sector s, qmb_sector_info* info);

/* Selects the irrep: chars[n_ext] (complex).  Computes every orbit's norm
 *   norm = sqrt(| sum_{i,j: g_i r = g_j r} conj(chi_i) chi_j |) / n_ext
 * (ComputeSRSNorms, exact_diagonalization/utils.cu:767-805), evaluated exactly
 * in FP64 as sqrt(n_ext |sum_{h in Stab(r)} chi(h)|) / n_ext, and the active
 * (norm >= tol_norm) subset that forms the Lanczos basis. */
QMB_API qmb_status qmb_sector_set_irrep(qmb_sector s, const double* chars, double tol_norm);

/* Orbit representatives in ascending order (SRS_states_min after sort/unique,
 * HeisenbergHamAbelianSymms_CUDA.cu:368-375, as strings instead of ranks). */
QMB_API qmb_status qmb_sector_reps(qmb_sector s, uint64_t* reps, int64_t cap);
/* Norms of all orbits for the selected irrep. */
QMB_API qmb_status qmb_sector_norms(qmb_sector s, double* norms, int64_t cap);
/* Orbit index of each active row. */
QMB_API qmb_status qmb_sector_active(qmb_sector s, int64_t* orbit_of_row, int64_t cap);
/* Reference-layout map sector rank -> (orbit, element) over all C(L, n_up)
 * strings, keeping the largest element where several reach one string: the
 * sequential outcome of ComputeOrbitIndices (exact_diagonalization/utils.cu:66-80). */
QMB_API qmb_status qmb_sector_orbit_map(qmb_sector s, uint32_t* orbit_indices /* [2*n_states] */,
                                int64_t cap);
/* Representative lookup: for strings t[n] of the sector, the orbit index
 * (or -1 if t is not in the sector) and the element e with g_e(t) = rep. */
QMB_API qmb_status qmb_sector_lookup(qmb_sector s, const uint64_t* t, int64_t n, int64_t* orbit,
                             int32_t* element);

/* =========================================================== Hamiltonians
 * Operator tables with the semantics of BuildHamiltonianXXZForAbelianGroup
 * (exact_diagonalization/utils.cu:83-184): for each term, the ops are applied
 * in order to the row's source string (Sm needs the spin up and lowers it; Sp
 * needs it down and raises it; Sz multiplies by +-1/2; others do nothing); a
 * result equal to the source adds to the diagonal, else the entry
 *   scalar * chi(g_t) * norm_t / norm_s
 * goes to the target's orbit unless that orbit is null. */
typedef struct {
    int n_terms;
    int n_col;              /* row length of op_code / op_site */
    const int* n_ops;       /* [n_terms] */
    const int* op_code;     /* [n_terms][n_col] */
    const int* op_site;     /* [n_terms][n_col] */
    const double* scalar;   /* complex [n_terms] */
} qmb_terms;

typedef struct qmb_ham_s* qmb_ham;

#define QMB_PREC_FP64 1  /* keep FP64 values */
#define QMB_PREC_FP32 2  /* keep FP32 values */

typedef struct {
    int64_t n_rows;
    int64_t nnz_offdiag;   /* stored off-diagonal entries */
    int64_t padded;        /* sliced-ELL slots including padding */
    int max_row;           /* largest off-diagonal count of a row */
    int is_complex;
    int n_codes;           /* distinct off-diagonal FP32 values (dictionary size) */
    int coded;             /* 1: FP32 off-diagonals packed as 8-bit code | 24-bit column */
    double bytes_fp64;     /* algorithmic bytes of one FP64 H*v (plain sliced-ELL entries) */
    double bytes_fp32;     /* algorithmic bytes of one FP32 H*v (plain sliced-ELL entries) */
    int coded_fp64;        /* 1: real FP64 off-diagonals packed the same way (one block) */
} qmb_ham_info;

/* Builds the matrix on the active rows of the sector's irrep, in sliced ELL
 * (32-row slices, column-major inside a slice) with a separate diagonal.
 * prec is a mask of QMB_PREC_*.  Replaces the launch of
 * HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:229-259. */
QMB_API qmb_status qmb_ham_create(qmb_sector s, const qmb_terms* terms, int prec, qmb_ham* out);
QMB_API qmb_status qmb_ham_destroy(qmb_ham h);
QMB_API qmb_status qmb_ham_get_info(qmb_ham h, qmb_ham_info* info);

/* Reference row-major layout over ALL orbits (slot 0 = diagonal, null rows
 * have track 0 and ind[row*W] = row), values FP64 (complex).  Rebuilds on
 * the GPU with the same rule.  QMB_ERR_ELL_OVERFLOW if a row needs more than
 * W slots (the reference would overwrite the next row). */
QMB_API qmb_status qmb_ham_export_ref(qmb_sector s, const qmb_terms* terms, int W, uint32_t* ind,
                              double* val /* complex [R*W] */, int16_t* track);

/* Brute-force layout of BuildHoppingHam_v2 (exact_diagonalization/
 * utils.cu:381-439) over the whole sector (column = sector rank). */
QMB_API qmb_status qmb_ham_export_nosym(int L, int n_up, const qmb_terms* terms, int W, uint32_t* ind,
                                double* val /* complex */, int16_t* track, int device);

/* y = H x on device vectors of the active basis.  prec selects the stored
 * values and the vector type: QMB_PREC_FP64 -> double (or complex double),
 * QMB_PREC_FP32 -> float (complex float).  stream may be 0. */
QMB_API qmb_status qmb_hv(qmb_ham h, int prec, const void* x_dev, void* y_dev, void* stream);
/* Same with host buffers: copies x in, multiplies, copies y out. */
QMB_API qmb_status qmb_hv_host(qmb_ham h, int prec, const void* x, void* y);
/* Matrix-free y = H x: every row regenerates its entries (flips, orbit search,
 * lookup) instead of reading stored ones. */
QMB_API qmb_status qmb_hv_matrix_free(qmb_ham h, int prec, const void* x_dev, void* y_dev, void* stream);

/* ================================================================ Lanczos */
#define QMB_MODE_FP64 0   /* FP64 vectors and values                              */
#define QMB_MODE_MIXED 1  /* FP32 vectors and values, FP64 reductions + FP64 refinement restart */
#define QMB_MODE_FP32 2   /* FP32 vectors and values, FP64 reductions, no refinement */

#define QMB_START_SPLITMIX 0 /* uniform(-1,1) from splitmix64(seed + i)                */
#define QMB_START_CURAND 1   /* curand_init(seed+i,0,0) + curand_uniform, as init_random_vec */

#define QMB_HV_STORED 0
#define QMB_HV_MATRIX_FREE 1

typedef struct {
    int mode;           /* QMB_MODE_* */
    int max_iter;       /* Krylov steps of the (first) phase; fixed count when tol <= 0 */
    int min_iter;
    double tol;         /* relative: stop when residual estimate < tol*|E| and dE < tol*|E| */
    int reorth;         /* full reorthogonalization against the stored basis: classical
                           Gram-Schmidt passes a step, 0..2; the second pass runs when
                           the first removed more than 1 - 1/sqrt(2) of the vector's
                           norm (Kahan-Parlett), every step with QMB_REORTH_ALWAYS=1 */
    int start;          /* QMB_START_* */
    uint64_t seed;
    int check_every;    /* convergence test interval (iterations) */
    int hv;             /* QMB_HV_STORED or QMB_HV_MATRIX_FREE */
    int refine_max_iter;/* FP64 steps of the refinement restart (mixed mode) */
    int want_vector;    /* 1: keep the ground-state vector (FP64) on the handle */
} qmb_lanczos_opts;

typedef struct {
    double E0;           /* lowest Ritz value (final phase) */
    double E0_low;       /* lowest Ritz value of the FP32 phase (mixed mode) */
    double residual;     /* ||H psi - E0 psi|| / ||psi|| in FP64 */
    double residual_ref; /* the reference's measure ||H psi - E psi|| / N */
    int iters;           /* Krylov steps, all phases */
    int iters_low;       /* FP32-phase steps */
    int n_hv;            /* matrix-vector products, all phases */
    int converged;
    double ms_total;     /* device time of the solve (CUDA events) */
    double ms_hv;        /* device time inside H*v kernels (-1: not measured) */
    double n_products;   /* H*v products of single problems computed (batches: active
                            sectors x coupling sets per step; single solves: n_hv) */
    double n_launches;   /* kernels of this library executed by the call (launches
                            plus kernel nodes run by its CUDA graphs) */
} qmb_lanczos_result;

QMB_API void qmb_lanczos_default_opts(qmb_lanczos_opts* o);

/* Ground state of the handle's matrix.  krylov_coeffs (optional, [max_iter])
 * receives the Ritz coefficients of the final phase, as eig_vec_Krylov_out
 * of LanczosEigVals_CUDA (exact_diagonalization/lanczos.cu:128-317). */
QMB_API qmb_status qmb_lanczos(qmb_ham h, const qmb_lanczos_opts* opts, qmb_lanczos_result* res,
                       double* krylov_coeffs, int64_t n_coeffs);
/* Copies the kept ground-state vector (FP64, complex if the matrix is). */
QMB_API qmb_status qmb_ground_state(qmb_ham h, void* psi /* host */, int64_t n);
/* Puts a vector (FP64, complex if the matrix is; host memory) on the handle
 * as its kept ground state, the counterpart of qmb_ground_state: a vector
 * saved from an earlier solve of the same sector irrep becomes the state of
 * qmb_expval without a new solve. */
QMB_API qmb_status qmb_set_ground_state(qmb_ham h, const void* psi /* host */, int64_t n);

/* LanczosEigVals_CUDA (exact_diagonalization/lanczos.h:20-32) on a
 * caller-owned reference-layout ELL in device memory: FP32 values, fixed
 * NIter steps, no reorthogonalization, cuRAND start vector from seed;
 * FP64 reductions and an FP64 tridiagonal eigensolve.  Writes E[0], the
 * Ritz coefficients (if krylov_out) and returns the residual
 * ||H psi - E psi|| / nobv through *residual (checkEigState path). */
QMB_API qmb_status qmb_lanczos_ref_ell(float* E, int n_iter, int nobv, int max_terms, long long seed,
                               const uint32_t* ind_dev, const void* val_dev, const int16_t* track_dev,
                               int is_complex, float* krylov_out, int check_eig_state,
                               float* residual);

/* qmb_lanczos_ref_ell without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate GPU memory while they
 * run -- a serving loop that reserved its memory budget up front, a process
 * under a hard per-process memory cap, or code beside a pooled allocator that
 * must not see cudaMalloc/cudaFree (both synchronise the whole device).
 *
 * Same arguments and results as qmb_lanczos_ref_ell, plus `stream` (a
 * cudaStream_t; NULL = the legacy default stream).  All work vectors, the
 * Lanczos scalars and the reduction scratch live in one static device array
 * of 12 MiB + 64 KiB per device, fixed when the library's device code is
 * loaded.  Limits: nobv <= 262144 rows and n_iter <= 1024 steps; larger sizes
 * return QMB_ERR_INVALID (use qmb_lanczos_ref_ell for them).
 *
 * Every call looks up the scratch's device address on the current device
 * (the first call on a device also loads the device code); make that first
 * call before any stream capture begins.  The host-side work arrays (about
 * 70 KB) are static too, not on the caller's stack.  The scratch is shared by every call on a device in
 * this process: calls that overlap on the GPU race on it.  This function
 * takes a process-wide lock and synchronises `stream` before it returns, so
 * host threads calling it are serialised. */
QMB_API qmb_status qmb_lanczos_ref_ell_noalloc(float* E, int n_iter, int nobv, int max_terms,
                                       long long seed, const uint32_t* ind_dev,
                                       const void* val_dev, const int16_t* track_dev,
                                       int is_complex, float* krylov_out, int check_eig_state,
                                       float* residual, void* stream);

/* LanczosEigenStateFromSeed (exact_diagonalization/lanczos.cu:31-104): the
 * ground state sum_j krylov[j] v_j of a finished qmb_lanczos_ref_ell solve,
 * regenerated from the same seed on the same reference-layout ELL.  The
 * Lanczos vectors are bit-identical to the solve's (same start, same
 * kernels); psi_dev receives nobv floats (complex: interleaved pairs).
 * krylov is the host array the solve wrote to krylov_out; trailing zeros
 * (a solve that broke down early) shorten the regeneration. */
QMB_API qmb_status qmb_eigvec_from_seed_ref(long long seed, void* psi_dev, const float* krylov, int n_iter,
                                    int nobv, int max_terms, const uint32_t* ind_dev,
                                    const void* val_dev, const int16_t* track_dev, int is_complex);

/* ============================================================== table files
 * Versioned binary files for reuse across runs, in place of the reference's
 * raw float dumps (WriteArrayToFile, utils/print_funcs.cu:73-90, called for
 * vals_mat.bin / ind_mat.bin at HeisenbergHamAbelianSymms_CUDA.cu:149-162),
 * which store indices as floats and carry no sizes or version.  A file has a
 * header (magic "QMBTABLE", format version, kind, kind-specific scalars), a
 * section table and 64-byte aligned payloads, each with a 64-bit checksum.
 * Files are written under a temporary name and renamed.  Errors:
 * QMB_ERR_IO (open, read, write), QMB_ERR_CORRUPT (checksums, truncation,
 * layout), QMB_ERR_UNSUPPORTED (newer format version or other byte order).
 *
 * qmb_sector_save / qmb_sector_load: group, representatives and the selected
 * irrep.  Loading skips the enumeration of all C(L, n_up) strings; it checks
 * that every stored representative is its orbit's minimum and recomputes the
 * irrep's norms on the device. */
QMB_API qmb_status qmb_sector_save(qmb_sector s, const char* path);
QMB_API qmb_status qmb_sector_load(const char* path, int device, qmb_sector* out);
/* qmb_ham_save / qmb_ham_load: the sliced-ELL matrix, its values in every
 * stored precision and its term tables.  The file records the sector and
 * irrep it was built for (group, representatives, characters, tolerance);
 * loading into a different one is QMB_ERR_INVALID. */
QMB_API qmb_status qmb_ham_save(qmb_ham h, const char* path);
QMB_API qmb_status qmb_ham_load(qmb_sector s, const char* path, qmb_ham* out);
/* Reference-layout ELL tables in host memory (ind [n_rows][width] uint32,
 * val [n_rows][width] float or complex float, track [n_rows] int16), the
 * tables LanczosEigVals_CUDA consumes.  qmb_ref_ell_load with all three
 * buffers NULL only reports the sizes; otherwise cap_rows must cover n_rows.
 * No GPU is needed for either call. */
QMB_API qmb_status qmb_ref_ell_save(const char* path, int64_t n_rows, int width, const uint32_t* ind,
                            const void* val, const int16_t* track, int is_complex);
QMB_API qmb_status qmb_ref_ell_load(const char* path, int64_t* n_rows, int* width, int* is_complex,
                            uint32_t* ind, void* val, int16_t* track, int64_t cap_rows);

/* ================================================================ observables
 * Zero-temperature expectation values out[2k] + i out[2k+1] =
 * <psi|A_k|psi> / <psi|psi> for n_ops operators on the handle's sector irrep.
 * Each A_k is a sum of products of Sz, S+, S- (and I) in the table form of
 * qmb_terms -- the form the reference's ComputeStaticExpValZeroT builds from a
 * ManyBodyOperator (HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:434-455): every
 * term's factors daggered (S+ <-> S-) in application order and its scalar
 * conjugated.  Replaces ComputeStaticExpValZeroT's rebuild + eigenvector
 * regeneration + ExpecValArbOperatorAbelianIrrepProjHeisenbergZeroT + reduce
 * (HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:421-601, utils.cu:442-550).
 *
 * psi_dev: the state on the device (FP64; complex double if the handle is
 * complex), or NULL for the ground state kept on the handle (qmb_lanczos with
 * want_vector, or qmb_set_ground_state).  Terms whose S+ and S- counts differ
 * change Sz and contribute zero.  Other operator codes are QMB_ERR_INVALID.
 * All operators are evaluated in one pass of one kernel per shared-memory
 * chunk of terms; sums are FP64 and deterministic. */
QMB_API qmb_status qmb_expval(qmb_ham h, int n_ops, const qmb_terms* ops, const void* psi_dev, double* out);

/* ============================================================== batches
 * Many coupling sets over many sectors of one model family:
 *   H(i, s) = c_xy[i] * A_s + c_z[i] * D_s
 * with A_s / D_s the hopping / diagonal parts of sector s (shared by all
 * coupling sets), c_xy / c_z per set.  All (set, sector) pairs run in one
 * batched Lanczos whose iterations are CUDA graphs.  Extends the serial sector
 * loop of HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:127-242. */
typedef struct qmb_batch_s* qmb_batch;

typedef struct {
    int n_sectors;
    const qmb_sector* sectors;      /* irreps already selected */
    const qmb_terms* terms_xy;      /* hopping part (off-diagonal entries) */
    const qmb_terms* terms_z;       /* diagonal part */
    int n_sets;
    int device;
} qmb_batch_desc;

typedef struct {
    int64_t rows_total;     /* sum over sectors of active rows */
    int64_t elems_total;    /* rows_total * n_sets */
    double bytes_hv_fp64;   /* algorithmic bytes of one batched H*v (all pairs) */
    double bytes_hv_fp32;
    int rows_per_block;     /* rows of one thread block */
    int sets_per_thread;    /* coupling sets handled by one thread */
    int set_stride;         /* sets per row in the device vector layout (padded) */
    int variant_fp32;       /* H*v kernel variant chosen by the tuner (-1: not tuned yet) */
    int variant_fp64;
    float tune_ms_fp32[8];  /* tuner timings of the variants, ms */
    float tune_ms_fp64[8];
    int ring_slots[2];      /* FP32 Krylov vectors the handle's ring holds now, real and
                               complex sectors (0: none yet); the ring starts at 128
                               (QMB_RING_START) and doubles when a solve needs more */
    int64_t nnz_total;      /* off-diagonal entries of the hopping parts, all sectors */
} qmb_batch_info;

QMB_API qmb_status qmb_batch_create(const qmb_batch_desc* desc, qmb_batch* out);
QMB_API qmb_status qmb_batch_destroy(qmb_batch b);
QMB_API qmb_status qmb_batch_get_info(qmb_batch b, qmb_batch_info* info);
/* Ground energies of all pairs: E0[set*n_sectors + sector].  c_xy, c_z are
 * host arrays [n_sets]; copied in, solved, E0 copied out. */
QMB_API qmb_status qmb_batch_solve(qmb_batch b, const double* c_xy, const double* c_z,
                           const qmb_lanczos_opts* opts, double* E0, qmb_lanczos_result* summary);
/* One batched y = H x over all pairs on device buffers in the layout of
 * qmb_batch_layout (FP64: double / complex double; FP32: float / complex
 * float).  prec: QMB_PREC_FP64 or QMB_PREC_FP32.  x_dev and y_dev must be
 * 16-byte aligned (64-byte alignment, as cudaMalloc gives, lets the fastest
 * kernel variants run). */
QMB_API qmb_status qmb_batch_hv(qmb_batch b, int prec, const void* x_dev, void* y_dev, void* stream);
/* Measurement: the batched Lanczos step's product kernel as a solve runs it
 * (K1: y = H x with the epilogue that reads v_{j-1}, writes v_j and y and
 * sums alpha), over both sector kinds, on the couplings of the last
 * qmb_batch_solve (zeros before the first).  reps (1..1000) steps from a
 * seeded start, each K1 launch bracketed by CUDA events, after one warm-up
 * step; the steps' update kernels run between them untimed.  *ms = mean K1
 * time of one step, *bytes = its algorithmic bytes (those of qmb_batch_hv plus
 * v_{j-1} read and v_j written for every (row, set)).  No reference
 * counterpart: the reference has no batched solver. */
QMB_API qmb_status qmb_batch_k1_time(qmb_batch b, int prec, int reps, double* ms, double* bytes);
/* Device vector layout: sectors of the real kind first, then those of the
 * complex kind (is_complex[s] tells which; real sectors that have fewer than
 * a quarter of the complex sectors' rows are stored and solved complex, with
 * zero imaginary parts); each sector is [row][set] with set stride
 * info.set_stride.  offsets[s] is the
 * start of caller sector s in scalars (a complex element counts 2);
 * offsets[n_sectors] is the total. */
QMB_API qmb_status qmb_batch_layout(qmb_batch b, int64_t* offsets /* [n_sectors+1] */,
                            int* is_complex /* [n_sectors] */);

#ifdef __cplusplus
}
#endif
#endif /* QMB_B200_H */
