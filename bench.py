"""Benchmark of the XXZ Lanczos ground-state path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric (the reference project's headline): H*v/s and HBM GB/s, mixed vs FP64
at |dE0| < 1e-9; batched sectors/s.  A "step" is one complete ground-state
solve of the workload (synthetic, seeded):

  batched            256 XXZ chains L=20, periodic, Delta ~ U(0,2), J ~ U(0.5,1.5)
                     (mt19937-64 seed 20261203 + rank), every momentum sector k=0..19
                     of Sz=0, one batched mixed-precision Lanczos (FP32 vectors/values,
                     FP64 scalars, FP64 refinement restart)

The single-sector workloads (L=16 without symmetry, L=24 k=0 even, L=32
J1-J2, 6x6) are parity tests at full size (tests/test_gpu_lanczos.py,
tests/test_gpu_configs.py).

`value` counts sector H*v products (one coupling set x one sector x one
product) per second of device time with inputs resident; `e2e` is the same
count over the wall time of the public C-ABI call that a step makes from host
buffers: qmb_batch_solve on the batch, with the step's couplings copied in
from pinned host memory and the energies copied out.  `e2e_with_setup` adds
building the 20 sectors and the batch from scratch to every step.  `--impl reference` times the
reference's own CPU H*v (SparseMatDenseVec_prod_EEL_host, compiled from its
sources into oracle/_ref) on the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(1, os.path.join(ROOT, "oracle"))

METRIC = "Hv/s and HBM GB/s, mixed vs FP64 at |dE0|<1e-9; batched sectors/s"
SEED = 20261203


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def couplings(n_sets: int, rank: int = 0):
    """Delta_i ~ U(0,2), J_i ~ U(0.5,1.5) from mt19937-64(seed), drawn in set order."""
    rng = np.random.Generator(np.random.MT19937(SEED + rank))
    d = np.empty(n_sets)
    j = np.empty(n_sets)
    for i in range(n_sets):
        d[i] = rng.uniform(0.0, 2.0)
        j[i] = rng.uniform(0.5, 1.5)
    return j, d


class Clocks:
    """nvidia-smi clock sampling during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.p = None
        import tempfile
        self.path = os.path.join(tempfile.gettempdir(), f"qmb_bench_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            # wait for nvidia-smi's first samples: its NVML start-up stalls
            # CUDA driver calls of this process for a while, which must not
            # fall into a timed step; sampling then runs throughout
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 10.0:
                time.sleep(0.1)
                try:
                    with open(self.path) as f:
                        if sum(1 for _ in f) >= 3:
                            break
                except OSError:
                    pass
            time.sleep(0.5)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.strip().split(",") for l in open(self.path) if l.strip()]
        except OSError:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[3:7]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def flush_l2(torch, buf):
    buf.add_(1.0)


# --------------------------------------------------------------- workloads
def batched_config(world: int, L: int = 20, n_sets: int = 256) -> dict:
    """The batched workload's `config`, the same for both arms.  Every Sz=0
    string lies in one orbit, and an orbit of d strings is active in d of the
    L momentum sectors, so the sectors hold C(L, L/2) rows together."""
    import math
    rows = math.comb(L, L // 2)
    return {
        "workload": f"batched: {n_sets} XXZ chains L={L} periodic, Delta~U(0,2), J~U(0.5,1.5) "
                    f"(mt19937-64 seed {SEED}), all k=0..{L - 1} of Sz=0, mixed precision",
        "n_sets": n_sets, "L": L, "sectors": L, "problems": n_sets * L,
        "rows_total": rows, "elements_per_hv": rows * n_sets,
        "l2_policy": "x and y of one batched H*v (complex FP32, %.0f MB each) exceed L2; "
                     "256 MB written between steps" % (rows * n_sets * 8 / 1e6),
        "parallelism": f"dp{world} (independent coupling sets per GPU)",
    }


def build_batched(q, L=20, n_sets=256):
    perm, ch = q.translation_group(L)
    secs = [q.Sector(L, L // 2, perm).set_irrep(ch[a]) for a in range(L)]
    bonds = q.chain_bonds(L)
    b = q.Batch(secs, q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"),
                n_sets)
    return secs, b


def time_k1(q, b, prec, reps=20):
    """The Lanczos step's product kernel as the solve runs it (K1: H x with
    the epilogue that reads v_{j-1} and writes v_j), CUDA events around each
    launch inside the library: (ms per step, algorithmic bytes)."""
    ms, byt = q._capi.C.c_double(), q._capi.C.c_double()
    q.check(q.lib().qmb_batch_k1_time(b.h, prec, reps, q._capi.C.byref(ms), q._capi.C.byref(byt)))
    return ms.value, byt.value


def time_batch_hv(torch, q, b, prec, reps=20):
    """Average device time of one batched H*v (CUDA events on the launch stream)."""
    off, cp = b.layout()
    tot = int(off[-1])
    dt = torch.float64 if prec == q._capi.PREC_FP64 else torch.float32
    x = torch.randn(tot, dtype=dt, device="cuda")
    y = torch.empty_like(x)
    st = torch.cuda.current_stream()
    sh = st.cuda_stream
    for _ in range(2):
        b.hv_dev(x.data_ptr(), y.data_ptr(), prec, sh)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        b.hv_dev(x.data_ptr(), y.data_ptr(), prec, sh)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def gather_bound(q, b, hv32_ms):
    """The batched FP32 product's x gathers against the device's bandwidth
    for that access pattern alone (qmb_l2_gather_probe): whole x rows of all
    sets (set stride x 8 bytes, complex FP32) read at scattered rows of a
    buffer of one sector's rows, as many rows as the product gathers."""
    A = q._capi
    info = b.info
    row_bytes = int(info.set_stride) * 8
    rows = int(info.rows_total) // max(1, len(b.sectors))
    gathers = int(info.nnz_total)
    gbs, ms = A.C.c_double(), A.C.c_double()
    q.check(q.lib().qmb_l2_gather_probe(rows, row_bytes, gathers, A.C.byref(gbs), A.C.byref(ms)))
    kern = gathers * row_bytes / (hv32_ms * 1e-3) / 1e9
    return {"probe": "qmb_l2_gather_probe: %d-byte rows at scattered rows of a %d-row buffer, %d gathers"
                     % (row_bytes, rows, gathers),
            "probe_gbs": gbs.value, "probe_ms": ms.value,
            "k_bhv_gather_bytes": gathers * row_bytes, "k_bhv_gather_gbs": kern,
            "k_bhv_frac_of_probe": kern / gbs.value}


def fp32_product_bytes(info):
    """Algorithmic bytes of one stored FP32 product in the handle's layout:
    x read once, y written once, the diagonal, and per off-diagonal a 32-bit
    column and an FP32 value (plain sliced ELL) or one 32-bit coded entry
    (8-bit value code and column, `info.coded`).  The second value is the plain
    layout's count for every handle, the convention of the H*v byte formula
    B_ell = N (nbar (4 + s_m) + s_m + 2 s_v)."""
    sv = 8 if info.is_complex else 4
    n, nnz = float(info.n_rows), float(info.nnz_offdiag)
    ell = float(info.bytes_fp32)
    if not int(info.coded):
        return ell, ell
    return nnz * 4 + n * (sv + 2 * sv), ell


def fp64_product_bytes(info):
    """fp32_product_bytes for the FP64 values (coded when `info.coded_fp64`)."""
    sv = 16 if info.is_complex else 8
    n, nnz = float(info.n_rows), float(info.nnz_offdiag)
    ell = float(info.bytes_fp64)
    if not int(info.coded_fp64):
        return ell, ell
    return nnz * 4 + n * (sv + 2 * sv), ell


def single_sector_hv(torch, q, reps=10):
    """Stored FP32 H*v of one large sector (L=32 J1-J2 chain, J2 = 0.5,
    Delta = 1, k = 0, spin-inversion even; 9,393,119 rows): CUDA-event time
    per product and its algorithmic bytes (qmb_ham_info.bytes_fp32)."""
    A = q._capi
    L = 32
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    J = [1.0] * L + [0.5] * L
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), J, J), prec=A.PREC_FP32)
    info = h.info
    x = torch.randn(int(info.n_rows), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    st = torch.cuda.current_stream()
    args = (h.h, A.PREC_FP32, A.C.c_void_p(x.data_ptr()), A.C.c_void_p(y.data_ptr()), A.C.c_void_p(st.cuda_stream))
    for _ in range(3):
        q.check(q.lib().qmb_hv(*args))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        q.check(q.lib().qmb_hv(*args))
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    peak, kind = load_peaks()
    byt, ell = fp32_product_bytes(info)
    gbs = byt / (ms * 1e-3) / 1e9
    out = {"workload": "L=32 J1-J2 chain, k=0, even (9,393,119 rows), stored FP32",
           "kernel": "k_hv<CbSellOp<float>> (coded entries, one column block)" if int(info.coded)
                     else "k_hv<SellOp<float>>",
           "rows": int(info.n_rows), "nnz": int(info.nnz_offdiag),
           "bytes": byt, "ms": ms, "achieved_gbs": gbs, "frac": gbs / peak,
           "bytes_ell_convention": ell, "frac_ell_convention": ell / (ms * 1e-3) / 1e9 / peak,
           "peak_source": kind}
    h.close()
    s.close()
    return out


def _averaged_sz_terms(ops_sites, L):
    """Distinct terms after averaging Sz-product terms over the L chain
    translations (factors on distinct sites ordered by site), per operator."""
    out = []
    for terms in ops_sites:
        keys = set()
        for sites in terms:
            for t in range(L):
                m = [(x + t) % L for x in sites]
                keys.add(tuple(sorted(m)) if len(set(m)) == len(m) else tuple(m))
        out.append(len(keys))
    return out


def observables(torch, q, reps=5):
    """Ground-state expectation values (qmb_expval) on the L=24 Heisenberg
    chain, k=0 (112,720 rows): the structure factor <Sz_q Sz_-q> at all 24 q
    (Fourier operators) and the 24 correlators <Sz_0 Sz_j>, 48 operators in one
    call.  Time of the whole call (host group averaging, chunk staging and the
    kernels) from CUDA events on the default stream, where it launches, and
    from the wall clock; work = rows x group-averaged terms.  Beside it the
    reference's member-loop rule (oracle restatement, one host thread) on
    <Sz_0 Sz_1> of the same state."""
    import oracle as O
    A = q._capi
    L = 24
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm).set_irrep(ch[0])
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L), 1.0, 1.0), prec=A.PREC_FP64)
    h.lanczos(mode=A.MODE_FP64, max_iter=300, tol=1e-12, want_vector=1, allow_unconverged=True)
    b = q.reciprocal_basis()
    ops, sites = [], []
    for n in range(L):
        kv = n * b[:, 0] / L
        f = q.multiply_terms(q.fourier_terms("Sz", kv, L, 1), q.fourier_terms("Sz", kv, L, 1, sign=-1))
        ops.append(q.operator_terms(f))
        sites.append([[x for _, x in fac] for _, fac in f])
    for j in range(L):
        ops.append(q.operator_terms([(1.0, [("Sz", 0), ("Sz", j)])]))
        sites.append([[0, j]])
    n_terms = int(np.sum(_averaged_sz_terms(sites, L)))
    rows = int(h.info.n_rows)
    h.expval(ops)
    st = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dev, wall = [], []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(st)
        v = h.expval(ops)
        e1.record(st)
        e1.synchronize()
        wall.append((time.perf_counter() - t0) * 1e3)
        dev.append(e0.elapsed_time(e1))
    ms = float(np.median(dev))
    corr = v[L:].real
    # the reference's rule on one host thread: every orbit member, one term
    g = O.Group(L, np.ascontiguousarray(perm, np.uint32), np.asarray(ch, np.complex128))
    sec = O.build_sector(g, L // 2)
    phi = np.zeros(sec.R, np.complex128)
    phi[O.active_rows(sec, 0)] = h.ground_state()
    tab = O.table_from_factors([(1.0, [(0, 0), (0, 1)])])
    t0 = time.perf_counter()
    v_cpu = O.expval_ref_rule(sec, tab, 0, phi, with_break=True)
    cpu_s = time.perf_counter() - t0
    evals = rows * n_terms
    out = {"workload": "L=24 Heisenberg chain ground state, k=0 (%d rows): S(q) at 24 q + 24 <Sz_0 Sz_j>, "
                       "48 operators, %d group-averaged terms" % (rows, n_terms),
           "kernel": "k_expval (+ k_expval_sum)", "ms_call": ms, "ms_wall": float(np.median(wall)),
           "row_term_evals_per_s": evals / (ms * 1e-3),
           "S_pi": float(v[L // 2].real), "SzSz_01": float(corr[1]),
           "SzSz_01_times_3L": float(3 * L * corr[1]),
           "cpu_reference_rule": {"operator": "<Sz_0 Sz_1>", "value": float(v_cpu.real),
                                  "row_member_term_evals": int(sec.R) * L, "s": cpu_s,
                                  "row_member_term_evals_per_s": sec.R * L / cpu_s, "cores": 1,
                                  "kind": "port"}}
    h.close()
    s.close()
    return out


def table_files(torch, q, reps=3):
    """Table files (qmb_sector_save/load, qmb_ham_save/load) against building
    from scratch: the L=32 J1-J2 chain sector (k=0, spin-inversion even;
    enumeration of C(32,16) strings) and the L=28 J1-J2 sector with its FP32
    matrix.  Wall times of the public calls (median of `reps` after one
    untimed round), file sizes, and whether the loaded tables and products
    are bit-identical to the built ones."""
    import tempfile
    A = q._capi

    def timed(f):
        f()
        ts, r = [], None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = f()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), r

    out = {}
    with tempfile.TemporaryDirectory() as d:
        for L, with_ham in ((32, False), (28, True)):
            perm, ch = q.translation_group(L)
            chars = q.with_spin_flip(ch[0], 1)
            t_build, s = timed(lambda: q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(chars))
            ps = os.path.join(d, f"L{L}.sector")
            t_save, _ = timed(lambda: s.save(ps))
            t_load, s2 = timed(lambda: q.Sector.load(ps))
            rec = {"rows": int(s.info.n_active), "orbits": int(s.info.n_orbits),
                   "sector_build_s": t_build, "sector_save_s": t_save, "sector_load_s": t_load,
                   "sector_file_mb": os.path.getsize(ps) / 1e6,
                   "sector_identical": bool(np.array_equal(s.reps(), s2.reps()))}
            if with_ham:
                J = [1.0] * L + [0.5] * L
                terms = q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), J, J)
                t_hb, h = timed(lambda: q.Hamiltonian(s, terms, prec=A.PREC_FP32))
                ph = os.path.join(d, f"L{L}.ham")
                t_hs, _ = timed(lambda: h.save(ph))
                t_hl, h2 = timed(lambda: q.Hamiltonian.load(s2, ph))
                x = np.random.default_rng(0).standard_normal(int(h.info.n_rows)).astype(np.float32)
                same = np.array_equal(h.hv_host(x, A.PREC_FP32), h2.hv_host(x, A.PREC_FP32))
                rec.update({"ham_build_s": t_hb, "ham_save_s": t_hs, "ham_load_s": t_hl,
                            "ham_file_mb": os.path.getsize(ph) / 1e6, "hv_identical": bool(same)})
            out[f"L{L}_j1j2_k0_even"] = rec
    return out


def single_sector_configs(torch, q):
    """The single-sector configurations, each one solve or product on one GPU
    (device times from the library's CUDA events; products from CUDA events
    on the launch stream):
      L=24 XXZ chain, Delta=0.5, k=0, spin-inversion even: FP64 vs mixed solve;
      L=32 J1-J2 chain, k=0, even: stored and matrix-free products, FP64 solve
        and mixed solves with two reorthogonalisation passes (stored and
        matrix-free);
      6x6 square lattice, k=(0,0), even: stored FP32 and matrix-free products."""
    A = q._capi
    st = torch.cuda.current_stream()

    def t_hv(h, prec, mf, reps):
        dt = torch.float64 if prec == A.PREC_FP64 else torch.float32
        n = int(h.info.n_rows)
        x = torch.randn(n, dtype=dt, device="cuda")
        y = torch.empty_like(x)
        f = q.lib().qmb_hv_matrix_free if mf else q.lib().qmb_hv
        args = (h.h, prec, A.C.c_void_p(x.data_ptr()), A.C.c_void_p(y.data_ptr()), A.C.c_void_p(st.cuda_stream))
        q.check(f(*args))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(reps):
            q.check(f(*args))
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def solve(h, reps=3, **kw):
        # one warm-up solve (it also sizes the handle's kept Lanczos buffers),
        # then the median of `reps`
        h.lanczos(**kw)
        rs = [h.lanczos(**kw) for _ in range(reps)]
        ms = sorted(x.ms_total for x in rs)
        r = rs[-1]
        return {"ms": ms[len(ms) // 2], "ms_all": [round(v, 2) for v in ms], "products": int(r.n_hv),
                "hv_per_s": r.n_hv / (ms[len(ms) // 2] * 1e-3),
                "iters": [int(r.iters_low), int(r.iters)], "E0": r.E0, "residual": r.residual}

    peak, _ = load_peaks()
    out = {}
    L = 24
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L), 1.0, 0.5))
    f64 = solve(h, mode=A.MODE_FP64, tol=1e-12)
    mix = solve(h, mode=A.MODE_MIXED, tol=1e-12)
    out["L24_xxz_d0.5_k0_even"] = {"rows": int(h.info.n_rows), "fp64": f64, "mixed": mix,
                                   "rel_dE0": abs(mix["E0"] - f64["E0"]) / abs(f64["E0"]),
                                   "hv_us_fp64": 1e3 * t_hv(h, A.PREC_FP64, False, 50),
                                   "hv_us_fp32": 1e3 * t_hv(h, A.PREC_FP32, False, 50)}
    h.close()
    s.close()
    L = 32
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    J = [1.0] * L + [0.5] * L
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), J, J))
    i = h.info
    ms64, ms32 = t_hv(h, A.PREC_FP64, False, 10), t_hv(h, A.PREC_FP32, False, 10)
    mf32 = t_hv(h, A.PREC_FP32, True, 3)
    f64 = solve(h, mode=A.MODE_FP64, tol=1e-12, max_iter=300)
    mix0 = solve(h, mode=A.MODE_MIXED, tol=1e-12, max_iter=300)
    f64r = solve(h, mode=A.MODE_FP64, tol=1e-12, max_iter=300, reorth=2)
    mix = solve(h, mode=A.MODE_MIXED, tol=1e-12, max_iter=300, reorth=2)
    mfr = solve(h, reps=1, mode=A.MODE_MIXED, tol=1e-12, max_iter=300, reorth=2, hv=A.HV_MATRIX_FREE)
    out["L32_j1j2_k0_even"] = {
        "rows": int(i.n_rows), "nnz": int(i.nnz_offdiag),
        "hv_ms_fp64": ms64, "hv_fp64_coded": int(i.coded_fp64),
        "hv_gbs_fp64": fp64_product_bytes(i)[0] / (ms64 * 1e-3) / 1e9,
        "hv_frac_fp64": fp64_product_bytes(i)[0] / (ms64 * 1e-3) / 1e9 / peak,
        "hv_frac_fp64_ell_convention": i.bytes_fp64 / (ms64 * 1e-3) / 1e9 / peak,
        "hv_ms_fp32": ms32, "hv_fp32_coded": int(i.coded),
        "hv_gbs_fp32": fp32_product_bytes(i)[0] / (ms32 * 1e-3) / 1e9,
        "hv_frac_fp32": fp32_product_bytes(i)[0] / (ms32 * 1e-3) / 1e9 / peak,
        "hv_frac_fp32_ell_convention": i.bytes_fp32 / (ms32 * 1e-3) / 1e9 / peak,
        "hv_ms_matrix_free_fp32": mf32,
        "fp64": f64, "mixed": mix0, "rel_dE0_no_reorth": abs(mix0["E0"] - f64["E0"]) / abs(f64["E0"]),
        "solve_speedup_mixed_over_fp64_no_reorth": f64["ms"] / mix0["ms"],
        "fp64_reorth2": f64r, "mixed_reorth2": mix, "rel_dE0": abs(mix["E0"] - f64r["E0"]) / abs(f64r["E0"]),
        "solve_speedup_mixed_over_fp64_reorth2": f64r["ms"] / mix["ms"],
        "mixed_reorth2_matrix_free": {"ms": mfr["ms"], "products": mfr["products"],
                                      "rel_dE0": abs(mfr["E0"] - f64["E0"]) / abs(f64["E0"])}}
    h.close()
    s.close()
    N = 6
    perm, ch = q.translation_group(N, N)
    t0 = time.perf_counter()
    s = q.Sector(N * N, N * N // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    t_sec = time.perf_counter() - t0
    h = q.Hamiltonian(s, q.xxz_terms(q.square_bonds(N, N), 1.0, 1.0), prec=A.PREC_FP32 | A.PREC_FP64)
    t_ham = time.perf_counter() - t0 - t_sec
    i = h.info
    ms32 = t_hv(h, A.PREC_FP32, False, 5)
    ms64 = t_hv(h, A.PREC_FP64, False, 3)
    mf32 = t_hv(h, A.PREC_FP32, True, 2)
    gathers = float(i.nnz_offdiag) * 32.0  # one 32-byte DRAM sector per gathered x element

    def once(**kw):
        r = h.lanczos(allow_unconverged=True, **kw)
        return {"ms": r.ms_total, "products": int(r.n_hv), "iters": [int(r.iters_low), int(r.iters)],
                "E0": r.E0, "E0_per_site": r.E0 / (N * N), "residual": r.residual,
                "converged": int(r.converged)}

    # the configuration as stated: 200 FP32 steps (FP64 reductions), then the
    # chosen mixed form (FP32 phase + FP64 restart) and a plain FP64 solve
    fp32_200 = once(mode=A.MODE_FP32, max_iter=200, tol=0.0)
    mixed = once(mode=A.MODE_MIXED, max_iter=200, tol=1e-12, refine_max_iter=200)
    fp64 = once(mode=A.MODE_FP64, max_iter=300, tol=1e-12)
    out["6x6_k00_even"] = {
        "rows": int(i.n_rows), "nnz": int(i.nnz_offdiag), "sector_build_s": t_sec, "ham_build_s": t_ham,
        "hv_ms_fp32": ms32, "hv_fp32_coded": int(i.coded),
        "hv_gbs_fp32": fp32_product_bytes(i)[0] / (ms32 * 1e-3) / 1e9,
        "hv_frac_fp32": fp32_product_bytes(i)[0] / (ms32 * 1e-3) / 1e9 / peak,
        "hv_frac_fp32_ell_convention": i.bytes_fp32 / (ms32 * 1e-3) / 1e9 / peak,
        "hv_sector_gbs_fp32": gathers / (ms32 * 1e-3) / 1e9,
        "hv_fp32_column_blocked": int(i.coded), "column_block_codes": int(i.n_codes),
        "hv_ms_fp64": ms64, "hv_gbs_fp64": i.bytes_fp64 / (ms64 * 1e-3) / 1e9,
        "hv_ms_matrix_free_fp32": mf32,
        "fp32_200_steps": fp32_200, "mixed": mixed, "fp64": fp64,
        "rel_dE0_mixed_vs_fp64": abs(mixed["E0"] - fp64["E0"]) / abs(fp64["E0"]),
        "rel_dE0_fp32_200_vs_fp64": abs(fp32_200["E0"] - fp64["E0"]) / abs(fp64["E0"]),
        "E0_per_site_published": -0.678872,
        "solve_speedup_mixed_over_fp64": fp64["ms"] / mixed["ms"]}
    h.close()
    s.close()
    # the L=16 chain without symmetry: FP64, 150 steps, full reorthogonalisation
    L = 16
    s = q.Sector(L, L // 2, np.arange(L, dtype=np.uint32)[None]).set_irrep([1.0])
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L), 1.0, 1.0))
    h.lanczos(mode=A.MODE_FP64, max_iter=150, tol=0.0, reorth=2, seed=SEED)
    r = h.lanczos(mode=A.MODE_FP64, max_iter=150, tol=0.0, reorth=2, seed=SEED)
    out["L16_nosym_fp64_150"] = {"rows": int(h.info.n_rows), "ms": r.ms_total, "products": int(r.n_hv),
                                 "E0": r.E0, "residual": r.residual}
    h.close()
    s.close()
    return out


def cpu_solve_baselines():
    """The oracle's FP64 Lanczos (lanczos_fp64: scipy CSR products, full
    reorthogonalisation through numpy/BLAS on all host threads) on the oracle's
    own matrices of two single-sector configurations, timed on the host:
      L=16 chain without symmetry (12,870 rows), 150 steps;
      L=24 XXZ chain, Delta=0.5, k=0, spin-inversion even (56,450 rows), 120
      steps (about twice what the GPU's FP64 solve needs).
    The matrix build is not timed.  Returns {name: {s, steps, E0, ...}}."""
    import oracle as O
    threads = os.cpu_count() or 1
    out = {}
    cases = []
    g = O.trivial_group(16)
    sec = O.build_sector(g, 8)
    t = O.xxz_terms(O.chain_bonds(16), 1.0, 1.0)
    cases.append(("L16_nosym_fp64_150", sec, t, 0, 150))
    g = O.translation_group(24, flip=True)
    sec = O.build_sector(g, 12)
    t = O.xxz_terms(O.chain_bonds(24), 1.0, 0.5)
    cases.append(("L24_xxz_d0.5_k0_even", sec, t, 0, 120))
    for name, sec, t, a, steps in cases:
        rows = O.active_rows(sec, a)
        rc, ind, val, tr = O.ell_terms(sec, t, a, 2 * t.H + 1)
        M = O.ell_to_csr(ind, val, tr, rows).real.tocsr()
        v0 = O.start_vector(SEED, M.shape[0])
        t0 = time.perf_counter()
        e0, al, be = O.lanczos_fp64(lambda v: M @ v, v0, steps, reorth=True)
        dt = time.perf_counter() - t0
        out[name] = {"rows": int(M.shape[0]), "steps": int(len(al)), "s": dt, "E0": e0,
                     "cores": threads, "kind": "port",
                     "sample": "oracle FP64 Lanczos with full reorthogonalisation (scipy CSR product on one "
                               "thread, numpy/BLAS reorthogonalisation on all threads)"}
    return out


def run_batched(args, torch, q, rank, world):
    A = q._capi
    # the single-sector configurations first, while the device memory is free
    # (the 6x6 matrix needs ~100 GB while it is built)
    configs = None if args.no_compare else single_sector_configs(torch, q)
    torch.cuda.empty_cache()
    L, n_sets = 20, 256
    J, D = couplings(n_sets, rank)
    secs, b = build_batched(q, L, n_sets)
    info = b.info
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device="cuda")
    opts = dict(mode=A.MODE_MIXED, max_iter=300, tol=1e-12, check_every=10, refine_max_iter=300,
                seed=SEED)

    def solve(mode):
        o = dict(opts, mode=mode)
        return b.solve(J, J * D, **o)

    dev_ms, hv_count, launches = [], [], 0
    # the clock sampler starts before the warm-up steps, so its start-up is
    # over by the first timed step
    with Clocks(torch.cuda.current_device()) as clk:
        for _ in range(args.warmup):
            solve(A.MODE_MIXED)
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush_l2(torch, flush)
            torch.cuda.synchronize()
            E_mix, r = solve(A.MODE_MIXED)
            dev_ms.append(r.ms_total)
            hv_count.append(r.n_products)
            launches += int(r.n_launches)
    clocks = clk.summary()
    # FP64 reference solve of the same problems, |dE0| of the mixed result
    # (after one warm-up FP64 solve, which sizes the FP64 workspace)
    if args.no_compare:
        E64, r64 = E_mix, r
    else:
        solve(A.MODE_FP64)
        flush_l2(torch, flush)
        torch.cuda.synchronize()
        E64, r64 = solve(A.MODE_FP64)
    rel = np.abs(E_mix - E64) / np.maximum(np.abs(E64), 1e-300)
    # per-kernel H*v times
    hv32_ms = time_batch_hv(torch, q, b, A.PREC_FP32)
    hv64_ms = time_batch_hv(torch, q, b, A.PREC_FP64)
    gather = gather_bound(q, b, hv32_ms)
    k1_32_ms, k1_32_bytes = time_k1(q, b, A.PREC_FP32)
    k1_64_ms, k1_64_bytes = time_k1(q, b, A.PREC_FP64)
    units = n_sets * L  # sector problems
    ms = float(np.mean(dev_ms))
    value = float(np.mean(hv_count)) / (ms * 1e-3)
    # end-to-end through the C ABI, per step: the step's couplings copied in
    # from pinned host memory, the solve, the energies copied out (one
    # qmb_batch_solve call on the batch built above, as a caller that solves
    # many coupling sets over the same sectors does)
    Jp = torch.from_numpy(np.ascontiguousarray(J)).pin_memory().numpy()
    JDp = torch.from_numpy(np.ascontiguousarray(J * D)).pin_memory().numpy()
    # one untimed solve first: the kernel timings above allocated and freed
    # their own scratch vectors in between
    b.solve(Jp, JDp, **opts)
    e2e_t = []
    for _ in range(args.steps):
        flush_l2(torch, flush)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E2, r2 = b.solve(Jp, JDp, **opts)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_t))
    # the same with the sectors and the batch built from scratch every step
    # (the batch above is released first, as a caller that rebuilds does:
    # otherwise its Krylov ring holds the memory the new batch sizes its own
    # ring from)
    info = b.info
    b.close()
    setup_t, build_t = [], []
    for _ in range(0 if args.no_compare else max(1, min(3, args.steps))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2, b2 = build_batched(q, L, n_sets)
        tb = time.perf_counter()
        E2, r2 = b2.solve(J, J * D, **opts)
        t1 = time.perf_counter()
        setup_t.append(t1 - t0)
        build_t.append(tb - t0)
        b2.close()
        for s in s2:
            s.close()
    e2e_setup = {"value": float(np.mean(hv_count)) / float(np.mean(setup_t)), "unit": "Hv/s",
                 "s_per_step": float(np.mean(setup_t)),
                 "s_steps": [round(v, 4) for v in setup_t],
                 "s_build_sectors_and_batch": [round(v, 4) for v in build_t]} if setup_t else None
    single = None if args.no_compare else single_sector_hv(torch, q)
    obs = None if args.no_compare else observables(torch, q)
    files = None if args.no_compare else table_files(torch, q)
    out = batched_config(world, L, n_sets)
    # the batch's own counts (equal to the closed form above)
    out["rows_total"], out["elements_per_hv"] = int(info.rows_total), int(info.elems_total)
    extra = {
        "sectors_per_s": units / (ms * 1e-3),
        "fp64_sectors_per_s": units / (r64.ms_total * 1e-3),
        "hv_products_per_solve": float(np.mean(hv_count)),
        "fp64_solve_ms": r64.ms_total, "fp64_hv_per_s": r64.n_products / (r64.ms_total * 1e-3),
        "hv_kernel_ms_fp32": hv32_ms, "hv_kernel_ms_fp64": hv64_ms,
        "hv_kernel_gbs_fp32": info.bytes_hv_fp32 / (hv32_ms * 1e-3) / 1e9,
        "hv_kernel_gbs_fp64": info.bytes_hv_fp64 / (hv64_ms * 1e-3) / 1e9,
        "hv_ratio_fp32_over_fp64": hv64_ms / hv32_ms,
        "k1_fp32": {"ms": k1_32_ms, "bytes": k1_32_bytes, "gbs": k1_32_bytes / (k1_32_ms * 1e-3) / 1e9},
        "k1_fp64": {"ms": k1_64_ms, "bytes": k1_64_bytes, "gbs": k1_64_bytes / (k1_64_ms * 1e-3) / 1e9},
        "gather_bound": gather,
        "max_rel_dE0_mixed_vs_fp64": float(rel.max()),
        "hv_tuner": {"timed": "each variant's K1 (Lanczos-step form) at step 1, minimum of 5 rounds",
                     "variant_fp32": int(info.variant_fp32), "variant_fp64": int(info.variant_fp64),
                     "ms_fp32": [round(v, 4) for v in info.tune_ms_fp32],
                     "ms_fp64": [round(v, 4) for v in info.tune_ms_fp64],
                     "variants": "k_bhv (slices a thread, unroll, min blocks/SM, hoisted row loads with "
                                 "per-set constants in shared memory): 0 (1,4,4,no) 1 (1,4,4,yes) "
                                 "2 (1,8,2,no) 3 (2,4,2,yes) 4 (2,2,3,yes) 5 (2,2,4,yes) "
                                 "6 (4,2,2,yes) 7 (4,1,2,yes)"},
        "e2e_steps_ms": [round(v * 1e3, 2) for v in e2e_t],
        "e2e_with_setup": e2e_setup,
        "single_sector_hv": single,
        "observables": obs,
        "table_files": files,
        "single_sector_configs": configs,
        "ms_steps": [round(float(v), 2) for v in dev_ms],
        "iters_mixed": [int(r.iters_low), int(r.iters)], "iters_fp64": int(r64.iters),
        "E0_min": float(E_mix.min()),
    }
    return dict(ms=ms, value=value, units_per_step=float(np.mean(hv_count)), out=out,
                extra=extra, clocks=clocks, e2e_s=e2e_s,
                e2e_value=float(np.mean(hv_count)) / e2e_s,
                h2d=2 * n_sets * 8, d2h=n_sets * L * 8, roof_bytes=k1_32_bytes, roof_ms=k1_32_ms,
                launches=launches,
                kernel="k_bhv in the Lanczos step form (K1: y = H w/beta - beta v_{j-1}, v_j stored, alpha "
                       "summed), FP32, one launch per step over all 20 sectors x 256 sets (the real momenta "
                       "k=0, 10 are solved in the complex kind); bytes: the product's plus v_{j-1} read and "
                       "v_j written",
                dtype="f32+f64")


def reference_tables(L=20, n_sets_sample=2):
    """Reference-layout FP32 ELLs of the batched workload (the first
    `n_sets_sample` coupling sets x all L momenta), built by the reference's
    own kernels (oracle/_ref, run on the host) from the oracle's group and
    term tables.  Nothing here loads the product library.  Returns a list of
    (ind, val, track, rows, W, k, set)."""
    import oracle as O
    R = O.ref()
    g = O.translation_group(L)
    perm = np.ascontiguousarray(g.perm, np.uint32)
    k = L // 2
    N = O.binom(L, k)
    G = L
    reps = np.zeros(N, np.uint32)
    srs = np.zeros(N * G, np.uint32)
    norms = np.zeros(N * G, np.float32)
    oi = np.zeros(2 * N, np.uint32)
    chf = np.ascontiguousarray(g.chars.astype(np.complex64)).view(np.float32).ravel()
    Rn = R.ref_build_srs_complex(L, k, G, perm, G, chf, reps, N, srs, norms, oi)
    J, D = couplings(n_sets_sample)
    tabs = []
    bonds = O.chain_bonds(L)
    W = 2 * L + 1
    for i in range(n_sets_sample):
        t = O.xxz_terms(bonds, J[i], J[i] * D[i])
        codes = np.ascontiguousarray(t.codes, np.int32)
        sites = np.ascontiguousarray(t.sites, np.int32)
        n_ops = np.ascontiguousarray(t.n_ops, np.int32)
        sc = np.ascontiguousarray(t.scalar.astype(np.complex64)).view(np.float32).ravel()
        for a in range(L):
            ind = np.zeros(Rn * W, np.uint32)
            val = np.zeros(2 * Rn * W, np.float32)
            tr = np.zeros(Rn, np.int16)
            R.ref_ham_terms_complex(L, k, G, Rn, srs, oi, G, chf, a, norms, 1e-5, t.H, t.n_col,
                                    n_ops, codes, sites, sc, W, ind, val, tr)
            tabs.append((ind, val, tr, Rn, W, a, i))
    return tabs


class ReferenceSweep:
    """One "step" of the reference's CPU H*v on the batched workload: its
    only CPU H*v, SparseMatDenseVec_prod_EEL_host (utils.cu:649-670, FP32),
    once over every sampled sector matrix, row blocks on `threads` host
    threads.  That function is float-only, so complex sectors (k != 0, L/2)
    are timed on the real parts of their values: the same index and vector
    traffic as the complex product, half of its arithmetic."""

    def __init__(self, threads=None, L=20, n_sets_sample=2):
        import ctypes as C
        import oracle as O
        self.R = O.ref()
        self.threads = threads or os.cpu_count() or 1
        tabs = reference_tables(L, n_sets_sample)
        self.n = len(tabs)
        self.rows = int(sum(t[3] for t in tabs))
        self.desc = (f"{self.n} sector matrices ({n_sets_sample} coupling sets x {L} momenta) of the "
                     f"L={L} batch, {self.rows} rows, one FP32 SparseMatDenseVec_prod_EEL_host per matrix "
                     f"a step on {self.threads} threads; complex sectors on their real parts")
        self._keep = []
        ptrs = {k: [] for k in ("ind", "val", "tr", "x", "y")}
        for j, (ind, val, tr, n, W, a, i) in enumerate(tabs):
            vr = np.ascontiguousarray(val.reshape(-1, 2)[:, 0])
            x = np.random.default_rng(j).standard_normal(n).astype(np.float32)
            y = np.zeros(n, np.float32)
            self._keep += [ind, vr, tr, x, y]
            for key, arr in zip(("ind", "val", "tr", "x", "y"), (ind, vr, tr, x, y)):
                ptrs[key].append(arr.ctypes.data)
        self._arr = {key: (C.c_void_p * self.n)(*v) for key, v in ptrs.items()}
        self.nobv = np.array([t[3] for t in tabs], np.int32)
        self.W = np.array([t[4] for t in tabs], np.int32)

    def step(self):
        a = self._arr
        self.R.ref_spmv_host_sweep(self.n, a["ind"], a["val"], a["tr"], a["x"], a["y"], self.nobv,
                                   self.W, self.threads)

    def run(self, steps, warmup):
        """Seconds of each of `steps` timed steps after `warmup` untimed ones."""
        for _ in range(warmup):
            self.step()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            self.step()
            ts.append(time.perf_counter() - t0)
        return ts


def cpu_reference_hv(seconds=10.0, threads=None):
    """The reference's CPU H*v (ReferenceSweep) repeated for about `seconds`.
    Returns (Hv/s, threads, sample description)."""
    sw = ReferenceSweep(threads)
    sw.run(0, 1)
    count, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        sw.step()
        count += sw.n
    dt = time.perf_counter() - t0
    return count / dt, sw.threads, f"{sw.desc}; {count} H*v in {dt:.1f} s"


def reference_arm(args):
    """bench.py --impl reference: the reference's own CPU H*v (ReferenceSweep)
    on the batched workload, `args.warmup` untimed and `args.steps` timed
    steps.  Returns the JSON line."""
    sw = ReferenceSweep()
    ts = sw.run(args.steps, args.warmup)
    s = float(np.mean(ts))
    v = sw.n / s
    return {"metric": METRIC, "value": v, "unit": "Hv/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * s,
            "ms_steps": [round(1e3 * t, 3) for t in ts],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": batched_config(args.gpus),
            "cpu_baseline": {"value": v, "unit": "Hv/s", "cores": sw.threads, "kind": "reference",
                             "sample": sw.desc},
            "e2e": {"value": v, "unit": "Hv/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def aggregate_ranks(torch, dist, ms, e2e_s, units, device):
    """Whole-job figures of a weak-scaling run: every rank solves its own
    coupling sets, the step time is the maximum over ranks and the work is
    the sum over ranks.  Returns (max ms, max end-to-end s, total units)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return ms, e2e_s, units
    t = torch.tensor([ms, e2e_s], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor([units], device=device, dtype=torch.float64)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(u[0])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="batched", choices=["batched"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--hv-only", action="store_true",
                    help="time only the batched H*v kernels (small device footprint, for profiling)")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the FP64 comparison solve and the end-to-end repeat")
    ap.add_argument("--profile-stored", choices=["l28", "l32", "l32-fp64", "6x6"], default=None,
                    help="two stored FP32 products (k_hv<SellOp<float>>) on the L=28 J1-J2 k=0 even "
                         "sector or the 6x6 k=(0,0) even sector, then exit (the launches the stored-product "
                         "DRAM traffic summary profiles)")
    ap.add_argument("--profile-k1", action="store_true",
                    help="build the L=20 batch and time 5 FP32 Lanczos-step products (K1), then exit "
                         "(the launches the K1 ncu summary profiles)")
    ap.add_argument("--profile-matrix-free", nargs="?", const="l32", choices=["l32", "6x6"], default=None,
                    help="matrix-free FP32 products on the L=32 J1-J2 k=0 even sector (default) or the 6x6 "
                         "k=(0,0) even sector, then exit (the launches the matrix-free ncu summaries profile)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(reference_arm(args)))
        return 0

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import qmbcuda_b200 as q

    if args.profile_stored:
        A = q._capi
        if args.profile_stored == "6x6":
            N = 6
            perm, ch = q.translation_group(N, N)
            s = q.Sector(N * N, N * N // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
            terms = q.xxz_terms(q.square_bonds(N, N), 1.0, 1.0)
        else:
            L = 28 if args.profile_stored == "l28" else 32
            perm, ch = q.translation_group(L)
            s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
            J = [1.0] * L + [0.5] * L
            terms = q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), J, J)
        f64 = args.profile_stored == "l32-fp64"
        prec = A.PREC_FP64 if f64 else A.PREC_FP32
        h = q.Hamiltonian(s, terms, prec=prec)
        x = torch.randn(int(h.info.n_rows), dtype=torch.float64 if f64 else torch.float32, device="cuda")
        y = torch.empty_like(x)
        for _ in range(2):
            q.check(q.lib().qmb_hv(h.h, prec, A.C.c_void_p(x.data_ptr()), A.C.c_void_p(y.data_ptr()), None))
        torch.cuda.synchronize()
        i = h.info
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            q.check(q.lib().qmb_hv(h.h, prec, A.C.c_void_p(x.data_ptr()), A.C.c_void_p(y.data_ptr()), None))
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 3
        byt, ell = fp64_product_bytes(i) if f64 else fp32_product_bytes(i)
        print(json.dumps({"profile": f"stored {'FP64' if f64 else 'FP32'} product, {args.profile_stored}",
                          "rows": int(i.n_rows), "nnz": int(i.nnz_offdiag), "bytes": byt, "bytes_ell_convention": ell,
                          "coded": int(i.coded_fp64 if f64 else i.coded), "ms": ms,
                          "frac": byt / (ms * 1e-3) / 1e9 / load_peaks()[0]}))
        return 0

    if args.profile_k1:
        secs, b = build_batched(q)
        ms, byt = time_k1(q, b, q._capi.PREC_FP32, reps=5)
        print(json.dumps({"profile": "K1 (Lanczos-step k_bhv), FP32, L=20 batch, 256 sets", "ms": ms, "bytes": byt,
                          "frac": byt / (ms * 1e-3) / 1e9 / load_peaks()[0]}))
        return 0

    if args.profile_matrix_free:
        A = q._capi
        if args.profile_matrix_free == "6x6":
            N = 6
            perm, ch = q.translation_group(N, N)
            s = q.Sector(N * N, N * N // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
            terms = q.xxz_terms(q.square_bonds(N, N), 1.0, 1.0)
            name = "6x6 square k=(0,0) even"
        else:
            L = 32
            perm, ch = q.translation_group(L)
            s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
            J = [1.0] * L + [0.5] * L
            terms = q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), J, J)
            name = "L=32 J1-J2 k=0 even"
        h = q.Hamiltonian(s, terms, prec=A.PREC_FP32)
        x = torch.randn(int(h.info.n_rows), dtype=torch.float32, device="cuda")
        y = torch.empty_like(x)
        args_mf = (h.h, A.PREC_FP32, A.C.c_void_p(x.data_ptr()), A.C.c_void_p(y.data_ptr()), None)
        for _ in range(2):
            q.check(q.lib().qmb_hv_matrix_free(*args_mf))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            q.check(q.lib().qmb_hv_matrix_free(*args_mf))
        e1.record()
        e1.synchronize()
        print(json.dumps({"profile": f"matrix-free FP32 product, {name}", "rows": int(h.info.n_rows),
                          "nnz": int(h.info.nnz_offdiag), "ms": e0.elapsed_time(e1) / 3}))
        return 0

    if args.hv_only:
        secs, b = build_batched(q)
        for prec in (q._capi.PREC_FP32, q._capi.PREC_FP64):
            ms = time_batch_hv(torch, q, b, prec, reps=max(1, args.steps))
            info = b.info
            byt = info.bytes_hv_fp32 if prec == q._capi.PREC_FP32 else info.bytes_hv_fp64
            print(json.dumps({"kernel": "k_bhv", "prec": "fp32" if prec == q._capi.PREC_FP32 else "fp64",
                              "ms": ms, "gbs": byt / (ms * 1e-3) / 1e9,
                              "tune_ms": list(info.tune_ms_fp32 if prec == q._capi.PREC_FP32 else info.tune_ms_fp64)}))
            if prec == q._capi.PREC_FP32:
                print(json.dumps({"gather_bound": gather_bound(q, b, ms)}))
        return 0
    if dist:
        dist.barrier()
    res = run_batched(args, torch, q, rank, world)
    ms, e2e_s, total_units = aggregate_ranks(torch, dist, res["ms"], res["e2e_s"], res["units_per_step"], "cuda")
    value = total_units / (ms * 1e-3)
    peak, peak_kind = load_peaks()
    achieved = res["roof_bytes"] / (res["roof_ms"] * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "batched_k1_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get("traffic_bytes_per_launch")
    line = {
        "metric": METRIC, "value": value, "unit": "Hv/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": res["dtype"], "data": "synthetic", "config": res["out"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": res["kernel"],
                     "peak_source": peak_kind},
        "e2e": {"value": total_units / e2e_s, "unit": "Hv/s",
                "h2d_bytes_per_step": res["h2d"], "d2h_bytes_per_step": res["d2h"]},
        "clocks": res["clocks"], "gpu_launches": res["launches"],
    }
    line.update(res["extra"])
    if rank == 0 and world == 1 and not args.no_compare:
        try:
            line["cpu_solve_baseline"] = cpu_solve_baselines()
        except Exception as e:  # scipy or the oracle build absent
            line["cpu_solve_baseline"] = {"unavailable": str(e)}
    if rank == 0 and world == 1:
        try:
            v, thr, sample = cpu_reference_hv(args.cpu_seconds)
            line["cpu_baseline"] = {"value": v, "unit": "Hv/s", "cores": thr, "kind": "reference",
                                    "sample": sample}
        except Exception as e:  # reference build absent
            line["cpu_baseline"] = {"value": None, "unit": "Hv/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
