"""The engine's reference-layout Lanczos against the reference's own GPU
Lanczos, LanczosEigVals_CUDA<T> (exact_diagonalization/lanczos.cu:128-317),
compiled unmodified for sm_100a into oracle/_ref/libqmb_ref_gpu.so
(oracle/Makefile, oracle/ref_gpu_harness.cu).

Both run NIter = 50 three-term Lanczos steps from the reference's cuRAND
start vector (seed 2212456, the reference's default) on the same
reference-layout ELL, exported by qmb_ham_export_ref; the reference in FP32
throughout (cuBLAS FP32 norms and dots, cuSOLVER FP32 syevd), the engine
with FP32 vectors and values and FP64 reductions and tridiagonal solve.  The
ground energies agree to FP32 level, 1e-5 relative (the floor the
reference's FP32 arithmetic sets), in a real and a complex momentum sector
of an L=12 and an L=20 chain.  The reference's allocations are padded (its
start-vector kernel writes one element past the end), and the test checks
that they were.
"""
import ctypes as C
import os

import numpy as np
import pytest

import qmbcuda_b200 as q

pytestmark = pytest.mark.gpu
A = q._capi
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_SO = os.path.join(ROOT, "oracle", "_ref", "libqmb_ref_gpu.so")
needs_ref_gpu = pytest.mark.skipif(not os.path.exists(_SO),
                                   reason="oracle/_ref/libqmb_ref_gpu.so not built (reference sources absent)")

_lib = None


def _ref():
    global _lib
    if _lib is None:
        L = C.CDLL(_SO)
        P = np.ctypeslib.ndpointer
        L.qmb_refgpu_lanczos.restype = C.c_int
        L.qmb_refgpu_lanczos.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_longlong,
                                         P(np.uint32, flags="C"), P(np.float32, flags="C"),
                                         P(np.int16, flags="C"), C.c_int, C.POINTER(C.c_float),
                                         P(np.float32, flags="C"), C.POINTER(C.c_float)]
        L.qmb_refgpu_padded_allocs.restype = C.c_longlong
        _lib = L
    return _lib


def _ell(L, a, Jz=1.0):
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm).set_irrep(ch[a])
    terms = q.xxz_terms(q.chain_bonds(L), 1.0, Jz)
    W = 2 * L + 1
    ind, val, tr = q.export_ref(s, terms, W)
    return s, ind, val, tr, W


@needs_ref_gpu
@pytest.mark.parametrize("L,a", [(12, 0), (12, 3), (20, 0), (20, 7)])
def test_engine_reference_lanczos_matches_the_reference_gpu_lanczos(L, a):
    import torch
    n_iter, seed = 50, 2212456
    s, ind, val, tr, W = _ell(L, a)
    R = ind.shape[0]
    cplx = a not in (0, L // 2)
    if cplx:
        vf = np.ascontiguousarray(val.astype(np.complex64).ravel()).view(np.float32)
    else:
        vf = np.ascontiguousarray(val.real.astype(np.float32).ravel())
    indf = np.ascontiguousarray(ind.ravel(), np.uint32)
    trf = np.ascontiguousarray(tr, np.int16)
    # the reference's own GPU Lanczos
    lib = _ref()
    before = lib.qmb_refgpu_padded_allocs()
    E_ref = C.c_float()
    res_ref = C.c_float()
    kry_ref = np.zeros(n_iter, np.float32)
    rc = lib.qmb_refgpu_lanczos(int(cplx), n_iter, R, W, seed, indf, vf, trf, 1, C.byref(E_ref), kry_ref,
                                C.byref(res_ref))
    assert rc == 0, rc
    assert lib.qmb_refgpu_padded_allocs() > before  # its allocations took the padded path
    # the engine's reference-layout Lanczos on the same tables
    dind = torch.tensor(indf.astype(np.int64)).to(torch.int32).cuda()
    dval = torch.tensor(vf).cuda()
    dtr = torch.tensor(trf).cuda()
    torch.cuda.synchronize()
    E = C.c_float()
    res = C.c_float()
    kry = np.zeros(n_iter, np.float32)
    q.check(q.lib().qmb_lanczos_ref_ell(C.byref(E), n_iter, R, W, seed, C.c_void_p(dind.data_ptr()),
                                        C.c_void_p(dval.data_ptr()), C.c_void_p(dtr.data_ptr()), int(cplx),
                                        A.ptr(kry), 1, C.byref(res)))
    assert abs(E.value - E_ref.value) <= 1e-5 * abs(E_ref.value), (E.value, E_ref.value)
    # both Ritz vectors are eigenvectors to FP32 accuracy (||H psi - E psi|| / nobv)
    assert res.value < 1e-4 and res_ref.value < 1e-4, (res.value, res_ref.value)
