"""The drop-in's symmetry operations as coordinate maps (host code, no GPU):
Tnm, Tnm_general, sigma_n_arb and GetElemProd of include/qmb/qmbcuda.hpp,
against the reference's rules (symmetries/SymmOperators.cu:21-137) restated
here in float32 numpy, and the element arrays SymmetryClass builds from them
(SymmetryClass::GetGroupElemArr with TranformGroupEls_ArmaToDev,
symmetries/SymmetryClass.cu:26-71 and utils/misc_funcs.cu:80-90: for an
element g mapping site q onto site g(q), the array holds arr[g(q)] = q).

Cases follow the reference's examples: Tnm_general_example,
Tnm_general_triangular_example and Tnm_general_square_example
(examples/examples.cu:549-662) with their lattices and shifts; the first
prints the old Tnm beside Tnm_general, which must agree."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "symm_check.cpp")
CUDA = "/usr/local/cuda"


@pytest.fixture(scope="module")
def maps(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("symm") / "symm_check")
    lib_dir = os.path.join(ROOT, "qmbcuda_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), SRC, "-o", exe, "-L", lib_dir, "-lqmb_b200",
           f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, check=True, timeout=60).stdout
    res = {}
    for line in out.splitlines():
        f = line.split()
        n = int(f[1])
        if f[0].endswith("_perm"):
            res[f[0]] = np.array([int(v) for v in f[2:]])
            assert len(res[f[0]]) == n
        else:
            v = np.array([float(x) for x in f[2:]], np.float32).reshape(n, 2)
            res[f[0]] = v
    return res


def _sites(N1, N2, A, x0=0.0, y0=0.0):
    """create_square / create_triangular (examples/examples.cu:200-238)."""
    A = np.asarray(A, np.float32)
    R = [(i * A[0, 0] + j * A[0, 1] + x0, i * A[1, 0] + j * A[1, 1] + y0) for i in range(N1) for j in range(N2)]
    return np.array(R, np.float32)


def _tnm(R, Nx, Ny, nx, ny):
    """Tnm (symmetries/SymmOperators.cu:46-60): shift, then fmod per axis."""
    R = R.astype(np.float32)
    return np.stack([np.fmod(R[:, 0] + np.float32(nx), np.float32(Nx)),
                     np.fmod(R[:, 1] + np.float32(ny), np.float32(Ny))], axis=1)


def _tnm_general(R, nx, ny, N1, N2, A):
    """Tnm_general (symmetries/SymmOperators.cu:62-126) in float32: shift by
    nx a1 + ny a2, coefficients in the basis from the Gram matrix
    [[1, a1.a2], [a1.a2, 1]], fmod by N1 / N2, a coefficient within 1e-3 of N
    set to 0, back to coordinates."""
    A = np.asarray(A, np.float32)
    a1 = A[:, 0]
    a2 = A[:, 1]
    w = np.float32(a1 @ a2)
    Winv = np.linalg.inv(np.array([[1, w], [w, 1]], np.float32)).astype(np.float32)
    out = []
    for x, y in R.astype(np.float32):
        r = np.array([x + nx * a1[0] + ny * a2[0], y + nx * a1[1] + ny * a2[1]], np.float32)
        c = Winv @ np.array([a1 @ r, a2 @ r], np.float32)
        c = np.array([np.fmod(c[0], np.float32(N1)), np.fmod(c[1], np.float32(N2))], np.float32)
        if abs(c[0] - N1) < 1e-3:
            c[0] = 0.0
        if abs(c[1] - N2) < 1e-3:
            c[1] = 0.0
        out.append(c[0] * a1 + c[1] * a2)
    return np.array(out, np.float32)


def _sigma(R, theta):
    """sigma_n_arb (symmetries/SymmOperators.cu:21-36): r - 2 n (n . r) with
    n the x unit vector rotated by theta degrees."""
    t = np.float32(theta * np.pi / 180.0)
    n = np.array([np.cos(t), np.sin(t)], np.float32)
    return (R - 2.0 * np.outer(R @ n, n)).astype(np.float32)


def _perm_of(R, TR, tol=1e-3):
    """Element array of the map q -> g(q) (TR[q] are the coordinates of g(q)):
    arr[g(q)] = q, with coordinates matched within 1e-3 as the reference does."""
    arr = -np.ones(len(R), np.int64)
    for q, t in enumerate(TR):
        d = np.abs(R - t).max(axis=1)
        m = np.nonzero(d < tol)[0]
        assert len(m) == 1
        arr[m[0]] = q
    assert (arr >= 0).all()
    return arr


SQ = [[1.0, 0.0], [0.0, 1.0]]
TRI = [[1.0, 0.5], [0.0, np.sqrt(3.0) / 2.0]]


@pytest.mark.parametrize("name,N1,N2,A,nx,ny", [
    ("tnm_general_square_4x6_11", 4, 6, SQ, 1, 1),
    ("tnm_general_triangular_4x6_11", 4, 6, TRI, 1, 1),
    ("tnm_general_triangular_4x6_32", 4, 6, TRI, 3, 2),
    ("tnm_general_square_6x4_14", 6, 4, SQ, 1, 4),
])
def test_tnm_general_matches_reference_rule(maps, name, N1, N2, A, nx, ny):
    R = _sites(N1, N2, A)
    want = _tnm_general(R, nx, ny, N1, N2, A)
    np.testing.assert_allclose(maps[name], want, atol=2e-5)
    p = maps[name + "_perm"]
    assert np.array_equal(p, _perm_of(R, want))
    assert sorted(p) == list(range(N1 * N2))  # a permutation of the sites


def test_tnm_and_tnm_general_agree_on_the_square_lattice(maps):
    """Tnm_general_example: the old square-lattice Tnm and Tnm_general."""
    R = _sites(4, 6, SQ)
    np.testing.assert_allclose(maps["tnm_square_4x6_11"], _tnm(R, 4, 6, 1, 1), atol=1e-6)
    np.testing.assert_allclose(maps["tnm_square_4x6_11"], maps["tnm_general_square_4x6_11"], atol=2e-5)
    assert np.array_equal(maps["tnm_square_4x6_11_perm"], maps["tnm_general_square_4x6_11_perm"])


@pytest.mark.parametrize("theta", [0, 45, 90, 135])
def test_reflections_match_reference_rule(maps, theta):
    R = _sites(4, 4, SQ, -1.5, -1.5)
    want = _sigma(R, theta)
    np.testing.assert_allclose(maps[f"sigma_{theta}"], want, atol=2e-5)
    p = maps[f"sigma_{theta}_perm"]
    assert np.array_equal(p, _perm_of(R, want))
    assert np.array_equal(p[p], np.arange(16))  # an involution


def test_element_products(maps):
    """GetElemProd(G2, G1) applies G2 first: two perpendicular reflections
    make the rotation by pi; the reflection x -> -x followed by C4 is the
    reflection across y = -x, whose normal is at 45 degrees."""
    R = _sites(4, 4, SQ, -1.5, -1.5)
    np.testing.assert_allclose(maps["prod_sigma_0_sigma_90"], -R, atol=2e-5)
    assert np.array_equal(maps["prod_sigma_0_sigma_90_perm"], _perm_of(R, -R))
    s0 = _sigma(R, 0)
    c4 = np.stack([-s0[:, 1], s0[:, 0]], axis=1)  # rotation by pi/2 about the origin
    np.testing.assert_allclose(maps["prod_sigma_0_c4"], c4, atol=2e-5)
    assert np.array_equal(maps["prod_sigma_0_c4_perm"], maps["sigma_45_perm"])
