"""GLL / Legendre tables against the reference's own known answers (CPU).

The reference tabulates closed forms (gauss.f90:134-331) and checks them at start-up with
gauss_lobatto_test / test_lobatto_mat / test_legendre_mat (gauss.f90:73-132,365-388,477-502,
called from main.f90:25-50).  Both the oracle's tables and the product library's tables (which the
kernels use) are computed from definitions; these tests pin them to the reference's closed forms and
self-checks.
"""
import math

import numpy as np
import pytest

S5 = math.sqrt(5.0)

# closed forms written in the reference (gauss.f90:172-217), expanded by its symmetry rules
KNOWN = {
    1: dict(x=[-1.0, 1.0], w=[1.0, 1.0],
            M=[[2 / 3, 1 / 3], [1 / 3, 2 / 3]], Minv=[[2.0, -1.0], [-1.0, 2.0]],
            D=[[-0.5, 0.5], [-0.5, 0.5]], Pmn=[[1.0, -1.0], [1.0, 1.0]],
            Pnm=[[0.5, 0.5], [-0.5, 0.5]]),
    2: dict(x=[-1.0, 0.0, 1.0], w=[1 / 3, 4 / 3, 1 / 3],
            M=[[4 / 15, 2 / 15, -1 / 15], [2 / 15, 16 / 15, 2 / 15], [-1 / 15, 2 / 15, 4 / 15]],
            Minv=[[4.5, -0.75, 1.5], [-0.75, 1.125, -0.75], [1.5, -0.75, 4.5]],
            D=[[-1.5, 2.0, -0.5], [-0.5, 0.0, 0.5], [0.5, -2.0, 1.5]],
            Pmn=[[1.0, -1.0, 1.0], [1.0, 0.0, -0.5], [1.0, 1.0, 1.0]],
            Pnm=[[1 / 6, 2 / 3, 1 / 6], [-0.5, 0.0, 0.5], [1 / 3, -2 / 3, 1 / 3]]),
    3: dict(x=[-1.0, -1 / S5, 1 / S5, 1.0], w=[1 / 6, 5 / 6, 5 / 6, 1 / 6],
            D=[[-3.0, 1.25 * (1 + S5), -1.25 * (-1 + S5), 0.5],
               [0.25 * (-1 - S5), 0.0, 0.5 * S5, -0.25 * (-1 + S5)],
               [0.25 * (-1 + S5), -0.5 * S5, 0.0, -0.25 * (-1 - S5)],
               [-0.5, 1.25 * (-1 + S5), -1.25 * (1 + S5), 3.0]],
            M=[[1 / 7, S5 / 42, -S5 / 42, 1 / 42], [S5 / 42, 5 / 7, 5 / 42, -S5 / 42],
               [-S5 / 42, 5 / 42, 5 / 7, S5 / 42], [1 / 42, -S5 / 42, S5 / 42, 1 / 7]]),
}


@pytest.fixture(scope="module", params=["oracle", "library"])
def tables(request, ora, pkg):
    if request.param == "oracle":
        return ora.gll_tables
    import ctypes as C

    def lib_tables(p):
        n = p + 1
        x, w = np.zeros(n), np.zeros(n)
        mats = [np.zeros((n, n), order="F") for _ in range(5)]
        dp = C.POINTER(C.c_double)
        rc = pkg.capi.load().mhd_gpu_gll_tables(p, *(a.ctypes.data_as(dp) for a in [x, w, *mats]))
        assert rc == 0
        return dict(x=x, w=w, M=mats[0], Minv=mats[1], D=mats[2], Pmn=mats[3], Pnm=mats[4])
    return lib_tables


@pytest.mark.parametrize("p", [1, 2, 3])
def test_closed_forms(tables, p):
    t = tables(p)
    for key, val in KNOWN[p].items():
        np.testing.assert_allclose(t[key], np.array(val), rtol=0, atol=4e-15, err_msg=key)


def test_quadrature_exactness(tables):
    """gauss_lobatto_test (gauss.f90:73-105): n-point rule exact for x^q, q <= 2n-3"""
    err = 0.0
    for n in range(1, 8):
        t = tables(n - 1)
        for q in range(0, 2 * n - 2):
            exact = (1.0 - (-1.0) ** (q + 1)) / (q + 1)
            approx = np.sum(t["x"] ** q * t["w"])
            err += abs(exact - approx) / (abs(exact) + 1.0)
    assert err < 1e-13


@pytest.mark.parametrize("p", range(0, 7))
def test_lobatto_matrix_identities(tables, p):
    """test_lobatto_mat (gauss.f90:365-388): Pmn Pnm = I, M Minv = I, D^(p+1) = 0, SBP"""
    t = tables(p)
    n = p + 1
    I = np.eye(n)
    assert np.abs(t["Pmn"] @ t["Pnm"] - I).max() < 1e-13
    assert np.abs(t["M"] @ t["Minv"] - I).max() < 1e-12
    assert np.abs(np.linalg.matrix_power(t["D"], n)).max() < 1e-9
    sbp = t["M"] @ t["D"] + t["D"].T @ t["M"]
    sbp[-1, -1] -= 1.0
    sbp[0, 0] += 1.0
    if p == 0:
        sbp[0, 0] = 0.0
    assert np.abs(sbp).max() < 1e-13


@pytest.mark.parametrize("p", range(0, 7))
def test_legendre_matrix_identities(ora, p):
    """test_legendre_mat (gauss.f90:477-502): nilpotent modal D and SBP with the trace vectors"""
    t = ora.legendre_tables(p)
    n = p + 1
    D, m, tl, tr = t["D"], t["m"], t["tl"], t["tr"]
    assert np.abs(np.linalg.matrix_power(D, n)).max() == 0.0
    mat = m[:, None] * D + (D.T) * m[None, :] - (np.outer(tr, tr) - np.outer(tl, tl))
    assert np.abs(mat).max() < 1e-13


def test_library_matches_oracle_tables(ora, pkg):
    import ctypes as C
    dp = C.POINTER(C.c_double)
    for p in range(0, 7):
        n = p + 1
        a = ora.gll_tables(p)
        x, w = np.zeros(n), np.zeros(n)
        mats = [np.zeros((n, n), order="F") for _ in range(5)]
        pkg.capi.load().mhd_gpu_gll_tables(p, *(q.ctypes.data_as(dp) for q in [x, w, *mats]))
        for key, val in zip(["x", "w", "M", "Minv", "D", "Pmn", "Pnm"], [x, w, *mats]):
            np.testing.assert_array_equal(val, a[key], err_msg=f"p={p} {key}")
