"""Locally divergence-free projector (LDF.f90) on the CPU.

* The oracle's projector (one-sided Jacobi SVD) matches the reference's construction with LAPACK
  DGESDD (LDF.f90:182-193; here scipy's bundled dgesdd) applied by the formula of LDF.f90:247-249.
* The identities the reference lists for it (LDF.f90:83-87): the result is divergence-free, the map
  is idempotent and self-adjoint in the modal mass inner product.
* The product library's dense nodal operator (symmetric-eigen route) equals the oracle's modal
  projector composed with the nodal transforms and the Piola scalings of DG_solver.f90:237-264.
"""
import numpy as np
import pytest
import scipy.linalg


def _gesdd_projector(p, ora):
    """LDF.f90:114-250 with LAPACK dgesdd, as an explicit (2n^2 x 2n^2) matrix on modal coefs"""
    lt = ora.legendre_tables(p)
    m, minv, D = lt["m"], lt["minv"], lt["D"]
    n = p + 1
    sq = np.sqrt(m)
    G = sq[:, None] * D / sq[None, :]
    U, L, _ = scipy.linalg.svd(G, lapack_driver="gesdd")
    den = L[:, None] ** 2 + L[None, :] ** 2
    den[-1, -1] = 1.0  # the zero singular pair: Ldagger(px+1,py+1) = 0 (LDF.f90:206-214)
    Ld = 1.0 / den
    Ld[-1, -1] = 0.0
    sqrtm2d = np.sqrt(np.outer(m, m))
    invm2d = np.outer(minv, minv)

    def apply(uu):
        u1, u2 = uu[:, :, 0], uu[:, :, 1]
        udiv = sqrtm2d * (U @ (Ld * (U.T @ (sqrtm2d * (D @ u1 + u2 @ D.T)) @ U)) @ U.T)
        return np.stack([u1 - invm2d * (D.T @ udiv), u2 - invm2d * (udiv @ D)], axis=2)

    P = np.zeros((2 * n * n, 2 * n * n))
    for c in range(2 * n * n):
        e = np.zeros(2 * n * n)
        e[c] = 1.0
        P[:, c] = apply(e.reshape((n, n, 2), order="F")).reshape(-1, order="F")
    return P


def _oracle_projector(p, ora):
    n = p + 1
    P = np.zeros((2 * n * n, 2 * n * n))
    for c in range(2 * n * n):
        e = np.zeros(2 * n * n)
        e[c] = 1.0
        P[:, c] = ora.ldf_apply(p, p, e).reshape(-1, order="F")
    return P


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6])
def test_oracle_projector_matches_dgesdd(ora, p):
    np.testing.assert_allclose(_oracle_projector(p, ora), _gesdd_projector(p, ora), rtol=0, atol=2e-13)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_projector_identities(ora, p):
    n = p + 1
    P = _oracle_projector(p, ora)
    assert np.abs(P @ P - P).max() < 1e-12  # idempotent (LDF.f90:86)
    m = ora.legendre_tables(p)["m"]
    M = np.kron(np.ones(2), np.outer(m, m).reshape(-1, order="F"))  # diag(M, M)
    MP = M[:, None] * P
    assert np.abs(MP - MP.T).max() < 1e-12  # self-adjoint in the mass inner product (LDF.f90:87)
    rng = np.random.default_rng(p)
    for _ in range(5):
        uu = rng.standard_normal((n, n, 2))
        out = ora.ldf_apply(p, p, uu)
        assert np.abs(ora.ldf_div(p, p, out)).max() < 1e-12  # divergence-free (LDF.f90:83-84)


def _nodal_from_oracle(p, hx, hy, ora):
    t = ora.gll_tables(p)
    n = p + 1
    Pnm, Pmn = t["Pnm"], t["Pmn"]
    N2 = 2 * n * n
    A = np.zeros((N2, N2))
    for c in range(N2):
        d = np.zeros(N2)
        d[c] = 1.0
        bx = d[: n * n].reshape((n, n), order="F") * (0.5 * hy)
        by = d[n * n:].reshape((n, n), order="F") * (0.5 * hx)
        uu = np.stack([Pnm @ bx @ Pnm.T, Pnm @ by @ Pnm.T], axis=2)
        uu = ora.ldf_apply(p, p, uu)
        ox = (2.0 / hy) * (Pmn @ uu[:, :, 0] @ Pmn.T)
        oy = (2.0 / hx) * (Pmn @ uu[:, :, 1] @ Pmn.T)
        A[:, c] = np.concatenate([ox.reshape(-1, order="F"), oy.reshape(-1, order="F")])
    return A


@pytest.mark.parametrize("p,hx,hy", [(1, 0.1, 0.1), (2, 2 * np.pi / 64, 2 * np.pi / 64),
                                     (3, 20 / 512, 20 / 512), (2, 0.05, 0.2), (3, 1.0, 0.3)])
def test_library_nodal_operator(ora, pkg, p, hx, hy):
    A_lib = pkg.ldf_operator(p, hx, hy)
    A_ref = _nodal_from_oracle(p, hx, hy, ora)
    np.testing.assert_allclose(A_lib, A_ref, rtol=0, atol=5e-13 * max(1.0, np.abs(A_ref).max()))
    assert np.abs(A_lib @ A_lib - A_lib).max() < 1e-11 * max(1.0, np.abs(A_lib).max())
