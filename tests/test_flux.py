"""Two-point fluxes of the oracle (CPU): the properties the reference's derivations rely on.

ESPP_HLL_flux_x (DG_solver.f90:894-1071), ec_flux_x/y (DG_solver.f90:1570-1650) and
log_avg_divisor (DG_solver.f90:1652-1681).
"""
import math

import numpy as np
import pytest


def phys_flux_x(w, g):
    rho, mx, my, mz, bx, by, bz, e = w
    vx, vy, vz = mx / rho, my / rho, mz / rho
    pm = 0.5 * (bx * bx + by * by + bz * bz)
    p = (g - 1) * (e - (0.5 * (mx * mx + my * my + mz * mz) / rho + pm))
    pt = p + pm
    bu = bx * vx + by * vy + bz * vz
    return np.array([mx, vx * mx - bx * bx + pt, vx * my - by * bx, vx * mz - bz * bx, 0.0,
                     -(bx * vy - by * vx), bz * vx - bx * vz, vx * (e + pt) - bx * bu])


def prim(w, g):
    rho, mx, my, mz, bx, by, bz, e = w
    vx, vy, vz = mx / rho, my / rho, mz / rho
    p = (g - 1) * (e - 0.5 * ((mx * mx + my * my + mz * mz) / rho + (bx * bx + by * by + bz * bz)))
    return np.array([rho, vx, vy, vz, bx, by, bz, 0.5 * rho / p])


def random_state(rng, g):
    rho = rng.uniform(0.5, 2.0)
    v = rng.normal(size=3)
    B = rng.normal(size=3)
    p = rng.uniform(0.2, 3.0)
    e = p / (g - 1) + 0.5 * rho * (v @ v) + 0.5 * (B @ B)
    return np.array([rho, rho * v[0], rho * v[1], rho * v[2], B[0], B[1], B[2], e])


@pytest.mark.parametrize("g", [5 / 3, 1.4])
def test_hll_consistency(ora, g):
    rng = np.random.default_rng(1)
    for _ in range(20):
        w = random_state(rng, g)
        nf, nb, sl, sr = ora.hll_flux_x(w, w, g)
        np.testing.assert_allclose(nf, phys_flux_x(w, g), rtol=1e-12, atol=1e-12)
        assert nb == pytest.approx(w[4], rel=1e-14)
        assert sl <= 0.0 <= sr


@pytest.mark.parametrize("g", [5 / 3, 1.4])
def test_ec_flux_consistency_and_symmetry(ora, g):
    rng = np.random.default_rng(2)
    for _ in range(20):
        w = random_state(rng, g)
        pw = prim(w, g)
        np.testing.assert_allclose(ora.ec_flux(pw, pw, g, "x"), phys_flux_x(w, g), rtol=1e-12, atol=1e-12)
        w2 = random_state(rng, g)
        pa, pb = prim(w, g), prim(w2, g)
        np.testing.assert_allclose(ora.ec_flux(pa, pb, g, "x"), ora.ec_flux(pb, pa, g, "x"), rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(ora.ec_flux(pa, pb, g, "y"), ora.ec_flux(pb, pa, g, "y"), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("a", [1.0, 3.7, 1e-3, 250.0])
def test_log_mean(ora, a):
    """0.5(a+b)/ff is the logarithmic mean (a-b)/(log a - log b), continuous across the series branch"""
    for rel in [1e-9, 1e-6, 1e-3, 0.011, 0.0119, 0.012, 0.05, 0.5, 3.0]:
        b = a * (1 + rel)
        ff = ora.log_avg_divisor(a, b)
        exact = (a - b) / (math.log(a) - math.log(b)) if rel > 1e-6 else None
        if exact is not None:
            assert 0.5 * (a + b) / ff == pytest.approx(exact, rel=1e-12)
        assert ff >= 1.0
