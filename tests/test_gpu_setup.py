"""Set-up and output next to the hot path (GPU): the initial state evaluated on the device
(mhd_gpu_init_problem, the init_by_fun_pri pattern of problems.f90:25-51) against the host set-up,
and the cell-average primitive output of save_tecbin_finite_volume (io.f90:75-86,
mhd_gpu_download_avg_primitive) against MHD_con2pri applied on the host.

The initial states agree to rounding (the device's sin/exp/sqrt are not glibc's: relative 1e-14 per
variable); the node coordinates and the primitive-to-conserved map are rounded exactly as the host
forms them.  The primitive output is bit-exact (same expression order, correctly rounded
operations, the same rounding to single precision).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SETUPS = [("ot2pi", {}), ("ot_unit", {"amp": 0.8}), ("vortex", {}), ("blast", {}), ("rotor", {"amp": 1.3}),
          ("alfven", {}), ("cloud_shock", {}), ("jet", {})]


def _make(pkg, name, kw):
    if name == "vortex":
        return pkg.problems.make(name)
    return pkg.problems.make(name, **kw)


@pytest.mark.parametrize("name,kw", SETUPS, ids=[s[0] for s in SETUPS])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_device_initial_state_matches_host(pkg, name, kw, p):
    prob = _make(pkg, name, kw)
    nx, ny = 13, 9
    ref = prob.initial_state(nx, ny, p)
    with pkg.DGSolver.for_problem(prob, nx, ny, p) as g:
        g.upload_state(0, np.zeros_like(ref))  # the device fill must overwrite everything
        g.init_problem(prob)
        got = g.download_state(0)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    inner = (slice(None),) * 3 + (slice(1, -1), slice(1, -1))
    for v in range(8):
        scale = max(np.abs(ref[v][inner[1:]]).max(), 1e-300)
        assert np.abs(got[v][inner[1:]] - ref[v][inner[1:]]).max() <= 1e-14 * scale, v


def test_blast_centre_parameter(pkg):
    prob = pkg.problems.make("blast")
    prob.params["center"] = (0.2, -0.1)
    nx = ny = 16
    ref = prob.initial_state(nx, ny, 2)
    with pkg.DGSolver.for_problem(prob, nx, ny, 2) as g:
        g.init_problem(prob)
        got = g.download_state(0)
    inner = (slice(None),) * 3 + (slice(1, -1), slice(1, -1))
    np.testing.assert_allclose(got[inner], ref[inner], rtol=1e-14, atol=0)


@pytest.mark.parametrize("name,p", [("rotor", 2), ("blast", 1), ("ot2pi", 3)])
def test_avg_primitive_output(pkg, name, p):
    prob = pkg.problems.make(name)
    nx, ny = 11, 7
    with pkg.DGSolver.for_problem(prob, nx, ny, p) as g:
        g.init_problem(prob)
        g.solve_begin(prob.final_T, prob.cfl)  # fills u_avg (initial post_process)
        g.advance(2)
        ua = g.download_avg()
        buf, vmin, vmax = g.download_avg_primitive()
    up = pkg.problems.con2pri(ua[:, 1:-1, 1:-1], prob.gamma).astype(np.float32)  # (8, nx, ny)
    exp = np.zeros((nx + 1, ny, 8), dtype=np.float32, order="F")
    exp[:nx, :, :] = np.moveaxis(up, 0, -1)
    np.testing.assert_array_equal(buf, exp)
    np.testing.assert_array_equal(vmin, up.reshape(8, -1).astype(np.float64).min(axis=1))
    np.testing.assert_array_equal(vmax, up.reshape(8, -1).astype(np.float64).max(axis=1))
