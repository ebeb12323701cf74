"""Boundary conditions of the cloud-shock and jet set-ups (problems.f90:425-595).

CPU: the oracle's ghost fills match a literal numpy transcription of the reference's loops on a
random state.  GPU: the library's fills match the oracle bit for bit (they are copies, sign flips
and a constant state), and two SSP-RK3 steps of each set-up match the oracle within the parity bar.
"""
import numpy as np
import pytest

from conftest import rel_l1


def reference_cloud_shock(u, state):
    """BC_cloud_shock (problems.f90:425-472) on u(8, n, n, 0:nx+1, 0:ny+1)"""
    u = u.copy(order="F")
    nx, ny = u.shape[3] - 2, u.shape[4] - 2
    for j in range(1, ny + 1):
        u[:, :, :, 0, j] = u[:, :, :, 1, j]
        u[:, :, :, nx + 1, j] = state[:, None, None]
    for i in range(1, nx + 1):
        u[:, :, :, i, 0] = u[:, :, :, i, 1]
        u[:, :, :, i, ny + 1] = u[:, :, :, i, ny]
    return u


def reference_jet(u, state):
    """BC_jet1_cell_ext (problems.f90:474-595) on u(8, n, n, 0:nx+1, 0:ny+1)"""
    u = u.copy(order="F")
    nx, ny, n = u.shape[3] - 2, u.shape[4] - 2, u.shape[1]
    for j in range(1, ny + 1):
        for l in range(n):
            for k in range(n):
                src = u[:, n - 1 - k, l, 1, j]
                u[:, k, l, 0, j] = src * np.array([1, -1, 1, 1, -1, 1, 1, 1])
        u[:, :, :, nx + 1, j] = u[:, :, :, nx, j]
    for i in range(1, nx + 1):
        if i <= nx // 10:
            u[:, :, :, i, 0] = state[:, None, None]
        else:
            u[:, :, :, i, 0] = u[:, :, :, i, 1]
        u[:, :, :, i, ny + 1] = u[:, :, :, i, ny]
    return u


CASES = [("cloud_shock", reference_cloud_shock, 12, 9), ("jet", reference_jet, 20, 7)]


def _random_state(nx, ny, p, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((8, p + 1, p + 1, nx + 2, ny + 2)))


@pytest.mark.parametrize("name,ref,nx,ny", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_oracle_bc_matches_reference_loops(pkg, ora, name, ref, nx, ny, p):
    prob = pkg.problems.make(name)
    o = ora.OracleSolver(nx, ny, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
    u = _random_state(nx, ny, p, 3)
    got = u.copy(order="F")
    o.apply_bc(got)
    np.testing.assert_array_equal(got, ref(u, np.asarray(prob.bc_state)))


def test_set_ups_match_the_reference_states(pkg):
    cs = pkg.problems.make("cloud_shock")
    x = np.array([0.3, 0.7, 0.8, 0.97])
    y = np.array([0.5, 0.9, 0.5, 0.5])
    up = pkg.problems.cloud_shock_pri(x, y, cs.gamma)
    assert up[0].tolist() == [3.86859, 1.0, 10.0, 1.0]  # post-shock, pre-shock, cloud, pre-shock
    jet = pkg.problems.make("jet")
    assert jet.gamma == 1.4 and jet.bc_kind == pkg.capi.BC_JET
    np.testing.assert_allclose(jet.bc_state[2], 1.4 * 800.0)  # nozzle momentum rho*v


@pytest.mark.gpu
@pytest.mark.parametrize("name,ref,nx,ny", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_gpu_bc_matches_oracle(pkg, ora, name, ref, nx, ny, p):
    prob = pkg.problems.make(name)
    o = ora.OracleSolver(nx, ny, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
    u = _random_state(nx, ny, p, 5)
    want = u.copy(order="F")
    o.apply_bc(want)
    with pkg.DGSolver.for_problem(prob, nx, ny, p) as g:
        g.upload_state(0, u)
        g.apply_bc(0)
        got = g.download_state(0)
    np.testing.assert_array_equal(got, want)  # corners are never filled: both keep the uploaded values


@pytest.mark.gpu
@pytest.mark.parametrize("rk", [1, 3])
@pytest.mark.parametrize("name,nx,ny,p", [("cloud_shock", 16, 16, 2), ("jet", 20, 30, 2)])
def test_gpu_steps_with_these_bcs_match_oracle(pkg, ora, name, nx, ny, p, rk):
    """with SSP-RK(1,1) the only stage is the final one, whose OEDG indicators read the ghost ring
    that the first stage forms on the device"""
    prob = pkg.problems.make(name)
    u0 = prob.initial_state(nx, ny, p)
    o = ora.OracleSolver(nx, ny, p, p, rk, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    st_o = o.solve(prob.final_T, prob.cfl, max_steps=2)
    with pkg.DGSolver.for_problem(prob, nx, ny, p, rk) as g:
        st = g.solve_execute(u0, prob.final_T, prob.cfl, max_steps=2)
        got = g.download_state(0)
    inner = (slice(None),) * 3 + (slice(1, -1), slice(1, -1))
    assert st["steps"] == 2 and st["retries"] == st_o["retries"]
    assert abs(st["t"] - st_o["t"]) <= 1e-14 * st_o["t"]
    assert rel_l1(got[inner], o.u_con[inner]).max() <= 1e-12
