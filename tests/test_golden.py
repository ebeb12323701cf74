"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py from the oracle).

CPU: the oracle reproduces every fixture (it is deterministic, so bit for bit) and the host set-up
reproduces the stored initial states.  GPU: the CUDA path, through the C ABI, matches the fixtures
within the parity bar (relative L1 <= 1e-12 per conserved variable).
"""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT, rel_l1

FIXTURES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FIXTURES]


def load(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def test_fixtures_exist():
    assert len(FIXTURES) == 4


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_setup_reproduces_initial_state(pkg, ora, path):
    d = load(path)
    prob = pkg.problems.make(str(d["problem"]))
    nx, ny, p = int(d["nx"]), int(d["ny"]), int(d["p"])
    u0 = prob.initial_state(nx, ny, p)
    inner = (slice(None),) * 3 + (slice(1, -1), slice(1, -1))
    np.testing.assert_array_equal(u0[inner], d["u_bc"][inner])


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_oracle_reproduces_fixture(pkg, ora, path):
    d = load(path)
    nx, ny, p = int(d["nx"]), int(d["ny"]), int(d["p"])
    prob = pkg.problems.make(str(d["problem"]))
    o = ora.OracleSolver(nx, ny, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
    u = np.asfortranarray(d["u_bc"].copy())
    ut, dl = o.semidiscretize(u)
    np.testing.assert_array_equal(ut, d["ut"])
    assert dl == d["dt_lim"]
    u1 = np.asfortranarray(d["u1_in"].copy())
    avg = np.full((8, nx + 2, ny + 2), np.nan, order="F")
    pp = o.post_process(u1, avg, 1, 1, float(d["pp_dt"]), 0, 1)
    np.testing.assert_array_equal(u1, d["u1_out"])
    assert pp["tot_ent"] == d["pp_tot_ent"] and pp["num_negcell"] == d["pp_num_negcell"]
    o.set_state(d["u_bc"][:, :, :, 1:-1, 1:-1])
    st = o.solve(prob.final_T, prob.cfl, max_steps=2)
    inner = (slice(None),) * 3 + (slice(1, -1), slice(1, -1))
    np.testing.assert_array_equal(o.u_con[inner], d["step2_u"][inner])
    assert st["t"] == d["step2_t"] and st["dt_lim"] == d["step2_dt_lim"]


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_gpu_matches_fixture(pkg, path):
    d = load(path)
    nx, ny, p = int(d["nx"]), int(d["ny"]), int(d["p"])
    prob = pkg.problems.make(str(d["problem"]))
    inner = (slice(None),) * 3 + (slice(1, -1), slice(1, -1))
    with pkg.DGSolver.for_problem(prob, nx, ny, p) as g:
        g.upload_state(0, d["u_bc"])
        dl = g.semidiscretize(1, 0)
        assert rel_l1(g.download_ut(1), d["ut"], floor_frac=1e-2).max() <= 1e-12
        assert abs(dl - float(d["dt_lim"])) <= 1e-13 * float(d["dt_lim"])
        g.upload_state(1, d["u1_in"])
        pp = g.post_process(1, 1, 1, float(d["pp_dt"]), 0, 1)
        m = np.isfinite(d["u1_out"])
        assert rel_l1(np.where(m, g.download_state(1), 0), np.where(m, d["u1_out"], 0)).max() <= 1e-12
        assert pp["num_negcell"] == int(d["pp_num_negcell"])
        st = g.solve_execute(d["u_bc"], prob.final_T, prob.cfl, max_steps=2)
        assert st["steps"] == int(d["step2_steps"])
        assert abs(st["t"] - float(d["step2_t"])) <= 1e-14 * float(d["step2_t"])
        assert rel_l1(g.download_state(0)[inner], d["step2_u"][inner]).max() <= 1e-12
