"""Serving loop (GPU): continuous batching returns, for every request, exactly the solve a plain
run gives, and the solve the oracle gives at the parity bar; admission respects the HBM budget; the
one-at-a-time mode serves the same queue."""
import numpy as np
import pytest

from conftest import rel_l1

pytestmark = pytest.mark.gpu

REQS = [("ot2pi", 12, 2, 0.0, 0.03), ("rotor", 10, 1, 0.0, 0.004), ("ot2pi", 8, 3, 0.01, 0.02),
        ("rotor", 14, 2, 0.02, 0.003), ("blast", 12, 1, 0.03, 0.0005), ("ot2pi", 16, 1, 0.05, 0.05)]


def _solo_avg(pkg, name, n, p, t_end):
    prob = pkg.problems.make(name)
    with pkg.DGSolver.for_problem(prob, n, n, p) as s:
        st = s.solve_execute(prob.initial_state(n, n, p), t_end, prob.cfl)
        return s.download_avg(), st


@pytest.mark.parametrize("batched", [True, False])
def test_served_results_identical_to_plain_runs(pkg, ora, batched):
    with pkg.Server(hbm_budget_bytes=8 << 30, tries_per_round=2, batched=batched) as srv:
        avgs = []
        for i, (name, n, p, arr, t_end) in enumerate(REQS):
            prob = pkg.problems.make(name)
            avgs.append(srv.submit(i, prob, n, n, p, prob.initial_state(n, n, p), arr, final_T=t_end,
                                   want_avg=True))
        srv.run(max_seconds=120)
        res = {r["id"]: r for r in srv.results()}
        assert sorted(res) == list(range(len(REQS)))
        for i, (name, n, p, arr, t_end) in enumerate(REQS):
            r = res[i]
            assert r["done"] == 1 and r["flags"] == 0 and r["error"] == 0
            assert r["finished"] >= r["admitted"] >= r["arrival"]
            ref_avg, st = _solo_avg(pkg, name, n, p, t_end)
            assert r["steps"] == st["steps"] and r["t"] == st["t"]
            m = np.isfinite(ref_avg)
            np.testing.assert_array_equal(avgs[i][m], ref_avg[m])
            if i < 3:  # and the oracle's run of the same request (cell averages of the final state)
                prob = pkg.problems.make(name)
                o = ora.OracleSolver(n, n, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
                o.set_state(prob.initial_state(n, n, p)[:, :, :, 1:-1, 1:-1])
                so = o.solve(t_end, prob.cfl)
                assert so["steps"] == r["steps"]
                inner = (slice(None), slice(1, -1), slice(1, -1))
                assert rel_l1(avgs[i][inner], o.u_avg[inner]).max() <= 1e-12
                o.close()
        st = srv.stats()
        assert st["admitted"] == st["retired"] == len(REQS) and st["rounds"] >= 1
        assert min(st[k] for k in ("admit_s", "launch_s", "wait_s", "retire_s", "idle_s")) >= 0.0


def test_admission_respects_budget(pkg):
    fp = pkg.footprint(16, 16, 2)
    with pkg.DGSolver(16, 16, 2) as s:
        assert s.device_bytes() == fp
    budget = int(2.5 * fp)  # at most two runs resident at a time
    with pkg.Server(hbm_budget_bytes=budget, tries_per_round=1) as srv:
        prob = pkg.problems.make("ot2pi")
        for i in range(5):
            srv.submit(i, prob, 16, 16, 2, prob.initial_state(16, 16, 2), 0.0, final_T=0.01)
        srv.run(max_seconds=1e-6)  # one round: two admitted, three waiting
        st = srv.pending()
        assert st["active"] == 2 and st["queued"] == 3 and st["used_bytes"] <= budget
        srv.run(max_seconds=120)
        res = srv.results()
        assert len(res) == 5 and all(r["done"] == 1 for r in res)
        assert srv.pending()["used_bytes"] == 0


@pytest.mark.parametrize("batched", [True, False])
def test_inadmissible_initial_value_is_reported(pkg, batched):
    """a run whose initial state has a negative cell-average density ends with
    MHD_FLAG_INIT_NEG_AVG and no steps (drive.f90:70), next to a healthy run that completes"""
    prob = pkg.problems.make("ot2pi")
    good = prob.initial_state(10, 10, 2)
    bad = good.copy(order="F")
    bad[0, :, :, 4, 5] = -1.0
    with pkg.Server(hbm_budget_bytes=8 << 30, tries_per_round=2, batched=batched) as srv:
        srv.submit(0, prob, 10, 10, 2, bad, 0.0, final_T=0.01)
        srv.submit(1, prob, 10, 10, 2, good, 0.0, final_T=0.01)
        srv.run(max_seconds=120)
        res = {r["id"]: r for r in srv.results()}
    assert res[0]["flags"] & pkg.capi.MHD_FLAG_INIT_NEG_AVG and res[0]["steps"] == 0 and res[0]["done"] == 0
    assert res[1]["done"] == 1 and res[1]["flags"] == 0
