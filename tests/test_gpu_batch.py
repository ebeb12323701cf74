"""Batched instances (GPU): every member of a batch computes exactly what it computes alone.

The batch runs the same kernel bodies over a flattened work list of all members' tiles, so the
identity is bitwise: a member advanced K tries inside a mixed batch (different degrees, problems,
gammas, mesh sizes) has the same state, time and entropy as the same instance advanced K steps on
its own.  Members can join and leave between advances.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIX = [("ot2pi", 20, 2, 1.0, None), ("rotor", 17, 1, 1.3, None), ("ot2pi", 12, 3, 0.7, 1.4),
       ("rotor", 24, 3, 0.6, 5.0 / 3.0), ("blast", 16, 2, 1.0, None), ("vortex", 10, 1, 1.0, None)]


def _make(pkg, name, n, p, amp, gamma):
    prob = pkg.problems.make(name, gamma=gamma, amp=amp) if name != "vortex" else pkg.problems.make(name)
    u0 = prob.initial_state(n, n, p)
    s = pkg.DGSolver.for_problem(prob, n, n, p)
    s.upload_state(0, u0)
    s.solve_begin(prob.final_T, prob.cfl)
    return s


def test_batch_members_identical_to_solo_runs(pkg):
    K = 6
    solo = []
    for spec in MIX:
        s = _make(pkg, *spec)
        st = s.advance(K)
        solo.append((s.download_state(0), st))
        s.close()
    with pkg.Batch() as b:
        members = [_make(pkg, *spec) for spec in MIX]
        for m in members:
            b.add(m)
        assert len(b) == len(MIX)
        b.advance(K)
        for m, (u_ref, st_ref) in zip(members, solo):
            st = b.status(m)
            assert st["retries"] == 0 and st_ref["retries"] == 0
            assert st["steps"] == st_ref["steps"] == K
            assert st["t"] == st_ref["t"] and st["dt_lim"] == st_ref["dt_lim"]
            assert st["tot_ent"] == st_ref["tot_ent"]
            assert st["num_negcell_total"] == st_ref["num_negcell_total"]
        for m in list(members):
            b.remove(m)
        for m, (u_ref, _) in zip(members, solo):
            np.testing.assert_array_equal(m.download_state(0), u_ref)
            m.close()


def test_members_join_and_leave(pkg):
    with pkg.Batch() as b:
        a = _make(pkg, "ot2pi", 16, 2, 1.0, None)
        c = _make(pkg, "rotor", 12, 1, 1.0, None)
        b.add(a)
        b.add(c)
        b.advance(3)
        b.remove(c)
        d = _make(pkg, "ot2pi", 14, 3, 0.8, None)  # a new degree group joins
        b.add(d)
        b.advance(2)
        assert b.status(a)["steps"] == 5 and b.status(d)["steps"] == 2
        assert c.status()["steps"] == 3  # the removed member kept its state
        c.advance(2)  # and runs on its own again
        assert c.status()["steps"] == 5
        ref = _make(pkg, "rotor", 12, 1, 1.0, None)
        ref.advance(5)
        np.testing.assert_array_equal(c.download_state(0), ref.download_state(0))
        for s in (a, d):
            b.remove(s)
            s.close()
        c.close()
        ref.close()


def test_finished_members_idle(pkg):
    with pkg.Batch() as b:
        prob = pkg.problems.make("ot2pi")
        s = pkg.DGSolver.for_problem(prob, 8, 8, 1)
        s.upload_state(0, prob.initial_state(8, 8, 1))
        s.solve_begin(0.02, prob.cfl)  # a few steps to the end time
        b.add(s)
        for _ in range(50):
            if b.advance(4) == 0:
                break
        st = b.status(s)
        assert st["done"] == 1 and abs(st["t"] - 0.02) < 1e-15
        steps = st["steps"]
        b.advance(3)
        assert b.status(s)["steps"] == steps
        b.remove(s)
        s.close()


def test_launch_then_wait_equals_advance(pkg):
    a1, a2 = _make(pkg, "ot2pi", 16, 2, 1.0, None), _make(pkg, "rotor", 12, 3, 1.0, None)
    r1, r2 = _make(pkg, "ot2pi", 16, 2, 1.0, None), _make(pkg, "rotor", 12, 3, 1.0, None)
    with pkg.Batch() as b, pkg.Batch() as ref:
        b.add(a1), b.add(a2), ref.add(r1), ref.add(r2)
        b.launch(3)
        with pytest.raises(pkg.MHDError):  # membership is frozen while a round is in flight
            b.remove(a1)
        assert b.wait() == 2
        ref.advance(3)
        for m, r in ((a1, r1), (a2, r2)):
            assert b.status(m) == ref.status(r)
        for s in (a1, a2):
            b.remove(s)
        for s in (r1, r2):
            ref.remove(s)
        np.testing.assert_array_equal(a1.download_state(0), r1.download_state(0))
        np.testing.assert_array_equal(a2.download_state(0), r2.download_state(0))
    for s in (a1, a2, r1, r2):
        s.close()


FLAG_MIX = [  # (name, n, p, rknstg, use_oedg, use_ldf, ent_offset)
    ("blast", 16, 2, 3, 1, 1, 1), ("blast", 12, 2, 3, 0, 1, 0), ("ot2pi", 14, 3, 3, 1, 0, 0),
    ("rotor", 12, 1, 3, 0, 0, 1), ("ot2pi", 10, 2, 2, 1, 1, 1), ("rotor", 10, 3, 1, 1, 1, 0),
    ("ot2pi", 12, 2, 5, 1, 1, 0),
]


def _make_flags(pkg, name, n, p, rknstg, oedg, ldf, ent_offset):
    prob = pkg.problems.make(name)
    s = pkg.DGSolver.for_problem(prob, n, n, p, rknstg)
    s.upload_state(0, prob.initial_state(n, n, p))
    s.solve_begin(prob.final_T, prob.cfl, oedg, ldf, ent_offset)
    return s


def test_members_with_mixed_solve_flags_identical_to_solo_runs(pkg):
    """members that differ in OEDG, LDF, the entropy offset and the SSP-RK scheme share a batch and
    still compute bit for bit what they compute alone"""
    K = 4
    solo = []
    for spec in FLAG_MIX:
        s = _make_flags(pkg, *spec)
        st = s.advance(K)
        solo.append((s.download_state(0), st))
        s.close()
    with pkg.Batch() as b:
        members = [_make_flags(pkg, *spec) for spec in FLAG_MIX]
        for m in members:
            b.add(m)
        b.advance(K)
        for m, (u_ref, st_ref) in zip(members, solo):
            st = b.status(m)
            assert st["retries"] == st_ref["retries"] == 0
            assert st["steps"] == st_ref["steps"] == K
            assert st["t"] == st_ref["t"] and st["dt_lim"] == st_ref["dt_lim"]
            assert st["tot_ent"] == st_ref["tot_ent"]
            assert st["num_negcell_total"] == st_ref["num_negcell_total"]
        for m in list(members):
            b.remove(m)
        for m, (u_ref, _) in zip(members, solo):
            np.testing.assert_array_equal(m.download_state(0), u_ref)
            m.close()


@pytest.mark.parametrize("rknstg", [3, 2, 5])
def test_batch_members_against_the_oracle(pkg, ora, rknstg):
    """each member of a mixed batch (degrees 1-3, different problems and meshes) against its own
    oracle run: the batched kernels themselves (residual2_batched, pp_*_batched,
    stage_end_bc_batched, ctl_batched) at the parity bar, not only through the solo path"""
    from conftest import rel_l1
    K = 4
    specs = [("ot2pi", 14, 2, 1.0, None), ("rotor", 12, 1, 1.2, None), ("blast", 10, 3, 1.0, None)]
    members, probs = [], []
    with pkg.Batch() as b:
        for name, n, p, amp, gamma in specs:
            prob = pkg.problems.make(name, gamma=gamma, amp=amp)
            s = pkg.DGSolver.for_problem(prob, n, n, p, rknstg)
            s.upload_state(0, prob.initial_state(n, n, p))
            s.solve_begin(prob.final_T, prob.cfl)
            b.add(s)
            members.append(s)
            probs.append(prob)
        b.advance(K)
        sts = [b.status(s) for s in members]
        for s in members:
            b.remove(s)
    for s, st, prob, (name, n, p, amp, gamma) in zip(members, sts, probs, specs):
        o = ora.OracleSolver(n, n, p, p, rknstg, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
        o.set_state(prob.initial_state(n, n, p)[:, :, :, 1:-1, 1:-1])
        so = o.solve(prob.final_T, prob.cfl, max_steps=K)
        assert st["steps"] == so["steps"] == K and st["retries"] == so["retries"]
        err = rel_l1(s.download_state(0)[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
        assert err.max() <= 1e-12, (name, p, err)
        assert abs(st["t"] - so["t"]) <= 1e-14 * so["t"]
        assert st["num_negcell_total"] == so["num_negcell_total"]
        o.close()
        s.close()
