"""GPU parity: the CUDA path through the C ABI against the CPU oracle on the same inputs.

Tolerances (FP64):
  * residual ut, post-processed states, one SSP-RK3 step: relative L1 per conserved variable
    <= 1e-12 (the one-step parity bar; observed differences are at the 1e-15 level, from FMA
    contraction and libm vs CUDA log/exp/sqrt rounding);
  * dt_lim, tot_ent: relative 1e-13;
  * integer outputs (neg_avg, num_negcell, retries, steps): exact.
"""
import numpy as np
import pytest

from conftest import rel_l1

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _ent_tol(u, gamma):
    """tolerance for the total entropy: 1e-13 relative times the conditioning of the pressure,
    max(E/p) over the nodes (p = (gamma-1)(E - kinetic - magnetic) loses that factor of relative
    accuracy, and the entropy depends on log p); ~4000 for the low-beta blast"""
    x = u[:, :, :, 1:-1, 1:-1]
    prs = (gamma - 1) * (x[7] - 0.5 * ((x[1] ** 2 + x[2] ** 2 + x[3] ** 2) / x[0] + (x[4] ** 2 + x[5] ** 2 + x[6] ** 2)))
    cond = np.max(np.abs(x[7]) / np.maximum(np.abs(prs), 1e-300))
    return 1e-13 * max(1.0, float(cond))


def _setup(pkg, ora, name, nx, ny, p, amp=1.0, rknstg=3):
    prob = pkg.problems.make(name, amp=amp)
    u0 = prob.initial_state(nx, ny, p)
    g = pkg.DGSolver.for_problem(prob, nx, ny, p, rknstg)
    o = ora.OracleSolver(nx, ny, p, p, rknstg, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
    return prob, u0, g, o


def _perturbed(u0, seed, scale=0.02, gamma=5.0 / 3.0):
    """interior perturbed node by node in primitive variables: density and pressure
    multiplicatively (they stay positive), velocity and field additively"""
    rng = np.random.default_rng(seed)
    u = u0.copy()
    inner = u[:, :, :, 1:-1, 1:-1]
    noise = rng.standard_normal(inner.shape)
    rho = inner[0]
    v = inner[1:4] / rho
    B = inner[4:7]
    prs = (gamma - 1) * (inner[7] - 0.5 * (rho * (v ** 2).sum(0) + (B ** 2).sum(0)))
    vs = 1.0 + np.abs(v).max()
    bs = 1.0 + np.abs(B).max()
    rho = rho * np.exp(scale * np.tanh(noise[0]))
    prs = prs * np.exp(scale * np.tanh(noise[7]))
    v = v + scale * vs * noise[1:4]
    B = B + scale * bs * noise[4:7] * np.sqrt(np.maximum(prs, 0.0) / (1.0 + (B ** 2).sum(0)))
    inner[0] = rho
    inner[1:4] = rho * v
    inner[4:7] = B
    inner[7] = prs / (gamma - 1) + 0.5 * (rho * (v ** 2).sum(0) + (B ** 2).sum(0))
    return u


CASES = [("ot2pi", 8, 8, 1), ("ot2pi", 12, 10, 2), ("ot2pi", 9, 7, 3), ("blast", 10, 12, 2),
         ("rotor", 11, 9, 2), ("vortex", 10, 10, 3), ("ot_unit", 17, 13, 1)]


@pytest.mark.parametrize("name,nx,ny,p", CASES)
def test_residual_parity(pkg, ora, name, nx, ny, p):
    prob, u0, g, o = _setup(pkg, ora, name, nx, ny, p)
    u = _perturbed(u0, seed=nx * 31 + p, gamma=prob.gamma)
    # ghosts by the solver's own BC on both sides
    g.upload_state(0, u)
    g.apply_bc(0)
    ug = g.download_state(0)
    uo = np.asfortranarray(u.copy())
    o.apply_bc(uo)
    inner_ghost = np.isfinite(uo)
    assert np.array_equal(np.isfinite(ug), inner_ghost)
    assert np.array_equal(ug[inner_ghost], uo[inner_ghost]), "BC fill must be bit-exact"
    dl_g = g.semidiscretize(1, 0)
    ut_g = g.download_ut(1)
    ut_o, dl_o = o.semidiscretize(uo)
    err = rel_l1(ut_g, ut_o, floor_frac=1e-2)
    assert err.max() <= TOL, err
    assert abs(dl_g - dl_o) <= 1e-13 * dl_o
    g.close()


@pytest.mark.parametrize("name,nx,ny,p", CASES)
@pytest.mark.parametrize("oedg,ldf,comput_ent,ent_offset", [(0, 1, 1, 0), (1, 1, 1, 0), (1, 0, 0, 0),
                                                           (0, 0, 1, 1), (1, 1, 1, 1)])
def test_post_process_parity(pkg, ora, name, nx, ny, p, oedg, ldf, comput_ent, ent_offset):
    prob, u0, g, o = _setup(pkg, ora, name, nx, ny, p)
    u = _perturbed(u0, seed=nx + 7 * p, scale=0.05, gamma=prob.gamma)
    uo = np.asfortranarray(u.copy())
    o.apply_bc(uo)
    g.upload_state(0, uo)
    avg_o = np.full((8, nx + 2, ny + 2), np.nan, order="F")
    ro = o.post_process(uo, avg_o, oedg, ldf, 1.3e-3, ent_offset, comput_ent)
    rg = g.post_process(0, oedg, ldf, 1.3e-3, ent_offset, comput_ent)
    assert rg["neg_avg"] == ro["neg_avg"]
    assert not ro["neg_avg"], "case must stay admissible"
    assert rg["num_negcell"] == ro["num_negcell"]
    if comput_ent and not ro["neg_avg"]:
        assert abs(rg["tot_ent"] - ro["tot_ent"]) <= _ent_tol(uo, prob.gamma) * abs(ro["tot_ent"])
    else:
        assert np.isnan(rg["tot_ent"]) and np.isnan(ro["tot_ent"])
    ug = g.download_state(0)
    m = np.isfinite(uo)
    err = rel_l1(np.where(m, ug, 0.0), np.where(m, uo, 0.0))
    assert err.max() <= TOL, err
    ag = g.download_avg()
    ma = np.isfinite(avg_o)
    assert rel_l1(np.where(ma, ag, 0), np.where(ma, avg_o, 0)).max() <= TOL
    g.close()


def _with_negative_nodes(u0, gamma):
    """blast state with nodal negative density / pressure in a few cells whose averages stay
    admissible: exercises both branches of the Zhang-Shu limiter (DG_solver.f90:544-600)"""
    u = np.asfortranarray(u0.copy())
    # thermal energy is p/(gamma-1) = 0.25 under a magnetic energy of ~398
    u[0, 0, 0, 3, 3] = -0.05   # negative density at a corner node
    u[7, 1, 1, 5, 6] -= 0.5    # negative pressure at the centre node, average stays positive
    u[7, 2, 0, 8, 2] -= 0.3    # negative pressure at an edge node
    u[0, 2, 2, 6, 9] = 1e-13   # density below PP_eps
    return u


@pytest.mark.parametrize("oedg", [0, 1])
def test_pp_limiter_parity(pkg, ora, oedg):
    prob, u0, g, o = _setup(pkg, ora, "blast", 10, 12, 2)
    uo = _with_negative_nodes(u0, prob.gamma)
    o.apply_bc(uo)
    g.upload_state(0, uo)
    avg_o = np.full((8, 12, 14), np.nan, order="F")
    ro = o.post_process(uo, avg_o, oedg, 1, 2e-3, 0, 1)
    rg = g.post_process(0, oedg, 1, 2e-3, 0, 1)
    assert not ro["neg_avg"] and not rg["neg_avg"]
    assert ro["num_negcell"] >= 1
    assert rg["num_negcell"] == ro["num_negcell"]
    assert abs(rg["tot_ent"] - ro["tot_ent"]) <= _ent_tol(uo, prob.gamma) * abs(ro["tot_ent"])
    ug = g.download_state(0)
    m = np.isfinite(uo)
    err = rel_l1(np.where(m, ug, 0.0), np.where(m, uo, 0.0))
    assert err.max() <= TOL, err
    g.close()


def test_inadmissible_average_flag(pkg, ora):
    """a state with negative cell averages: both report neg_avg (the state itself is then
    unspecified, because the step is discarded) and neither reports an entropy"""
    prob, u0, g, o = _setup(pkg, ora, "blast", 10, 12, 2)
    uo = np.asfortranarray(u0.copy())
    uo[7, :, :, 3, 4] = 0.0  # zero energy under B ~ 28: negative pressure average in one cell
    uo[7, :, :, 7, 9] = 10.0
    o.apply_bc(uo)
    g.upload_state(0, uo)
    avg_o = np.full((8, 12, 14), np.nan, order="F")
    ro = o.post_process(uo, avg_o, 1, 1, 1e-3, 0, 1)
    rg = g.post_process(0, 1, 1, 1e-3, 0, 1)
    assert ro["neg_avg"] and rg["neg_avg"]
    assert rg["num_negcell"] == ro["num_negcell"] == 0
    assert np.isnan(rg["tot_ent"]) and np.isnan(ro["tot_ent"])
    g.close()


@pytest.mark.parametrize("name,nx,ny,p", CASES)
@pytest.mark.parametrize("rknstg", [3])
def test_one_step_parity(pkg, ora, name, nx, ny, p, rknstg):
    """after one SSP-RK3 step: relative L1 <= 1e-12 per conserved variable"""
    prob, u0, g, o = _setup(pkg, ora, name, nx, ny, p, rknstg=rknstg)
    sg = g.solve_execute(u0, prob.final_T, prob.cfl, max_steps=1)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, prob.cfl, max_steps=1)
    assert so["status"] == 0 and sg["flags"] == 0
    assert sg["steps"] == so["steps"] == 1
    assert sg["retries"] == so["retries"]
    assert abs(sg["t"] - so["t"]) <= 1e-14 * so["t"]
    assert abs(sg["dt_lim"] - so["dt_lim"]) <= 1e-13 * so["dt_lim"]
    ug = g.download_state(0)[:, :, :, 1:-1, 1:-1]
    uo = o.u_con[:, :, :, 1:-1, 1:-1]
    err = rel_l1(ug, uo)
    assert err.max() <= TOL, err
    g.close()


@pytest.mark.parametrize("rknstg", [1, 2, 5])
def test_other_rk_schemes(pkg, ora, rknstg):
    prob, u0, g, o = _setup(pkg, ora, "ot2pi", 10, 10, 2, rknstg=rknstg)
    sg = g.solve_execute(u0, prob.final_T, 0.1, max_steps=3)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, 0.1, max_steps=3)
    assert sg["steps"] == so["steps"] == 3
    err = rel_l1(g.download_state(0)[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
    assert err.max() <= 1e-12, err
    g.close()


def test_multi_step_blast_limiter_counts(pkg, ora):
    """blast: the PP limiter is active; limiter counts and states follow the oracle"""
    prob, u0, g, o = _setup(pkg, ora, "blast", 24, 24, 2)
    sg = g.solve_execute(u0, prob.final_T, prob.cfl, max_steps=10)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, prob.cfl, max_steps=10)
    assert sg["steps"] == so["steps"] == 10
    assert sg["retries"] == so["retries"]
    assert sg["num_negcell_total"] == so["num_negcell_total"]
    err = rel_l1(g.download_state(0)[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
    assert err.max() <= 1e-11, err
    ug = g.download_state(0)[:, :, :, 1:-1, 1:-1]
    assert ug[0].min() > 0
    g.close()


def test_retry_path(pkg, ora):
    """an over-large CFL makes an average inadmissible; both re-try with the golden-ratio shrink.
    The re-tries fall in steps 2-4 (2, 1 and 4 of them), after accepted steps, so the recomputed
    residual of u_con reads u_con's ghost ring as the reference leaves it: filled when the solve
    starts and not refreshed on acceptance (drive.f90:100-105, 304-311)."""
    prob, u0, g, o = _setup(pkg, ora, "blast", 16, 16, 2)
    cfl = 10.0
    sg = g.solve_execute(u0, prob.final_T, cfl, max_steps=4)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, cfl, max_steps=4)
    assert so["retries"] > 0
    assert sg["retries"] == so["retries"]
    assert sg["steps"] == so["steps"]
    assert abs(sg["t"] - so["t"]) <= 1e-13 * so["t"]
    err = rel_l1(g.download_state(0)[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
    assert err.max() <= 1e-11, err
    g.close()


def test_ot_full_run_small(pkg, ora):
    """Orszag-Tang 16x16 p=2 to t=0.5 (the plain-method config shape on a small mesh)"""
    prob, u0, g, o = _setup(pkg, ora, "ot2pi", 16, 16, 2)
    sg = g.solve_execute(u0, prob.final_T, prob.cfl)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, prob.cfl)
    assert sg["done"] == 1 and sg["steps"] == so["steps"]
    assert abs(sg["t"] - so["t"]) <= 1e-15 * so["t"]  # the clipped final step: t within an ulp or two
    err = rel_l1(g.download_state(0)[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
    assert err.max() <= 1e-10, err
    assert abs(sg["tot_ent"] - so["tot_ent"]) <= 1e-12 * abs(so["tot_ent"])
    g.close()


def test_ot_config_full_run(pkg, ora):
    """the reference's own CPU configuration end to end: Orszag-Tang on 64x64 quads, degree 2,
    SSP-RK3, CFL 0.2, OEDG + LDF + positivity, to t = 0.5 (561 steps); measured agreement is
    ~2e-15 relative L1 per variable and ~3e-16 in the total entropy"""
    prob, u0, g, o = _setup(pkg, ora, "ot2pi", 64, 64, 2)
    sg = g.solve_execute(u0, prob.final_T, prob.cfl)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, prob.cfl)
    assert so["status"] == 0 and sg["flags"] == 0 and sg["done"] == 1
    assert sg["steps"] == so["steps"] and sg["retries"] == so["retries"]
    assert abs(sg["t"] - so["t"]) <= 1e-15 * so["t"]  # the clipped final step: t within an ulp or two
    err = rel_l1(g.download_state(0)[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
    assert err.max() <= TOL, err
    assert abs(sg["tot_ent"] - so["tot_ent"]) <= 1e-13 * abs(so["tot_ent"])
    g.close()


def test_blast_config_hundred_steps(pkg, ora):
    """the low-beta blast configuration (p = 2, gamma = 1.4, PP limiter on thousands of cells per
    step) on 48x48 for 100 steps: identical limiter counts and relative L1 <= 1e-10.  The flow is
    chaotic at the round-off level: differences grow about tenfold every 8 steps after step 60
    (1e-14 at step 40, 7e-12 at step 100, 1e-5 at step 200), and the oracle perturbed by one ulp
    in one energy value departs from itself in the same way, so a full run to t = 0.01 is not a
    parity case"""
    prob, u0, g, o = _setup(pkg, ora, "blast", 48, 48, 2)
    sg = g.solve_execute(u0, prob.final_T, prob.cfl, max_steps=100)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, prob.cfl, max_steps=100)
    assert sg["steps"] == so["steps"] == 100 and sg["retries"] == so["retries"]
    assert sg["num_negcell_total"] == so["num_negcell_total"] > 10000
    err = rel_l1(g.download_state(0)[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
    assert err.max() <= 1e-10, err
    g.close()


@pytest.mark.parametrize("rknstg,oedg,expect", [(3, 1, 18), (3, 0, 16), (2, 1, 14), (1, 1, 10), (5, 1, 30)])
def test_step_graph_kernel_count(pkg, rknstg, oedg, expect):
    """kernel launches of one captured try: 3 (step begin, re-try residual, dt with the first
    stage's pseudo-time) + per stage ([combination for SSP-RK(5,4) stages > 1], [boundary fill
    before loop 1 for stages > 1], loop 1, [final stage: global sums and face indicators with
    OEDG, limiter], stage end with the boundary fill (and the entropy sum in the final stage),
    residual) + step end"""
    prob = pkg.problems.make("ot2pi")
    with pkg.DGSolver.for_problem(prob, 8, 8, 2, rknstg) as g:
        with pytest.raises(pkg.MHDError):
            g.step_graph_kernels()  # no graph before the first advance
        g.upload_state(0, prob.initial_state(8, 8, 2))
        g.solve_begin(prob.final_T, prob.cfl, oedg, 1, 0)
        g.advance(1)
        assert g.step_graph_kernels() == expect


PIPELINE_FLAGS = [(3, 1, 1, 1), (3, 0, 1, 0), (3, 1, 0, 0), (3, 0, 0, 1), (1, 1, 1, 1), (2, 1, 1, 1)]


@pytest.mark.parametrize("name,n,p", [("blast", 16, 2), ("ot2pi", 12, 3)])
@pytest.mark.parametrize("rknstg,oedg,ldf,ent_offset", PIPELINE_FLAGS)
def test_pipeline_flag_parity(pkg, ora, name, n, p, rknstg, oedg, ldf, ent_offset):
    """three steps of the device time-step pipeline against the oracle for the solve flags:
    OEDG off (the final stage limits without the indicators), LDF off, and the entropy-offset
    limiter, whose cell entropies are formed in the same loop-1 pass that forms stage 1"""
    prob, u0, g, o = _setup(pkg, ora, name, n, n, p, rknstg=rknstg)
    sg = g.solve_execute(u0, prob.final_T, prob.cfl, oedg, ldf, ent_offset, max_steps=3)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    so = o.solve(prob.final_T, prob.cfl, oedg, ldf, ent_offset, max_steps=3)
    assert so["status"] == 0 and sg["flags"] == 0
    assert sg["steps"] == so["steps"] == 3 and sg["retries"] == so["retries"]
    assert sg["num_negcell_total"] == so["num_negcell_total"]
    assert abs(sg["t"] - so["t"]) <= 1e-14 * so["t"]
    ug = g.download_state(0)
    assert abs(sg["tot_ent"] - so["tot_ent"]) <= _ent_tol(ug, prob.gamma) * abs(so["tot_ent"])
    err = rel_l1(ug[:, :, :, 1:-1, 1:-1], o.u_con[:, :, :, 1:-1, 1:-1])
    assert err.max() <= TOL, err
    g.close()
