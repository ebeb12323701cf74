"""Generate the golden fixtures of tests/golden/ from the CPU oracle (strict build).

The reference ships no golden vectors and cannot be run here (no Fortran compiler), so these
fixtures freeze the oracle's outputs on small, seeded inputs:

  * the initial state (problems.py set-up, ghost ring filled by the problem's BC);
  * DG_semidiscretize of it: ut and dt_lim;
  * post_process of the first SSP-RK3 stage state with OEDG + LDF + entropy;
  * the state, t, dt_lim and total entropy after two SSP-RK3 steps of solve_execute.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = {
    # name: (problem, nx, ny, p)
    "ot2pi_6x5_p2": ("ot2pi", 6, 5, 2),
    "blast_8x8_p1": ("blast", 8, 8, 1),
    "vortex_5x6_p3": ("vortex", 5, 6, 3),
    "rotor_7x7_p2": ("rotor", 7, 7, 2),
}


def generate(name):
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    from oracle import oracle as ora
    prob_name, nx, ny, p = CASES[name]
    prob = pkg.problems.make(prob_name)
    u0 = prob.initial_state(nx, ny, p)
    o = ora.OracleSolver(nx, ny, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
    u_bc = np.asfortranarray(u0.copy())
    o.apply_bc(u_bc)
    ut, dt_lim = o.semidiscretize(u_bc)
    # a stage state: U1 = U0 + dt L(U0), with ghosts, then post_process(OEDG, LDF, entropy)
    dt = prob.cfl * dt_lim
    u1 = np.asfortranarray(u_bc.copy())
    u1[:, :, :, 1:-1, 1:-1] = u_bc[:, :, :, 1:-1, 1:-1] + dt * ut
    o.apply_bc(u1)
    u1_in = u1.copy()
    avg = np.full((8, nx + 2, ny + 2), np.nan, order="F")
    pp = o.post_process(u1, avg, 1, 1, dt, 0, 1)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    st = o.solve(prob.final_T, prob.cfl, max_steps=2)
    return dict(problem=prob_name, nx=nx, ny=ny, p=p, gamma=prob.gamma, domain=np.array(prob.domain),
                bc_kind=prob.bc_kind, u_bc=u_bc, ut=ut, dt_lim=dt_lim, pp_dt=dt, u1_in=u1_in,
                u1_out=u1, avg1=avg, pp_tot_ent=pp["tot_ent"], pp_num_negcell=pp["num_negcell"],
                step2_u=o.u_con.copy(), step2_t=st["t"], step2_dt_lim=st["dt_lim"],
                step2_tot_ent=st["tot_ent"], step2_steps=st["steps"])


def main():
    for name in CASES:
        d = generate(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print(name, "written")


if __name__ == "__main__":
    main()
