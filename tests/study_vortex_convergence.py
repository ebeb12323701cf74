"""Convergence study of the device solver on the smooth isentropic MHD vortex (GPU; not collected by
pytest -- run it directly).

The scope table's vortex configuration: [-10,10]^2 periodic, rho = 1, bulk velocity (1, 1),
kappa = mu = 1, p_inf = 1, gamma = 5/3; SSP-RK3, CFL 0.6, OEDG + LDF + positivity limiter on;
meshes 64^2 .. 512^2 at degrees 1-3, to one period (t = 20), where the exact solution is the
initial state again.  The errors are the reference's norms for its smooth test problems
(compute_error_smooth1D, problems.f90:697-741): the GLL-quadrature L2 norm of the error summed
over the eight conserved variables, and the max norm over nodes and variables.

    python tests/study_vortex_convergence.py [--meshes 64,128,256,512] [--degrees 1,2,3]
                                             [--final-time 20] [--no-oedg] [--no-ldf] [--json out.json]

--no-oedg / --no-ldf switch the OEDG damping / the LDF projection off (the discretisation's own
order on a smooth solution, without the damping that dominates the error on coarse meshes).
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def errors(pkg, u, n, p, T, w):
    """(L2, max) of the interior state u against the exact vortex at time T"""
    prob = pkg.problems.make("vortex")
    ex = pkg.problems.vortex_exact(n, n, p, T)
    h = (prob.domain[1] - prob.domain[0]) / n
    W = 0.25 * h * h * np.outer(w, w)
    d = u - ex
    l2 = math.sqrt(float(np.einsum("sklij,kl->", d * d, W)))
    return l2, float(np.abs(d).max())


def run(pkg, n, p, T, oedg=True, ldf=True):
    prob = pkg.problems.make("vortex")
    t0 = time.perf_counter()
    with pkg.DGSolver.for_problem(prob, n, n, p) as g:
        g.init_problem(prob)
        g.solve_begin(T, prob.cfl, oedg, ldf, False)
        st = g.advance(0, check_every=256)
        u = g.download_state(0)[:, :, :, 1:-1, 1:-1]
    wall = time.perf_counter() - t0
    assert st["flags"] == 0 and st["done"] == 1, st
    return u, st, wall


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--meshes", default="64,128,256,512")
    ap.add_argument("--degrees", default="1,2,3")
    ap.add_argument("--final-time", type=float, default=20.0)
    ap.add_argument("--no-oedg", action="store_true")
    ap.add_argument("--no-ldf", action="store_true")
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    meshes = [int(x) for x in a.meshes.split(",")]
    rows = []
    for p in (int(x) for x in a.degrees.split(",")):
        w = pkg.problems.gll_nodes(p)[1]
        prev = None
        for n in meshes:
            u, st, wall = run(pkg, n, p, a.final_time, not a.no_oedg, not a.no_ldf)
            l2, mx = errors(pkg, u, n, p, a.final_time, w)
            row = dict(p=p, n=n, steps=st["steps"], retries=st["retries"], l2=l2, max=mx, wall_s=wall)
            if prev:
                row["order_l2"] = math.log2(prev["l2"] / l2)
                row["order_max"] = math.log2(prev["max"] / mx)
            rows.append(row)
            prev = row
            print(json.dumps(row), flush=True)
    print("\n| p | mesh | steps | L2 error | order | max error | order |")
    print("|---|---|---|---|---|---|---|")
    for r in rows:
        o2 = f"{r['order_l2']:.2f}" if "order_l2" in r else "-"
        om = f"{r['order_max']:.2f}" if "order_max" in r else "-"
        print(f"| {r['p']} | {r['n']}^2 | {r['steps']} | {r['l2']:.3e} | {o2} | {r['max']:.3e} | {om} |")
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
