"""How much can batching gain on the served request mix?  (GPU; not collected by pytest -- run it
directly.)

Serving many runs at once can only remove the time a run spends below the GPU's throughput: a
mesh too small to fill the device is latency-bound when it runs alone (its step costs the launch
and synchronisation floor of about 18 kernels), while a large mesh already runs at the device's
full rate.  This script measures, for every (problem, N, p) of a grid spanning the served mix,

  * the solo step time of the device-resident driver (CUDA-graph steps, CUDA events), and
  * the time step dt the run takes at its CFL (from the device's own first steps),

and then draws requests from the scope table's served distribution (problem in {OT, rotor, blast},
N log-uniform in [n_lo, n_hi], p uniform in {1,2,3}, t_end uniform in [0.05, 0.5] x the problem's
horizon), giving each request

  * T_solo  = steps x solo step time (interpolated in log N), and
  * T_ideal = steps x 3 x DOFs / R_peak, the time at the best throughput measured on the grid.

sum(T_solo) / sum(T_ideal) bounds the solves/s gain of any batched or served form over one run at a
time on this mix (Amdahl: a batch cannot make a run faster than the device's peak rate).  R_peak is
the best rate of the grid, or --device-peak (the rate a mesh that fills the GPU reaches, e.g. the
512x512 p=3 vortex), which bounds a batch of small meshes that together fill the GPU.

    python tests/study_serving_bound.py [--n-lo 32] [--n-hi 512] [--samples 20000] [--device-peak R]
                                        [--json out]
"""
import argparse
import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

HORIZON = {"ot2pi": 0.5, "rotor": 0.15, "blast": 0.01}
MESHES = [32, 48, 64, 96, 128, 192, 256, 384, 512]


def measure(pkg, name, n, p, steps=20):
    import torch
    prob = pkg.problems.make(name)
    with pkg.DGSolver.for_problem(prob, n, n, p) as s:
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)
        s.init_problem(prob)
        s.solve_begin(prob.final_T, prob.cfl)
        s.advance(3)
        t0 = s.status()["t"]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            e0.record(st)
        r = s.advance(steps, check_every=steps)
        with torch.cuda.stream(st):
            e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        dt = (r["t"] - t0) / steps
    return ms, dt


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-lo", type=int, default=32)
    ap.add_argument("--n-hi", type=int, default=512)
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--device-peak", type=float, default=0.0, help="DOF-stage/s (0: the grid's best)")
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    grid = {}
    for name in HORIZON:
        for p in (1, 2, 3):
            for n in MESHES:
                if a.n_lo <= n <= a.n_hi or n in (a.n_lo, a.n_hi):
                    ms, dt = measure(pkg, name, n, p)
                    grid[(name, p, n)] = (ms, dt)
                    print(json.dumps(dict(problem=name, p=p, n=n, ms_per_step=ms, dt=dt,
                                          dof_stage_per_s=3 * 8 * n * n * (p + 1) ** 2 / (ms * 1e-3))), flush=True)
    peak = max(3 * 8 * n * n * (p + 1) ** 2 / (ms * 1e-3) for (name, p, n), (ms, dt) in grid.items())
    peak = max(peak, a.device_peak)

    def interp(name, p, n, k):  # k = 0: ms per step, 1: dt x n (dt scales as 1/n)
        ns = sorted(m for (nm, pp, m) in grid if nm == name and pp == p)
        xs = np.log([float(m) for m in ns])
        ys = [grid[(name, p, m)][0] if k == 0 else grid[(name, p, m)][1] * m for m in ns]
        return float(np.interp(math.log(n), xs, ys))

    rng = np.random.default_rng(a.seed)
    t_solo = t_ideal = 0.0
    for _ in range(a.samples):
        name = list(HORIZON)[int(rng.integers(0, 3))]
        n = int(round(math.exp(rng.uniform(math.log(a.n_lo), math.log(a.n_hi)))))
        p = int(rng.integers(1, 4))
        t_end = float(rng.uniform(0.05, 0.5)) * HORIZON[name]
        steps = math.ceil(t_end / (interp(name, p, n, 1) / n))
        t_solo += steps * interp(name, p, n, 0) * 1e-3
        t_ideal += steps * 3 * 8 * n * n * (p + 1) ** 2 / peak
    out = dict(n_lo=a.n_lo, n_hi=a.n_hi, samples=a.samples, peak_dof_stage_per_s=peak,
               mean_solo_s=t_solo / a.samples, mean_ideal_s=t_ideal / a.samples, bound=t_solo / t_ideal)
    print(json.dumps(out))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(dict(grid={f"{k[0]}_p{k[1]}_n{k[2]}": v for k, v in grid.items()}, summary=out), f, indent=1)


if __name__ == "__main__":
    main()
