"""Batched against one-after-another on homogeneous batches (GPU; not collected by pytest -- run it
directly).

The batched kernels run every member of a degree group in shared persistent launches, the single
instance kernels one run at a time.  For each case COUNT runs of the same problem, mesh and degree
are stepped STEPS SSP-RK3 steps one after another (each run's own CUDA graph), then the same runs
from the same initial states as one batch; both timed with CUDA events.  Batches of small meshes
gain (a run alone cannot fill the GPU); batches of large meshes show what the batched form of the
kernels costs against the single-instance form.

    python tests/study_batch_efficiency.py [--cases vortex:256:3:16,vortex:64:3:256,...] [--steps 4]
                                           [--batched-only]

--batched-only skips the one-after-another leg (for a launch list of the batched kernels).
"""
import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

DEFAULT = "vortex:256:3:16,vortex:64:3:256,vortex:64:2:256,vortex:512:3:2"


def trial(pkg, torch, name, n, p, count, steps, batched_only):
    prob = pkg.problems.make(name)
    runs = [pkg.DGSolver.for_problem(prob, n, n, p) for _ in range(count)]
    dofs = count * 8 * n * n * (p + 1) ** 2

    def start():  # initial state, then one untimed step each (kernels loaded, each run's graph built)
        for r in runs:
            r.init_problem(prob)
            r.solve_begin(prob.final_T, prob.cfl)
            r.advance(1)
        torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms_solo = None
    if not batched_only:
        start()
        e0.record()
        for r in runs:
            r.advance(steps, check_every=steps)
        e1.record()
        torch.cuda.synchronize()
        ms_solo = e0.elapsed_time(e1)
    start()
    b = pkg.Batch()
    for r in runs:
        b.add(r)
    b.advance(0)  # tables and the batch graph, untimed
    torch.cuda.synchronize()
    e0.record()
    b.advance(steps)
    e1.record()
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1)
    for r in list(runs):
        b.remove(r)
    b.close()
    for r in runs:
        r.close()
    su = 3 * dofs * steps
    out = dict(case=f"{count} x {name} {n}^2 p={p}", steps=steps,
               batched_dof_stage_per_s=su / ms_b * 1e3, batched_ms_per_step=ms_b / steps)
    if ms_solo is not None:
        out.update(one_after_another_dof_stage_per_s=su / ms_solo * 1e3,
                   one_after_another_ms_per_run_step=ms_solo / steps / count)
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default=DEFAULT, help="problem:N:p:count,...")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--batched-only", action="store_true")
    a = ap.parse_args()
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    for c in a.cases.split(","):
        name, n, p, count = c.split(":")
        trial(pkg, torch, name, int(n), int(p), int(count), a.steps, a.batched_only)


if __name__ == "__main__":
    main()
