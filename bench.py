"""Benchmark of the B200 per-stage DG update for 2D ideal MHD.

Metric: FP64 DOF-stage updates per second (DOF = element x GLL node x conserved variable; one
SSP-RK3 time step = 3 stage updates of every DOF).  Workload (default): the smooth isentropic MHD
vortex on [-10,10]^2, periodic, 512x512 elements, degree 3 (16 GLL nodes per element, 33.5 M DOFs),
gamma = 5/3, SSP-RK3, CFL 0.6, OEDG + LDF + positivity limiter on -- the largest single-GPU
configuration of the vortex convergence study.  Synthetic input: the analytic initial condition.

Legs in one JSON line:
  value     device-resident time steps (mhd_gpu_advance), state resident in HBM;
  e2e       the same steps through the C ABI with host buffers: per step the Fortran-layout state is
            uploaded from pinned host memory, one step runs, and the state is downloaded;
  roofline  the dominant kernel (the DG residual) timed live with CUDA events on the solver's stream;
  cpu_baseline  the CPU oracle (OpenMP, all host threads) on a bounded sample of the same workload.
Multi-GPU: replicas only (independent instances, no exchange); value = sum over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (problem, n, p, use_oedg, use_ldf)
    "vortex512_p3": ("vortex", 512, 3, True, True),
    "vortex256_p3": ("vortex", 256, 3, True, True),
    "blast400_p2": ("blast", 400, 2, True, True),
    "ot64_p2": ("ot2pi", 64, 2, True, True),
}


FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12  # 148 SMs x 64 FP64 FMA/clk x 2 x 1.965 GHz

# the set-up parameters of each workload's problem (problems.make), repeated here so that the CPU
# baseline arm can describe its workload without importing anything that loads the CUDA library
PROBLEM_CFL = {"vortex": 0.6, "blast": 0.6, "ot2pi": 0.2}


def workload_config(name, n_gpus):
    """the `config` object of the JSON line, identical in both arms"""
    prob_name, n, p, oedg, ldf = WORKLOADS[name]
    dofs = 8 * n * n * (p + 1) ** 2
    return {"workload": name, "problem": prob_name, "mesh": f"{n}x{n}", "degree": p, "dofs": dofs,
            "rk": "SSP-RK3", "cfl": PROBLEM_CFL[prob_name], "oedg": oedg, "ldf": ldf, "pp": True,
            "parallelism": f"replicas{n_gpus}", "l2": l2_note(dofs * 8 * (n + 2) ** 2 / n ** 2)}


def l2_note(state_bytes, l2_bytes=126e6):
    mb = state_bytes / 1e6
    if state_bytes > l2_bytes:
        return "inputs larger than L2 (state %.0f MB per stage buffer, L2 126 MB)" % mb
    return "inputs fit in L2 (state %.1f MB per stage buffer); not flushed between steps" % mb


def fp64_gemm_tflops(device, n=8192, reps=4):
    """FP64 throughput measured on this GPU: a cuBLAS DGEMM (torch.matmul, float64) of n x n x n,
    timed with CUDA events after one warm-up; the denominator of the FP64 roofline (the kernels
    of the step use the FP64 FMA pipe, which the DGEMM figure bounds from above)"""
    import torch
    a = torch.rand(n, n, dtype=torch.float64, device=device)
    b = torch.rand(n, n, dtype=torch.float64, device=device)
    c = torch.matmul(a, b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record()
    for _ in range(reps):
        torch.matmul(a, b, out=c)
    e1.record()
    torch.cuda.synchronize(device)
    t = e0.elapsed_time(e1) * 1e-3 / reps
    del a, b, c
    return 2.0 * n ** 3 / t / 1e12


def algo_counts():
    with open(os.path.join(ROOT, "ALGO_COUNTS.json")) as f:
        return json.load(f)["per_degree"]


def measured_traffic(workload, kernel):
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            return json.load(f)[workload][kernel]["bytes_per_launch"]
    except Exception:
        return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (MEASURED_PEAKS.json absent: earlier STREAM-copy measurement on this pool)"


# ------------------------------------------------------------------------------ clocks sampling
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------ distributed
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    import datetime
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist, rank, ws, local


def max_over_ranks(dist, x, device=None):
    """max of a scalar over all ranks (the multi-GPU timing rule)"""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(dofs, steps, world, ms_max):
    """whole-job DOF-stage updates/s: 3 stage updates per SSP-RK3 step, summed over the replicas,
    over the slowest rank's device time"""
    return 3.0 * dofs * steps * world / (ms_max * 1e-3)


def barrier(dist, device=None):
    if dist is not None:
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ------------------------------------------------------------------------------ CPU legs
def cpu_sample(prob_name, n, p, use_oedg, use_ldf, budget_s=15.0, max_steps=50, threads=None):
    """time whole SSP-RK3 steps of the oracle (fast build, OpenMP) on the workload mesh"""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    from oracle import oracle as ora
    prob = pkg.problems.make(prob_name)
    u0 = prob.initial_state(n, n, p, nodes=ora.gll_tables(p)["x"])
    nthreads = threads or os.cpu_count()
    o = ora.OracleSolver(n, n, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state,
                         fast=True, threads=nthreads)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    o.solve(prob.final_T, prob.cfl, use_oedg, use_ldf, max_steps=1)  # prologue + 1 warm step
    t0 = time.perf_counter()
    o.solve(prob.final_T, prob.cfl, use_oedg, use_ldf, max_steps=1, resume=True)
    t1 = time.perf_counter() - t0
    k = max(1, min(max_steps, int(budget_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    o.solve(prob.final_T, prob.cfl, use_oedg, use_ldf, max_steps=k, resume=True)
    el = time.perf_counter() - t0
    dofs = 8 * n * n * (p + 1) ** 2
    o.close()
    return {"value": 3 * dofs * k / el, "unit": "DOF-stage/s", "cores": nthreads,
            "kind": "port", "sample": f"{k} SSP-RK3 steps of the full {n}x{n} p={p} mesh "
                                      f"(oracle -O3 -march=native, OpenMP {nthreads} threads)",
            "seconds": el}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference's path (no Fortran compiler here)."""
    if int(os.environ.get("RANK", "0")) != 0:  # under torchrun only rank 0 times the CPU path
        return
    prob_name, n, p, oedg, ldf = WORKLOADS[args.workload]
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    from oracle import oracle as ora
    prob = pkg.problems.make(prob_name)
    # the initial state at the oracle's own GLL nodes: nothing on this arm loads the CUDA library
    u0 = prob.initial_state(n, n, p, nodes=ora.gll_tables(p)["x"])
    nthreads = os.cpu_count()
    o = ora.OracleSolver(n, n, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state,
                         fast=True, threads=nthreads)
    o.set_state(u0[:, :, :, 1:-1, 1:-1])
    o.solve(prob.final_T, prob.cfl, oedg, ldf, max_steps=1)
    for _ in range(args.warmup):
        o.solve(prob.final_T, prob.cfl, oedg, ldf, max_steps=1, resume=True)
    t0 = time.perf_counter()
    o.solve(prob.final_T, prob.cfl, oedg, ldf, max_steps=args.steps, resume=True)
    el = time.perf_counter() - t0
    dofs = 8 * n * n * (p + 1) ** 2
    val = 3 * dofs * args.steps / el
    line = {
        "impl": "reference", "metric": "FP64 DOF-stage updates/s", "value": val, "unit": "DOF-stage/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic initial condition)",
        "config": workload_config(args.workload, args.gpus),
        "cpu_baseline": {"value": val, "unit": "DOF-stage/s", "cores": nthreads, "kind": "port",
                         "sample": f"{args.steps} SSP-RK3 steps of the full mesh per timed run "
                                   "(C restatement of the reference, -O3 -march=native, OpenMP; the "
                                   "Fortran reference cannot be compiled: no Fortran compiler)"},
        "e2e": {"value": val, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------ serving leg
HORIZON = {"ot2pi": 0.5, "rotor": 0.15, "blast": 0.01}


def make_requests(n_req, rate, seed, n_lo, n_hi, t_scale):
    """seeded request stream: Poisson arrivals at `rate`/s; problem in {OT, rotor, blast}; mesh N^2
    with N log-uniform in [n_lo, n_hi]; degree uniform in {1,2,3}; t_end uniform in [0.05, 0.5] x
    the problem's horizon (x t_scale)"""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(n_req):
        t += rng.exponential(1.0 / rate)
        name = ["ot2pi", "rotor", "blast"][int(rng.integers(0, 3))]
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        p = int(rng.integers(1, 4))
        t_end = float(rng.uniform(0.05, 0.5)) * HORIZON[name] * t_scale
        reqs.append(dict(id=i, name=name, n=n, p=p, t_end=t_end, arrival=t))
    return reqs


def serve(pkg, reqs, batched, budget, tries_per_round=2):
    srv = pkg.Server(budget, max_active=4096, tries_per_round=tries_per_round, batched=batched)
    for r in reqs:
        prob = pkg.problems.make(r["name"])
        srv.submit(r["id"], prob, r["n"], r["n"], r["p"], r["u0"], r["arrival"], final_T=r["t_end"])
    t0 = time.perf_counter()
    srv.run()
    wall = time.perf_counter() - t0
    res = srv.results()
    stats = srv.stats()
    srv.close()
    tts = np.array([x["finished"] - x["arrival"] for x in res])
    makespan = max(x["finished"] for x in res) - min(x["arrival"] for x in res)
    ok = sum(1 for x in res if x["done"] == 1 and x["flags"] == 0 and x["error"] == 0)
    # steady state: completions between the 10 % and the 90 % mark over that window (the ramp-up
    # and the tail, where the last runs execute nearly alone, left out)
    fin = np.sort(np.array([x["finished"] for x in res]))
    i10, i90 = int(0.1 * len(fin)), int(0.9 * len(fin)) - 1
    steady = (i90 - i10) / (fin[i90] - fin[i10]) if i90 > i10 and fin[i90] > fin[i10] else None
    return {"solves_per_s": len(res) / makespan, "steady_solves_per_s": steady,
            "p50_tts_s": float(np.percentile(tts, 50)),
            "p99_tts_s": float(np.percentile(tts, 99)), "completed": ok, "requests": len(reqs),
            "wall_s": wall, "steps": int(sum(x["steps"] for x in res)),
            "host_s": {k: round(stats[k], 4) for k in ("admit_s", "launch_s", "wait_s", "retire_s", "idle_s")},
            "rounds": stats["rounds"], "graph_captures": stats["graph_captures"]}


def pinned_copy(a):
    """a copy of the Fortran-ordered array `a` in pinned host memory (so that its upload is an
    asynchronous DMA instead of a copy through a staging buffer that blocks the host)"""
    import torch
    buf = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    out = buf.numpy().reshape(a.shape, order="F")
    out[...] = a  # the view's base chain holds the tensor, so the pinned buffer lives as long as it
    return out


def serve_leg(pkg, n_req, rates, n_hi, t_scale, seed=7, n_lo=32, budget=64 << 30):
    """one request stream served at each arrival rate in `rates`, batched and one run at a time,
    after an untimed pass of each (first-touch costs: module loading, the arena reservation).  The
    requests (problem, mesh, degree, t_end) are the same at every rate; only the Poisson arrival
    times scale with 1/rate.  Initial states sit in pinned host memory, as a serving host would
    keep its request buffers."""
    base = make_requests(n_req, 1.0, seed, n_lo, n_hi, t_scale)
    for r in base:
        r["u0"] = pinned_copy(pkg.problems.make(r["name"]).initial_state(r["n"], r["n"], r["p"]))
    # the untimed pass: the first requests at the fastest rate (base arrivals are at 1/s)
    warm = [dict(r, arrival=r["arrival"] / max(rates)) for r in base[: max(4, min(64, n_req // 8))]]
    serve(pkg, warm, True, budget)
    serve(pkg, warm, False, budget)
    out = {"stream": f"{n_req} requests, Poisson arrivals, seed {seed}, N log-uniform [{n_lo},{n_hi}], "
                     f"p in 1..3, problem in {{OT, rotor, blast}}, t_end U[0.05,0.5] x horizon x {t_scale:g}"}
    for rate in rates:
        reqs = [dict(r, arrival=r["arrival"] / rate) for r in base]
        b = serve(pkg, reqs, True, budget)
        q = serve(pkg, reqs, False, budget)
        bs, qs = b["steady_solves_per_s"], q["steady_solves_per_s"]
        out[f"rate_{rate:g}"] = {"batched": b, "one_at_a_time": q,
                                 "speedup_solves_per_s": b["solves_per_s"] / q["solves_per_s"],
                                 "speedup_steady": bs / qs if bs and qs else None}
    return out


# the served configuration of the scope table (N up to 512; t_end scaled by 0.05 so that the largest
# runs finish in seconds), and a stream of 1,000 small meshes with the scope table's t_end at two
# arrival rates (one that a single run at a time cannot keep up with, one that saturates both
# modes), where packing runs into one launch pays most
SERVE_STREAMS = {"spec_N32-512": dict(n_req=64, rates=[200.0], n_hi=512, t_scale=0.05),
                 "small_N32-96": dict(n_req=1000, rates=[100.0, 2000.0], n_hi=96, t_scale=1.0)}


def batched_leg(pkg, n_runs=512, steps=4, seed=11, n_lo=32, n_hi=256, sample=8):
    """the batched configuration of the scope table: n_runs independent runs (N ~ U[n_lo, n_hi],
    p ~ U{1,2,3}, IC in {OT, rotor}, amplitude ~ U[0.5, 1.5], gamma in {5/3, 1.4}), initial states
    evaluated on the device.  Timed with CUDA events: `steps` steps of every run one after another
    (each run's own CUDA graph), then the same from the same initial states as one batch (shared
    persistent launches, one CUDA graph per try); one untimed step and the graph captures come
    first in both.  `identical` counts sampled runs whose final state is bitwise the same both ways."""
    import torch
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n_runs):
        name = ["ot2pi", "rotor"][int(rng.integers(0, 2))]
        specs.append(dict(name=name, n=int(rng.integers(n_lo, n_hi + 1)), p=int(rng.integers(1, 4)),
                          amp=float(rng.uniform(0.5, 1.5)), gamma=[5.0 / 3.0, 1.4][int(rng.integers(0, 2))]))
    probs = [pkg.problems.make(sp["name"], gamma=sp["gamma"], amp=sp["amp"]) for sp in specs]
    runs = [pkg.DGSolver.for_problem(pr, sp["n"], sp["n"], sp["p"]) for pr, sp in zip(probs, specs)]
    dofs = sum(8 * sp["n"] ** 2 * (sp["p"] + 1) ** 2 for sp in specs)

    def start():  # initial state, then one untimed step each (loads kernels, builds each run's graph)
        for r, pr in zip(runs, probs):
            r.init_problem(pr)
            r.solve_begin(pr.final_T, pr.cfl)
            r.advance(1)
        torch.cuda.synchronize()

    # the calls below return only when their work is done, so events recorded on the default stream
    # just before and just after bracket it on the device
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start()
    e0.record()
    tries_solo = 0
    for r in runs:
        st = r.advance(steps, check_every=steps)
        tries_solo += st["steps"] + st["retries"]
    e1.record()
    torch.cuda.synchronize()
    ms_solo = e0.elapsed_time(e1)
    ref = [runs[i].download_state(0) for i in range(sample)]
    start()
    b = pkg.Batch()
    for r in runs:
        b.add(r)
    b.advance(0)  # uploads the tables and captures the batch graph, untimed
    torch.cuda.synchronize()
    e0.record()
    b.advance(steps)
    e1.record()
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1)
    sts = [b.status(r) for r in runs]
    for r in list(runs):
        b.remove(r)
    b.close()
    same = sum(int(np.array_equal(runs[i].download_state(0), ref[i], equal_nan=True)) for i in range(sample))
    for r in runs:
        r.close()
    stage_updates = 3 * dofs * steps
    return {"runs": n_runs, "dofs": dofs, "steps": steps,
            "batched": {"ms": ms_b, "dof_stage_per_s": stage_updates / (ms_b * 1e-3)},
            "one_after_another": {"ms": ms_solo, "dof_stage_per_s": stage_updates / (ms_solo * 1e-3)},
            "speedup": ms_solo / ms_b, "identical": f"{same}/{sample}",
            "retries": int(sum(s["retries"] for s in sts)),
            "config": f"{n_runs} runs, seed {seed}, N ~ U[{n_lo},{n_hi}], p ~ U{{1,2,3}}, IC in {{OT, rotor}}, "
                      f"amp ~ U[0.5,1.5], gamma in {{5/3, 1.4}}, {steps} SSP-RK3 steps each"}


# ------------------------------------------------------------------------------ GPU leg
def run_ours(args):
    import torch
    dist, rank, ws, local = dist_setup()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    prob_name, n, p, oedg, ldf = WORKLOADS[args.workload]
    prob = pkg.problems.make(prob_name)
    assert prob.cfl == PROBLEM_CFL[prob_name]
    u0 = prob.initial_state(n, n, p)
    dofs = 8 * n * n * (p + 1) ** 2
    stream = torch.cuda.Stream(device=device)
    solver = pkg.DGSolver.for_problem(prob, n, n, p)
    solver.set_stream(stream.cuda_stream)
    solver.upload_state(0, u0)
    solver.solve_begin(prob.final_T, prob.cfl, oedg, ldf, False)

    # ---- value: device-resident steps ----
    # clocks are sampled from the start of the warm-up (already under load) to the end of the
    # timed region
    sampler = ClockSampler(device.index)
    sampler.start()
    solver.advance(args.warmup)
    st0 = solver.status()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    with torch.cuda.stream(stream):
        ev0.record(stream)
    st_run = solver.advance(args.steps, check_every=max(1, args.steps))
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize(device)
    barrier(dist, device)
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    tries = st_run["steps"] - st0["steps"] + st_run["retries"] - st0["retries"]
    kernels_per_try = solver.step_graph_kernels()  # kernel nodes of the captured try graph
    ms_max = max_over_ranks(dist, ms, device)
    steps_done = st_run["steps"] - st0["steps"]

    # ---- roofline: the residual kernel timed alone on the same stream ----
    nrep = 20
    solver.semidiscretize(1, 0)
    ek0, ek1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    with torch.cuda.stream(stream):
        ek0.record(stream)
    lib = solver.lib
    for _ in range(nrep):
        lib.mhd_gpu_semidiscretize(solver.h, 1, 0, None)
    with torch.cuda.stream(stream):
        ek1.record(stream)
    torch.cuda.synchronize(device)
    t_res = ek0.elapsed_time(ek1) / nrep * 1e-3
    nodes = n * n * (p + 1) ** 2
    res_bytes = 2 * 64 * nodes  # read u (8 doubles/node) + write ut (8 doubles/node)
    hbm_peak, peak_kind = peaks()
    fp64_meas = fp64_gemm_tflops(device)
    achieved = res_bytes / t_res / 1e9
    counts = algo_counts()[str(p)]
    res_flops = counts["residual_per_element"]["total"] * n * n
    step_flops = counts["rk3_per_dof_stage"]["total"] * 3 * dofs

    # ---- e2e: host buffers through the C ABI, per step upload + step + download ----
    e2e = None
    if not args.no_e2e:
        host = torch.empty(u0.size, dtype=torch.float64, pin_memory=True)
        host_np = host.numpy().reshape(u0.shape, order="F")
        host_np[...] = u0
        out = torch.empty(u0.size, dtype=torch.float64, pin_memory=True)
        out_np = out.numpy().reshape(u0.shape, order="F")
        k_e2e = max(1, min(args.steps, 5))
        solver.upload_state(0, host_np)
        solver.solve_begin(prob.final_T, prob.cfl, oedg, ldf, False)
        solver.step()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            solver.upload_state(0, host_np)
            solver.step()
            solver.download_state(0, out_np)
        el = time.perf_counter() - t0
        el = max_over_ranks(dist, el, device)
        e2e = {"value": 3 * dofs * k_e2e * ws / el, "unit": "DOF-stage/s",
               "h2d_bytes_per_step": int(u0.nbytes), "d2h_bytes_per_step": int(u0.nbytes) + 64,
               "steps": k_e2e, "ms_per_step": 1e3 * el / k_e2e}

    roof_fp64 = {"bound": "fp64", "kernel": "residual_kernel", "achieved": res_flops / t_res / 1e12,
                 "peak": fp64_meas, "unit": "TFLOP/s", "frac": res_flops / t_res / 1e12 / fp64_meas,
                 "traffic": measured_traffic(args.workload, "residual_kernel"),
                 "algorithmic_flops_per_launch": res_flops, "algorithmic_bytes_per_launch": res_bytes,
                 "launch_ms": t_res * 1e3,
                 "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 (float64), CUDA events "
                                "(MEASURED_PEAKS.json has no FP64 figure)",
                 "nominal_peak": FP64_NOMINAL_TFLOPS,
                 "frac_of_nominal": res_flops / t_res / 1e12 / FP64_NOMINAL_TFLOPS,
                 "counting": "ALGO_COUNTS.json (log, /, sqrt count 1)"}
    roof_hbm = {"bound": "hbm", "kernel": "residual_kernel", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": measured_traffic(args.workload, "residual_kernel"),
                "algorithmic_bytes_per_launch": res_bytes, "launch_ms": t_res * 1e3, "peak_source": peak_kind}
    fp64_binds = res_flops / (fp64_meas * 1e12) >= res_bytes / (hbm_peak * 1e9)
    roof_main, roof_other = (roof_fp64, roof_hbm) if fp64_binds else (roof_hbm, roof_fp64)

    line = None
    if rank == 0:
        value = aggregate_value(dofs, steps_done, ws, ms_max)
        line = {
            "metric": "FP64 DOF-stage updates/s", "value": value, "unit": "DOF-stage/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / max(1, steps_done), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic initial condition)",
            "config": workload_config(args.workload, ws),
            "tries": tries,
            "gpu_launches": kernels_per_try * tries,
            # the binding side of the residual's roofline (the longer of flops at the FP64 peak
            # and bytes at the HBM peak) is the headline; the other side is reported beside it
            "roofline": roof_main,
            "roofline_other": roof_other,
            "step_roofline": {"algorithmic_flops_per_step": step_flops,
                              "algorithmic_bytes_per_step": 32 * 3 * dofs,
                              "roof_ms": max(step_flops / (fp64_meas * 1e12),
                                             32 * 3 * dofs / (hbm_peak * 1e9)) * 1e3,
                              "frac": max(step_flops / (fp64_meas * 1e12),
                                          32 * 3 * dofs / (hbm_peak * 1e9)) * 1e3 / (ms_max / max(1, steps_done))},
            "clocks": clocks,
        }
        if e2e:
            line["e2e"] = e2e
        t_leg = time.perf_counter()

        def progress(leg):  # wall time of each extra leg, on stderr (stdout carries the JSON line)
            nonlocal t_leg
            now = time.perf_counter()
            print(f"bench: {leg} leg {now - t_leg:.1f} s", file=sys.stderr, flush=True)
            t_leg = now

        if not args.no_batched and ws == 1:
            line["batched"] = batched_leg(pkg)
            progress("batched")
        if not args.no_serve and ws == 1:
            line["served"] = {}
            for k, kw in SERVE_STREAMS.items():
                line["served"][k] = serve_leg(pkg, **kw)
                progress(f"served {k}")
        if not args.no_cpu and ws == 1:
            line["cpu_baseline"] = cpu_sample(prob_name, n, p, oedg, ldf, budget_s=args.cpu_budget)
            progress("cpu baseline")
        print(json.dumps(line), flush=True)
    solver.close()
    if dist:
        barrier(dist, device)
        dist.destroy_process_group()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="vortex512_p3", choices=sorted(WORKLOADS))
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
