"""Per-degree tuning of the stage kernels on the GPU at hand.

    python pp-es-dg-mhd_b200/autotune.py [--what residual|post|all] [--jobs J]

Two groups of build-time knobs, each a macro per degree p = 1, 2, 3:

  residual  MHD_RES2_CFG<p> = TX, TY, threads, CTAs per SM of the residual tile (csrc/residual.cuh;
            a tile holds at most (threads / 32) * (32 / (p+1)^2) elements, one lane per node).
            Timed: the residual alone, CUDA events over 20 launches.  Written to
            csrc/residual2_tuned.h.
  post      MHD_PP_CFG<p> = threads, CTAs per SM of the loop-1 and loop-3 kernels, and
            MHD_SIG_CFG<p> = TX, TY, CTAs per SM of the OEDG indicator kernel (csrc/post.cuh).
            Timed: whole device-resident SSP-RK3 steps (OEDG + LDF + PP), CUDA events over 10
            steps, since those kernels share the step with the residual.  Written to
            csrc/post_tuned.h.

The library is built once per candidate set (set i takes candidate i of every degree), in parallel;
each set is timed in its own process on a vortex mesh of about 33 M DOFs per degree, and the
fastest candidate per degree is written to the group's header, which the next build picks up
(build.py rebuilds when it changes).  A set that does not build (a tile that does not fit one CTA's
shared memory, for instance) is skipped.  Needs a GPU for the timing.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build as B  # noqa: E402

# group -> macro(s) -> per degree the candidates; set i takes candidate i of every degree
GROUPS = {
    "residual": {
        "MHD_RES2_CFG": {  # 128 threads at 4, 5 and 6 CTAs per SM (128, 102, 85 registers), 256 at 3
            1: [(8, 4, 128, 4), (8, 4, 128, 5), (8, 4, 128, 6), (8, 8, 256, 3)],
            2: [(4, 3, 128, 4), (4, 3, 128, 5), (4, 3, 128, 6), (6, 4, 256, 3)],
            3: [(4, 2, 128, 4), (4, 2, 128, 5), (4, 2, 128, 6), (8, 2, 256, 3)],
        },
    },
    "post": {  # sets 1 and 2 vary the indicator kernel, set 3 loops 1 and 3, against set 0
        "MHD_PP_CFG": {
            1: [(256, 4), (256, 4), (256, 4), (128, 8)],
            2: [(256, 4), (256, 4), (256, 4), (128, 8)],
            3: [(256, 4), (256, 4), (256, 4), (128, 8)],
        },
        "MHD_SIG_CFG": {
            1: [(8, 8, 3), (8, 8, 4), (8, 4, 4), (8, 8, 3)],
            2: [(8, 4, 3), (8, 4, 4), (4, 4, 4), (8, 4, 3)],
            3: [(4, 4, 2), (4, 4, 4), (4, 4, 3), (4, 4, 2)],
        },
    },
}
HEADERS = {"residual": "residual2_tuned.h", "post": "post_tuned.h"}
CANDIDATES = GROUPS["residual"]["MHD_RES2_CFG"]  # the residual tiles (checked by the CPU tests)
MESHES = {1: 724, 2: 512, 3: 512}  # vortex, about 33 M DOFs each


def nsets(group):
    counts = {len(c) for m in GROUPS[group].values() for c in m.values()}
    assert len(counts) == 1, "every macro of a group needs the same number of candidates"
    return counts.pop()


def build_set(group, i, tmp):
    hdr = os.path.join(tmp, f"{group}{i}.h")
    with open(hdr, "w") as f:
        for macro, per_p in GROUPS[group].items():
            for p, cands in per_p.items():
                f.write(f"#define {macro}{p} {', '.join(map(str, cands[i]))}\n")
    objs = []
    try:
        for src in B.SOURCES:
            obj = os.path.join(tmp, f"{group}{i}_{os.path.splitext(src)[0]}.o")
            cmd = [B.nvcc(), *B.NVCC_FLAGS, "-include", hdr, "-I", os.path.join(B.ROOT, "include"),
                   "-x", "cu" if src.endswith(".cu") else "c++", "-c", os.path.join(B.CSRC, src), "-o", obj]
            subprocess.run(cmd, check=True, capture_output=True)
            objs.append(obj)
        lib = os.path.join(tmp, f"{group}{i}.so")
        subprocess.run([B.nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib, *objs,
                        "-lcudart"], check=True, capture_output=True)
        return lib
    except subprocess.CalledProcessError:
        return None


TIMER = r"""
import json, sys
sys.path.insert(0, sys.argv[2])
import torch
import __graft_entry__ as ge
pkg = ge.load_package()
pkg.capi.load(sys.argv[1])
what = sys.argv[4]
out = {}
for p, n in json.loads(sys.argv[3]).items():
    prob = pkg.problems.make("vortex")
    s = pkg.DGSolver.for_problem(prob, n, n, int(p))
    st = torch.cuda.Stream()
    s.set_stream(st.cuda_stream)
    s.init_problem(prob)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if what == "residual":
        s.apply_bc(0)
        for _ in range(3):
            s.lib.mhd_gpu_semidiscretize(s.h, 1, 0, None)
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            e0.record(st)
        for _ in range(20):
            s.lib.mhd_gpu_semidiscretize(s.h, 1, 0, None)
        with torch.cuda.stream(st):
            e1.record(st)
        torch.cuda.synchronize()
        out[p] = e0.elapsed_time(e1) / 20
    else:
        s.solve_begin(prob.final_T, prob.cfl, True, True, False)
        s.advance(3)
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            e0.record(st)
        r = s.advance(10, check_every=10)
        with torch.cuda.stream(st):
            e1.record(st)
        torch.cuda.synchronize()
        out[p] = e0.elapsed_time(e1) / 10
    s.close()
print(json.dumps(out))
"""


def tune(group, jobs):
    n = nsets(group)
    with tempfile.TemporaryDirectory() as tmp:
        with ThreadPoolExecutor(jobs) as ex:
            libs = list(ex.map(lambda i: build_set(group, i, tmp), range(n)))
        times = {}
        for i, lib in enumerate(libs):
            if lib is None:
                print(f"{group} set {i}: does not build, skipped", flush=True)
                continue
            r = subprocess.run([sys.executable, "-c", TIMER, lib, B.ROOT, json.dumps(MESHES), group],
                               capture_output=True, text=True)
            if r.returncode:
                print(f"{group} set {i}: timing failed, skipped\n{r.stderr[-400:]}", flush=True)
                continue
            times[i] = {int(p): ms for p, ms in json.loads(r.stdout.strip().splitlines()[-1]).items()}
            print(f"{group} set {i}: {times[i]}", flush=True)
    if not times:
        sys.exit(f"no {group} candidate set could be timed")
    write_header(group, times)


MARGIN = 0.01  # run-to-run spread of these timings on one GPU


def pick(times, p):
    """the fastest set for degree p; set 0 (the incumbent) unless another beats it by more than
    MARGIN, so that timing noise does not swap in a candidate with more spilled registers"""
    best = min(times, key=lambda i: times[i][p])
    if 0 in times and times[best][p] >= (1.0 - MARGIN) * times[0][p]:
        return 0
    return best


def write_header(group, times):
    """times[set][p] in ms -> the group's header with the chosen candidate per degree"""
    unit = "residual ms per launch" if group == "residual" else "ms per SSP-RK3 step (OEDG + LDF + PP)"
    lines = [f"// {HEADERS[group]} -- written by autotune.py: the fastest candidate per degree on this GPU",
             f"// ({unit}, vortex mesh of about 33 M DOFs; set 0 stays unless another is faster by more",
             f"// than {100 * MARGIN:.0f} %)."]
    for p in (1, 2, 3):
        best = pick(times, p)
        for i in sorted(times):
            knobs = "; ".join(f"{m} {GROUPS[group][m][p][i]}" for m in GROUPS[group])
            lines.append(f"//   p={p} {knobs}: {times[i][p]:.4f} ms{'  <- chosen' if i == best else ''}")
        for macro, per_p in GROUPS[group].items():
            lines += [f"#ifndef {macro}{p}", f"#define {macro}{p} {', '.join(map(str, per_p[p][best]))}", "#endif"]
    path = os.path.join(B.CSRC, HEADERS[group])
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(open(path).read())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--what", default="all", choices=["residual", "post", "all"])
    ap.add_argument("--jobs", type=int, default=4)
    args = ap.parse_args()
    for group in (["residual", "post"] if args.what == "all" else [args.what]):
        tune(group, args.jobs)
        B.build()  # the next group is timed with this group's choice built in


if __name__ == "__main__":
    main()
