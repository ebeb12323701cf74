"""Per-degree tuning of the residual kernel on the GPU at hand.

    python pp-es-dg-mhd_b200/autotune.py [--out PATH] [--jobs J]

Builds the library once per candidate set (every set gives each degree p = 1, 2, 3 one tile
configuration TX, TY, threads, CTAs per SM -- the MHD_RES2_CFG<p> macros of csrc/residual.cuh; a
tile holds at most (threads / 32) * (32 / (p+1)^2) elements, one lane per node), times the residual
of each degree on a large mesh with CUDA events (each set in its own process), and writes the
fastest configuration per degree as a header (csrc/residual2_tuned.h by default), which the next
build picks up.  Candidates whose tile does not
fit one CTA's shared memory fail to compile and are skipped.  Needs a GPU for the timing.
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

# (TX, TY, NT, MINB) per degree; set i takes candidate i of every degree
CANDIDATES = {
    1: [(8, 8, 256, 2), (8, 4, 128, 4), (8, 6, 192, 3), (16, 4, 256, 2)],
    2: [(6, 4, 256, 2), (4, 3, 128, 4), (6, 3, 192, 3), (8, 3, 256, 2)],
    3: [(4, 4, 256, 2), (4, 2, 128, 4), (4, 3, 192, 3), (8, 2, 256, 2)],
}
MESHES = {1: 724, 2: 512, 3: 512}  # vortex, about 33 M DOFs each


def build_set(i, tmp):
    hdr = os.path.join(tmp, f"cfg{i}.h")
    with open(hdr, "w") as f:
        for p, cands in CANDIDATES.items():
            f.write(f"#define MHD_RES2_CFG{p} {', '.join(map(str, cands[i]))}\n")
    objs = []
    try:
        for src in B.SOURCES:
            obj = os.path.join(tmp, f"set{i}_{os.path.splitext(src)[0]}.o")
            cmd = [B.nvcc(), *B.NVCC_FLAGS, "-include", hdr, "-I", os.path.join(B.ROOT, "include"),
                   "-x", "cu" if src.endswith(".cu") else "c++", "-c", os.path.join(B.CSRC, src), "-o", obj]
            subprocess.run(cmd, check=True, capture_output=True)
            objs.append(obj)
        lib = os.path.join(tmp, f"set{i}.so")
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
out = {}
for p, n in json.loads(sys.argv[3]).items():
    prob = pkg.problems.make("vortex")
    s = pkg.DGSolver.for_problem(prob, n, n, int(p))
    st = torch.cuda.Stream()
    s.set_stream(st.cuda_stream)
    s.init_problem(prob)
    s.apply_bc(0)
    for _ in range(3):
        s.lib.mhd_gpu_semidiscretize(s.h, 1, 0, None)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        e0.record(st)
    for _ in range(20):
        s.lib.mhd_gpu_semidiscretize(s.h, 1, 0, None)
    with torch.cuda.stream(st):
        e1.record(st)
    torch.cuda.synchronize()
    out[p] = e0.elapsed_time(e1) / 20
    s.close()
print(json.dumps(out))
"""


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(B.CSRC, "residual2_tuned.h"))
    ap.add_argument("--jobs", type=int, default=4)
    args = ap.parse_args()
    nsets = len(CANDIDATES[1])
    with tempfile.TemporaryDirectory() as tmp:
        with ThreadPoolExecutor(args.jobs) as ex:
            libs = list(ex.map(lambda i: build_set(i, tmp), range(nsets)))
        times = {}
        for i, lib in enumerate(libs):
            if lib is None:
                print(f"set {i}: does not build, skipped", flush=True)
                continue
            r = subprocess.run([sys.executable, "-c", TIMER, lib, B.ROOT, json.dumps(MESHES)],
                               capture_output=True, text=True)
            if r.returncode:
                print(f"set {i}: timing failed, skipped\n{r.stderr[-400:]}", flush=True)
                continue
            times[i] = {int(p): ms for p, ms in json.loads(r.stdout.strip().splitlines()[-1]).items()}
            print(f"set {i}: {times[i]}", flush=True)
    if not times:
        sys.exit("no candidate set could be timed")
    lines = ["// residual2_tuned.h -- written by autotune.py: residual tile per degree, fastest of the",
             "// candidates timed on this GPU (residual ms per launch, vortex mesh of about 33 M DOFs)."]
    for p in (1, 2, 3):
        best = min(times, key=lambda i: times[i][p])
        for i in sorted(times):
            lines.append(f"//   p={p} {CANDIDATES[p][i]}: {times[i][p]:.4f} ms{'  <- chosen' if i == best else ''}")
        lines += [f"#ifndef MHD_RES2_CFG{p}", f"#define MHD_RES2_CFG{p} {', '.join(map(str, CANDIDATES[p][best]))}",
                  "#endif"]
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(open(args.out).read())


if __name__ == "__main__":
    main()
