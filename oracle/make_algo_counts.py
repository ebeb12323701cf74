"""Build oracle/flop_count.cpp (the oracle compiled with an operation-counting double) and write
ALGO_COUNTS.json at the repository root: the algorithmic FP64 operation counts per element / per
DOF-stage that bench.py's FP64 roofline uses.  Measurement infrastructure only.

    python oracle/make_algo_counts.py
"""
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def main():
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    exe = os.path.join(HERE, "_build", "flop_count")
    subprocess.run(["g++", "-std=c++17", "-O1", "-w", "-I", HERE, os.path.join(HERE, "flop_count.cpp"),
                    "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    data = json.loads(out)
    data["generated_by"] = "oracle/make_algo_counts.py (oracle/flop_count.cpp)"
    with open(os.path.join(ROOT, "ALGO_COUNTS.json"), "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")
    return data


if __name__ == "__main__":
    d = main()
    for p, v in d["per_degree"].items():
        print(p, "residual/element", v["residual_per_element"]["total"],
              "rk3/DOF-stage", round(v["rk3_per_dof_stage"]["total"], 2))
