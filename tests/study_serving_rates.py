"""The small-mesh served stream at several arrival rates (GPU; not collected by pytest -- run it
directly).

The bench serves the stream of small meshes (N log-uniform in [32, 96], p in 1..3, problem in
{OT, rotor, blast}, unshortened t_end) at 100 and 2000 requests/s.  This study serves the same
requests (the first REQUESTS of the bench's seeded stream) at other arrival rates, batched and one
run at a time, and prints one JSON line per rate: solves/s overall and between the 10 % and 90 %
completion marks, p50/p99 time-to-solution, and the host's admission time.

    python tests/study_serving_rates.py [--rates 10,100,500,2000] [--requests 1000]
"""
import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="10,100,500,2000", help="arrival rates, requests/s")
    ap.add_argument("--requests", type=int, default=1000)
    a = ap.parse_args()
    import bench
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    rates = [float(r) for r in a.rates.split(",")]
    kw = dict(bench.SERVE_STREAMS["small_N32-96"])
    kw.update(n_req=a.requests, rates=rates)
    out = bench.serve_leg(pkg, **kw)
    keep = ("solves_per_s", "steady_solves_per_s", "p50_tts_s", "p99_tts_s", "completed", "wall_s")
    for rate in rates:
        r = out[f"rate_{rate:g}"]
        line = {"stream": out["stream"], "rate": rate}
        for mode in ("batched", "one_at_a_time"):
            line[mode] = {k: r[mode][k] for k in keep}
            line[mode]["admit_s"] = r[mode]["host_s"]["admit_s"]
        line["speedup_solves_per_s"] = r["speedup_solves_per_s"]
        line["speedup_steady"] = r["speedup_steady"]
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
