"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/mhd_oracle.c`` with gcc into ``oracle/_build/libmhd_oracle.so``.
Two flavours are built:

* ``libmhd_oracle.so``      -- ``-O2 -ffp-contract=off``: every operation rounded as written in
  the reference source; used as the parity checker.
* ``libmhd_oracle_fast.so`` -- ``-O3 -march=native -ffp-contract=fast``: the same source built the
  way the reference's README builds itself (``gfortran -O3 -march=native``); used only as the timed
  CPU baseline.

The reference itself (Fortran 2008) cannot be compiled on this machine: no gfortran/ifx/flang and
no LAPACK are installed, so ``oracle/_ref`` stays empty.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
SRC = os.path.join(HERE, "mhd_oracle.c")

FLAVOURS = {
    "libmhd_oracle.so": ["-O2", "-ffp-contract=off", "-fno-fast-math"],
    "libmhd_oracle_fast.so": ["-O3", "-march=native", "-ffp-contract=fast", "-fno-fast-math"],
}


def build(force: bool = False, verbose: bool = False) -> dict:
    os.makedirs(BUILD, exist_ok=True)
    out = {}
    for name, flags in FLAVOURS.items():
        target = os.path.join(BUILD, name)
        out[name] = target
        if (not force and os.path.exists(target)
                and os.path.getmtime(target) >= max(os.path.getmtime(SRC),
                                                     os.path.getmtime(SRC[:-1] + "h"))):
            continue
        cmd = ["gcc", "-std=c11", "-shared", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-variable",
               "-Wno-unused-but-set-variable", *flags, SRC, "-o", target + ".tmp", "-lm"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(target + ".tmp", target)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
