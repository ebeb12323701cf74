"""The C-ABI library loads and exports every function include/mhd_gpu.h declares (CPU, no GPU compute)."""
import ctypes as C
import os
import re

import numpy as np

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mhd_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mhd_(?:gpu|batch|server)_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported(pkg):
    lib = C.CDLL(pkg.capi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares exactly the header's functions
    assert sorted(pkg.capi.SIGNATURES) == names


def test_status_strings(pkg):
    cap = pkg.capi
    assert cap.status_string(0) == "ok"
    assert "average" in cap.status_string(cap.MHD_FLAG_NEG_AVG)
    assert "CUDA" in cap.status_string(cap.MHD_ERR_CUDA)


def test_host_only_entry_points(pkg):
    lib = pkg.capi.load()
    dp = C.POINTER(C.c_double)
    x = np.zeros(4)
    assert lib.mhd_gpu_gll_tables(3, x.ctypes.data_as(dp), None, None, None, None, None, None) == 0
    assert lib.mhd_gpu_gll_tables(7, x.ctypes.data_as(dp), None, None, None, None, None, None) < 0
    A = np.zeros((32, 32))
    assert lib.mhd_gpu_ldf_operator(3, 0.1, 0.1, A.ctypes.data_as(dp)) == 0
    assert lib.mhd_gpu_ldf_operator(3, -0.1, 0.1, A.ctypes.data_as(dp)) < 0


def test_create_rejects_bad_arguments_before_touching_a_device(pkg):
    lib = pkg.capi.load()
    h = C.c_void_p()
    # unsupported degree / unequal degrees / bad rknstg / bad domain
    assert lib.mhd_gpu_create(8, 8, 4, 4, 3, 0.0, 1.0, 0.0, 1.0, 1.4, 0, None, C.byref(h)) == pkg.capi.MHD_ERR_UNSUPPORTED
    assert lib.mhd_gpu_create(8, 8, 2, 1, 3, 0.0, 1.0, 0.0, 1.0, 1.4, 0, None, C.byref(h)) == pkg.capi.MHD_ERR_UNSUPPORTED
    assert lib.mhd_gpu_create(8, 8, 2, 2, 4, 0.0, 1.0, 0.0, 1.0, 1.4, 0, None, C.byref(h)) == pkg.capi.MHD_ERR_UNSUPPORTED
    assert lib.mhd_gpu_create(8, 8, 2, 2, 3, 1.0, 0.0, 0.0, 1.0, 1.4, 0, None, C.byref(h)) == pkg.capi.MHD_ERR_INVALID
    assert lib.mhd_gpu_create(8, 8, 2, 2, 3, 0.0, 1.0, 0.0, 1.0, 1.4, 2, None, C.byref(h)) == pkg.capi.MHD_ERR_INVALID
    assert not h.value


def test_struct_layouts_match_the_header(pkg, tmp_path):
    """the ctypes mirrors of the header's structs have the C sizes and field offsets (gcc-compiled probe)"""
    import subprocess
    cap = pkg.capi
    structs = {"mhd_gpu_status": cap.Status, "mhd_request": cap.Request,
               "mhd_request_result": cap.RequestResult, "mhd_server_stats": cap.ServerStats,
               "mhd_log_entry": cap.LogEntry}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "mhd_gpu.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_set_up_entry_points_reject_bad_arguments(pkg):
    lib = pkg.capi.load()
    assert lib.mhd_gpu_set_log(None, 16, 0) == pkg.capi.MHD_ERR_INVALID
    n = C.c_int()
    assert lib.mhd_gpu_read_log(None, None, 0, C.byref(n), None) == pkg.capi.MHD_ERR_INVALID
    assert lib.mhd_gpu_init_problem(None, 0, None, 0) == pkg.capi.MHD_ERR_INVALID
    assert lib.mhd_gpu_download_avg_primitive(None, None, None, None) == pkg.capi.MHD_ERR_INVALID


def test_every_problem_has_a_device_initial_state(pkg):
    for name in ("ot2pi", "ot_unit", "vortex", "blast", "rotor", "alfven", "cloud_shock", "jet"):
        pid, params = pkg.problems.make(name).device_ic()
        assert 0 <= pid <= 7 and len(params) in (1, 2, 5)


def test_autotune_candidates_are_well_formed():
    """every candidate set of the residual autotuner gives each degree whole warps within one CTA"""
    import importlib.util
    spec = importlib.util.spec_from_file_location("autotune", os.path.join(ROOT, "pp-es-dg-mhd_b200", "autotune.py"))
    at = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(at)
    sets = {len(c) for c in at.CANDIDATES.values()}
    assert len(sets) == 1  # set i takes candidate i of every degree
    for p, cands in at.CANDIDATES.items():
        for tx, ty, nt, minb in cands:
            # one lane per node: a warp holds 32 // (p+1)^2 elements
            assert nt % 32 == 0 and nt <= 1024 and tx >= 1 and ty >= 1 and minb >= 1
            assert tx * ty <= (nt // 32) * (32 // (p + 1) ** 2)


def test_tuned_header_defines_every_degree():
    path = os.path.join(ROOT, "pp-es-dg-mhd_b200", "csrc", "residual2_tuned.h")
    if not os.path.exists(path):
        return
    text = open(path).read()
    for p in (1, 2, 3):
        m = re.search(rf"#define MHD_RES2_CFG{p} (\d+), (\d+), (\d+), (\d+)", text)
        assert m, p
        tx, ty, nt, minb = map(int, m.groups())
        assert nt % 32 == 0 and tx * ty <= (nt // 32) * (32 // (p + 1) ** 2)


def test_noalloc_rejects_misaligned_and_overlapping_buffers_on_the_host(pkg):
    """mhd_gpu_semidiscretize_noalloc checks its caller's pointers before any CUDA call: the
    pointers below are never dereferenced (no GPU here)."""
    lib = pkg.capi.load()
    base = 1 << 24
    bad = pkg.capi.MHD_ERR_INVALID
    # 8-byte aligned but not 16-byte aligned: an offset into a caller's own pool
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 8, 8, 0.1, 0.1, 1.4, C.c_void_p(base + 8),
                                              C.c_void_p(base + (1 << 20)), None, None) == bad
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 8, 8, 0.1, 0.1, 1.4, C.c_void_p(base),
                                              C.c_void_p(base + (1 << 20) + 8), None, None) == bad
    # ut overlapping u (either order)
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 8, 8, 0.1, 0.1, 1.4, C.c_void_p(base),
                                              C.c_void_p(base + 4096), None, None) == bad
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 8, 8, 0.1, 0.1, 1.4, C.c_void_p(base + 4096),
                                              C.c_void_p(base), None, None) == bad
