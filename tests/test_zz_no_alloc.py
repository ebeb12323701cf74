"""The allocation-free residual entry point (mhd_gpu_semidiscretize_noalloc) against the regular one.

Some callers cannot let this library allocate device memory: hosts that reserved their whole
device-memory budget up front in their own pool, devices whose allocations are capped by an external
manager, and time-critical loops that cannot take the device-wide synchronisation an allocation may
cause.  For them the library offers one entry point that works on caller-owned device buffers and
keeps its only scratch (the dt_lim reduction cell) in a static device array.

This test (GPU) fills a state through a regular solver handle, runs the regular
mhd_gpu_semidiscretize on it, then calls the allocation-free entry point twice in a row through the
C ABI, writing into a buffer this test owns, and compares ut and dt_lim each time.  The tolerance is
the parity bar of the other GPU tests: relative L1 <= 1e-12 per conserved variable, dt_lim relative
1e-13.  A second case runs in a fresh child process in which the allocation-free call is the first
call into the library (so the call itself does the device set-up) and checks it against the CPU
oracle; the file runs last in the suite, after every other GPU test.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import rel_l1

pytestmark = pytest.mark.gpu


def _blocked_to_fortran(flat, nx, ny, p):
    n = p + 1
    a = flat.reshape(ny, nx, 8, n, n)          # [j][i][var][l][k]
    return np.asfortranarray(a.transpose(2, 4, 3, 1, 0))  # (8, k, l, i, j)


@pytest.mark.parametrize("name,nx,ny,p", [("ot2pi", 16, 12, 2), ("vortex", 10, 9, 3), ("blast", 12, 12, 1)])
def test_noalloc_residual_matches_regular_entry_point(pkg, name, nx, ny, p):
    import torch
    prob = pkg.problems.make(name)
    u0 = prob.initial_state(nx, ny, p)
    lib = pkg.capi.load()
    with pkg.DGSolver.for_problem(prob, nx, ny, p) as g:
        g.upload_state(0, u0)
        g.apply_bc(0)
        dl_ref = g.semidiscretize(1, 0)
        ut_ref = g.download_ut(1)
        g.synchronize()
        u_dev = g.state_device_ptr(0)
        hx = (prob.domain[1] - prob.domain[0]) / nx
        hy = (prob.domain[3] - prob.domain[2]) / ny
        ut_buf = torch.full((nx * ny * 8 * (p + 1) ** 2,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        for call in range(2):
            dl = C.c_double(0.0)
            rc = lib.mhd_gpu_semidiscretize_noalloc(p, nx, ny, hx, hy, prob.gamma, C.c_void_p(u_dev),
                                                    C.c_void_p(ut_buf.data_ptr()), C.byref(dl), None)
            assert rc == 0, pkg.capi.status_string(rc)
            torch.cuda.synchronize()
            ut = _blocked_to_fortran(ut_buf.cpu().numpy(), nx, ny, p)
            err = rel_l1(ut, ut_ref)
            assert err.max() <= 1e-12, (call, err)
            assert abs(dl.value - dl_ref) <= 1e-13 * dl_ref, (call, dl.value, dl_ref)
            ut_buf.fill_(float("nan"))


def test_noalloc_rejects_sizes_beyond_its_limits(pkg):
    lib = pkg.capi.load()
    bogus = C.c_void_p(16)  # never dereferenced: the call must reject before touching the GPU
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 4097, 8, 0.1, 0.1, 1.4, bogus, bogus, None, None) == pkg.capi.MHD_ERR_UNSUPPORTED
    assert lib.mhd_gpu_semidiscretize_noalloc(4, 8, 8, 0.1, 0.1, 1.4, bogus, bogus, None, None) == pkg.capi.MHD_ERR_UNSUPPORTED
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 8, 8, -0.1, 0.1, 1.4, bogus, bogus, None, None) == pkg.capi.MHD_ERR_INVALID
    # pointers that are never dereferenced: misaligned (odd multiple of 8 bytes) and overlapping
    base = 1 << 24
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 8, 8, 0.1, 0.1, 1.4, C.c_void_p(base + 8),
                                              C.c_void_p(base + (1 << 20)), None, None) == pkg.capi.MHD_ERR_INVALID
    assert lib.mhd_gpu_semidiscretize_noalloc(2, 8, 8, 0.1, 0.1, 1.4, C.c_void_p(base),
                                              C.c_void_p(base + 4096), None, None) == pkg.capi.MHD_ERR_INVALID


def _fortran_to_blocked(u):
    """(8, k, l, i, j) Fortran layout -> flat element-blocked [j][i][var][l][k]"""
    return np.ascontiguousarray(u.transpose(4, 3, 0, 2, 1)).reshape(-1)


def _first_call_in_a_fresh_process():
    """child process: the allocation-free residual is the first call into the library"""
    import torch
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    from oracle import oracle as ora
    name, nx, ny, p = "ot2pi", 12, 10, 2
    prob = pkg.problems.make(name)
    u = np.asfortranarray(prob.initial_state(nx, ny, p))
    o = ora.OracleSolver(nx, ny, p, p, 3, *prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)
    o.apply_bc(u)
    ut_ref, dl_ref = o.semidiscretize(u)
    lib = pkg.capi.load()
    u_dev = torch.from_numpy(_fortran_to_blocked(u)).cuda()
    ut_dev = torch.full((nx * ny * 8 * (p + 1) ** 2,), float("nan"), dtype=torch.float64, device="cuda")
    hx = (prob.domain[1] - prob.domain[0]) / nx
    hy = (prob.domain[3] - prob.domain[2]) / ny
    for call in range(2):
        dl = C.c_double(0.0)
        rc = lib.mhd_gpu_semidiscretize_noalloc(p, nx, ny, hx, hy, prob.gamma, C.c_void_p(u_dev.data_ptr()),
                                                C.c_void_p(ut_dev.data_ptr()), C.byref(dl), None)
        assert rc == 0, pkg.capi.status_string(rc)
        torch.cuda.synchronize()
        ut = _blocked_to_fortran(ut_dev.cpu().numpy(), nx, ny, p)
        err = rel_l1(ut, ut_ref, floor_frac=1e-2)
        assert err.max() <= 1e-12, (call, err)
        assert abs(dl.value - dl_ref) <= 1e-13 * dl_ref, (call, dl.value, dl_ref)
        ut_dev.fill_(float("nan"))
    print("fresh-process no-alloc ok")


def test_noalloc_first_call_in_a_fresh_process_sets_the_device_up():
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--fresh-process"], cwd=here,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "fresh-process no-alloc ok" in r.stdout


if __name__ == "__main__" and "--fresh-process" in sys.argv:
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    _first_call_in_a_fresh_process()
