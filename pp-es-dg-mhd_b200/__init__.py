"""pp_es_dg_mhd_b200 -- B200 (sm_100a) per-stage DG update for 2D ideal MHD.

Host-side mirror of the reference's solver interface (YueWu2002/PP-ES-DG-MHD), over the C ABI of
include/mhd_gpu.h:

    reference (Fortran)                                   here
    init_DG_solver(nx,ny,px,py,rknstg,l,r,b,t)            DGSolver(nx, ny, p, rknstg, domain, gamma, bc)
      DG_solver.f90:47
    post_process(u, u_avg, neg_avg, num_negcell, ...)     DGSolver.post_process(slot, ...)
      DG_solver.f90:128
    DG_semidiscretize(ut(:,s), dt_lim, u)                 DGSolver.semidiscretize(stage, slot)
      DG_solver.f90:663
    BC_handle(u, ...)            drive.f90:25             DGSolver.apply_bc(slot)
    stage update                 drive.f90:130-275        DGSolver.rk_combine(stage, dt)
    step acceptance              drive.f90:304-311        DGSolver.rk_accept()
    solve_execute(final_T, CFL, use_oedg, use_LDF,        DGSolver.solve_execute(...)
                  ent_offset)    drive.f90:32
    finalize_DG_solver           DG_solver.f90:109        DGSolver.close()

State arrays cross the boundary in the reference's Fortran layouts (numpy, order='F').
The reference stops the program (`error stop`) on fatal conditions; here those raise MHDError.
All compute runs in the CUDA library; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import capi, problems
from .capi import (BC_EXTRAPOLATE, BC_FIXED, BC_PERIODIC, BC_XEXTRAP_YPER, MHDError, Status)

__all__ = ["DGSolver", "Batch", "Server", "footprint", "MHDError", "capi", "problems", "BC_PERIODIC", "BC_EXTRAPOLATE",
           "BC_FIXED", "BC_XEXTRAP_YPER", "library_path", "ldf_operator"]

_dp = C.POINTER(C.c_double)


def library_path():
    return capi.LIB_PATH


def _p(a):
    return a.ctypes.data_as(_dp)


def ldf_operator(p, hx, hy):
    """Dense nodal LDF operator of the library (host-only, no GPU needed)."""
    n2 = 2 * (p + 1) ** 2
    A = np.zeros((n2, n2), order="F")
    rc = capi.load().mhd_gpu_ldf_operator(int(p), float(hx), float(hy), _p(A))
    if rc:
        raise MHDError("mhd_gpu_ldf_operator", rc)
    return A


def _check(fn, rc, fatal_flags=True):
    if rc < 0 or (fatal_flags and rc & (capi.MHD_FLAG_PP_RELIMIT | capi.MHD_FLAG_DT_COLLAPSE |
                                        capi.MHD_FLAG_INIT_NEG_AVG | capi.MHD_FLAG_DEVICE_WAIT)):
        raise MHDError(fn, rc)
    return rc


class DGSolver:
    """One solver instance (the reference's DG_solver_m module state, but per object)."""

    def __init__(self, nx, ny, p, rknstg=3, domain=(0.0, 1.0, 0.0, 1.0), gamma=5.0 / 3.0,
                 bc_kind=BC_PERIODIC, bc_state=None):
        self.lib = capi.load()
        self.nx, self.ny, self.p, self.rknstg = nx, ny, p, rknstg
        self.domain, self.gamma, self.bc_kind = tuple(domain), gamma, bc_kind
        n = p + 1
        self.shape_u = (8, n, n, nx + 2, ny + 2)
        self.shape_ut = (8, n, n, nx, ny)
        self.shape_avg = (8, nx + 2, ny + 2)
        st = None
        if bc_state is not None:
            self._bc = np.ascontiguousarray(bc_state, dtype=np.float64)
            st = _p(self._bc)
        h = C.c_void_p()
        rc = self.lib.mhd_gpu_create(nx, ny, p, p, rknstg, *map(float, domain), float(gamma), bc_kind,
                                     st, C.byref(h))
        _check("mhd_gpu_create", rc)
        self.h = h

    @classmethod
    def for_problem(cls, prob, nx, ny, p, rknstg=3):
        return cls(nx, ny, p, rknstg, prob.domain, prob.gamma, prob.bc_kind, prob.bc_state)

    # -------------------------------------------------------------------------- life cycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def device_bytes(self):
        b = C.c_size_t()
        _check("mhd_gpu_device_bytes", self.lib.mhd_gpu_device_bytes(self.h, C.byref(b)))
        return b.value

    def set_stream(self, stream_handle):
        _check("mhd_gpu_set_stream", self.lib.mhd_gpu_set_stream(self.h, C.c_void_p(stream_handle)))

    def synchronize(self):
        _check("mhd_gpu_synchronize", self.lib.mhd_gpu_synchronize(self.h))

    # -------------------------------------------------------------------------- geometry
    def nodes(self):
        xx = np.zeros((self.p + 1, self.nx), order="F")
        yy = np.zeros((self.p + 1, self.ny), order="F")
        _check("mhd_gpu_nodes", self.lib.mhd_gpu_nodes(self.h, _p(xx), _p(yy)))
        return xx, yy

    def ldf_operator(self):
        return ldf_operator(self.p, (self.domain[1] - self.domain[0]) / self.nx,
                            (self.domain[3] - self.domain[2]) / self.ny)

    # -------------------------------------------------------------------------- transfers
    def upload_state(self, slot, u):
        u = np.asfortranarray(u, dtype=np.float64)
        assert u.shape == self.shape_u, (u.shape, self.shape_u)
        _check("mhd_gpu_upload_state", self.lib.mhd_gpu_upload_state(self.h, slot, _p(u)))

    def download_state(self, slot, out=None):
        if out is None:
            out = np.empty(self.shape_u, order="F")
        _check("mhd_gpu_download_state", self.lib.mhd_gpu_download_state(self.h, slot, _p(out)))
        return out

    def upload_ut(self, stage, ut):
        ut = np.asfortranarray(ut, dtype=np.float64)
        assert ut.shape == self.shape_ut
        _check("mhd_gpu_upload_ut", self.lib.mhd_gpu_upload_ut(self.h, stage, _p(ut)))

    def download_ut(self, stage, out=None):
        if out is None:
            out = np.empty(self.shape_ut, order="F")
        _check("mhd_gpu_download_ut", self.lib.mhd_gpu_download_ut(self.h, stage, _p(out)))
        return out

    def download_avg(self):
        out = np.empty(self.shape_avg, order="F")
        _check("mhd_gpu_download_avg", self.lib.mhd_gpu_download_avg(self.h, _p(out)))
        return out

    def state_device_ptr(self, slot):
        p = _dp()
        _check("mhd_gpu_state_device_ptr", self.lib.mhd_gpu_state_device_ptr(self.h, slot, C.byref(p)))
        return C.cast(p, C.c_void_p).value

    # -------------------------------------------------------------------------- reference calls
    def init_problem(self, prob):
        """the initial state of a problems-module set-up, evaluated on the GPU into slot 0"""
        pid, params = prob.device_ic()
        arr = (C.c_double * max(1, len(params)))(*params)
        _check("mhd_gpu_init_problem", self.lib.mhd_gpu_init_problem(self.h, pid, arr, len(params)))

    def download_avg_primitive(self):
        """(buffer_var(nx+1, ny, 8) float32 Fortran order, var_min(8), var_max(8)) as
        save_tecbin_finite_volume forms them from u_avg"""
        buf = np.empty((self.nx + 1, self.ny, 8), dtype=np.float32, order="F")
        vmin, vmax = np.empty(8), np.empty(8)
        _check("mhd_gpu_download_avg_primitive",
               self.lib.mhd_gpu_download_avg_primitive(self.h, buf.ctypes.data_as(C.POINTER(C.c_float)), _p(vmin),
                                                       _p(vmax)))
        return buf, vmin, vmax

    def apply_bc(self, slot):
        _check("mhd_gpu_apply_bc", self.lib.mhd_gpu_apply_bc(self.h, slot))

    def post_process(self, slot, apply_oedg, apply_ldf, oedg_dt, ent_offset, comput_ent):
        neg, nneg = C.c_int(), C.c_int()
        tot = C.c_double()
        rc = self.lib.mhd_gpu_post_process(self.h, slot, int(apply_oedg), int(apply_ldf),
                                           float(oedg_dt), int(ent_offset), int(comput_ent),
                                           C.byref(neg), C.byref(nneg), C.byref(tot))
        _check("mhd_gpu_post_process", rc, fatal_flags=False)
        return dict(neg_avg=bool(neg.value), num_negcell=nneg.value, tot_ent=tot.value,
                    pp_relimit_fail=bool(rc & capi.MHD_FLAG_PP_RELIMIT))

    def semidiscretize(self, ut_stage, slot):
        d = C.c_double()
        _check("mhd_gpu_semidiscretize", self.lib.mhd_gpu_semidiscretize(self.h, ut_stage, slot, C.byref(d)))
        return d.value

    def rk_combine(self, stage, dt):
        _check("mhd_gpu_rk_combine", self.lib.mhd_gpu_rk_combine(self.h, stage, float(dt)))

    def rk_accept(self):
        """u_con = uRK_con(:, rknstg) on the interior (drive.f90:304-311)"""
        _check("mhd_gpu_rk_accept", self.lib.mhd_gpu_rk_accept(self.h))

    # -------------------------------------------------------------------------- driver
    def solve_begin(self, final_T, cfl, use_oedg=True, use_ldf=True, ent_offset=False):
        te, dl = C.c_double(), C.c_double()
        rc = self.lib.mhd_gpu_solve_begin(self.h, float(final_T), float(cfl), int(use_oedg),
                                          int(use_ldf), int(ent_offset), C.byref(te), C.byref(dl))
        _check("mhd_gpu_solve_begin", rc)
        return dict(tot_ent=te.value, dt_lim=dl.value)

    def step(self):
        st = Status()
        rc = self.lib.mhd_gpu_step(self.h, C.byref(st))
        _check("mhd_gpu_step", rc)
        return st.as_dict()

    def advance(self, max_steps=0, check_every=16, raise_on_flags=True):
        st = Status()
        rc = self.lib.mhd_gpu_advance(self.h, int(max_steps), int(check_every), C.byref(st))
        _check("mhd_gpu_advance", rc, fatal_flags=raise_on_flags)
        return st.as_dict()

    def step_graph_kernels(self):
        """kernel launches in one try of a time step (the nodes of the captured step graph)"""
        n = C.c_int()
        _check("mhd_gpu_step_graph_kernels", self.lib.mhd_gpu_step_graph_kernels(self.h, C.byref(n)))
        return n.value

    def set_log(self, capacity=4096, diagnostics=False):
        """keep the driver log on the device (mhd_gpu_set_log); capacity 0 turns it off"""
        _check("mhd_gpu_set_log", self.lib.mhd_gpu_set_log(self.h, int(capacity), int(diagnostics)))

    def read_log(self):
        """(records, dropped): every log record not yet read, oldest first, as dicts (the stage
        prints of drive.f90:285-294 and the (t, tot_ent) log of drive.f90:74,314)"""
        n, dropped = C.c_int(), C.c_longlong()
        _check("mhd_gpu_read_log", self.lib.mhd_gpu_read_log(self.h, None, 0, C.byref(n), C.byref(dropped)))
        arr = (capi.LogEntry * max(1, n.value))()
        _check("mhd_gpu_read_log", self.lib.mhd_gpu_read_log(self.h, arr, n.value, C.byref(n), C.byref(dropped)))
        return [arr[i].as_dict() for i in range(n.value)], dropped.value

    def status(self):
        st = Status()
        rc = self.lib.mhd_gpu_get_status(self.h, C.byref(st))
        _check("mhd_gpu_get_status", rc, fatal_flags=False)
        return st.as_dict()

    def solve_execute(self, u0, final_T, cfl, use_oedg=True, use_ldf=True, ent_offset=False,
                      max_steps=0):
        """solve_execute (drive.f90:32-343) from the initial state u0 (Fortran layout)."""
        self.upload_state(0, u0)
        info = self.solve_begin(final_T, cfl, use_oedg, use_ldf, ent_offset)
        st = self.advance(max_steps)
        st["initial"] = info
        return st


class Batch:
    """Many independent solver instances advanced together (mhd_batch_*).

    Members are DGSolver objects already through solve_begin.  Each member computes exactly what
    it would compute alone; the batch only packs their work into shared launches."""

    def __init__(self):
        self.lib = capi.load()
        h = C.c_void_p()
        _check("mhd_batch_create", self.lib.mhd_batch_create(C.byref(h)))
        self.h = h
        self.members = []

    def add(self, solver):
        _check("mhd_batch_add", self.lib.mhd_batch_add(self.h, solver.h))
        self.members.append(solver)

    def remove(self, solver):
        _check("mhd_batch_remove", self.lib.mhd_batch_remove(self.h, solver.h))
        self.members.remove(solver)

    def __len__(self):
        n = C.c_int()
        _check("mhd_batch_size", self.lib.mhd_batch_size(self.h, C.byref(n)))
        return n.value

    def advance(self, tries=1):
        """`tries` batched tries; returns the number of members neither done nor failed"""
        n = C.c_int()
        _check("mhd_batch_advance", self.lib.mhd_batch_advance(self.h, int(tries), C.byref(n)))
        return n.value

    def launch(self, tries=1):
        """queue `tries` batched tries and return at once (membership is frozen until wait)"""
        _check("mhd_batch_launch", self.lib.mhd_batch_launch(self.h, int(tries)))

    def wait(self):
        """finish the launched round; returns the number of members neither done nor failed"""
        n = C.c_int()
        _check("mhd_batch_wait", self.lib.mhd_batch_wait(self.h, C.byref(n)))
        return n.value

    def status(self, solver):
        st = Status()
        rc = self.lib.mhd_batch_member_status(self.h, solver.h, C.byref(st))
        _check("mhd_batch_member_status", rc, fatal_flags=False)
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_batch_destroy(self.h)
            self.h = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def footprint(nx, ny, p, rknstg=3):
    """device bytes one instance needs (host-only)"""
    b = C.c_size_t()
    _check("mhd_gpu_footprint", capi.load().mhd_gpu_footprint(nx, ny, p, rknstg, C.byref(b)))
    return b.value


class Server:
    """Continuous-batching request loop (mhd_server_*): admits runs by HBM footprint, keeps them
    resident, advances all active runs in one batch, retires finished runs."""

    def __init__(self, hbm_budget_bytes, max_active=1024, tries_per_round=4, batched=True):
        self.lib = capi.load()
        h = C.c_void_p()
        _check("mhd_server_create", self.lib.mhd_server_create(int(hbm_budget_bytes), int(max_active),
                                                               int(tries_per_round), int(batched), C.byref(h)))
        self.h = h
        self._keep = []  # host buffers must outlive the runs

    def submit(self, rid, prob, nx, ny, p, u0, arrival, final_T=None, rknstg=3, use_oedg=True,
               use_ldf=True, ent_offset=False, want_avg=False):
        u0 = np.asfortranarray(u0, dtype=np.float64)
        r = capi.Request()
        r.id = rid
        r.nx, r.ny, r.p, r.rknstg = nx, ny, p, rknstg
        r.left, r.right, r.bottom, r.top = map(float, prob.domain)
        r.gamma = prob.gamma
        r.bc_kind = prob.bc_kind
        if prob.bc_state is not None:
            for v in range(8):
                r.bc_state8[v] = float(prob.bc_state[v])
        r.final_T = prob.final_T if final_T is None else final_T
        r.cfl = prob.cfl
        r.use_oedg, r.use_ldf, r.ent_offset = int(use_oedg), int(use_ldf), int(ent_offset)
        r.arrival = float(arrival)
        r.u0 = u0.ctypes.data
        avg = None
        if want_avg:
            avg = np.empty((8, nx + 2, ny + 2), order="F")
            r.u_avg_out = avg.ctypes.data
        self._keep.append((u0, avg))
        _check("mhd_server_submit", self.lib.mhd_server_submit(self.h, C.byref(r)))
        return avg

    def run(self, max_seconds=0.0):
        _check("mhd_server_run", self.lib.mhd_server_run(self.h, float(max_seconds)))

    def results(self):
        n = C.c_int()
        self.lib.mhd_server_results(self.h, None, 0, C.byref(n))
        arr = (capi.RequestResult * max(1, n.value))()
        self.lib.mhd_server_results(self.h, arr, n.value, C.byref(n))
        return [arr[i].as_dict() for i in range(n.value)]

    def stats(self):
        st = capi.ServerStats()
        _check("mhd_server_get_stats", self.lib.mhd_server_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def pending(self):
        q, a, u = C.c_int(), C.c_int(), C.c_size_t()
        self.lib.mhd_server_pending(self.h, C.byref(q), C.byref(a), C.byref(u))
        return dict(queued=q.value, active=a.value, used_bytes=u.value)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
