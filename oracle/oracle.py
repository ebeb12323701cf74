"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this module.  It mirrors
the reference's Fortran interface (init_DG_solver / post_process / DG_semidiscretize /
solve_execute, DG_solver.f90:47,128,663 and drive.f90:32) over numpy arrays in the reference's
Fortran layouts:

    u      (8, px+1, py+1, nx+2, ny+2)   order='F'   (ghost ring included)
    ut     (8, px+1, py+1, nx, ny)       order='F'
    u_avg  (8, nx+2, ny+2)               order='F'
"""
import ctypes as C
import os

import numpy as np

from . import build_oracle

BC_PERIODIC, BC_EXTRAPOLATE, BC_FIXED, BC_XEXTRAP_YPER, BC_CLOUD_SHOCK, BC_JET = 0, 1, 2, 3, 4, 5

_libs = {}
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous)
    return a.ctypes.data_as(_dp)


def lib(fast: bool = False):
    name = "libmhd_oracle_fast.so" if fast else "libmhd_oracle.so"
    if name not in _libs:
        paths = build_oracle.build()
        L = C.CDLL(paths[name])
        L.ora_create.restype = C.c_void_p
        L.ora_create.argtypes = [C.c_int] * 5 + [C.c_double] * 5 + [C.c_int, _dp]
        L.ora_destroy.argtypes = [C.c_void_p]
        for f in ("ora_size_u", "ora_size_ut", "ora_size_avg"):
            getattr(L, f).restype = C.c_long
            getattr(L, f).argtypes = [C.c_void_p]
        L.ora_u_con.restype = _dp
        L.ora_u_con.argtypes = [C.c_void_p]
        L.ora_u_avg.restype = _dp
        L.ora_u_avg.argtypes = [C.c_void_p]
        L.ora_ut_con.restype = _dp
        L.ora_ut_con.argtypes = [C.c_void_p, C.c_int]
        L.ora_urk_con.restype = _dp
        L.ora_urk_con.argtypes = [C.c_void_p, C.c_int]
        L.ora_nodes.argtypes = [C.c_void_p, _dp, _dp]
        L.ora_gll_tables.argtypes = [C.c_int] + [_dp] * 7
        L.ora_legendre_tables.argtypes = [C.c_int] + [_dp] * 5
        L.ora_ldf_tables.argtypes = [C.c_int, C.c_int] + [_dp] * 5
        L.ora_ldf_apply.argtypes = [C.c_int, C.c_int, _dp]
        L.ora_ldf_div.argtypes = [C.c_int, C.c_int, _dp, _dp]
        L.ora_hll_flux_x.argtypes = [_dp, _dp, C.c_double, _dp, _dp, _dp, _dp]
        L.ora_ec_flux_x.argtypes = [_dp, _dp, C.c_double, _dp]
        L.ora_ec_flux_y.argtypes = [_dp, _dp, C.c_double, _dp]
        L.ora_log_avg_divisor.restype = C.c_double
        L.ora_log_avg_divisor.argtypes = [C.c_double, C.c_double]
        L.ora_apply_bc.argtypes = [C.c_void_p, _dp]
        L.ora_post_process.argtypes = [C.c_void_p, _dp, _dp, _ip, _ip, C.c_int, C.c_int, C.c_double,
                                       C.c_int, C.c_int, _dp, _ip]
        L.ora_semidiscretize.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.ora_rk_combine.restype = C.c_double
        L.ora_rk_combine.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, _dp]
        L.ora_solve.restype = C.c_int
        L.ora_solve.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                C.c_int, _dp]
        L.ora_solve_resume.restype = C.c_int
        L.ora_solve_resume.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_int, _dp]
        L.ora_set_threads.argtypes = [C.c_int]
        L.ora_get_threads.restype = C.c_int
        _libs[name] = L
    return _libs[name]


# ----------------------------------------------------------------------------------- tables
def gll_tables(p):
    n = p + 1
    x, w = np.zeros(n), np.zeros(n)
    M, Minv, D, Pmn, Pnm = (np.zeros((n, n), order="F") for _ in range(5))
    rc = lib().ora_gll_tables(p, *(_ptr(a) for a in (x, w, M, Minv, D, Pmn, Pnm)))
    if rc:
        raise ValueError(f"gll_tables: p={p} unsupported")
    return dict(x=x, w=w, M=M, Minv=Minv, D=D, Pmn=Pmn, Pnm=Pnm)


def legendre_tables(p):
    n = p + 1
    m, minv, tl, tr = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    D = np.zeros((n, n), order="F")
    lib().ora_legendre_tables(p, _ptr(m), _ptr(minv), _ptr(D), _ptr(tl), _ptr(tr))
    return dict(m=m, minv=minv, D=D, tl=tl, tr=tr)


def ldf_tables(px, py):
    Lx, Ly = np.zeros(px + 1), np.zeros(py + 1)
    Ux = np.zeros((px + 1, px + 1), order="F")
    Uy = np.zeros((py + 1, py + 1), order="F")
    Ld = np.zeros((px + 1, py + 1), order="F")
    lib().ora_ldf_tables(px, py, _ptr(Lx), _ptr(Ux), _ptr(Ly), _ptr(Uy), _ptr(Ld))
    return dict(Lx=Lx, Ux=Ux, Ly=Ly, Uy=Uy, Ldagger=Ld)


def ldf_apply(px, py, uu):
    uu = np.asfortranarray(np.array(uu, dtype=np.float64).reshape((px + 1, py + 1, 2), order="F"))
    lib().ora_ldf_apply(px, py, _ptr(uu))
    return uu


def ldf_div(px, py, uu):
    uu = np.asfortranarray(np.array(uu, dtype=np.float64).reshape((px + 1, py + 1, 2), order="F"))
    out = np.zeros((px + 1, py + 1), order="F")
    lib().ora_ldf_div(px, py, _ptr(uu), _ptr(out))
    return out


def hll_flux_x(wl, wr, gamma):
    wl = np.ascontiguousarray(wl, dtype=np.float64)
    wr = np.ascontiguousarray(wr, dtype=np.float64)
    nf = np.zeros(8)
    nb, sl, sr = C.c_double(), C.c_double(), C.c_double()
    lib().ora_hll_flux_x(_ptr(wl), _ptr(wr), gamma, _ptr(nf), C.byref(nb), C.byref(sl), C.byref(sr))
    return nf, nb.value, sl.value, sr.value


def ec_flux(pl, pr, gamma, direction="x"):
    pl = np.ascontiguousarray(pl, dtype=np.float64)
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    out = np.zeros(8)
    f = lib().ora_ec_flux_x if direction == "x" else lib().ora_ec_flux_y
    f(_ptr(pl), _ptr(pr), gamma, _ptr(out))
    return out


def log_avg_divisor(a, b):
    return lib().ora_log_avg_divisor(a, b)


# ----------------------------------------------------------------------------------- solver
class OracleSolver:
    """Mirror of the reference's module-level solver (DG_solver_m + drive_m) on the CPU."""

    def __init__(self, nx, ny, px, py, rknstg, left, right, bottom, top, gamma,
                 bc_kind=BC_PERIODIC, bc_state=None, fast=False, threads=None):
        self.L = lib(fast)
        if threads:
            self.L.ora_set_threads(int(threads))
        st = None
        if bc_state is not None:
            self._bc = np.ascontiguousarray(bc_state, dtype=np.float64)
            st = _ptr(self._bc)
        self.h = self.L.ora_create(nx, ny, px, py, rknstg, left, right, bottom, top, gamma,
                                   bc_kind, st)
        if not self.h:
            raise ValueError("oracle: invalid solver parameters")
        self.nx, self.ny, self.px, self.py, self.rknstg = nx, ny, px, py, rknstg
        self.gamma = gamma
        self.shape_u = (8, px + 1, py + 1, nx + 2, ny + 2)
        self.shape_ut = (8, px + 1, py + 1, nx, ny)
        self.shape_avg = (8, nx + 2, ny + 2)

    def close(self):
        if getattr(self, "h", None):
            self.L.ora_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _view(self, p, shape):
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(shape, order="F")

    @property
    def u_con(self):
        return self._view(self.L.ora_u_con(self.h), self.shape_u)

    @property
    def u_avg(self):
        return self._view(self.L.ora_u_avg(self.h), self.shape_avg)

    def ut_con(self, stage):
        return self._view(self.L.ora_ut_con(self.h, stage), self.shape_ut)

    def urk_con(self, stage):
        return self._view(self.L.ora_urk_con(self.h, stage), self.shape_u)

    def nodes(self):
        xx = np.zeros((self.px + 1, self.nx), order="F")
        yy = np.zeros((self.py + 1, self.ny), order="F")
        self.L.ora_nodes(self.h, _ptr(xx), _ptr(yy))
        return xx, yy

    def apply_bc(self, u):
        assert u.flags.f_contiguous and u.shape == self.shape_u
        self.L.ora_apply_bc(self.h, _ptr(u))

    def post_process(self, u, u_avg, apply_oedg, apply_ldf, oedg_dt, ent_offset, comput_ent):
        assert u.flags.f_contiguous and u_avg.flags.f_contiguous
        neg, nneg, relim = C.c_int(), C.c_int(), C.c_int()
        tot = C.c_double()
        self.L.ora_post_process(self.h, _ptr(u), _ptr(u_avg), C.byref(neg), C.byref(nneg),
                                int(apply_oedg), int(apply_ldf), float(oedg_dt), int(ent_offset),
                                int(comput_ent), C.byref(tot), C.byref(relim))
        return dict(neg_avg=bool(neg.value), num_negcell=nneg.value, tot_ent=tot.value,
                    pp_relimit_fail=bool(relim.value))

    def semidiscretize(self, u, ut=None):
        if ut is None:
            ut = np.zeros(self.shape_ut, order="F")
        d = C.c_double()
        self.L.ora_semidiscretize(self.h, _ptr(ut), C.byref(d), _ptr(u))
        return ut, d.value

    def rk_combine(self, stage, dt, t, t_rk):
        t_rk = np.ascontiguousarray(t_rk, dtype=np.float64)
        tr = self.L.ora_rk_combine(self.h, stage, dt, t, _ptr(t_rk))
        return tr, t_rk

    def set_state(self, u_interior_or_full):
        """Copy a state (with or without ghost ring) into u_con."""
        u = self.u_con
        a = np.asarray(u_interior_or_full)
        if a.shape == self.shape_u:
            u[...] = a
        else:
            u[:, :, :, 1:-1, 1:-1] = a

    def solve(self, final_T, cfl, use_oedg=True, use_ldf=True, ent_offset=False, max_steps=0,
              resume=False):
        out = np.zeros(7)
        rc = self.L.ora_solve_resume(self.h, final_T, cfl, int(use_oedg), int(use_ldf),
                                     int(ent_offset), int(max_steps), int(resume), _ptr(out))
        return dict(status=rc, t=out[0], dt_lim=out[1], tot_ent=out[2], steps=int(out[3]),
                    retries=int(out[4]), dt=out[5], num_negcell_total=int(out[6]))


def threads():
    return lib().ora_get_threads()
