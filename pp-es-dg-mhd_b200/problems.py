"""Host-side set-ups: initial conditions, boundary kinds and domains (the role of problems.f90).

Initial values are evaluated on the host at the GLL nodes and handed to the solver in the
reference's Fortran layout u(8, px+1, py+1, 0:nx+1, 0:ny+1) (ghost ring NaN), exactly as
init_by_fun_pri (problems.f90:25-51) fills u_con before solve_execute.

Problems
  ot2pi     Orszag-Tang on [0,2pi]^2 (rho=gamma^2, p=gamma, u=-sin y, v=sin x, Bx=-sin y,
            By=sin 2x), periodic.  Not in the reference (its OT is the [0,1]^2 scaled form).
  ot_unit   the reference's OrszagTang_init_pri (problems.f90:155-168) on [0,1]^2, periodic.
  vortex    smooth isentropic MHD vortex on [-10,10]^2, periodic, with exact advected solution.
            Not in the reference; pressure from d(p + B_phi^2/2)/dr = rho v_phi^2/r - B_phi^2/r.
  blast     low-beta blast wave on [-0.5,0.5]^2 with extrapolation ("outflow") ghosts
            (BC_YeeSjogreen pattern, problems.f90:386-423); the reference's Blast_init_pri
            (problems.f90:201-218) is the same state centred at (0.5,0.5) on [0,1]^2.
  rotor     the reference's Rotor_init_pri (problems.f90:170-199) with BC_rotor fixed ghosts
            (problems.f90:597-654), gamma = 1.4.
  alfven    the reference's smooth_alfven_init_fun (problems.f90:74-98), periodic.
  cloud_shock  cloud_shock_init_pri (problems.f90:220-247) with BC_cloud_shock (:425-472).
  jet       jet1_init_pri (problems.f90:249-257) with BC_jet1_cell_ext (:474-595), gamma 1.4.
An amplitude factor `amp` scales velocity and magnetic field perturbations (ot2pi, rotor).
"""
import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import capi

PI = math.pi


def gll_nodes(p):
    """GLL nodes and weights of degree p from the library's tables (no GPU needed)."""
    n = p + 1
    x, w = np.zeros(n), np.zeros(n)
    rc = capi.load().mhd_gpu_gll_tables(p, x.ctypes.data_as(C.POINTER(C.c_double)),
                                        w.ctypes.data_as(C.POINTER(C.c_double)), None, None, None,
                                        None, None)
    if rc:
        raise capi.MHDError("mhd_gpu_gll_tables", rc)
    return x, w


def node_coords(nx, ny, p, domain, nodes=None):
    """xx(p+1, nx), yy(p+1, ny) exactly as init_DG_solver computes them (DG_solver.f90:93-106).
    nodes: the p+1 GLL nodes to use (default: the library's tables)."""
    left, right, bottom, top = domain
    q = gll_nodes(p)[0] if nodes is None else np.asarray(nodes, dtype=np.float64)
    hx = (right - left) / nx
    hy = (top - bottom) / ny
    i = np.arange(1, nx + 1)
    j = np.arange(1, ny + 1)
    xx = (0.5 * hx) * q[:, None] + (left + (i - 0.5) * hx)[None, :]
    yy = (0.5 * hy) * q[:, None] + (bottom + (j - 0.5) * hy)[None, :]
    return np.asfortranarray(xx), np.asfortranarray(yy)


def pri2con(up, gamma):
    """MHD_pri2con (MHD_PDE.f90:58-70), vectorised over trailing axes."""
    uc = np.empty_like(up)
    uc[0] = up[0]
    uc[1] = up[0] * up[1]
    uc[2] = up[0] * up[2]
    uc[3] = up[0] * up[3]
    uc[4] = up[4]
    uc[5] = up[5]
    uc[6] = up[6]
    uc[7] = up[7] / (gamma - 1.0) + 0.5 * (up[0] * (up[1] ** 2 + up[2] ** 2 + up[3] ** 2)
                                           + (up[4] ** 2 + up[5] ** 2 + up[6] ** 2))
    return uc


def con2pri(uc, gamma):
    """MHD_con2pri (MHD_PDE.f90:44-56)."""
    up = np.empty_like(uc)
    up[0] = uc[0]
    up[1] = uc[1] / uc[0]
    up[2] = uc[2] / uc[0]
    up[3] = uc[3] / uc[0]
    up[4:7] = uc[4:7]
    up[7] = (gamma - 1.0) * (uc[7] - 0.5 * ((uc[1] ** 2 + uc[2] ** 2 + uc[3] ** 2) / uc[0]
                                             + (uc[4] ** 2 + uc[5] ** 2 + uc[6] ** 2)))
    return up


# ------------------------------------------------------------------------------ primitive ICs
def ot2pi_pri(x, y, gamma, amp=1.0):
    z = np.zeros_like(x)
    return np.stack([z + gamma ** 2, -amp * np.sin(y), amp * np.sin(x), z,
                     -amp * np.sin(y), amp * np.sin(2.0 * x), z, z + gamma])


def ot_unit_pri(x, y, gamma, amp=1.0):
    z = np.zeros_like(x)
    s4 = math.sqrt(4.0 * PI)
    return np.stack([z + 25.0 / (36.0 * PI), -amp * np.sin(2 * PI * y), amp * np.sin(2 * PI * x), z,
                     -amp * np.sin(2 * PI * y) / s4, amp * np.sin(4 * PI * x) / s4, z,
                     z + 5.0 / (12.0 * PI)])


def vortex_pri(x, y, gamma, kappa=1.0, mu=1.0, p_inf=1.0, bulk=(1.0, 1.0)):
    r2 = x * x + y * y
    e = np.exp(0.5 * (1.0 - r2))
    a, b = kappa / (2 * PI), mu / (2 * PI)
    z = np.zeros_like(x)
    # p = p_inf + e^{1-r^2} (b^2 (1 - r^2) - a^2) / 2  solves the radial balance above
    p = p_inf + 0.5 * e * e * (b * b * (1.0 - r2) - a * a)
    return np.stack([z + 1.0, bulk[0] - a * e * y, bulk[1] + a * e * x, z, -b * e * y, b * e * x, z, p])


def blast_pri(x, y, gamma, amp=1.0, center=(0.0, 0.0)):
    z = np.zeros_like(x)
    inside = (x - center[0]) ** 2 + (y - center[1]) ** 2 < 0.01
    return np.stack([z + 1.0, z, z, z, z + 100.0 / math.sqrt(4 * PI), z, z,
                     np.where(inside, 1000.0, 0.1)])


def rotor_pri(x, y, gamma, amp=1.0):
    r0, r1, u0 = 0.1, 0.115, 2.0 * amp
    r = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2)
    f = (r1 - r) / (r1 - r0)
    rho = np.where(r < r0, 10.0, np.where(r < r1, 1.0 + 9 * f, 1.0))
    vx = np.where(r < r0, -(u0 / r0) * (y - 0.5), np.where(r < r1, -(u0 / r0) * (y - 0.5) * f, 0.0))
    vy = np.where(r < r0, (u0 / r0) * (x - 0.5), np.where(r < r1, (u0 / r0) * (x - 0.5) * f, 0.0))
    z = np.zeros_like(x)
    return np.stack([rho, vx, vy, z, z + amp * 5.0 / math.sqrt(4 * PI), z, z, z + 1.0])


def cloud_shock_pri(x, y, gamma, amp=1.0):
    """cloud_shock_init_pri (problems.f90:220-247), the reference's "original formulation" values"""
    post = np.array([3.86859, 0.0, 0.0, 0.0, 0.0, 2.1826182, -2.1826182, 167.345])
    pre = np.array([1.0, -11.2536, 0.0, 0.0, 0.0, 0.56418958, 0.56418958, 1.0])
    left = x < 0.6
    u = np.where(left[None], post.reshape((8,) + (1,) * x.ndim), pre.reshape((8,) + (1,) * x.ndim))
    cloud = (~left) & ((x - 0.8) ** 2 + (y - 0.5) ** 2 <= 0.15 ** 2)
    u[0] = np.where(cloud, 10.0, u[0])
    return u


def jet_pri(x, y, gamma, amp=1.0):
    """jet1_init_pri (problems.f90:249-257): the ambient state"""
    z = np.zeros_like(x)
    return np.stack([z + 0.1 * gamma, z, z, z, z, z + math.sqrt(200.0), z, z + 1.0])


def alfven_pri(x, y, gamma, amp=1.0):
    al = PI / 6.0
    xp = x * math.cos(al) + y * math.sin(al)
    vp = 0.1 * amp * np.sin(2 * PI * xp)
    uz = 0.1 * amp * np.cos(2 * PI * xp)
    z = np.zeros_like(x)
    return np.stack([z + 1.0, vp * (-math.sin(al)), vp * math.cos(al), uz,
                     math.cos(al) - vp * math.sin(al), math.sin(al) + vp * math.cos(al), uz, z + 0.1])


@dataclass
class Problem:
    name: str
    domain: tuple
    gamma: float
    bc_kind: int
    final_T: float
    cfl: float
    pri_fn: object
    params: dict = field(default_factory=dict)
    bc_state: object = None

    def device_ic(self):
        """(problem id, parameters) of mhd_gpu_init_problem for this set-up"""
        ids = {"ot2pi": capi.IC_OT2PI, "ot_unit": capi.IC_OT_UNIT, "vortex": capi.IC_VORTEX,
               "blast": capi.IC_BLAST, "rotor": capi.IC_ROTOR, "alfven": capi.IC_ALFVEN,
               "cloud_shock": capi.IC_CLOUD_SHOCK, "jet": capi.IC_JET}
        if self.name == "vortex":
            kw = dict(kappa=1.0, mu=1.0, p_inf=1.0, bulk=(1.0, 1.0))
            kw.update(self.params)
            return ids["vortex"], [kw["kappa"], kw["mu"], kw["p_inf"], kw["bulk"][0], kw["bulk"][1]]
        if self.name == "blast":
            c = self.params.get("center", (0.0, 0.0))
            return ids["blast"], [c[0], c[1]]
        return ids[self.name], [self.params.get("amp", 1.0)]

    def initial_state(self, nx, ny, p, nodes=None):
        """u(8, p+1, p+1, nx+2, ny+2) Fortran order, interior from the IC, ghost ring NaN.
        nodes: the p+1 GLL nodes to evaluate at (default: the library's tables; a caller that must
        not load the library passes its own, e.g. the CPU baseline)."""
        xx, yy = node_coords(nx, ny, p, self.domain, nodes)
        n = p + 1
        X = np.broadcast_to(xx[:, None, :, None], (n, n, nx, ny))
        Y = np.broadcast_to(yy[None, :, None, :], (n, n, nx, ny))
        up = self.pri_fn(np.array(X), np.array(Y), self.gamma, **self.params)
        uc = pri2con(up, self.gamma)
        u = np.full((8, n, n, nx + 2, ny + 2), np.nan, order="F")
        u[:, :, :, 1:-1, 1:-1] = uc
        return u


def make(name, gamma=None, amp=1.0, **kw):
    """Problem set-up by name (see module docstring)."""
    if name == "ot2pi":
        g = 5.0 / 3.0 if gamma is None else gamma
        return Problem(name, (0.0, 2 * PI, 0.0, 2 * PI), g, capi.BC_PERIODIC, 0.5, 0.2, ot2pi_pri,
                       {"amp": amp})
    if name == "ot_unit":
        g = 5.0 / 3.0 if gamma is None else gamma
        return Problem(name, (0.0, 1.0, 0.0, 1.0), g, capi.BC_PERIODIC, 0.5, 0.6, ot_unit_pri,
                       {"amp": amp})
    if name == "vortex":
        g = 5.0 / 3.0 if gamma is None else gamma
        return Problem(name, (-10.0, 10.0, -10.0, 10.0), g, capi.BC_PERIODIC, 20.0, 0.6, vortex_pri, kw)
    if name == "blast":
        g = 1.4 if gamma is None else gamma
        return Problem(name, (-0.5, 0.5, -0.5, 0.5), g, capi.BC_EXTRAPOLATE, 0.01, 0.6, blast_pri,
                       {"amp": amp})
    if name == "rotor":
        g = 1.4 if gamma is None else gamma
        st = pri2con(np.array([1.0, 0.0, 0.0, 0.0, amp * 5.0 / math.sqrt(4 * PI), 0.0, 0.0, 1.0]), g)
        return Problem(name, (0.0, 1.0, 0.0, 1.0), g, capi.BC_FIXED, 0.15, 0.6, rotor_pri,
                       {"amp": amp}, bc_state=st)
    if name == "cloud_shock":  # main.f90:141-155
        g = 5.0 / 3.0 if gamma is None else gamma
        st = pri2con(np.array([1.0, -11.2536, 0.0, 0.0, 0.0, 0.56418958, 0.56418958, 1.0]), g)
        return Problem(name, (0.0, 1.0, 0.0, 1.0), g, capi.BC_CLOUD_SHOCK, 0.06, 0.6, cloud_shock_pri, {},
                       bc_state=st)
    if name == "jet":  # main.f90:156-169; nx must be a multiple of 10 (the nozzle is the first nx/10)
        g = 1.4 if gamma is None else gamma
        st = pri2con(np.array([g, 0.0, 800.0, 0.0, 0.0, math.sqrt(200.0), 0.0, 1.0]), g)
        return Problem(name, (0.0, 0.5, 0.0, 1.5), g, capi.BC_JET, 2.0e-3, 0.6, jet_pri, {}, bc_state=st)
    if name == "alfven":
        g = 5.0 / 3.0 if gamma is None else gamma
        return Problem(name, (0.0, 1.0 / math.cos(PI / 6.0), 0.0, 1.0 / math.sin(PI / 6.0)), g,
                       capi.BC_PERIODIC, 5.0, 0.6, alfven_pri, {"amp": amp})
    raise ValueError(f"unknown problem {name!r}")


def vortex_exact(nx, ny, p, t, gamma=5.0 / 3.0, **kw):
    """Exact conserved state of the advected vortex at time t (interior, (8,n,n,nx,ny))."""
    prob = make("vortex", gamma=gamma, **kw)
    xx, yy = node_coords(nx, ny, p, prob.domain)
    n = p + 1
    L = 20.0
    X = np.broadcast_to(xx[:, None, :, None], (n, n, nx, ny)) - t * 1.0
    Y = np.broadcast_to(yy[None, :, None, :], (n, n, nx, ny)) - t * 1.0
    X = (X + 10.0) % L - 10.0
    Y = (Y + 10.0) % L - 10.0
    return pri2con(vortex_pri(X, Y, gamma, **kw), gamma)
