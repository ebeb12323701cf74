// setup.cuh -- set-up and output next to the hot path (included by mhd_gpu.cu).
//
//   init_problem_kernel  the initial state at the GLL nodes on the device: the pattern of
//                        init_by_fun_pri (problems.f90:25-51) -- primitive state at each interior
//                        node, MHD_pri2con (MHD_PDE.f90:58-70) -- for the set-ups of the package's
//                        problems module; the ghost ring is NaN, as the host set-up leaves it.
//   avg_primitive_kernel the cell-average output of save_tecbin_finite_volume (io.f90:75-86):
//                        MHD_con2pri (MHD_PDE.f90:44-56) of every interior u_avg, rounded to
//                        single precision into buffer_var(nx+1, ny, 8), with per-variable min/max.
#pragma once
#include "common.cuh"

namespace mhd {

enum ProblemId : int {
  IC_OT2PI = 0, IC_OT_UNIT = 1, IC_VORTEX = 2, IC_BLAST = 3, IC_ROTOR = 4, IC_ALFVEN = 5, IC_CLOUD_SHOCK = 6, IC_JET = 7
};

struct ProblemParams {
  int id;
  double amp;                   // ot2pi, ot_unit, rotor, alfven
  double kappa, mu, p_inf, bx0, by0;  // vortex (bulk velocity bx0, by0)
  double cx, cy;                // blast centre
};

constexpr double IC_PI = 3.14159265358979323846;

// primitive state (rho, vx, vy, vz, Bx, By, Bz, p) at (x, y)
__device__ __forceinline__ void problem_pri(const ProblemParams& pp, double x, double y, double gamma, double* w) {
  for (int v = 0; v < 8; ++v) w[v] = 0.0;
  switch (pp.id) {
    case IC_OT2PI:  // Orszag-Tang on [0, 2pi]^2
      w[0] = gamma * gamma;
      w[1] = -pp.amp * sin(y);
      w[2] = pp.amp * sin(x);
      w[4] = -pp.amp * sin(y);
      w[5] = pp.amp * sin(2.0 * x);
      w[7] = gamma;
      break;
    case IC_OT_UNIT: {  // OrszagTang_init_pri (problems.f90:155-168)
      const double s4 = sqrt(4.0 * IC_PI);
      w[0] = 25.0 / (36.0 * IC_PI);
      w[1] = -pp.amp * sin(2 * IC_PI * y);
      w[2] = pp.amp * sin(2 * IC_PI * x);
      w[4] = -pp.amp * sin(2 * IC_PI * y) / s4;
      w[5] = pp.amp * sin(4 * IC_PI * x) / s4;
      w[7] = 5.0 / (12.0 * IC_PI);
      break;
    }
    case IC_VORTEX: {  // isentropic MHD vortex; p from the radial balance of the package docs
      const double r2 = x * x + y * y;
      const double e = exp(0.5 * (1.0 - r2));
      const double a = pp.kappa / (2 * IC_PI), b = pp.mu / (2 * IC_PI);
      w[0] = 1.0;
      w[1] = pp.bx0 - a * e * y;
      w[2] = pp.by0 + a * e * x;
      w[4] = -b * e * y;
      w[5] = b * e * x;
      w[7] = pp.p_inf + 0.5 * e * e * (b * b * (1.0 - r2) - a * a);
      break;
    }
    case IC_BLAST: {  // Blast_init_pri (problems.f90:201-218), centred at (cx, cy)
      const bool inside = (x - pp.cx) * (x - pp.cx) + (y - pp.cy) * (y - pp.cy) < 0.01;
      w[0] = 1.0;
      w[4] = 100.0 / sqrt(4 * IC_PI);
      w[7] = inside ? 1000.0 : 0.1;
      break;
    }
    case IC_ROTOR: {  // Rotor_init_pri (problems.f90:170-199)
      const double r0 = 0.1, r1 = 0.115, u0 = 2.0 * pp.amp;
      const double r = sqrt((x - 0.5) * (x - 0.5) + (y - 0.5) * (y - 0.5));
      const double f = (r1 - r) / (r1 - r0);
      w[0] = r < r0 ? 10.0 : (r < r1 ? 1.0 + 9 * f : 1.0);
      w[1] = r < r0 ? -(u0 / r0) * (y - 0.5) : (r < r1 ? -(u0 / r0) * (y - 0.5) * f : 0.0);
      w[2] = r < r0 ? (u0 / r0) * (x - 0.5) : (r < r1 ? (u0 / r0) * (x - 0.5) * f : 0.0);
      w[4] = pp.amp * 5.0 / sqrt(4 * IC_PI);
      w[7] = 1.0;
      break;
    }
    case IC_CLOUD_SHOCK:  // cloud_shock_init_pri (problems.f90:220-247), "original formulation"
      if (x < 0.6) {
        w[0] = 3.86859;
        w[5] = 2.1826182;
        w[6] = -2.1826182;
        w[7] = 167.345;
      } else {
        w[0] = ((x - 0.8) * (x - 0.8) + (y - 0.5) * (y - 0.5) <= 0.15 * 0.15) ? 10.0 : 1.0;
        w[1] = -11.2536;
        w[5] = 0.56418958;
        w[6] = 0.56418958;
        w[7] = 1.0;
      }
      break;
    case IC_JET:  // jet1_init_pri (problems.f90:249-257)
      w[0] = 0.1 * gamma;
      w[5] = sqrt(200.0);
      w[7] = 1.0;
      break;
    default: {  // smooth_alfven_init_fun (problems.f90:74-98)
      const double al = IC_PI / 6.0, ca = cos(al), sa = sin(al);
      const double xp = x * ca + y * sa;
      const double vp = 0.1 * pp.amp * sin(2 * IC_PI * xp);
      const double uz = 0.1 * pp.amp * cos(2 * IC_PI * xp);
      w[0] = 1.0;
      w[1] = vp * (-sa);
      w[2] = vp * ca;
      w[3] = uz;
      w[4] = ca - vp * sa;
      w[5] = sa + vp * ca;
      w[6] = uz;
      w[7] = 0.1;
      break;
    }
  }
}

// One thread per (element of the ghosted grid, node).  The node coordinates are rounded exactly as
// init_DG_solver forms them (DG_solver.f90:93-106): (hx/2)*x_k + (left + (i-1/2)*hx), no FMA.
template <int P>
__global__ void __launch_bounds__(256) init_problem_kernel(double* __restrict__ u, Geo g, ProblemParams pp,
                                                           double left, double bottom) {
  constexpr int N = P + 1, NN = N * N, EB = 8 * NN;
  const long long nelg = (long long)(g.nx + 2) * (g.ny + 2);
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= nelg * NN) return;
  const long long e = it / NN;
  const int q = (int)(it - e * NN), k = q % N, l = q / N;
  const int j = (int)(e / (g.nx + 2)), i = (int)(e - (long long)j * (g.nx + 2));
  double* dst = u + e * EB + q;
  if (i < 1 || i > g.nx || j < 1 || j > g.ny) {
    for (int v = 0; v < 8; ++v) dst[v * NN] = __longlong_as_double(0x7ff8000000000000LL);  // quiet NaN
    return;
  }
  const DegConst& dc = c_deg[P];
  const double x = __dadd_rn(__dmul_rn(0.5 * g.hx, dc.qx[k]), __dadd_rn(left, __dmul_rn(i - 0.5, g.hx)));
  const double y = __dadd_rn(__dmul_rn(0.5 * g.hy, dc.qx[l]), __dadd_rn(bottom, __dmul_rn(j - 0.5, g.hy)));
  double w[8];
  problem_pri(pp, x, y, g.gamma, w);
  // MHD_pri2con (MHD_PDE.f90:58-70)
  const double gm1 = g.gamma - 1.0;
  const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(w[1], w[1]), __dmul_rn(w[2], w[2])), __dmul_rn(w[3], w[3]));
  const double b2 = __dadd_rn(__dadd_rn(__dmul_rn(w[4], w[4]), __dmul_rn(w[5], w[5])), __dmul_rn(w[6], w[6]));
  dst[0 * NN] = w[0];
  dst[1 * NN] = __dmul_rn(w[0], w[1]);
  dst[2 * NN] = __dmul_rn(w[0], w[2]);
  dst[3 * NN] = __dmul_rn(w[0], w[3]);
  dst[4 * NN] = w[4];
  dst[5 * NN] = w[5];
  dst[6 * NN] = w[6];
  dst[7 * NN] = __dadd_rn(__ddiv_rn(w[7], gm1), __dmul_rn(0.5, __dadd_rn(__dmul_rn(w[0], v2), b2)));
}

// One thread per interior cell.  out = buffer_var(nx+1, ny, 8) (Fortran order, single precision);
// its column nx+1, which the reference allocates but never fills, is written as zero.  mm holds the
// ordered encodings of the per-variable minima (mm[0..7]) and maxima (mm[8..15]) of the rounded
// values, as the reference takes them (io.f90:81-84).
__global__ void __launch_bounds__(256) avg_primitive_kernel(const double* __restrict__ u_avg, Geo g,
                                                            float* __restrict__ out, unsigned long long* mm) {
  const int nx = g.nx, ny = g.ny;
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= (long long)(nx + 1) * ny) return;
  const int j = (int)(it / (nx + 1)), i = (int)(it - (long long)j * (nx + 1));  // 0-based, i = nx: unused column
  const long long plane = (long long)(nx + 1) * ny;
  if (i == nx) {
    for (int v = 0; v < 8; ++v) out[v * plane + it] = 0.0f;
    return;
  }
  const double* uc = u_avg + ((long long)(j + 1) * (nx + 2) + (i + 1)) * 8;
  double up[8];
  up[0] = uc[0];
  up[1] = __ddiv_rn(uc[1], uc[0]);
  up[2] = __ddiv_rn(uc[2], uc[0]);
  up[3] = __ddiv_rn(uc[3], uc[0]);
  up[4] = uc[4];
  up[5] = uc[5];
  up[6] = uc[6];
  const double m2 = __dadd_rn(__dadd_rn(__dmul_rn(uc[1], uc[1]), __dmul_rn(uc[2], uc[2])), __dmul_rn(uc[3], uc[3]));
  const double b2 = __dadd_rn(__dadd_rn(__dmul_rn(uc[4], uc[4]), __dmul_rn(uc[5], uc[5])), __dmul_rn(uc[6], uc[6]));
  up[7] = __dmul_rn(g.gamma - 1.0, __dsub_rn(uc[7], __dmul_rn(0.5, __dadd_rn(__ddiv_rn(m2, uc[0]), b2))));
  for (int v = 0; v < 8; ++v) {
    const float f = __double2float_rn(up[v]);
    out[v * plane + it] = f;
    const unsigned long long enc = ord_enc((double)f);
    atomicMin(mm + v, enc);
    atomicMax(mm + 8 + v, enc);
  }
}

}  // namespace mhd
