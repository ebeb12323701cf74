// tables.h -- host-side construction of the 1-D GLL / Legendre tables and of the dense nodal LDF
// operator.  Everything is computed in extended precision (long double) from the definitions and
// rounded once to double.
#pragma once

namespace mhd {
namespace tables {

// gauss_lobatto + gauss_lobatto_matrix (gauss.f90:17-71,134-331) for p in 0..6.
// x, w: n = p+1 entries; M, Minv, D, Pmn, Pnm: n*n column-major.  Returns 0 on success.
int gll(int p, double* x, double* w, double* M, double* Minv, double* D, double* Pmn, double* Pnm);

// Rows of powers of the nodal differentiation matrix: R0[kk*n + k] = (D^kk)(0,k),
// RN[kk*n + k] = (D^kk)(n-1,k), kk = 0..p.
int dpow_rows(int p, double* R0, double* RN);

// Dense nodal operator of post_process's LDF step for px = py = p on an hx x hy element
// (DG_solver.f90:237-264 with LDF.f90:114-250):  [Bx;By]_new - avg = A ([Bx;By] - avg),
// A is (2n^2)x(2n^2) column-major, node index k + n*l, Bx block first.
int ldf_nodal_operator(int p, double hx, double hy, double* A);

}  // namespace tables
}  // namespace mhd
