/*
 * mhd_oracle.c -- CPU restatement (the oracle) of the reference's per-stage DG update.
 *
 * TEST INFRASTRUCTURE ONLY: the correctness checker and timed CPU baseline; the product path
 * never links or calls it.  Each routine cites the reference file:line it restates.  The
 * expression order of the Fortran source is kept (left-to-right evaluation, the same clamps),
 * and the file is compiled with -ffp-contract=off so that every operation is rounded as
 * written.  Reductions that the reference performs with OpenMP (order depends on the thread
 * count there) are done here in a fixed row order so that the oracle is deterministic.
 *
 * Parity status: "parity unpinned" against a run of the reference (no Fortran compiler exists
 * on this machine); pinned only through the reference's own known answers (table identities,
 * closed-form table entries, LDF projector identities) and physical invariants.
 */
#include "mhd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Extended precision for the one-time tables.  A counting build (oracle/flop_count.cpp) defines
 * ORA_LDBL_DEFINED before replacing `double` by an operation-counting type. */
#ifndef ORA_LDBL_DEFINED
typedef long double ldbl;
#endif
/* hook for counting min/max as one operation each (empty in the normal builds) */
#ifndef ORA_COUNT_MINMAX
#define ORA_COUNT_MINMAX()
#endif

#define NQMAX 7          /* max nodes per direction (p<=6), gauss.f90:34-64 */
#define NNMAX (NQMAX * NQMAX)

static const double PP_eps = 1.0e-11;   /* DG_solver.f90:17 */
static const double OEDG_eps = 1.0e-8;  /* DG_solver.f90:148 */

static inline double dmax(double a, double b) {
  ORA_COUNT_MINMAX();
  return a > b ? a : b;
}
static inline double dmin(double a, double b) {
  ORA_COUNT_MINMAX();
  return a < b ? a : b;
}
static inline int imax(int a, int b) { return a > b ? a : b; }

/* _macro_prs_ (DG_solver.f90:125) */
static inline double prs_macro(double rho, double mx, double my, double mz, double bx, double by,
                               double bz, double e_tot, double gamma) {
  return (gamma - 1.0) * (e_tot - 0.5 * ((mx * mx + my * my + mz * mz) / rho + (bx * bx + by * by + bz * bz)));
}
/* _macro_ent_ (DG_solver.f90:126) */
static inline double ent_macro(double rho, double prs, double gamma) {
  return -(rho * (log(prs) - gamma * log(rho)) / (gamma - 1.0));
}

/* ------------------------------------------------------------------------------------------ */
/* 1-D tables (gauss.f90).  The reference tabulates closed forms for p<=6; here the same        */
/* matrices are computed from their definitions in extended precision and rounded once.        */
/* ------------------------------------------------------------------------------------------ */

static void legendre_all(int N, ldbl x, ldbl *P, ldbl *dP) {
  /* P[k] = P_k(x), dP[k] = P_k'(x), k=0..N (recurrence as gauss.f90:390-434 states it) */
  P[0] = 1.0L;
  dP[0] = 0.0L;
  if (N >= 1) {
    P[1] = x;
    dP[1] = 1.0L;
  }
  for (int k = 2; k <= N; ++k) {
    P[k] = ((2 * k - 1) * x * P[k - 1] - (k - 1) * P[k - 2]) / k;
    dP[k] = dP[k - 2] + (2 * k - 1) * P[k - 1];
  }
}

static int invert_ld(int n, const ldbl *A, ldbl *Ainv) {
  /* Gauss-Jordan with partial pivoting, column-major n x n */
  ldbl W[NQMAX][2 * NQMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      W[i][j] = A[i + n * j];
      W[i][n + j] = (i == j) ? 1.0L : 0.0L;
    }
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (fabsl(W[r][c]) > fabsl(W[piv][c])) piv = r;
    if (W[piv][c] == 0.0L) return -1;
    if (piv != c)
      for (int j = 0; j < 2 * n; ++j) {
        ldbl t = W[c][j];
        W[c][j] = W[piv][j];
        W[piv][j] = t;
      }
    ldbl d = W[c][c];
    for (int j = 0; j < 2 * n; ++j) W[c][j] /= d;
    for (int r = 0; r < n; ++r)
      if (r != c) {
        ldbl f = W[r][c];
        if (f != 0.0L)
          for (int j = 0; j < 2 * n; ++j) W[r][j] -= f * W[c][j];
      }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) Ainv[i + n * j] = W[i][n + j];
  return 0;
}

/* GLL nodes/weights (gauss.f90:17-71) and nodal matrices (gauss.f90:134-331), extended precision */
static int gll_tables_ld(int p, ldbl *x, ldbl *w, ldbl *M, ldbl *Minv,
                         ldbl *D, ldbl *Pmn, ldbl *Pnm) {
  const int n = p + 1, N = p;
  if (p < 0 || p > 6) return -1;
  ldbl P[NQMAX + 1], dP[NQMAX + 1];
  if (p == 0) {
    x[0] = 0.0L;
    w[0] = 2.0L;
  } else {
    x[0] = -1.0L;
    x[N] = 1.0L;
    const ldbl pi = 3.141592653589793238462643383279502884L;
    for (int i = 1; i < N; ++i) {
      ldbl xi = -cosl(pi * i / N);
      for (int it = 0; it < 200; ++it) {
        legendre_all(N, xi, P, dP);
        /* f = P_N'(x), f' = P_N''(x) from the Legendre equation */
        ldbl f = dP[N];
        ldbl fp = (2.0L * xi * dP[N] - N * (N + 1) * P[N]) / (1.0L - xi * xi);
        ldbl dx = f / fp;
        xi -= dx;
        if (fabsl(dx) < 1e-30L) break;
      }
      x[i] = xi;
    }
    for (int i = 0; i < n / 2; ++i) { /* exact symmetry of the node set */
      ldbl a = 0.5L * (x[N - i] - x[i]);
      x[i] = -a;
      x[N - i] = a;
    }
    if (n % 2 == 1) x[N / 2] = 0.0L;
    for (int i = 0; i < n; ++i) {
      legendre_all(N, x[i], P, dP);
      w[i] = 2.0L / (N * (N + 1) * P[N] * P[N]);
    }
  }
  /* Pmn(i,j) = P_j(x_i): evaluation of Legendre modes at the nodes */
  for (int i = 0; i < n; ++i) {
    legendre_all(N, x[i], P, dP);
    for (int j = 0; j < n; ++j) Pmn[i + n * j] = P[j];
  }
  if (invert_ld(n, Pmn, Pnm)) return -2;
  /* exact mass matrix of the Lagrange basis: M = Pnm^T diag(2/(2m+1)) Pnm */
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      ldbl acc = 0.0L;
      for (int m = 0; m < n; ++m) acc += Pnm[m + n * i] * Pnm[m + n * j] * (2.0L / (2 * m + 1));
      M[i + n * j] = acc;
    }
  if (invert_ld(n, M, Minv)) return -3;
  /* D(i,j) = l_j'(x_i) */
  if (p == 0) {
    D[0] = 0.0L;
  } else {
    ldbl PN[NQMAX];
    for (int i = 0; i < n; ++i) {
      legendre_all(N, x[i], P, dP);
      PN[i] = P[N];
    }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        if (i != j)
          D[i + n * j] = PN[i] / (PN[j] * (x[i] - x[j]));
        else if (i == 0)
          D[i + n * j] = -(ldbl)(N * (N + 1)) / 4.0L;
        else if (i == N)
          D[i + n * j] = (ldbl)(N * (N + 1)) / 4.0L;
        else
          D[i + n * j] = 0.0L;
      }
  }
  return 0;
}

int ora_gll_tables(int p, double *x, double *w, double *M, double *Minv, double *D, double *Pmn,
                   double *Pnm) {
  ldbl lx[NQMAX], lw[NQMAX], lM[NNMAX], lMi[NNMAX], lD[NNMAX], lPmn[NNMAX], lPnm[NNMAX];
  int rc = gll_tables_ld(p, lx, lw, lM, lMi, lD, lPmn, lPnm);
  if (rc) return rc;
  int n = p + 1;
  for (int i = 0; i < n; ++i) {
    if (x) x[i] = (double)lx[i];
    if (w) w[i] = (double)lw[i];
  }
  for (int i = 0; i < n * n; ++i) {
    if (M) M[i] = (double)lM[i];
    if (Minv) Minv[i] = (double)lMi[i];
    if (D) D[i] = (double)lD[i];
    if (Pmn) Pmn[i] = (double)lPmn[i];
    if (Pnm) Pnm[i] = (double)lPnm[i];
  }
  return 0;
}

/* gauss_legendre_matrix (gauss.f90:436-475) */
int ora_legendre_tables(int p, double *m, double *minv, double *D, double *tl, double *tr) {
  if (p < 0 || p > 6) return -1;
  int n = p + 1;
  for (int j = 0; j < n; ++j) {
    if (m) m[j] = 1.0 / (j + 0.5);
    if (minv) minv[j] = j + 0.5;
    if (tr) tr[j] = 1.0;
    if (tl) tl[j] = (j % 2 == 0) ? 1.0 : -1.0;
    if (D) {
      for (int i = 0; i < j; ++i) D[i + n * j] = ((j - i) % 2 == 1) ? 2.0 * i + 1.0 : 0.0;
      for (int i = j; i < n; ++i) D[i + n * j] = 0.0;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* LDF projector (LDF.f90)                                                                     */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int px, py;
  double Lx[NQMAX], Ly[NQMAX];
  double mx[NQMAX], my[NQMAX], invmx[NQMAX], invmy[NQMAX];
  double sqrtm2d[NNMAX], invm2d[NNMAX]; /* (px+1,py+1) */
  double Dx[NNMAX], Dy[NNMAX];
  double Ux[NNMAX], Uy[NNMAX];
  double Ldagger[NNMAX];
} ldf_t;

/* Singular value decomposition G = U diag(L) V^T of a small square matrix, L descending.
 * Replaces LAPACK DGESDD('A',...) (LDF.f90:182-193).  One-sided Jacobi (Hestenes) on G^T in
 * extended precision: G^T V = W diag(L)  =>  G = V diag(L) W^T, so the left singular vectors
 * of G are the accumulated rotations V.  The projector built from (U, L) is invariant to the
 * sign and in-eigenspace basis freedom of U. */
static void svd_left(int n, const double *G, double *U, double *L) {
  ldbl A[NQMAX][NQMAX], V[NQMAX][NQMAX]; /* A[c][r]: column c of G^T = row c of G */
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) {
      A[c][r] = G[c + n * r]; /* (G^T)(r,c) = G(c,r) */
      V[c][r] = (c == r) ? 1.0L : 0.0L;
    }
  for (int sweep = 0; sweep < 100; ++sweep) {
    int rotated = 0;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        ldbl al = 0, be = 0, ga = 0;
        for (int r = 0; r < n; ++r) {
          al += A[p][r] * A[p][r];
          be += A[q][r] * A[q][r];
          ga += A[p][r] * A[q][r];
        }
        if (ga == 0.0L || fabsl(ga) <= 1e-30L * sqrtl(al * be)) continue;
        rotated = 1;
        ldbl zeta = (be - al) / (2.0L * ga);
        ldbl t = (zeta >= 0 ? 1.0L : -1.0L) / (fabsl(zeta) + sqrtl(1.0L + zeta * zeta));
        ldbl c = 1.0L / sqrtl(1.0L + t * t), s = c * t;
        for (int r = 0; r < n; ++r) {
          ldbl ap = A[p][r], aq = A[q][r];
          A[p][r] = c * ap - s * aq;
          A[q][r] = s * ap + c * aq;
          ldbl vp = V[p][r], vq = V[q][r];
          V[p][r] = c * vp - s * vq;
          V[q][r] = s * vp + c * vq;
        }
      }
    if (!rotated) break;
  }
  ldbl sv[NQMAX];
  int order[NQMAX];
  for (int c = 0; c < n; ++c) {
    ldbl acc = 0;
    for (int r = 0; r < n; ++r) acc += A[c][r] * A[c][r];
    sv[c] = sqrtl(acc);
    order[c] = c;
  }
  for (int a = 0; a < n; ++a) /* sort descending (DGESDD order) */
    for (int b = a + 1; b < n; ++b)
      if (sv[order[b]] > sv[order[a]]) {
        int t = order[a];
        order[a] = order[b];
        order[b] = t;
      }
  for (int c = 0; c < n; ++c) {
    L[c] = (double)sv[order[c]];
    for (int r = 0; r < n; ++r) U[r + n * c] = (double)V[order[c]][r];
  }
}

/* LDF_projector%init (LDF.f90:114-217) */
static int ldf_init(ldf_t *P, int px, int py) {
  if (px < 0 || py < 0 || px > 6 || py > 6) return -1;
  memset(P, 0, sizeof(*P));
  P->px = px;
  P->py = py;
  int nx = px + 1, ny = py + 1;
  double tl[NQMAX], tr[NQMAX];
  ora_legendre_tables(px, P->mx, P->invmx, P->Dx, tl, tr);
  ora_legendre_tables(py, P->my, P->invmy, P->Dy, tl, tr);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) P->sqrtm2d[i + nx * j] = sqrt(P->mx[i] * P->my[j]);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) P->invm2d[i + nx * j] = P->invmx[i] * P->invmy[j];
  double sqx[NQMAX], sqy[NQMAX], Gx[NNMAX], Gy[NNMAX];
  for (int i = 0; i < nx; ++i) sqx[i] = sqrt(P->mx[i]);
  for (int i = 0; i < ny; ++i) sqy[i] = sqrt(P->my[i]);
  for (int j = 0; j < nx; ++j)
    for (int i = 0; i < nx; ++i) Gx[i + nx * j] = sqx[i] * P->Dx[i + nx * j] / sqx[j];
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < ny; ++i) Gy[i + ny * j] = sqy[i] * P->Dy[i + ny * j] / sqy[j];
  svd_left(nx, Gx, P->Ux, P->Lx);
  svd_left(ny, Gy, P->Uy, P->Ly);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      if (i < px || j < py) /* 1-based: i<=px .or. j<=py */
        P->Ldagger[i + nx * j] = 1.0 / (P->Lx[i] * P->Lx[i] + P->Ly[j] * P->Ly[j]);
      else
        P->Ldagger[i + nx * j] = 0.0;
    }
  return 0;
}

/* C(a x c) = A(a x b) * B(b x c), column-major, inner sum ascending */
static void mm(int a, int b, int c, const double *A, const double *B, double *C) {
  for (int j = 0; j < c; ++j)
    for (int i = 0; i < a; ++i) {
      double acc = 0.0;
      for (int m = 0; m < b; ++m) acc += A[i + a * m] * B[m + b * j];
      C[i + a * j] = acc;
    }
}
static void transpose(int a, int b, const double *A, double *At) {
  for (int j = 0; j < b; ++j)
    for (int i = 0; i < a; ++i) At[j + b * i] = A[i + a * j];
}

/* LDF_projector%apply (LDF.f90:219-250), combined form of :247-249 */
static void ldf_apply(const ldf_t *P, double *uu) {
  const int nx = P->px + 1, ny = P->py + 1, nn = nx * ny;
  double *u1 = uu, *u2 = uu + nn;
  double t1[NNMAX], t2[NNMAX], t3[NNMAX], DyT[NNMAX], UxT[NNMAX], UyT[NNMAX], DxT[NNMAX], udiv[NNMAX];
  transpose(ny, ny, P->Dy, DyT);
  transpose(nx, nx, P->Ux, UxT);
  transpose(ny, ny, P->Uy, UyT);
  transpose(nx, nx, P->Dx, DxT);
  /* sqrtm2d * (matmul(Dx, uu1) + matmul(uu2, transpose(Dy))) */
  mm(nx, nx, ny, P->Dx, u1, t1);
  mm(nx, ny, ny, u2, DyT, t2);
  for (int i = 0; i < nn; ++i) t1[i] = P->sqrtm2d[i] * (t1[i] + t2[i]);
  /* matmul(matmul(transpose(Ux), .), Uy) */
  mm(nx, nx, ny, UxT, t1, t2);
  mm(nx, ny, ny, t2, P->Uy, t3);
  /* Ldagger * . */
  for (int i = 0; i < nn; ++i) t3[i] = P->Ldagger[i] * t3[i];
  /* matmul(matmul(Ux, .), transpose(Uy)) */
  mm(nx, nx, ny, P->Ux, t3, t1);
  mm(nx, ny, ny, t1, UyT, t2);
  for (int i = 0; i < nn; ++i) udiv[i] = P->sqrtm2d[i] * t2[i];
  /* uu1 -= invm2d * matmul(transpose(Dx), udiv);  uu2 -= invm2d * matmul(udiv, Dy) */
  mm(nx, nx, ny, DxT, udiv, t1);
  mm(nx, ny, ny, udiv, P->Dy, t2);
  for (int i = 0; i < nn; ++i) {
    u1[i] = u1[i] - P->invm2d[i] * t1[i];
    u2[i] = u2[i] - P->invm2d[i] * t2[i];
  }
}

int ora_ldf_tables(int px, int py, double *Lx, double *Ux, double *Ly, double *Uy, double *Ldagger) {
  ldf_t P;
  if (ldf_init(&P, px, py)) return -1;
  int nx = px + 1, ny = py + 1;
  if (Lx) memcpy(Lx, P.Lx, sizeof(double) * nx);
  if (Ly) memcpy(Ly, P.Ly, sizeof(double) * ny);
  if (Ux) memcpy(Ux, P.Ux, sizeof(double) * nx * nx);
  if (Uy) memcpy(Uy, P.Uy, sizeof(double) * ny * ny);
  if (Ldagger) memcpy(Ldagger, P.Ldagger, sizeof(double) * nx * ny);
  return 0;
}
int ora_ldf_apply(int px, int py, double *uu) {
  ldf_t P;
  if (ldf_init(&P, px, py)) return -1;
  ldf_apply(&P, uu);
  return 0;
}
/* LDF_projector%div (LDF.f90:252-260) */
int ora_ldf_div(int px, int py, const double *uu, double *udiv) {
  ldf_t P;
  if (ldf_init(&P, px, py)) return -1;
  int nx = px + 1, ny = py + 1, nn = nx * ny;
  double DyT[NNMAX], t[NNMAX];
  transpose(ny, ny, P.Dy, DyT);
  mm(nx, nx, ny, P.Dx, uu, udiv);
  mm(nx, ny, ny, uu + nn, DyT, t);
  for (int i = 0; i < nn; ++i) udiv[i] = udiv[i] + t[i];
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Two-point fluxes                                                                            */
/* ------------------------------------------------------------------------------------------ */

/* log_avg_divisor (DG_solver.f90:1652-1681) */
double ora_log_avg_divisor(double LL, double RR) {
  const double eps = 1.4e-4;
  const double a0 = 1.0, a1 = 1.0 / 3.0, a2 = 1.0 / 5.0, a3 = 1.0 / 7.0;
  double zeta = LL / RR;
  double f = (zeta - 1.0) / (zeta + 1.0);
  double u = f * f;
  if (u < eps) return a0 + u * (a1 + u * (a2 + u * a3));
  return 0.5 * log(zeta) / f;
}

/* ec_flux_x (DG_solver.f90:1570-1609); p = (rho,vx,vy,vz,bx,by,bz,beta) */
void ora_ec_flux_x(const double *pl, const double *pr, double gamma, double *flux) {
  double rho_l = pl[0], vx_l = pl[1], vy_l = pl[2], vz_l = pl[3], bx_l = pl[4], by_l = pl[5], bz_l = pl[6], beta_l = pl[7];
  double rho_r = pr[0], vx_r = pr[1], vy_r = pr[2], vz_r = pr[3], bx_r = pr[4], by_r = pr[5], bz_r = pr[6], beta_r = pr[7];
  double rho_bar = 0.5 * (rho_l + rho_r);
  double vx_bar = 0.5 * (vx_l + vx_r);
  double vy_bar = 0.5 * (vy_l + vy_r);
  double vz_bar = 0.5 * (vz_l + vz_r);
  double bx_bar = 0.5 * (bx_l + bx_r);
  double by_bar = 0.5 * (by_l + by_r);
  double bz_bar = 0.5 * (bz_l + bz_r);
  double beta_bar = 0.5 * (beta_l + beta_r);
  double v_sq_bar = 0.5 * ((vx_l * vx_l + vy_l * vy_l + vz_l * vz_l) + (vx_r * vx_r + vy_r * vy_r + vz_r * vz_r));
  double b_sq_bar = 0.5 * ((bx_l * bx_l + by_l * by_l + bz_l * bz_l) + (bx_r * bx_r + by_r * by_r + bz_r * bz_r));
  double betavx_bar = 0.5 * (beta_l * vx_l + beta_r * vx_r);
  double betavy_bar = 0.5 * (beta_l * vy_l + beta_r * vy_r);
  double betavz_bar = 0.5 * (beta_l * vz_l + beta_r * vz_r);
  double rho_hat = rho_bar / ora_log_avg_divisor(rho_l, rho_r);
  double beta_hat = beta_bar / ora_log_avg_divisor(beta_l, beta_r);
  flux[0] = rho_hat * vx_bar;
  flux[1] = vx_bar * flux[0] - bx_bar * bx_bar + 0.5 * (b_sq_bar + rho_bar / beta_bar);
  flux[2] = vy_bar * flux[0] - bx_bar * by_bar + 0.0;
  flux[3] = vz_bar * flux[0] - bx_bar * bz_bar + 0.0;
  flux[4] = 0.0;
  flux[5] = (betavx_bar * by_bar - betavy_bar * bx_bar) / beta_bar;
  flux[6] = (betavx_bar * bz_bar - betavz_bar * bx_bar) / beta_bar;
  flux[7] = 0.5 * (1.0 / ((gamma - 1.0) * beta_hat) - v_sq_bar) * flux[0] +
            (vx_bar * flux[1] + vy_bar * flux[2] + vz_bar * flux[3]) +
            (bx_bar * flux[4] + by_bar * flux[5] + bz_bar * flux[6]) - 0.5 * vx_bar * b_sq_bar +
            (vx_bar * bx_bar + vy_bar * by_bar + vz_bar * bz_bar) * bx_bar;
}

/* ec_flux_y (DG_solver.f90:1611-1650) */
void ora_ec_flux_y(const double *pl, const double *pr, double gamma, double *flux) {
  double rho_l = pl[0], vx_l = pl[1], vy_l = pl[2], vz_l = pl[3], bx_l = pl[4], by_l = pl[5], bz_l = pl[6], beta_l = pl[7];
  double rho_r = pr[0], vx_r = pr[1], vy_r = pr[2], vz_r = pr[3], bx_r = pr[4], by_r = pr[5], bz_r = pr[6], beta_r = pr[7];
  double rho_bar = 0.5 * (rho_l + rho_r);
  double vx_bar = 0.5 * (vx_l + vx_r);
  double vy_bar = 0.5 * (vy_l + vy_r);
  double vz_bar = 0.5 * (vz_l + vz_r);
  double bx_bar = 0.5 * (bx_l + bx_r);
  double by_bar = 0.5 * (by_l + by_r);
  double bz_bar = 0.5 * (bz_l + bz_r);
  double beta_bar = 0.5 * (beta_l + beta_r);
  double v_sq_bar = 0.5 * ((vx_l * vx_l + vy_l * vy_l + vz_l * vz_l) + (vx_r * vx_r + vy_r * vy_r + vz_r * vz_r));
  double b_sq_bar = 0.5 * ((bx_l * bx_l + by_l * by_l + bz_l * bz_l) + (bx_r * bx_r + by_r * by_r + bz_r * bz_r));
  double betavx_bar = 0.5 * (beta_l * vx_l + beta_r * vx_r);
  double betavy_bar = 0.5 * (beta_l * vy_l + beta_r * vy_r);
  double betavz_bar = 0.5 * (beta_l * vz_l + beta_r * vz_r);
  double rho_hat = rho_bar / ora_log_avg_divisor(rho_l, rho_r);
  double beta_hat = beta_bar / ora_log_avg_divisor(beta_l, beta_r);
  flux[0] = rho_hat * vy_bar;
  flux[1] = vx_bar * flux[0] - by_bar * bx_bar + 0.0;
  flux[2] = vy_bar * flux[0] - by_bar * by_bar + 0.5 * (b_sq_bar + rho_bar / beta_bar);
  flux[3] = vz_bar * flux[0] - by_bar * bz_bar + 0.0;
  flux[4] = (betavy_bar * bx_bar - betavx_bar * by_bar) / beta_bar;
  flux[5] = 0.0;
  flux[6] = (betavy_bar * bz_bar - betavz_bar * by_bar) / beta_bar;
  flux[7] = 0.5 * (1.0 / ((gamma - 1.0) * beta_hat) - v_sq_bar) * flux[0] +
            (vx_bar * flux[1] + vy_bar * flux[2] + vz_bar * flux[3]) +
            (bx_bar * flux[4] + by_bar * flux[5] + bz_bar * flux[6]) - 0.5 * vy_bar * b_sq_bar +
            (vx_bar * bx_bar + vy_bar * by_bar + vz_bar * bz_bar) * by_bar;
}

/* ESPP_HLL_flux_x (DG_solver.f90:894-1071) */
void ora_hll_flux_x(const double *w_l, const double *w_r, double gamma, double *nflux, double *nBn,
                    double *sl_out, double *sr_out) {
  double rho_l = w_l[0], mx_l = w_l[1], my_l = w_l[2], mz_l = w_l[3], bx_l = w_l[4], by_l = w_l[5], bz_l = w_l[6], e_tot_l = w_l[7];
  double rho_r = w_r[0], mx_r = w_r[1], my_r = w_r[2], mz_r = w_r[3], bx_r = w_r[4], by_r = w_r[5], bz_r = w_r[6], e_tot_r = w_r[7];
  double inv_rho_l = 1.0 / rho_l, inv_rho_r = 1.0 / rho_r;
  double vx_l = inv_rho_l * mx_l, vx_r = inv_rho_r * mx_r;
  double vy_l = inv_rho_l * my_l, vy_r = inv_rho_r * my_r;
  double vz_l = inv_rho_l * mz_l, vz_r = inv_rho_r * mz_r;
  double e_knt_l = 0.5 * inv_rho_l * (mx_l * mx_l + my_l * my_l + mz_l * mz_l);
  double e_knt_r = 0.5 * inv_rho_r * (mx_r * mx_r + my_r * my_r + mz_r * mz_r);
  double ey_l = bz_l * vx_l - bx_l * vz_l, ey_r = bz_r * vx_r - bx_r * vz_r;
  double ez_l = bx_l * vy_l - by_l * vx_l, ez_r = bx_r * vy_r - by_r * vx_r;
  double b_sq_l = bx_l * bx_l + by_l * by_l + bz_l * bz_l;
  double b_sq_r = bx_r * bx_r + by_r * by_r + bz_r * bz_r;
  double p_mag_l = 0.5 * b_sq_l, p_mag_r = 0.5 * b_sq_r;
  double p_fld_l = dmax((gamma - 1.0) * (e_tot_l - (e_knt_l + p_mag_l)), PP_eps);
  double p_fld_r = dmax((gamma - 1.0) * (e_tot_r - (e_knt_r + p_mag_r)), PP_eps);
  double p_tot_l = p_fld_l + p_mag_l, p_tot_r = p_fld_r + p_mag_r;
  double b_dot_u_l = bx_l * vx_l + by_l * vy_l + bz_l * vz_l;
  double b_dot_u_r = bx_r * vx_r + by_r * vy_r + bz_r * vz_r;
  double snc_sq_l = gamma * p_fld_l * inv_rho_l, snc_sq_r = gamma * p_fld_r * inv_rho_r;
  double alfven_sq_l = b_sq_l * inv_rho_l, alfven_sq_r = b_sq_r * inv_rho_r;
  double sum_sq_l = snc_sq_l + alfven_sq_l, sum_sq_r = snc_sq_r + alfven_sq_r;
  double cfx_l = sqrt(0.5 * (sum_sq_l + sqrt(dmax(sum_sq_l * sum_sq_l - 4 * snc_sq_l * inv_rho_l * (bx_l * bx_l), 0.0))));
  double cfx_r = sqrt(0.5 * (sum_sq_r + sqrt(dmax(sum_sq_r * sum_sq_r - 4 * snc_sq_r * inv_rho_r * (bx_r * bx_r), 0.0))));
  double inv_theta_l = rho_l / p_fld_l, inv_theta_r = rho_r / p_fld_r;
  double phi_l = inv_theta_l * b_dot_u_l, phi_r = inv_theta_r * b_dot_u_r;
  double sp_ent_l = log(p_fld_l) - gamma * log(rho_l);
  double sp_ent_r = log(p_fld_r) - gamma * log(rho_r);
  double ent_fun_l = -rho_l * sp_ent_l / (gamma - 1.0);
  double ent_fun_r = -rho_r * sp_ent_r / (gamma - 1.0);
  double ent_flux_l = ent_fun_l * vx_l, ent_flux_r = ent_fun_r * vx_r;
  double flux_l[8], flux_r[8], entv_l[8], entv_r[8];
  flux_l[0] = mx_l;
  flux_l[1] = vx_l * mx_l - bx_l * bx_l + p_tot_l;
  flux_l[2] = vx_l * my_l - by_l * bx_l;
  flux_l[3] = vx_l * mz_l - bz_l * bx_l;
  flux_l[4] = 0.0;
  flux_l[5] = -ez_l;
  flux_l[6] = ey_l;
  flux_l[7] = vx_l * (e_tot_l + p_tot_l) - bx_l * b_dot_u_l;
  flux_r[0] = mx_r;
  flux_r[1] = vx_r * mx_r - bx_r * bx_r + p_tot_r;
  flux_r[2] = vx_r * my_r - by_r * bx_r;
  flux_r[3] = vx_r * mz_r - bz_r * bx_r;
  flux_r[4] = 0.0;
  flux_r[5] = -ez_r;
  flux_r[6] = ey_r;
  flux_r[7] = vx_r * (e_tot_r + p_tot_r) - bx_r * b_dot_u_r;
  entv_l[0] = (gamma - sp_ent_l) / (gamma - 1.0) - e_knt_l / p_fld_l;
  entv_l[1] = mx_l / p_fld_l;
  entv_l[2] = my_l / p_fld_l;
  entv_l[3] = mz_l / p_fld_l;
  entv_l[4] = inv_theta_l * bx_l;
  entv_l[5] = inv_theta_l * by_l;
  entv_l[6] = inv_theta_l * bz_l;
  entv_l[7] = -inv_theta_l;
  entv_r[0] = (gamma - sp_ent_r) / (gamma - 1.0) - e_knt_r / p_fld_r;
  entv_r[1] = mx_r / p_fld_r;
  entv_r[2] = my_r / p_fld_r;
  entv_r[3] = mz_r / p_fld_r;
  entv_r[4] = inv_theta_r * bx_r;
  entv_r[5] = inv_theta_r * by_r;
  entv_r[6] = inv_theta_r * bz_r;
  entv_r[7] = -inv_theta_r;
  double sqrt_rho_l = sqrt(rho_l), sqrt_rho_r = sqrt(rho_r);
  double sum_sqrt_rho = sqrt_rho_l + sqrt_rho_r;
  double vx_roe = (vx_l * sqrt_rho_l + vx_r * sqrt_rho_r) / sum_sqrt_rho;
  double db_aux = sqrt((bx_l - bx_r) * (bx_l - bx_r) + (by_l - by_r) * (by_l - by_r) + (bz_l - bz_r) * (bz_l - bz_r)) / sum_sqrt_rho;
  double sl_pp = dmin(vx_l, vx_roe) - cfx_l - db_aux;
  double sr_pp = dmax(vx_r, vx_roe) + cfx_r + db_aux;
  double dot_a = 0.0, dot_bl = 0.0, dot_br = 0.0;
  for (int s = 0; s < 8; ++s) dot_a += (entv_r[s] - entv_l[s]) * (w_r[s] - w_l[s]);
  for (int s = 0; s < 8; ++s) dot_bl += entv_l[s] * (flux_r[s] - flux_l[s]);
  for (int s = 0; s < 8; ++s) dot_br += entv_r[s] * (flux_r[s] - flux_l[s]);
  double a_form = dmax(dot_a, 0.0) + 1e-8;
  double bl_form = (ent_flux_r - ent_flux_l) - dot_bl - phi_l * (bx_r - bx_l);
  double br_form = (ent_flux_r - ent_flux_l) - dot_br - phi_r * (bx_r - bx_l);
  double al_form = dmax(bl_form / a_form, 0.0);
  double ar_form = dmax(br_form / a_form, 0.0);
  double aa_form = sqrt(al_form * ar_form);
  double sl_es = -(ar_form + aa_form);
  double sr_es = +(al_form + aa_form);
  double sl = dmin(dmin(sl_es, sl_pp), 0.0);
  double sr = dmax(dmax(sr_es, sr_pp), 0.0);
  double dslr = sr - sl;
  double wei_l = sr / dslr, wei_r = -sl / dslr;
  for (int s = 0; s < 8; ++s) nflux[s] = wei_l * flux_l[s] + wei_r * flux_r[s] + ((sl * sr) / dslr) * (w_r[s] - w_l[s]);
  *nBn = wei_l * bx_l + wei_r * bx_r;
  *sl_out = sl;
  *sr_out = sr;
}

/* swap_xy (DG_solver.f90:1556-1568) */
static inline void swap_xy(const double *in, double *out) {
  out[0] = in[0];
  out[1] = in[2];
  out[2] = in[1];
  out[3] = in[3];
  out[4] = in[5];
  out[5] = in[4];
  out[6] = in[6];
  out[7] = in[7];
}

/* ------------------------------------------------------------------------------------------ */
/* Solver state (DG_solver.f90:6-43 module data)                                               */
/* ------------------------------------------------------------------------------------------ */
struct ora_solver {
  int nx, ny, px, py, nqx, nqy, nn, rknstg, bc_kind;
  double left, right, bottom, top, hx, hy, gamma;
  double bc_state[8];
  double qx_x[NQMAX], qw_x[NQMAX], qx_y[NQMAX], qw_y[NQMAX];
  double diff_x[NNMAX], diff_y[NNMAX], M_x[NNMAX], Minv_x[NNMAX], M_y[NNMAX], Minv_y[NNMAX];
  double Pmn_x[NNMAX], Pnm_x[NNMAX], Pmn_y[NNMAX], Pnm_y[NNMAX];
  ldf_t ldf;
  double *u_avg, *u_con, *ut_con, *uRK_con;
  double *sxl, *sxr, *syd, *syu, *nflux_x, *nflux_y, *nB_x, *nB_y;
  double *sigsum_x, *sigsum_y;
  double *cell_ent_DG, *cell_ent_FV;
  unsigned char *cell_ent_nan;
  double *rowbuf; /* per-row partial sums (deterministic reductions) */
  double run_t, run_dt, run_dt_lim, run_tot_ent; /* driver scalars kept between ora_solve_resume calls */
};

long ora_size_u(const ora_solver *s) { return 8L * s->nn * (s->nx + 2) * (s->ny + 2); }
long ora_size_ut(const ora_solver *s) { return 8L * s->nn * s->nx * s->ny; }
long ora_size_avg(const ora_solver *s) { return 8L * (s->nx + 2) * (s->ny + 2); }
double *ora_u_con(ora_solver *s) { return s->u_con; }
double *ora_ut_con(ora_solver *s, int st) { return s->ut_con + (long)(st - 1) * ora_size_ut(s); }
double *ora_urk_con(ora_solver *s, int st) { return s->uRK_con + (long)(st - 1) * ora_size_u(s); }
double *ora_u_avg(ora_solver *s) { return s->u_avg; }

/* element block (i,j) of a ghosted array (i in 0..nx+1, j in 0..ny+1) */
static inline double *EB(const ora_solver *s, double *u, int i, int j) {
  return u + 8L * s->nn * (i + (long)(s->nx + 2) * j);
}
static inline const double *EBc(const ora_solver *s, const double *u, int i, int j) {
  return u + 8L * s->nn * (i + (long)(s->nx + 2) * j);
}
/* interior block of ut (i in 1..nx, j in 1..ny) */
static inline double *UTB(const ora_solver *s, double *ut, int i, int j) {
  return ut + 8L * s->nn * ((i - 1) + (long)s->nx * (j - 1));
}
#define NODE(s_, v, k, l) ((v) + 8 * ((k) + (s_)->nqx * (l)))

static double *nan_alloc(long n) {
  double *p = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  if (!p) return NULL;
  double q = NAN;
  for (long i = 0; i < n; ++i) p[i] = q;
  return p;
}

/* init_DG_solver (DG_solver.f90:47-107) plus BC selection */
ora_solver *ora_create(int nx, int ny, int px, int py, int rknstg, double left, double right,
                       double bottom, double top, double gamma, int bc_kind, const double *bc_state8) {
  if (nx < 1 || ny < 1 || px < 0 || py < 0 || px > 6 || py > 6) return NULL;
  if (!(rknstg == 1 || rknstg == 2 || rknstg == 3 || rknstg == 5)) return NULL;
  ora_solver *s = (ora_solver *)calloc(1, sizeof(ora_solver));
  s->nx = nx;
  s->ny = ny;
  s->px = px;
  s->py = py;
  s->nqx = px + 1;
  s->nqy = py + 1;
  s->nn = s->nqx * s->nqy;
  s->rknstg = rknstg;
  s->left = left;
  s->right = right;
  s->bottom = bottom;
  s->top = top;
  s->gamma = gamma;
  s->bc_kind = bc_kind;
  for (int v = 0; v < 8; ++v) {
    if (bc_state8)
      s->bc_state[v] = bc_state8[v];
    else
      s->bc_state[v] = NAN;
  }
  ora_gll_tables(px, s->qx_x, s->qw_x, s->M_x, s->Minv_x, s->diff_x, s->Pmn_x, s->Pnm_x);
  ora_gll_tables(py, s->qx_y, s->qw_y, s->M_y, s->Minv_y, s->diff_y, s->Pmn_y, s->Pnm_y);
  ldf_init(&s->ldf, px, py);
  s->hx = (right - left) / nx;
  s->hy = (top - bottom) / ny;
  s->u_avg = nan_alloc(ora_size_avg(s));
  s->u_con = nan_alloc(ora_size_u(s));
  s->ut_con = nan_alloc(ora_size_ut(s) * rknstg);
  s->uRK_con = nan_alloc(ora_size_u(s) * rknstg);
  s->sxl = nan_alloc((long)s->nqy * (nx + 1) * ny);
  s->sxr = nan_alloc((long)s->nqy * (nx + 1) * ny);
  s->syd = nan_alloc((long)s->nqx * nx * (ny + 1));
  s->syu = nan_alloc((long)s->nqx * nx * (ny + 1));
  s->nflux_x = nan_alloc(8L * s->nqy * (nx + 1) * ny);
  s->nflux_y = nan_alloc(8L * s->nqx * nx * (ny + 1));
  s->nB_x = nan_alloc((long)s->nqy * (nx + 1) * ny);
  s->nB_y = nan_alloc((long)s->nqx * nx * (ny + 1));
  s->sigsum_x = nan_alloc(8L * (nx + 1) * ny);
  s->sigsum_y = nan_alloc(8L * nx * (ny + 1));
  s->cell_ent_DG = nan_alloc((long)(nx + 2) * (ny + 2));
  s->cell_ent_FV = nan_alloc((long)(nx + 2) * (ny + 2));
  s->cell_ent_nan = (unsigned char *)malloc((size_t)(nx + 2) * (ny + 2));
  memset(s->cell_ent_nan, 1, (size_t)(nx + 2) * (ny + 2));
  s->rowbuf = (double *)calloc(16L * (ny + 2), sizeof(double));
  return s;
}

void ora_destroy(ora_solver *s) {
  if (!s) return;
  free(s->u_avg);
  free(s->u_con);
  free(s->ut_con);
  free(s->uRK_con);
  free(s->sxl);
  free(s->sxr);
  free(s->syd);
  free(s->syu);
  free(s->nflux_x);
  free(s->nflux_y);
  free(s->nB_x);
  free(s->nB_y);
  free(s->sigsum_x);
  free(s->sigsum_y);
  free(s->cell_ent_DG);
  free(s->cell_ent_FV);
  free(s->cell_ent_nan);
  free(s->rowbuf);
  free(s);
}

/* node coordinates (DG_solver.f90:101-106) */
void ora_nodes(const ora_solver *s, double *xx, double *yy) {
  for (int i = 1; i <= s->nx; ++i)
    for (int k = 0; k < s->nqx; ++k)
      xx[k + s->nqx * (i - 1)] = (0.5 * s->hx) * s->qx_x[k] + (s->left + (i - 0.5) * s->hx);
  for (int j = 1; j <= s->ny; ++j)
    for (int l = 0; l < s->nqy; ++l)
      yy[l + s->nqy * (j - 1)] = (0.5 * s->hy) * s->qx_y[l] + (s->bottom + (j - 0.5) * s->hy);
}

void ora_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int ora_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------------------------ */
/* Boundary conditions (problems.f90)                                                          */
/* ------------------------------------------------------------------------------------------ */
void ora_apply_bc(ora_solver *s, double *u) {
  const int nx = s->nx, ny = s->ny, nq = s->nn;
  const size_t blk = sizeof(double) * 8 * nq;
  switch (s->bc_kind) {
    case ORA_BC_PERIODIC: /* problems.f90:312-348 */
#pragma omp parallel for schedule(static)
      for (int j = 1; j <= ny; ++j) {
        memcpy(EB(s, u, 0, j), EB(s, u, nx, j), blk);
        memcpy(EB(s, u, nx + 1, j), EB(s, u, 1, j), blk);
      }
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= nx; ++i) {
        memcpy(EB(s, u, i, 0), EB(s, u, i, ny), blk);
        memcpy(EB(s, u, i, ny + 1), EB(s, u, i, 1), blk);
      }
      break;
    case ORA_BC_EXTRAPOLATE: /* problems.f90:386-423 */
#pragma omp parallel for schedule(static)
      for (int j = 1; j <= ny; ++j)
        for (int l = 0; l < s->nqy; ++l)
          for (int k = 0; k < s->nqx; ++k)
            for (int v = 0; v < 8; ++v) {
              EB(s, u, 0, j)[NODE(s, v, k, l)] = EB(s, u, 1, j)[NODE(s, v, 0, l)];
              EB(s, u, nx + 1, j)[NODE(s, v, k, l)] = EB(s, u, nx, j)[NODE(s, v, s->px, l)];
            }
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= nx; ++i)
        for (int l = 0; l < s->nqy; ++l)
          for (int k = 0; k < s->nqx; ++k)
            for (int v = 0; v < 8; ++v) {
              EB(s, u, i, 0)[NODE(s, v, k, l)] = EB(s, u, i, 1)[NODE(s, v, k, 0)];
              EB(s, u, i, ny + 1)[NODE(s, v, k, l)] = EB(s, u, i, ny)[NODE(s, v, k, s->py)];
            }
      break;
    case ORA_BC_FIXED: /* problems.f90:597-654 with the given conserved state */
#pragma omp parallel for schedule(static)
      for (int j = 1; j <= ny; ++j)
        for (int q = 0; q < nq; ++q)
          for (int v = 0; v < 8; ++v) {
            EB(s, u, 0, j)[v + 8 * q] = s->bc_state[v];
            EB(s, u, nx + 1, j)[v + 8 * q] = s->bc_state[v];
          }
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= nx; ++i)
        for (int q = 0; q < nq; ++q)
          for (int v = 0; v < 8; ++v) {
            EB(s, u, i, 0)[v + 8 * q] = s->bc_state[v];
            EB(s, u, i, ny + 1)[v + 8 * q] = s->bc_state[v];
          }
      break;
    case ORA_BC_XEXTRAP_YPER: /* problems.f90:350-384 */
#pragma omp parallel for schedule(static)
      for (int j = 1; j <= ny; ++j)
        for (int l = 0; l < s->nqy; ++l)
          for (int k = 0; k < s->nqx; ++k)
            for (int v = 0; v < 8; ++v) {
              EB(s, u, 0, j)[NODE(s, v, k, l)] = EB(s, u, 1, j)[NODE(s, v, 0, l)];
              EB(s, u, nx + 1, j)[NODE(s, v, k, l)] = EB(s, u, nx, j)[NODE(s, v, s->px, l)];
            }
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= nx; ++i) {
        memcpy(EB(s, u, i, 0), EB(s, u, i, ny), blk);
        memcpy(EB(s, u, i, ny + 1), EB(s, u, i, 1), blk);
      }
      break;
    case ORA_BC_CLOUD_SHOCK: /* problems.f90:449-471: copies, and the inflow state on the right */
#pragma omp parallel for schedule(static)
      for (int j = 1; j <= ny; ++j) {
        memcpy(EB(s, u, 0, j), EB(s, u, 1, j), blk);
        for (int q = 0; q < nq; ++q)
          for (int v = 0; v < 8; ++v) EB(s, u, nx + 1, j)[v + 8 * q] = s->bc_state[v];
      }
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= nx; ++i) {
        memcpy(EB(s, u, i, 0), EB(s, u, i, 1), blk);
        memcpy(EB(s, u, i, ny + 1), EB(s, u, i, ny), blk);
      }
      break;
    case ORA_BC_JET: /* problems.f90:502-593 */
#pragma omp parallel for schedule(static)
      for (int j = 1; j <= ny; ++j) {
        /* left: mirror of element 1 in x (node k <- px-k), normal momentum and field negated */
        for (int l = 0; l < s->nqy; ++l)
          for (int k = 0; k < s->nqx; ++k)
            for (int v = 0; v < 8; ++v) {
              const double x = EB(s, u, 1, j)[NODE(s, v, s->px - k, l)];
              EB(s, u, 0, j)[NODE(s, v, k, l)] = (v == 1 || v == 4) ? -x : x;
            }
        /* right: copy element nx */
        memcpy(EB(s, u, nx + 1, j), EB(s, u, nx, j), blk);
      }
#pragma omp parallel for schedule(static)
      for (int i = 1; i <= nx; ++i) {
        if (i <= nx / 10) { /* the nozzle (the reference requires nx to be a multiple of 10) */
          for (int q = 0; q < nq; ++q)
            for (int v = 0; v < 8; ++v) EB(s, u, i, 0)[v + 8 * q] = s->bc_state[v];
        } else {
          memcpy(EB(s, u, i, 0), EB(s, u, i, 1), blk);
        }
        memcpy(EB(s, u, i, ny + 1), EB(s, u, i, ny), blk);
      }
      break;
    default:
      break;
  }
}

/* ------------------------------------------------------------------------------------------ */
/* post_process (DG_solver.f90:128-661)                                                        */
/* ------------------------------------------------------------------------------------------ */
static void oedg_sigsum_xface(const ora_solver *s, const double *uthis, const double *uleft, int v,
                              double *out) {
  /* DG_solver.f90:309-343 for one variable */
  const int px = s->px, py = s->py, nqx = s->nqx, nqy = s->nqy;
  const double hx = s->hx, hy = s->hy;
  double dll[NNMAX], drr[NNMAX], tmp[NNMAX], jump[NQMAX], jt[NQMAX];
  double Dxs[NNMAX], Dys[NNMAX];
  for (int q = 0; q < nqx * nqx; ++q) Dxs[q] = (2.0 / hx) * s->diff_x[q];
  for (int q = 0; q < nqy * nqy; ++q) Dys[q] = (2.0 / hy) * s->diff_y[q];
  for (int l = 0; l < nqy; ++l)
    for (int k = 0; k < nqx; ++k) {
      dll[k + nqx * l] = uleft[NODE(s, v, k, l)];
      drr[k + nqx * l] = uthis[NODE(s, v, k, l)];
    }
  double total = 0.0;
  int fac_kk = 1;
  double hx_pow_kk = 1.0;
  for (int kk = 0; kk <= px; ++kk) {
    for (int l = 0; l < nqy; ++l) jump[l] = drr[0 + nqx * l] - dll[px + nqx * l];
    int fac_ll = 1;
    double hx_pow = hx_pow_kk;
    for (int ll = 0; ll <= imax(px, py) - kk; ++ll) {
      int mm_ = kk + ll;
      double L1 = 0.0;
      for (int l = 0; l < nqy; ++l) L1 += (0.5 * s->qw_y[l]) * fabs(jump[l]);
      double coef = ((2 * mm_ + 1) * hx_pow) / (double)(2 * imax(2 * px - 1, 1) * fac_kk * fac_ll);
      total = total + coef * L1;
      if (ll < py) {
        mm(nqy, nqy, 1, Dys, jump, jt);
        memcpy(jump, jt, sizeof(double) * nqy);
        fac_ll = fac_ll * (ll + 1);
        hx_pow = hx_pow * hx;
      }
    }
    if (kk < px) {
      mm(nqx, nqx, nqy, Dxs, dll, tmp);
      memcpy(dll, tmp, sizeof(double) * nqx * nqy);
      mm(nqx, nqx, nqy, Dxs, drr, tmp);
      memcpy(drr, tmp, sizeof(double) * nqx * nqy);
      fac_kk = fac_kk * (kk + 1);
      hx_pow_kk = hx_pow_kk * hx;
    }
  }
  *out = total;
}

static void oedg_sigsum_yface(const ora_solver *s, const double *uthis, const double *ubott, int v,
                              double *out) {
  /* DG_solver.f90:373-407 for one variable */
  const int px = s->px, py = s->py, nqx = s->nqx, nqy = s->nqy;
  const double hx = s->hx, hy = s->hy;
  double ddd[NNMAX], duu[NNMAX], tmp[NNMAX], jump[NQMAX], jt[NQMAX];
  double Dxs[NNMAX], DysT[NNMAX];
  for (int q = 0; q < nqx * nqx; ++q) Dxs[q] = (2.0 / hx) * s->diff_x[q];
  for (int a = 0; a < nqy; ++a)
    for (int b = 0; b < nqy; ++b) DysT[a + nqy * b] = (2.0 / hy) * s->diff_y[b + nqy * a];
  for (int l = 0; l < nqy; ++l)
    for (int k = 0; k < nqx; ++k) {
      ddd[k + nqx * l] = ubott[NODE(s, v, k, l)];
      duu[k + nqx * l] = uthis[NODE(s, v, k, l)];
    }
  double total = 0.0;
  int fac_ll = 1;
  double hy_pow_ll = 1.0;
  for (int ll = 0; ll <= py; ++ll) {
    for (int k = 0; k < nqx; ++k) jump[k] = duu[k + nqx * 0] - ddd[k + nqx * py];
    int fac_kk = 1;
    double hy_pow = hy_pow_ll;
    for (int kk = 0; kk <= imax(px, py) - ll; ++kk) {
      int mm_ = kk + ll;
      double L1 = 0.0;
      for (int k = 0; k < nqx; ++k) L1 += (0.5 * s->qw_x[k]) * fabs(jump[k]);
      double coef = ((2 * mm_ + 1) * hy_pow) / (double)(2 * imax(2 * py - 1, 1) * fac_kk * fac_ll);
      total = total + coef * L1;
      if (kk < px) {
        mm(nqx, nqx, 1, Dxs, jump, jt);
        memcpy(jump, jt, sizeof(double) * nqx);
        fac_kk = fac_kk * (kk + 1);
        hy_pow = hy_pow * hy;
      }
    }
    if (ll < py) {
      mm(nqx, nqy, nqy, ddd, DysT, tmp);
      memcpy(ddd, tmp, sizeof(double) * nqx * nqy);
      mm(nqx, nqy, nqy, duu, DysT, tmp);
      memcpy(duu, tmp, sizeof(double) * nqx * nqy);
      fac_ll = fac_ll * (ll + 1);
      hy_pow_ll = hy_pow_ll * hy;
    }
  }
  *out = total;
}

void ora_post_process(ora_solver *s, double *u, double *u_avg, int *neg_avg_out, int *num_negcell_out,
                      int apply_oedg, int apply_ldf, double oedg_dt, int ent_offset, int comput_ent,
                      double *tot_ent_out, int *pp_relimit_fail_out) {
  const int nx = s->nx, ny = s->ny, px = s->px, py = s->py, nqx = s->nqx, nqy = s->nqy, nq = s->nn;
  const double gamma = s->gamma, hx = s->hx, hy = s->hy;
  int neg_avg = 0, num_negcell = 0, relimit_fail = 0;
  double tot_ent = 0.0;
  double u_avg_global[8] = {0}, u_vari_global[8] = {0};
  double *rowsum = s->rowbuf; /* (ny+2) x 16 */

  /* loop 1: cell averages, admissibility, LDF (DG_solver.f90:161-277) */
#pragma omp parallel for schedule(static) reduction(| : neg_avg)
  for (int j = 0; j <= ny + 1; ++j) {
    double racc[8] = {0};
    for (int i = 0; i <= nx + 1; ++i) {
      if (!((i >= 1 && i <= nx) || (j >= 1 && j <= ny))) continue;
      double uc[8 * NNMAX], ua[8];
      memcpy(uc, EB(s, u, i, j), sizeof(double) * 8 * nq);
      for (int v = 0; v < 8; ++v) ua[v] = 0.0;
      for (int l = 0; l < nqy; ++l)
        for (int k = 0; k < nqx; ++k)
          for (int v = 0; v < 8; ++v) ua[v] = ua[v] + (0.25 * s->qw_x[k] * s->qw_y[l]) * uc[NODE(s, v, k, l)];
      double den_avg = ua[0];
      double prs_avg = prs_macro(ua[0], ua[1], ua[2], ua[3], ua[4], ua[5], ua[6], ua[7], gamma);
      if (den_avg < PP_eps || prs_avg < PP_eps) {
        neg_avg = 1;
        continue;
      }
      int cell_nan = 1;
      double cell_ent = NAN, ent_avg = NAN;
      if (ent_offset) {
        ent_avg = ent_macro(den_avg, prs_avg, gamma);
        double rho[NNMAX], prs[NNMAX];
        int flag = 1;
        for (int l = 0; l < nqy; ++l)
          for (int k = 0; k < nqx; ++k) {
            const double *w = uc + 8 * (k + nqx * l);
            rho[k + nqx * l] = w[0];
            prs[k + nqx * l] = prs_macro(w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], gamma);
            flag = flag && (rho[k + nqx * l] >= PP_eps) && (prs[k + nqx * l] >= PP_eps);
          }
        if (flag) {
          cell_nan = 0;
          cell_ent = 0.0;
          for (int l = 0; l < nqy; ++l)
            for (int k = 0; k < nqx; ++k)
              cell_ent = cell_ent + (0.25 * hx * hy * s->qw_x[k] * s->qw_y[l]) * ent_macro(rho[k + nqx * l], prs[k + nqx * l], gamma);
        }
      }
      if ((i >= 1 && i <= nx) && (j >= 1 && j <= ny))
        for (int v = 0; v < 8; ++v) racc[v] = racc[v] + (hx * hy) * ua[v];
      if (apply_ldf) {
        double mag_val[2 * NNMAX], mag_coef[2 * NNMAX], t1[NNMAX], PnmyT[NNMAX], PmnyT[NNMAX];
        for (int l = 0; l < nqy; ++l)
          for (int k = 0; k < nqx; ++k) {
            mag_val[k + nqx * l] = (0.5 * hy) * (uc[NODE(s, 4, k, l)] - ua[4]);
            mag_val[nq + k + nqx * l] = (0.5 * hx) * (uc[NODE(s, 5, k, l)] - ua[5]);
          }
        transpose(nqy, nqy, s->Pnm_y, PnmyT);
        transpose(nqy, nqy, s->Pmn_y, PmnyT);
        for (int c = 0; c < 2; ++c) {
          mm(nqx, nqx, nqy, s->Pnm_x, mag_val + c * nq, t1);
          mm(nqx, nqy, nqy, t1, PnmyT, mag_coef + c * nq);
        }
        ldf_apply(&s->ldf, mag_coef);
        for (int c = 0; c < 2; ++c) {
          mm(nqx, nqx, nqy, s->Pmn_x, mag_coef + c * nq, t1);
          mm(nqx, nqy, nqy, t1, PmnyT, mag_val + c * nq);
        }
        for (int l = 0; l < nqy; ++l)
          for (int k = 0; k < nqx; ++k) {
            uc[NODE(s, 4, k, l)] = (2.0 / hy) * mag_val[k + nqx * l] + ua[4];
            uc[NODE(s, 5, k, l)] = (2.0 / hx) * mag_val[nq + k + nqx * l] + ua[5];
          }
      }
      long ce = i + (long)(nx + 2) * j;
      s->cell_ent_FV[ce] = ent_avg;
      s->cell_ent_DG[ce] = cell_ent;
      s->cell_ent_nan[ce] = (unsigned char)cell_nan;
      memcpy(EB(s, u, i, j), uc, sizeof(double) * 8 * nq);
      for (int v = 0; v < 8; ++v) u_avg[v + 8 * (i + (long)(nx + 2) * j)] = ua[v];
    }
    for (int v = 0; v < 8; ++v) rowsum[16 * j + v] = racc[v];
  }
  for (int j = 0; j <= ny + 1; ++j)
    for (int v = 0; v < 8; ++v) u_avg_global[v] = u_avg_global[v] + rowsum[16 * j + v];

  if (apply_oedg) {
    /* global variation (DG_solver.f90:282-294) */
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= ny; ++j) {
      double rmax[8] = {0};
      for (int i = 1; i <= nx; ++i) {
        const double *uc = EBc(s, u, i, j);
        for (int q = 0; q < nq; ++q)
          for (int v = 0; v < 8; ++v) rmax[v] = dmax(rmax[v], fabs(uc[v + 8 * q] - u_avg_global[v]));
      }
      for (int v = 0; v < 8; ++v) rowsum[16 * j + 8 + v] = rmax[v];
    }
    for (int j = 1; j <= ny; ++j)
      for (int v = 0; v < 8; ++v) u_vari_global[v] = dmax(u_vari_global[v], rowsum[16 * j + 8 + v]);
    /* face jump indicators (DG_solver.f90:295-358, 359-422) */
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx + 1; ++i)
        for (int v = 0; v < 8; ++v)
          oedg_sigsum_xface(s, EBc(s, u, i, j), EBc(s, u, i - 1, j), v, &s->sigsum_x[v + 8 * ((i - 1) + (long)(nx + 1) * (j - 1))]);
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i)
      for (int j = 1; j <= ny + 1; ++j)
        for (int v = 0; v < 8; ++v)
          oedg_sigsum_yface(s, EBc(s, u, i, j), EBc(s, u, i, j - 1), v, &s->sigsum_y[v + 8 * ((i - 1) + (long)nx * (j - 1))]);
  }

  /* loop 3: OEDG damping, PP limiter, entropy (DG_solver.f90:428-656) */
  if (!neg_avg) {
#pragma omp parallel for schedule(static) reduction(+ : num_negcell) reduction(| : relimit_fail)
    for (int j = 1; j <= ny; ++j) {
      double rent = 0.0;
      for (int i = 1; i <= nx; ++i) {
        double uc[8 * NNMAX], ua[8];
        memcpy(uc, EB(s, u, i, j), sizeof(double) * 8 * nq);
        memcpy(ua, &u_avg[8 * (i + (long)(nx + 2) * j)], sizeof(double) * 8);
        if (apply_oedg) { /* DG_solver.f90:448-524 */
          double maxeig_x = 0.0, maxeig_y = 0.0, vec_delta[8];
          for (int l = 0; l < nqy; ++l)
            for (int k = 0; k < nqx; ++k) {
              const double *w = uc + 8 * (k + nqx * l);
              double rho = dmax(w[0], PP_eps);
              double mx = w[1], my = w[2], mz = w[3], bx = w[4], by = w[5], bz = w[6], e_tot = w[7];
              double inv_rho = 1.0 / rho;
              double vx = inv_rho * mx, vy = inv_rho * my;
              double e_knt = 0.5 * inv_rho * (mx * mx + my * my + mz * mz);
              double b_sq = bx * bx + by * by + bz * bz;
              double p_mag = 0.5 * b_sq;
              double p_fld = dmax((gamma - 1.0) * (e_tot - (e_knt + p_mag)), PP_eps);
              double snc_sq = gamma * p_fld * inv_rho;
              double alfven_sq = b_sq * inv_rho;
              double sum_sq = snc_sq + alfven_sq;
              double sum_sqsq = sum_sq * sum_sq;
              double coef = 4 * snc_sq * inv_rho;
              maxeig_x = dmax(maxeig_x, fabs(vx) + sqrt(0.5 * dmax(sum_sq + sqrt(dmax(sum_sqsq - coef * (bx * bx), 0.0)), 0.0)));
              maxeig_y = dmax(maxeig_y, fabs(vy) + sqrt(0.5 * dmax(sum_sq + sqrt(dmax(sum_sqsq - coef * (by * by), 0.0)), 0.0)));
            }
          double dmaxv = -DBL_MAX;
          for (int v = 0; v < 8; ++v) {
            if (u_vari_global[v] > OEDG_eps)
              vec_delta[v] = ((maxeig_x / hx) * (s->sigsum_x[v + 8 * ((i - 1) + (long)(nx + 1) * (j - 1))] + s->sigsum_x[v + 8 * (i + (long)(nx + 1) * (j - 1))]) +
                              (maxeig_y / hy) * (s->sigsum_y[v + 8 * ((i - 1) + (long)nx * (j - 1))] + s->sigsum_y[v + 8 * ((i - 1) + (long)nx * j)])) /
                             u_vari_global[v];
            else
              vec_delta[v] = 0.0;
            dmaxv = dmax(dmaxv, vec_delta[v]);
          }
          double theta = exp(-oedg_dt * dmaxv);
          for (int v = 0; v < 8; ++v)
            for (int q = 0; q < nq; ++q) uc[v + 8 * q] = ua[v] + theta * (uc[v + 8 * q] - ua[v]);
        }
        { /* PP limiter (DG_solver.f90:528-603) */
          int neg_node = 0;
          double theta = 0.0;
          double den_avg = ua[0];
          double prs_avg = prs_macro(ua[0], ua[1], ua[2], ua[3], ua[4], ua[5], ua[6], ua[7], gamma);
          double den_min = DBL_MAX;
          for (int q = 0; q < nq; ++q) den_min = dmin(den_min, uc[8 * q]);
          if (den_min < PP_eps) {
            neg_node = 1;
            theta = dmax(dmin((den_avg - PP_eps) / (den_avg - den_min), 1.0), 0.0);
            for (int q = 0; q < nq; ++q) uc[8 * q] = ua[0] + theta * (uc[8 * q] - ua[0]);
            for (int q = 0; q < nq; ++q) uc[8 * q] = dmax(uc[8 * q], PP_eps);
          }
          double prs_min = DBL_MAX;
          for (int q = 0; q < nq; ++q) {
            const double *w = uc + 8 * q;
            prs_min = dmin(prs_min, prs_macro(w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], gamma));
          }
          if (prs_min < PP_eps) {
            neg_node = 1;
            theta = dmax(dmin((prs_avg - PP_eps) / (prs_avg - prs_min), 1.0), 0.0);
            for (int q = 0; q < nq; ++q)
              for (int v = 0; v < 8; ++v) uc[v + 8 * q] = ua[v] + theta * (uc[v + 8 * q] - ua[v]);
            int it_count = 0;
            for (;;) {
              prs_min = DBL_MAX;
              for (int q = 0; q < nq; ++q) {
                const double *w = uc + 8 * q;
                prs_min = dmin(prs_min, prs_macro(w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], gamma));
              }
              if (prs_min < 0.99 * PP_eps) {
                if (it_count > 1) {
                  relimit_fail = 1; /* the reference stops the program here */
                  break;
                }
                theta = 0.6 * theta;
                for (int q = 0; q < nq; ++q)
                  for (int v = 0; v < 8; ++v) uc[v + 8 * q] = ua[v] + theta * (uc[v + 8 * q] - ua[v]);
              } else {
                break;
              }
              it_count = it_count + 1;
            }
          }
          if (neg_node) num_negcell = num_negcell + 1;
        }
        long ce = i + (long)(nx + 2) * j;
        if (ent_offset && !s->cell_ent_nan[ce]) { /* DG_solver.f90:606-633 */
          double cell_ent_old = s->cell_ent_DG[ce], ent_avg = s->cell_ent_FV[ce];
          double cell_ent_new = 0.0;
          for (int l = 0; l < nqy; ++l)
            for (int k = 0; k < nqx; ++k) {
              const double *w = uc + 8 * (k + nqx * l);
              cell_ent_new = cell_ent_new + (0.25 * hx * hy * s->qw_x[k] * s->qw_y[l]) *
                                                ent_macro(w[0], dmax(prs_macro(w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], gamma), PP_eps), gamma);
            }
          if (cell_ent_new > cell_ent_old) {
            double theta = dmax(dmin((cell_ent_old - ent_avg) / (cell_ent_new - ent_avg), 1.0), 0.0);
            for (int q = 0; q < nq; ++q)
              for (int v = 0; v < 8; ++v) uc[v + 8 * q] = ua[v] + theta * (uc[v + 8 * q] - ua[v]);
          }
        }
        if (comput_ent) { /* DG_solver.f90:635-649 */
          double cell_ent_final = 0.0;
          for (int l = 0; l < nqy; ++l)
            for (int k = 0; k < nqx; ++k) {
              const double *w = uc + 8 * (k + nqx * l);
              cell_ent_final = cell_ent_final + (0.25 * hx * hy * s->qw_x[k] * s->qw_y[l]) *
                                                    ent_macro(w[0], dmax(prs_macro(w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], gamma), PP_eps), gamma);
            }
          rent = rent + cell_ent_final;
        }
        memcpy(EB(s, u, i, j), uc, sizeof(double) * 8 * nq);
      }
      rowsum[16 * j] = rent;
    }
    for (int j = 1; j <= ny; ++j) tot_ent = tot_ent + rowsum[16 * j];
  }
  if (neg_avg || !comput_ent) tot_ent = NAN;
  *neg_avg_out = neg_avg;
  *num_negcell_out = neg_avg ? 0 : num_negcell;
  *tot_ent_out = tot_ent;
  if (pp_relimit_fail_out) *pp_relimit_fail_out = relimit_fail;
}

/* ------------------------------------------------------------------------------------------ */
/* DG_semidiscretize (DG_solver.f90:663-892)                                                   */
/* ------------------------------------------------------------------------------------------ */
void ora_semidiscretize(ora_solver *s, double *ut, double *dt_lim_out, const double *u) {
  const int nx = s->nx, ny = s->ny, px = s->px, py = s->py, nqx = s->nqx, nqy = s->nqy, nq = s->nn;
  const double gamma = s->gamma, hx = s->hx, hy = s->hy;
  double dt_lim = DBL_MAX;
  /* x faces (DG_solver.f90:680-692) */
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx + 1; ++i)
      for (int l = 0; l < nqy; ++l) {
        double wl[8], wr[8];
        for (int v = 0; v < 8; ++v) {
          wl[v] = EBc(s, u, i - 1, j)[NODE(s, v, px, l)];
          wr[v] = EBc(s, u, i, j)[NODE(s, v, 0, l)];
        }
        long f = l + (long)nqy * ((i - 1) + (long)(nx + 1) * (j - 1));
        ora_hll_flux_x(wl, wr, gamma, &s->nflux_x[8 * f], &s->nB_x[f], &s->sxl[f], &s->sxr[f]);
      }
  /* y faces (DG_solver.f90:693-713) */
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= ny + 1; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nqx; ++k) {
        double a[8], b[8], t1[8], t2[8], tf[8];
        for (int v = 0; v < 8; ++v) {
          a[v] = EBc(s, u, i, j - 1)[NODE(s, v, k, py)];
          b[v] = EBc(s, u, i, j)[NODE(s, v, k, 0)];
        }
        swap_xy(a, t1);
        swap_xy(b, t2);
        long f = k + (long)nqx * ((i - 1) + (long)nx * (j - 1));
        ora_hll_flux_x(t1, t2, gamma, tf, &s->nB_y[f], &s->syd[f], &s->syu[f]);
        swap_xy(tf, &s->nflux_y[8 * f]);
      }
  /* element loop (DG_solver.f90:717-889) */
#pragma omp parallel for schedule(static) reduction(min : dt_lim)
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      const double *uc = EBc(s, u, i, j);
      double rho[NNMAX], bx[NNMAX], by[NNMAX], bz[NNMAX], vx[NNMAX], vy[NNMAX], vz[NNMAX], beta[NNMAX], divB[NNMAX];
      double utc[8 * NNMAX], GP[8 * NNMAX], flux[2][8 * NNMAX];
      double max_sigma_x = 0.0, max_sigma_y = 0.0;
      for (int l = 0; l < nqy; ++l)
        for (int k = 0; k < nqx; ++k) {
          int q = k + nqx * l;
          const double *w = uc + 8 * q;
          rho[q] = w[0];
          double mx = w[1], my = w[2], mz = w[3];
          bx[q] = w[4];
          by[q] = w[5];
          bz[q] = w[6];
          double e_tot = w[7];
          double inv_rho = 1.0 / rho[q];
          vx[q] = inv_rho * mx;
          vy[q] = inv_rho * my;
          vz[q] = inv_rho * mz;
          double e_knt = 0.5 * inv_rho * (mx * mx + my * my + mz * mz);
          double ex = by[q] * vz[q] - bz[q] * vy[q];
          double ey = bz[q] * vx[q] - bx[q] * vz[q];
          double ez = bx[q] * vy[q] - by[q] * vx[q];
          double b_sq = bx[q] * bx[q] + by[q] * by[q] + bz[q] * bz[q];
          double p_mag = 0.5 * b_sq;
          double p_fld = dmax((gamma - 1.0) * (e_tot - (e_knt + p_mag)), PP_eps);
          beta[q] = 0.5 * rho[q] / p_fld;
          double p_tot = p_fld + p_mag;
          double b_dot_u = bx[q] * vx[q] + by[q] * vy[q] + bz[q] * vz[q];
          double snc_sq = gamma * p_fld * inv_rho;
          double alfven_sq = b_sq * inv_rho;
          double sum_sq = snc_sq + alfven_sq;
          double coef = 4 * snc_sq * inv_rho;
          max_sigma_x = dmax(max_sigma_x, fabs(vx[q]) + sqrt(0.5 * dmax(sum_sq + sqrt(dmax(sum_sq * sum_sq - coef * (bx[q] * bx[q]), 0.0)), 0.0)));
          max_sigma_y = dmax(max_sigma_y, fabs(vy[q]) + sqrt(0.5 * dmax(sum_sq + sqrt(dmax(sum_sq * sum_sq - coef * (by[q] * by[q]), 0.0)), 0.0)));
          double *F = flux[0] + 8 * q, *G = flux[1] + 8 * q, *gp = GP + 8 * q;
          F[0] = mx;
          F[1] = vx[q] * mx - bx[q] * bx[q] + p_tot;
          F[2] = vx[q] * my - by[q] * bx[q] + 0.0;
          F[3] = vx[q] * mz - bz[q] * bx[q] + 0.0;
          F[4] = 0.0;
          F[5] = -ez;
          F[6] = ey;
          F[7] = vx[q] * (e_tot + p_tot) - bx[q] * b_dot_u;
          G[0] = my;
          G[1] = vy[q] * mx - bx[q] * by[q] + 0.0;
          G[2] = vy[q] * my - by[q] * by[q] + p_tot;
          G[3] = vy[q] * mz - bz[q] * by[q] + 0.0;
          G[4] = ez;
          G[5] = 0.0;
          G[6] = -ex;
          G[7] = vy[q] * (e_tot + p_tot) - by[q] * b_dot_u;
          gp[0] = 0.0;
          gp[1] = bx[q];
          gp[2] = by[q];
          gp[3] = bz[q];
          gp[4] = vx[q];
          gp[5] = vy[q];
          gp[6] = vz[q];
          gp[7] = b_dot_u;
        }
      /* dt for linear stability (DG_solver.f90:806) */
      double smax_x = max_sigma_x, smax_y = max_sigma_y;
      {
        double mxr = -DBL_MAX, mnl = DBL_MAX, myu = -DBL_MAX, mnd = DBL_MAX;
        for (int l = 0; l < nqy; ++l) {
          mxr = dmax(mxr, s->sxr[l + (long)nqy * ((i - 1) + (long)(nx + 1) * (j - 1))]);
          mnl = dmin(mnl, s->sxl[l + (long)nqy * (i + (long)(nx + 1) * (j - 1))]);
        }
        for (int k = 0; k < nqx; ++k) {
          myu = dmax(myu, s->syu[k + (long)nqx * ((i - 1) + (long)nx * (j - 1))]);
          mnd = dmin(mnd, s->syd[k + (long)nqx * ((i - 1) + (long)nx * j)]);
        }
        smax_x = dmax(dmax(max_sigma_x, mxr), -mnl);
        smax_y = dmax(dmax(max_sigma_y, myu), -mnd);
      }
      double dtl = 1.0 / ((2 * px + 1) * smax_x / hx + (2 * py + 1) * smax_y / hy);
      dt_lim = dmin(dt_lim, dtl);
      for (int q = 0; q < 8 * nq; ++q) utc[q] = 0.0;
      /* divB = (2/hx) Dx bx + (2/hy) by Dy^T (DG_solver.f90:813) */
      for (int l = 0; l < nqy; ++l)
        for (int k = 0; k < nqx; ++k) {
          double a = 0.0, b = 0.0;
          for (int r = 0; r < nqx; ++r) a += s->diff_x[k + nqx * r] * bx[r + nqx * l];
          for (int m = 0; m < nqy; ++m) b += by[k + nqx * m] * s->diff_y[l + nqy * m];
          divB[k + nqx * l] = (2.0 / hx) * a + (2.0 / hy) * b;
        }
      /* flux differencing (DG_solver.f90:828-851) */
      for (int l = 0; l < nqy; ++l)
        for (int k = 0; k < nqx; ++k) {
          int q = k + nqx * l;
          double dkk = 2.0 * (2.0 / hx) * s->diff_x[k + nqx * k];
          double dll = 2.0 * (2.0 / hy) * s->diff_y[l + nqy * l];
          for (int v = 0; v < 8; ++v)
            utc[v + 8 * q] = utc[v + 8 * q] - dkk * flux[0][v + 8 * q] - dll * flux[1][v + 8 * q] - divB[q] * GP[v + 8 * q];
          double pk[8] = {rho[q], vx[q], vy[q], vz[q], bx[q], by[q], bz[q], beta[q]};
          for (int r = 0; r < k; ++r) {
            int qr = r + nqx * l;
            double pr[8] = {rho[qr], vx[qr], vy[qr], vz[qr], bx[qr], by[qr], bz[qr], beta[qr]};
            double ec[8];
            ora_ec_flux_x(pk, pr, gamma, ec);
            double ckr = 2.0 * (2.0 / hx) * s->diff_x[k + nqx * r];
            double crk = 2.0 * (2.0 / hx) * s->diff_x[r + nqx * k];
            for (int v = 0; v < 8; ++v) utc[v + 8 * q] = utc[v + 8 * q] - ckr * ec[v];
            for (int v = 0; v < 8; ++v) utc[v + 8 * qr] = utc[v + 8 * qr] - crk * ec[v];
          }
          for (int m = 0; m < l; ++m) {
            int qs = k + nqx * m;
            double ps[8] = {rho[qs], vx[qs], vy[qs], vz[qs], bx[qs], by[qs], bz[qs], beta[qs]};
            double ec[8];
            ora_ec_flux_y(pk, ps, gamma, ec);
            double cls = 2.0 * (2.0 / hy) * s->diff_y[l + nqy * m];
            double csl = 2.0 * (2.0 / hy) * s->diff_y[m + nqy * l];
            for (int v = 0; v < 8; ++v) utc[v + 8 * q] = utc[v + 8 * q] - cls * ec[v];
            for (int v = 0; v < 8; ++v) utc[v + 8 * qs] = utc[v + 8 * qs] - csl * ec[v];
          }
        }
      /* x-face terms (DG_solver.f90:872-875) */
      for (int l = 0; l < nqy; ++l) {
        long f0 = l + (long)nqy * ((i - 1) + (long)(nx + 1) * (j - 1));
        long f1 = l + (long)nqy * (i + (long)(nx + 1) * (j - 1));
        int q0 = 0 + nqx * l, q1 = px + nqx * l;
        double c0 = (2.0 / hx) / s->qw_x[0], c1 = (2.0 / hx) / s->qw_x[px];
        for (int v = 0; v < 8; ++v)
          utc[v + 8 * q0] = utc[v + 8 * q0] - c0 * (flux[0][v + 8 * q0] - s->nflux_x[v + 8 * f0] + GP[v + 8 * q0] * (bx[q0] - s->nB_x[f0]));
        for (int v = 0; v < 8; ++v)
          utc[v + 8 * q1] = utc[v + 8 * q1] + c1 * (flux[0][v + 8 * q1] - s->nflux_x[v + 8 * f1] + GP[v + 8 * q1] * (bx[q1] - s->nB_x[f1]));
      }
      /* y-face terms (DG_solver.f90:879-882) */
      for (int k = 0; k < nqx; ++k) {
        long f0 = k + (long)nqx * ((i - 1) + (long)nx * (j - 1));
        long f1 = k + (long)nqx * ((i - 1) + (long)nx * j);
        int q0 = k + nqx * 0, q1 = k + nqx * py;
        double c0 = (2.0 / hy) / s->qw_y[0], c1 = (2.0 / hy) / s->qw_y[py];
        for (int v = 0; v < 8; ++v)
          utc[v + 8 * q0] = utc[v + 8 * q0] - c0 * (flux[1][v + 8 * q0] - s->nflux_y[v + 8 * f0] + GP[v + 8 * q0] * (by[q0] - s->nB_y[f0]));
        for (int v = 0; v < 8; ++v)
          utc[v + 8 * q1] = utc[v + 8 * q1] + c1 * (flux[1][v + 8 * q1] - s->nflux_y[v + 8 * f1] + GP[v + 8 * q1] * (by[q1] - s->nB_y[f1]));
      }
      memcpy(UTB(s, ut, i, j), utc, sizeof(double) * 8 * nq);
    }
  *dt_lim_out = dt_lim;
}

/* ------------------------------------------------------------------------------------------ */
/* SSP-RK stage combination (drive.f90:130-275)                                                */
/* ------------------------------------------------------------------------------------------ */
double ora_rk_combine(ora_solver *s, int st, double dt, double t, double *t_rk) {
  const int nx = s->nx, ny = s->ny;
  const long nb = 8L * s->nn;
  double *u = s->u_con;
  double *r[6] = {0};
  double *k[6] = {0};
  for (int q = 1; q <= s->rknstg; ++q) {
    r[q] = ora_urk_con(s, q);
    k[q] = ora_ut_con(s, q);
  }
  const int R = s->rknstg;
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      const double *uc = EB(s, u, i, j);
      double *o = EB(s, r[st], i, j);
      const double *k1 = k[1] ? UTB(s, k[1], i, j) : NULL;
      const double *k2 = (R >= 2) ? UTB(s, k[2], i, j) : NULL;
      const double *k3 = (R >= 3) ? UTB(s, k[3], i, j) : NULL;
      const double *k4 = (R >= 4) ? UTB(s, k[4], i, j) : NULL;
      const double *k5 = (R >= 5) ? UTB(s, k[5], i, j) : NULL;
      const double *r1 = EB(s, r[1], i, j);
      const double *r2 = (R >= 2) ? EB(s, r[2], i, j) : NULL;
      const double *r3 = (R >= 3) ? EB(s, r[3], i, j) : NULL;
      const double *r4 = (R >= 4) ? EB(s, r[4], i, j) : NULL;
      for (long q = 0; q < nb; ++q) {
        double val;
        if (R == 1 || (st == 1 && R <= 3)) {
          val = uc[q] + dt * k1[q];
        } else if (R == 2) {
          val = 0.5 * uc[q] + 0.5 * (r1[q] + dt * k2[q]);
        } else if (R == 3) {
          if (st == 2)
            val = 0.75 * uc[q] + 0.25 * (r1[q] + dt * k2[q]);
          else
            val = (1.0 / 3.0) * uc[q] + (2.0 / 3.0) * (r2[q] + dt * k3[q]);
        } else { /* SSP-RK(5,4) */
          switch (st) {
            case 1: val = uc[q] + (0.391752226571890 * dt) * k1[q]; break;
            case 2: val = 0.444370493651235 * uc[q] + 0.555629506348765 * r1[q] + (0.368410593050371 * dt) * k2[q]; break;
            case 3: val = 0.620101851488403 * uc[q] + 0.379898148511597 * r2[q] + (0.251891774271694 * dt) * k3[q]; break;
            case 4: val = 0.178079954393132 * uc[q] + 0.821920045606868 * r3[q] + (0.544974750228521 * dt) * k4[q]; break;
            default:
              val = 0.517231671970585 * r2[q] + 0.096059710526147 * r3[q] + (0.063692468666290 * dt) * k4[q] + 0.386708617503269 * r4[q] + (0.226007483236906 * dt) * k5[q];
              break;
          }
        }
        o[q] = val;
      }
    }
  /* pseudo-time of the stage */
  double tr;
  if (R == 1 || (st == 1 && R <= 3)) tr = t + dt * 1.0;
  else if (R == 2) tr = 0.5 * t + 0.5 * (t_rk[1] + dt * 1.0);
  else if (R == 3) tr = (st == 2) ? 0.75 * t + 0.25 * (t_rk[1] + dt * 1.0) : (1.0 / 3.0) * t + (2.0 / 3.0) * (t_rk[2] + dt * 1.0);
  else {
    switch (st) {
      case 1: tr = t + (0.391752226571890 * dt) * 1.0; break;
      case 2: tr = 0.444370493651235 * t + 0.555629506348765 * t_rk[1] + (0.368410593050371 * dt) * 1.0; break;
      case 3: tr = 0.620101851488403 * t + 0.379898148511597 * t_rk[2] + (0.251891774271694 * dt) * 1.0; break;
      case 4: tr = 0.178079954393132 * t + 0.821920045606868 * t_rk[3] + (0.544974750228521 * dt) * 1.0; break;
      default:
        tr = 0.517231671970585 * t_rk[2] + 0.096059710526147 * t_rk[3] + (0.063692468666290 * dt) * 1.0 + 0.386708617503269 * t_rk[4] + (0.226007483236906 * dt) * 1.0;
        break;
    }
  }
  t_rk[st] = tr;
  return tr;
}

/* integer power as Fortran's x**n with integer n (binary exponentiation) */
static double powi(double x, int n) {
  double r = 1.0;
  int first = 1;
  double b = x;
  while (n > 0) {
    if (n & 1) {
      r = first ? b : r * b;
      first = 0;
    }
    n >>= 1;
    if (n) b = b * b;
  }
  return r;
}

/* solve_execute (drive.f90:32-343) */
int ora_solve(ora_solver *s, double final_T, double cfl, int use_oedg, int use_ldf, int ent_offset,
              int max_steps, double *out) {
  return ora_solve_resume(s, final_T, cfl, use_oedg, use_ldf, ent_offset, max_steps, 0, out);
}

int ora_solve_resume(ora_solver *s, double final_T, double cfl, int use_oedg, int use_ldf, int ent_offset,
                     int max_steps, int resume, double *out) {
  const int R = s->rknstg;
  double cfl_rk = (R <= 3) ? 1.0 : 1.508;
  double t = 0.0, dt = 0.0, dt_lim = 0.0, tot_ent = 0.0, t_rk[6] = {0};
  int neg_avg = 0, num_negcell = 0, relimit = 0;
  long total_negcell = 0;
  int steps = 0, retries = 0, status = ORA_OK;
  int flag = 1;
  if (resume) {
    t = s->run_t;
    dt = s->run_dt;
    dt_lim = s->run_dt_lim;
    tot_ent = s->run_tot_ent;
    goto loop;
  }
  /* drive.f90:68-73 */
  ora_apply_bc(s, s->u_con);
  ora_post_process(s, s->u_con, s->u_avg, &neg_avg, &num_negcell, 0, use_ldf, 0.0, 0, 1, &tot_ent, &relimit);
  if (neg_avg) {
    status = ORA_ERR_INIT_NEG_AVG;
    goto done;
  }
  ora_apply_bc(s, s->u_con);
  ora_semidiscretize(s, ora_ut_con(s, 1), &dt_lim, s->u_con);
loop:;
  flag = 1;
  while (flag) {
    if (max_steps > 0 && steps >= max_steps) break;
    steps++;
    int try_num = 0, try_again = 1;
    while (try_again) {
      try_again = 0;
      try_num++;
      if (try_num > 10 || dt_lim < 1e-14) {
        status = ORA_ERR_DT_COLLAPSE;
        goto done;
      } else if (try_num > 1) {
        retries++;
        ora_semidiscretize(s, ora_ut_con(s, 1), &dt_lim, s->u_con);
      }
      if (try_num <= 1)
        dt = cfl_rk * cfl * dt_lim;
      else
        dt = powi(sqrt(1.25) - 0.5, try_num - 1) * dt;
      if (t + dt >= final_T) {
        dt = final_T - t;
        flag = 0;
      } else {
        flag = 1;
      }
      for (int st = 1; st <= R; ++st) {
        int rk_final = (st == R);
        ora_rk_combine(s, st, dt, t, t_rk);
        double *urk = ora_urk_con(s, st);
        ora_apply_bc(s, urk);
        ora_post_process(s, urk, s->u_avg, &neg_avg, &num_negcell, use_oedg && rk_final, use_ldf, dt, ent_offset, rk_final, &tot_ent, &relimit);
        if (relimit) {
          status = ORA_ERR_PP_RELIMIT;
          goto done;
        }
        if (neg_avg) {
          try_again = 1;
          break;
        }
        ora_apply_bc(s, urk);
        total_negcell += num_negcell;
        ora_semidiscretize(s, ora_ut_con(s, (st % R) + 1), &dt_lim, urk);
      }
    }
    /* accept (drive.f90:304-312): interior only, ghosts of u_con keep their old values */
    {
      const int nx = s->nx, ny = s->ny;
      double *last = ora_urk_con(s, R);
#pragma omp parallel for schedule(static)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) memcpy(EB(s, s->u_con, i, j), EB(s, last, i, j), sizeof(double) * 8 * s->nn);
    }
    t = t_rk[R];
  }
done:
  s->run_t = t;
  s->run_dt = dt;
  s->run_dt_lim = dt_lim;
  s->run_tot_ent = tot_ent;
  if (out) {
    out[0] = t;
    out[1] = dt_lim;
    out[2] = tot_ent;
    out[3] = steps;
    out[4] = retries;
    out[5] = dt;
    out[6] = (double)total_negcell;
  }
  return status;
}
