// tables.cpp -- host tables for the DG-MHD kernels, computed in long double from their
// definitions:
//   GLL nodes: +-1 and the roots of P_N' (Newton on the Legendre equation); weights
//   2/(N(N+1) P_N(x)^2); Pmn(i,j) = P_j(x_i); Pnm = Pmn^-1; the exact Lagrange mass matrix
//   M = Pnm^T diag(2/(2m+1)) Pnm; D(i,j) = l_j'(x_i).
//   LDF projector (LDF.f90:1-60 derivation): S_1d = G G^T with G = sqrt(m) D_modal sqrt(m)^-1,
//   diagonalised here by a cyclic Jacobi eigen-solver (the reference uses LAPACK DGESDD on G;
//   the projector depends only on the eigenpairs of G G^T, not on that choice).
#include "tables.h"

#include <cmath>
#include <cstring>

namespace mhd {
namespace tables {
namespace {

constexpr int NMAX = 7;
typedef long double ld;

void legendre(int N, ld x, ld* P, ld* dP) {
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

bool invert(int n, const ld* A, ld* Ai) {
  ld W[NMAX][2 * NMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      W[i][j] = A[i + n * j];
      W[i][n + j] = (i == j) ? 1.0L : 0.0L;
    }
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (fabsl(W[r][c]) > fabsl(W[piv][c])) piv = r;
    if (W[piv][c] == 0.0L) return false;
    for (int j = 0; j < 2 * n; ++j) {
      ld t = W[c][j];
      W[c][j] = W[piv][j];
      W[piv][j] = t;
    }
    const ld d = W[c][c];
    for (int j = 0; j < 2 * n; ++j) W[c][j] /= d;
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const ld f = W[r][c];
      for (int j = 0; j < 2 * n; ++j) W[r][j] -= f * W[c][j];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) Ai[i + n * j] = W[i][n + j];
  return true;
}

struct Gll {
  int n;
  ld x[NMAX], w[NMAX], M[NMAX * NMAX], Minv[NMAX * NMAX], D[NMAX * NMAX], Pmn[NMAX * NMAX], Pnm[NMAX * NMAX];
};

bool gll_ld(int p, Gll& t) {
  if (p < 0 || p > 6) return false;
  const int n = p + 1, N = p;
  t.n = n;
  ld P[NMAX + 1], dP[NMAX + 1];
  if (p == 0) {
    t.x[0] = 0.0L;
    t.w[0] = 2.0L;
  } else {
    const ld pi = 3.141592653589793238462643383279502884L;
    t.x[0] = -1.0L;
    t.x[N] = 1.0L;
    for (int i = 1; i < N; ++i) {
      ld xi = -cosl(pi * i / N);
      for (int it = 0; it < 100; ++it) {
        legendre(N, xi, P, dP);
        const ld f = dP[N];
        const ld fp = (2.0L * xi * dP[N] - N * (N + 1) * P[N]) / (1.0L - xi * xi);
        const ld step = f / fp;
        xi -= step;
        if (fabsl(step) < 1e-30L) break;
      }
      t.x[i] = xi;
    }
    for (int i = 0; i < n / 2; ++i) {
      const ld a = 0.5L * (t.x[N - i] - t.x[i]);
      t.x[i] = -a;
      t.x[N - i] = a;
    }
    if (n % 2) t.x[N / 2] = 0.0L;
    for (int i = 0; i < n; ++i) {
      legendre(N, t.x[i], P, dP);
      t.w[i] = 2.0L / (N * (N + 1) * P[N] * P[N]);
    }
  }
  for (int i = 0; i < n; ++i) {
    legendre(N, t.x[i], P, dP);
    for (int j = 0; j < n; ++j) t.Pmn[i + n * j] = P[j];
  }
  if (!invert(n, t.Pmn, t.Pnm)) return false;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      ld a = 0.0L;
      for (int m = 0; m < n; ++m) a += t.Pnm[m + n * i] * t.Pnm[m + n * j] * (2.0L / (2 * m + 1));
      t.M[i + n * j] = a;
    }
  if (!invert(n, t.M, t.Minv)) return false;
  if (p == 0) {
    t.D[0] = 0.0L;
  } else {
    ld PN[NMAX];
    for (int i = 0; i < n; ++i) {
      legendre(N, t.x[i], P, dP);
      PN[i] = P[N];
    }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        ld d;
        if (i != j) d = PN[i] / (PN[j] * (t.x[i] - t.x[j]));
        else if (i == 0) d = -(ld)(N * (N + 1)) / 4.0L;
        else if (i == N) d = (ld)(N * (N + 1)) / 4.0L;
        else d = 0.0L;
        t.D[i + n * j] = d;
      }
  }
  return true;
}

// symmetric eigen-decomposition S = V diag(lam) V^T, eigenvalues sorted descending
void sym_eig_desc(int n, const ld* S, ld* V, ld* lam) {
  ld A[NMAX][NMAX], Q[NMAX][NMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      A[i][j] = S[i + n * j];
      Q[i][j] = (i == j) ? 1.0L : 0.0L;
    }
  for (int sweep = 0; sweep < 100; ++sweep) {
    ld off = 0.0L;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) off += A[i][j] * A[i][j];
    if (off < 1e-60L) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        if (A[p][q] == 0.0L) continue;
        const ld th = (A[q][q] - A[p][p]) / (2.0L * A[p][q]);
        const ld t = (th >= 0 ? 1.0L : -1.0L) / (fabsl(th) + sqrtl(th * th + 1.0L));
        const ld c = 1.0L / sqrtl(t * t + 1.0L), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p,q
          const ld akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p,q
          const ld apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const ld qkp = Q[k][p], qkq = Q[k][q];
          Q[k][p] = c * qkp - s * qkq;
          Q[k][q] = s * qkp + c * qkq;
        }
      }
  }
  int ord[NMAX];
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b)
      if (A[ord[b]][ord[b]] > A[ord[a]][ord[a]]) {
        const int t = ord[a];
        ord[a] = ord[b];
        ord[b] = t;
      }
  for (int c = 0; c < n; ++c) {
    lam[c] = A[ord[c]][ord[c]];
    for (int r = 0; r < n; ++r) V[r + n * c] = Q[r][ord[c]];
  }
}

// C(a x c) = A(a x b) B(b x c)
void mm(int a, int b, int c, const ld* A, const ld* B, ld* C) {
  for (int j = 0; j < c; ++j)
    for (int i = 0; i < a; ++i) {
      ld s = 0.0L;
      for (int m = 0; m < b; ++m) s += A[i + a * m] * B[m + b * j];
      C[i + a * j] = s;
    }
}
void tr(int n, const ld* A, ld* At) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) At[j + n * i] = A[i + n * j];
}

}  // namespace

int gll(int p, double* x, double* w, double* M, double* Minv, double* D, double* Pmn, double* Pnm) {
  Gll t;
  if (!gll_ld(p, t)) return -1;
  const int n = p + 1;
  for (int i = 0; i < n; ++i) {
    if (x) x[i] = (double)t.x[i];
    if (w) w[i] = (double)t.w[i];
  }
  for (int i = 0; i < n * n; ++i) {
    if (M) M[i] = (double)t.M[i];
    if (Minv) Minv[i] = (double)t.Minv[i];
    if (D) D[i] = (double)t.D[i];
    if (Pmn) Pmn[i] = (double)t.Pmn[i];
    if (Pnm) Pnm[i] = (double)t.Pnm[i];
  }
  return 0;
}

int dpow_rows(int p, double* R0, double* RN) {
  Gll t;
  if (!gll_ld(p, t)) return -1;
  const int n = p + 1;
  ld Pk[NMAX * NMAX], T[NMAX * NMAX];
  for (int i = 0; i < n * n; ++i) Pk[i] = (i % (n + 1) == 0) ? 1.0L : 0.0L;  // identity
  for (int kk = 0; kk <= p; ++kk) {
    for (int k = 0; k < n; ++k) {
      R0[kk * n + k] = (double)Pk[0 + n * k];
      RN[kk * n + k] = (double)Pk[(n - 1) + n * k];
    }
    mm(n, n, n, t.D, Pk, T);
    std::memcpy(Pk, T, sizeof(T));
  }
  return 0;
}

int ldf_nodal_operator(int p, double hx, double hy, double* A) {
  Gll t;
  if (p < 1 || !gll_ld(p, t)) return -1;
  const int n = p + 1, nn = n * n, n2 = 2 * nn;
  // modal (Legendre) tables: m_j = 1/(j+1/2), D(i,j) = 2i+1 for i<j with j-i odd (gauss.f90:436-475)
  ld m[NMAX], minv[NMAX], Dm[NMAX * NMAX], G[NMAX * NMAX], S[NMAX * NMAX], U[NMAX * NMAX], lam[NMAX];
  for (int j = 0; j < n; ++j) {
    m[j] = 1.0L / (j + 0.5L);
    minv[j] = j + 0.5L;
    for (int i = 0; i < n; ++i) Dm[i + n * j] = (i < j && ((j - i) % 2 == 1)) ? (ld)(2 * i + 1) : 0.0L;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) G[i + n * j] = sqrtl(m[i]) * Dm[i + n * j] / sqrtl(m[j]);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      ld s = 0.0L;
      for (int k = 0; k < n; ++k) s += G[i + n * k] * G[j + n * k];
      S[i + n * j] = s;
    }
  sym_eig_desc(n, S, U, lam);
  ld Ld[NMAX * NMAX], sq2[NMAX * NMAX], im2[NMAX * NMAX];  // (n x n)
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      Ld[i + n * j] = (i < n - 1 || j < n - 1) ? 1.0L / (lam[i] + lam[j]) : 0.0L;
      sq2[i + n * j] = sqrtl(m[i] * m[j]);
      im2[i + n * j] = minv[i] * minv[j];
    }
  ld UT[NMAX * NMAX], DmT[NMAX * NMAX], PnmT[NMAX * NMAX], PmnT[NMAX * NMAX];
  tr(n, U, UT);
  tr(n, Dm, DmT);
  tr(n, t.Pnm, PnmT);
  tr(n, t.Pmn, PmnT);
  for (int col = 0; col < n2; ++col) {
    ld d[2 * NMAX * NMAX] = {0};
    d[col] = 1.0L;
    ld c1[NMAX * NMAX], c2[NMAX * NMAX], a[NMAX * NMAX], b[NMAX * NMAX], e[NMAX * NMAX];
    // contravariant Piola map and nodal -> modal (DG_solver.f90:238-248)
    for (int q = 0; q < nn; ++q) {
      a[q] = (0.5L * hy) * d[q];
      b[q] = (0.5L * hx) * d[nn + q];
    }
    mm(n, n, n, t.Pnm, a, e);
    mm(n, n, n, e, PnmT, c1);
    mm(n, n, n, t.Pnm, b, e);
    mm(n, n, n, e, PnmT, c2);
    // correction of LDF.f90:247-249
    ld div[NMAX * NMAX], w1[NMAX * NMAX], w2[NMAX * NMAX];
    mm(n, n, n, Dm, c1, w1);
    mm(n, n, n, c2, DmT, w2);
    for (int q = 0; q < nn; ++q) div[q] = sq2[q] * (w1[q] + w2[q]);
    mm(n, n, n, UT, div, w1);
    mm(n, n, n, w1, U, w2);
    for (int q = 0; q < nn; ++q) w2[q] *= Ld[q];
    mm(n, n, n, U, w2, w1);
    mm(n, n, n, w1, UT, w2);
    for (int q = 0; q < nn; ++q) div[q] = sq2[q] * w2[q];
    mm(n, n, n, DmT, div, w1);
    mm(n, n, n, div, Dm, w2);
    for (int q = 0; q < nn; ++q) {
      c1[q] -= im2[q] * w1[q];
      c2[q] -= im2[q] * w2[q];
    }
    // modal -> nodal and inverse Piola map (DG_solver.f90:254-263)
    mm(n, n, n, t.Pmn, c1, e);
    mm(n, n, n, e, PmnT, a);
    mm(n, n, n, t.Pmn, c2, e);
    mm(n, n, n, e, PmnT, b);
    for (int q = 0; q < nn; ++q) {
      A[q + n2 * col] = (double)((2.0L / hy) * a[q]);
      A[nn + q + n2 * col] = (double)((2.0L / hx) * b[q]);
    }
  }
  return 0;
}

}  // namespace tables
}  // namespace mhd
