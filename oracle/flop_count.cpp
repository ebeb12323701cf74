// flop_count.cpp -- algorithmic FP64 operation counts of the hot path (TEST/MEASUREMENT
// INFRASTRUCTURE ONLY).
//
// Compiles the oracle (mhd_oracle.c) as C++ with `double` replaced by `Counted`, a double that
// counts every arithmetic operation performed on it, and runs one residual, the post-process
// variants of an SSP-RK3 step and one stage combination on a small periodic Orszag-Tang mesh.
// Counting convention (as the reference's source is written): + - * min max abs = 1 each,
// / sqrt log exp = 1 each; comparisons, negation and loads/stores are free.  Built sequentially
// (no OpenMP), so the counts are exact and deterministic.  Output: JSON on stdout.
//
//   g++ -std=c++17 -O1 -I oracle oracle/flop_count.cpp -o oracle/_build/flop_count
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

struct Counters {
  long long add = 0, mul = 0, div = 0, sqrt_ = 0, log_ = 0, exp_ = 0, minmax = 0, abs_ = 0;
  long long total() const { return add + mul + div + sqrt_ + log_ + exp_ + minmax + abs_; }
};
static Counters g_cnt;

struct Counted {
  double v;
  Counted() = default;
  Counted(double x) : v(x) {}
  Counted(long double x) : v((double)x) {}
  Counted(float x) : v(x) {}
  Counted(int x) : v(x) {}
  Counted(long x) : v((double)x) {}
  operator double() const { return v; }
  Counted& operator+=(Counted o) { ++g_cnt.add; v += o.v; return *this; }
  Counted& operator-=(Counted o) { ++g_cnt.add; v -= o.v; return *this; }
  Counted& operator*=(Counted o) { ++g_cnt.mul; v *= o.v; return *this; }
  Counted& operator/=(Counted o) { ++g_cnt.div; v /= o.v; return *this; }
  Counted operator-() const { return Counted(-v); }
  Counted operator+() const { return *this; }
};
#define CNT_BIN(op, field)                                                              \
  inline Counted operator op(Counted a, Counted b) { ++g_cnt.field; return Counted(a.v op b.v); } \
  inline Counted operator op(Counted a, double b) { ++g_cnt.field; return Counted(a.v op b); }    \
  inline Counted operator op(double a, Counted b) { ++g_cnt.field; return Counted(a op b.v); }    \
  inline Counted operator op(Counted a, int b) { ++g_cnt.field; return Counted(a.v op b); }       \
  inline Counted operator op(int a, Counted b) { ++g_cnt.field; return Counted(a op b.v); }
CNT_BIN(+, add)
CNT_BIN(-, add)
CNT_BIN(*, mul)
CNT_BIN(/, div)
#define CNT_CMP(op)                                                      \
  inline bool operator op(Counted a, Counted b) { return a.v op b.v; }   \
  inline bool operator op(Counted a, double b) { return a.v op b; }      \
  inline bool operator op(double a, Counted b) { return a op b.v; }      \
  inline bool operator op(Counted a, int b) { return a.v op b; }         \
  inline bool operator op(int a, Counted b) { return a op b.v; }
CNT_CMP(<)
CNT_CMP(>)
CNT_CMP(<=)
CNT_CMP(>=)
CNT_CMP(==)
CNT_CMP(!=)
inline Counted sqrt(Counted a) { ++g_cnt.sqrt_; return Counted(std::sqrt(a.v)); }
inline Counted log(Counted a) { ++g_cnt.log_; return Counted(std::log(a.v)); }
inline Counted exp(Counted a) { ++g_cnt.exp_; return Counted(std::exp(a.v)); }
inline Counted fabs(Counted a) { ++g_cnt.abs_; return Counted(std::fabs(a.v)); }

typedef long double ldbl;
#define ORA_LDBL_DEFINED 1
#define ORA_COUNT_MINMAX() (++g_cnt.minmax)
#define double Counted
#include "mhd_oracle.c"
#undef double

static void ot_state(ora_solver* s, double gamma) {
  // Orszag-Tang on [0,2pi]^2 at the GLL nodes, conserved variables, interior only
  const int nx = s->nx, ny = s->ny, nq = s->nqx;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int l = 0; l < nq; ++l)
        for (int k = 0; k < nq; ++k) {
          double x = (0.5 * s->hx.v) * s->qx_x[k].v + (s->left.v + (i - 0.5) * s->hx.v);
          double y = (0.5 * s->hy.v) * s->qx_y[l].v + (s->bottom.v + (j - 0.5) * s->hy.v);
          double rho = gamma * gamma, vx = -std::sin(y), vy = std::sin(x), bx = -std::sin(y), by = std::sin(2 * x);
          double e = gamma / (gamma - 1.0) + 0.5 * (rho * (vx * vx + vy * vy) + bx * bx + by * by);
          Counted* w = EB(s, s->u_con, i, j) + 8 * (k + nq * l);
          w[0] = rho; w[1] = rho * vx; w[2] = rho * vy; w[3] = 0.0; w[4] = bx; w[5] = by; w[6] = 0.0; w[7] = e;
        }
}

static void emit(const char* key, const Counters& c, double per, bool last) {
  printf("      \"%s\": {\"total\": %.3f, \"add\": %.3f, \"mul\": %.3f, \"div\": %.3f, \"sqrt\": %.3f, "
         "\"log\": %.3f, \"exp\": %.3f, \"minmax\": %.3f, \"abs\": %.3f}%s\n",
         key, c.total() / per, c.add / per, c.mul / per, c.div / per, c.sqrt_ / per, c.log_ / per,
         c.exp_ / per, c.minmax / per, c.abs_ / per, last ? "" : ",");
}

int main() {
  const int nx = 8, ny = 8;
  const double gamma = 5.0 / 3.0, PI = 3.14159265358979323846;
  printf("{\n  \"convention\": \"operations as written in the reference source: + - * min max abs / sqrt log exp "
         "count 1 each; comparisons and negation free\",\n  \"mesh\": \"Orszag-Tang [0,2pi]^2 8x8 periodic\",\n"
         "  \"per_degree\": {\n");
  for (int p = 1; p <= 3; ++p) {
    ora_solver* s = ora_create(nx, ny, p, p, 3, 0.0, 2 * PI, 0.0, 2 * PI, gamma, ORA_BC_PERIODIC, NULL);
    ot_state(s, gamma);
    ora_apply_bc(s, s->u_con);
    const double E = nx * ny, NN = (p + 1) * (p + 1);
    Counters c_res, c_pp, c_ppf, c_cmb;
    Counted dt_lim;
    g_cnt = Counters();
    ora_semidiscretize(s, ora_ut_con(s, 1), &dt_lim, s->u_con);
    c_res = g_cnt;
    // post_process as in a non-final stage: LDF + PP, no OEDG, no entropy
    Counted* u1 = ora_urk_con(s, 1);
    memcpy(u1, s->u_con, sizeof(Counted) * ora_size_u(s));
    int neg, nneg, rel;
    Counted te;
    g_cnt = Counters();
    ora_post_process(s, u1, s->u_avg, &neg, &nneg, 0, 1, 0.0, 0, 0, &te, &rel);
    c_pp = g_cnt;
    // post_process of the final stage: OEDG + LDF + PP + entropy
    memcpy(u1, s->u_con, sizeof(Counted) * ora_size_u(s));
    g_cnt = Counters();
    ora_post_process(s, u1, s->u_avg, &neg, &nneg, 1, 1, 1e-3, 0, 1, &te, &rel);
    c_ppf = g_cnt;
    // stage combination of stage 2 (u, uRK1, ut2)
    memcpy(ora_ut_con(s, 2), ora_ut_con(s, 1), sizeof(Counted) * ora_size_ut(s));
    Counted trk[6] = {0, 0, 0, 0, 0, 0};
    g_cnt = Counters();
    ora_rk_combine(s, 2, 1e-3, 0.0, trk);
    c_cmb = g_cnt;
    printf("    \"%d\": {\n      \"nodes_per_element\": %d,\n", p, (int)NN);
    emit("residual_per_element", c_res, E, false);
    emit("post_process_stage_per_element", c_pp, E, false);
    emit("post_process_final_stage_per_element", c_ppf, E, false);
    emit("combine_per_dof", c_cmb, E * NN * 8, false);
    // SSP-RK3 step: 3 residuals, 2 non-final + 1 final post_process, 3 combines (the third has
    // the same operation count as the second)
    Counters step;
    step.add = 3 * c_res.add + 2 * c_pp.add + c_ppf.add + 3 * c_cmb.add;
    step.mul = 3 * c_res.mul + 2 * c_pp.mul + c_ppf.mul + 3 * c_cmb.mul;
    step.div = 3 * c_res.div + 2 * c_pp.div + c_ppf.div + 3 * c_cmb.div;
    step.sqrt_ = 3 * c_res.sqrt_ + 2 * c_pp.sqrt_ + c_ppf.sqrt_ + 3 * c_cmb.sqrt_;
    step.log_ = 3 * c_res.log_ + 2 * c_pp.log_ + c_ppf.log_ + 3 * c_cmb.log_;
    step.exp_ = 3 * c_res.exp_ + 2 * c_pp.exp_ + c_ppf.exp_ + 3 * c_cmb.exp_;
    step.minmax = 3 * c_res.minmax + 2 * c_pp.minmax + c_ppf.minmax + 3 * c_cmb.minmax;
    step.abs_ = 3 * c_res.abs_ + 2 * c_pp.abs_ + c_ppf.abs_ + 3 * c_cmb.abs_;
    emit("rk3_per_dof_stage", step, E * NN * 8 * 3, true);
    printf("    }%s\n", p < 3 ? "," : "");
    ora_destroy(s);
  }
  printf("  }\n}\n");
  return 0;
}
