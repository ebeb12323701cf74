// post.cuh -- post_process (DG_solver.f90:128-661) as sm_100a kernels.
//
//   pp_avg_ldf_kernel   loop 1 (DG_solver.f90:161-277): cell averages of every interior and
//                       non-corner ghost element, admissibility of the average, the LDF projection
//                       of (Bx,By) as one dense nodal operator, and (for OEDG) per-block partial
//                       sums of the average plus max/min of the post-LDF interior values.
//   pp_reduce_kernel    the global average sum (fixed order) and u_vari_global (DG_solver.f90:282-294):
//                       max|u - g| = max(umax - g, g - umin) because rounding is monotone.
//   pp_sigsum_kernel    the OEDG face jump indicators OEDG_sigsum_x/y (DG_solver.f90:295-422).
//   pp_limit_kernel     loop 3 (DG_solver.f90:428-656): OEDG damping, Zhang-Shu positivity
//                       scaling with its bounded re-limit loop, entropy-offset limiting, cell
//                       entropy (block partials, fixed order).
//   pp_entsum_kernel    total entropy from the partials (fixed order).
#pragma once
#include "common.cuh"

namespace mhd {

constexpr int PP_NT = 256;

template <int P>
struct PPCfg {
  static constexpr int N = P + 1, NN = N * N, EB = 8 * NN, N2 = 2 * NN;
  static constexpr int TE = (P == 1) ? 64 : (P == 2 ? 32 : 16);  // elements per CTA
};

// ---------------------------------------------------------------------------------------------
// Zhang-Shu positivity (DG_solver.f90:528-603), entropy-offset limiting (:606-633) and the cell
// entropy (:635-649) of the elements a CTA holds in shared memory (s_u [e][var][node], s_avg
// [e][8]).  Node-parallel: node pressures and entropies take one thread per node; the per-element
// decisions take one lane per element; the rare re-limit loop stays serial per element.
// mask (may be NULL = all) selects the elements to limit; cell-entropy arrays are indexed from
// ebase; the CTA's entropy partial (elements in order) goes to *ent_out.
// ---------------------------------------------------------------------------------------------
template <int P>
__device__ __forceinline__ void limit_elements(double* s_u, const double* s_avg, const unsigned char* mask, int ne,
                                               long long ebase, const Geo& g, Ctrl* ctrl, int ent_offset,
                                               int comput_ent, const double* __restrict__ cell_ent_DG,
                                               const double* __restrict__ cell_ent_FV,
                                               const unsigned char* __restrict__ cell_ent_nan,
                                               double* __restrict__ ent_out) {
  using C = PPCfg<P>;
  constexpr int N = C::N, NN = C::NN, EB = C::EB, TE = C::TE;
  constexpr double BIG = 1.7976931348623157e308;
  __shared__ double l_nd[TE * NN];
  __shared__ double l_thd[TE], l_thp[TE];
  __shared__ int l_cnt;
  const int tid = threadIdx.x;
  const double gamma = g.gamma;
  const DegConst& dc = c_deg[P];
  if (tid == 0) l_cnt = 0;
  // density: theta from the minimum nodal density (DG_solver.f90:538-553)
  if (tid < ne) {
    double th = -1.0;
    if (!mask || mask[tid]) {
      const double* x = s_u + tid * EB;
      double den_min = BIG;
      for (int q = 0; q < NN; ++q) den_min = fmin(den_min, x[q]);
      if (den_min < PP_EPS) {
        const double da = s_avg[tid * 8];
        th = fmax(fmin((da - PP_EPS) / (da - den_min), 1.0), 0.0);
      }
    }
    l_thd[tid] = th;
  }
  __syncthreads();
  for (int it = tid; it < ne * NN; it += PP_NT) {
    const int e = it / NN, q = it - e * NN;
    const double th = l_thd[e];
    if (th >= 0.0) {
      const double a0 = s_avg[e * 8];
      double x = s_u[e * EB + q];
      x = a0 + th * (x - a0);
      s_u[e * EB + q] = fmax(x, PP_EPS);
    }
  }
  __syncthreads();
  // pressure: nodal pressures in parallel, theta from their minimum (DG_solver.f90:556-571)
  for (int it = tid; it < ne * NN; it += PP_NT) {
    const int e = it / NN, q = it - e * NN;
    if (mask && !mask[e]) continue;
    const double* x = s_u + e * EB + q;
    l_nd[it] = prs_of(x[0], x[NN], x[2 * NN], x[3 * NN], x[4 * NN], x[5 * NN], x[6 * NN], x[7 * NN], gamma);
  }
  __syncthreads();
  if (tid < ne) {
    double th = -1.0;
    if (!mask || mask[tid]) {
      double pmin = BIG;
      for (int q = 0; q < NN; ++q) pmin = fmin(pmin, l_nd[tid * NN + q]);
      if (pmin < PP_EPS) {
        const double* a = s_avg + tid * 8;
        const double pa = prs_of(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], gamma);
        th = fmax(fmin((pa - PP_EPS) / (pa - pmin), 1.0), 0.0);
      }
      if (l_thd[tid] >= 0.0 || th >= 0.0) atomicAdd(&l_cnt, 1);  // neg_node (DG_solver.f90:602)
    }
    l_thp[tid] = th;
  }
  __syncthreads();
  for (int it = tid; it < ne * EB; it += PP_NT) {
    const int e = it / EB;
    const double th = l_thp[e];
    if (th >= 0.0) {
      const double a = s_avg[e * 8 + (it - e * EB) / NN];
      s_u[it] = a + th * (s_u[it] - a);
    }
  }
  __syncthreads();
  if (tid < ne) {
    double* x = s_u + tid * EB;
    const double* a = s_avg + tid * 8;
    double theta = l_thp[tid];
    if (theta >= 0.0) {  // re-check after the FP-inexact theta (DG_solver.f90:573-599), rare
      for (int it_count = 0;; ++it_count) {  // bounded: at most two extra shrinks
        double prs_min = BIG;
        for (int q = 0; q < NN; ++q)
          prs_min = fmin(prs_min, prs_of(x[q], x[NN + q], x[2 * NN + q], x[3 * NN + q], x[4 * NN + q], x[5 * NN + q], x[6 * NN + q], x[7 * NN + q], gamma));
        if (!(prs_min < 0.99 * PP_EPS)) break;
        if (it_count > 1) {
          atomicOr(&ctrl->pp_relimit, 1);
          break;
        }
        theta = 0.6 * theta;
        for (int v = 0; v < 8; ++v)
          for (int q = 0; q < NN; ++q) x[v * NN + q] = a[v] + theta * (x[v * NN + q] - a[v]);
      }
    }
    const long long ce = ebase + tid;
    if (ent_offset && (!mask || mask[tid]) && !cell_ent_nan[ce]) {  // DG_solver.f90:606-633
      const double old = cell_ent_DG[ce], eavg = cell_ent_FV[ce];
      double nw = 0.0;
      for (int l = 0; l < N; ++l)
        for (int k = 0; k < N; ++k) {
          const int q = k + N * l;
          const double pq = fmax(prs_of(x[q], x[NN + q], x[2 * NN + q], x[3 * NN + q], x[4 * NN + q], x[5 * NN + q], x[6 * NN + q], x[7 * NN + q], gamma), PP_EPS);
          nw = nw + (0.25 * g.hx * g.hy * dc.qw[k] * dc.qw[l]) * ent_of(x[q], pq, gamma);
        }
      if (nw > old) {
        const double th = fmax(fmin((old - eavg) / (nw - eavg), 1.0), 0.0);
        for (int v = 0; v < 8; ++v)
          for (int q = 0; q < NN; ++q) x[v * NN + q] = a[v] + th * (x[v * NN + q] - a[v]);
      }
    }
  }
  __syncthreads();
  if (comput_ent) {  // DG_solver.f90:635-649
    for (int it = tid; it < ne * NN; it += PP_NT) {
      const int e = it / NN, q = it - e * NN;
      if (mask && !mask[e]) continue;
      const int k = q % N, l = q / N;
      const double* x = s_u + e * EB + q;
      const double pq = fmax(prs_of(x[0], x[NN], x[2 * NN], x[3 * NN], x[4 * NN], x[5 * NN], x[6 * NN], x[7 * NN], gamma), PP_EPS);
      l_nd[it] = (0.25 * g.hx * g.hy * dc.qw[k] * dc.qw[l]) * ent_of(x[0], pq, gamma);
    }
    __syncthreads();
    if (tid == 0) {
      double tot = 0.0;
      for (int e = 0; e < ne; ++e) {
        if (mask && !mask[e]) continue;
        double ce = 0.0;
        for (int q = 0; q < NN; ++q) ce = ce + l_nd[e * NN + q];
        tot = tot + ce;
      }
      *ent_out = tot;
    }
  }
  __syncthreads();
  if (tid == 0 && l_cnt) atomicAdd(&ctrl->num_negcell, l_cnt);
}

// ---------------------------------------------------------------------------------------------
// loop 1: averages + admissibility + LDF.  A CTA owns TE consecutive element blocks of the
// ghosted grid (one contiguous run of memory).
// ---------------------------------------------------------------------------------------------
//
// limit = 1 fuses loop 3 for a stage without OEDG and without the entropy sum: the interior
// elements of the chunk are limited in shared memory before the one write-back.  The reference
// skips loop 3 altogether when any element has an inadmissible average (neg_avg); here other CTAs
// may already have limited their elements by then.  That is only allowed where the stage result
// is discarded on neg_avg (the time-step pipeline re-tries the step from u_con), so the stand-alone
// post_process never fuses.
template <int P>
__device__ __forceinline__ void pp_avg_ldf_chunk(double* __restrict__ u, double* __restrict__ u_avg,
                                                 const Geo& g, Ctrl* ctrl, long long chunk, int apply_ldf,
                                                 int need_global, int ent_offset,
                                                 double* __restrict__ partial_out,  // 8 doubles
                                                 double* __restrict__ cell_ent_DG,
                                                 double* __restrict__ cell_ent_FV,
                                                 unsigned char* __restrict__ cell_ent_nan, int limit = 0) {
  using C = PPCfg<P>;
  constexpr int N = C::N, NN = C::NN, EB = C::EB, N2 = C::N2, TE = C::TE;
  __shared__ __align__(16) double s_u[TE * EB];
  __shared__ double s_out[TE * N2];
  __shared__ double s_avg[TE * 8];
  __shared__ double s_A[N2 * N2];
  __shared__ unsigned char s_valid[TE], s_inner[TE];
  __shared__ double s_mx[8 * (PP_NT / 32)], s_mn[8 * (PP_NT / 32)];
  const int tid = threadIdx.x;
  const int nx = g.nx, ny = g.ny, NXG = nx + 2;
  const long long total = (long long)NXG * (ny + 2);
  const long long e0 = chunk * TE;
  const int ne = (int)min((long long)TE, total - e0);
  const DegConst& dc = c_deg[P];

  for (int it = tid; it < ne * EB / 2; it += PP_NT)
    reinterpret_cast<double2*>(s_u)[it] = reinterpret_cast<const double2*>(u + e0 * EB)[it];
  if (apply_ldf)
    for (int it = tid; it < N2 * N2; it += PP_NT) s_A[it] = __ldg(g.ldfA + it);
  if (tid < TE) {
    const long long e = e0 + tid;
    int valid = 0, inner = 0;
    if (tid < ne) {
      const int j = (int)(e / NXG), i = (int)(e - (long long)j * NXG);
      const bool ii = (i >= 1 && i <= nx), jj = (j >= 1 && j <= ny);
      valid = ii || jj;  // DG_solver.f90:165 (corners are skipped)
      inner = ii && jj;
    }
    s_valid[tid] = (unsigned char)valid;
    s_inner[tid] = (unsigned char)inner;
  }
  __syncthreads();

  // cell averages: ua(s) += (0.25*qw_x(k)*qw_y(l)) * u(s,k,l), l outer, k inner (DG_solver.f90:177-184)
  for (int it = tid; it < TE * 8; it += PP_NT) {
    const int e = it >> 3, v = it & 7;
    if (!s_valid[e]) continue;
    const double* x = s_u + e * EB + v * NN;
    double a = 0.0;
#pragma unroll
    for (int l = 0; l < N; ++l)
#pragma unroll
      for (int k = 0; k < N; ++k) a = a + (0.25 * dc.qw[k] * dc.qw[l]) * x[k + N * l];
    s_avg[it] = a;
  }
  __syncthreads();

  // admissibility of the average; cell entropy for the entropy-offset limiter (DG_solver.f90:186-224)
  if (tid < TE && s_valid[tid]) {
    const double* a = s_avg + tid * 8;
    const double den = a[0];
    const double prs = prs_of(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], g.gamma);
    if (den < PP_EPS || prs < PP_EPS) {
      // inadmissible average: the reference leaves this element unwritten (DG_solver.f90:189-193)
      atomicOr(&ctrl->neg_avg, 1);
      s_valid[tid] = 0;
      s_inner[tid] = 0;
    }
    if (ent_offset) {
      const long long e = e0 + tid;
      const double* x = s_u + tid * EB;
      bool flag = true;
      double ce = 0.0;
      for (int q = 0; q < NN; ++q) {
        const double pq = prs_of(x[q], x[NN + q], x[2 * NN + q], x[3 * NN + q], x[4 * NN + q], x[5 * NN + q], x[6 * NN + q], x[7 * NN + q], g.gamma);
        flag = flag && (x[q] >= PP_EPS) && (pq >= PP_EPS);
      }
      if (flag) {
        for (int l = 0; l < N; ++l)
          for (int k = 0; k < N; ++k) {
            const int q = k + N * l;
            const double pq = prs_of(x[q], x[NN + q], x[2 * NN + q], x[3 * NN + q], x[4 * NN + q], x[5 * NN + q], x[6 * NN + q], x[7 * NN + q], g.gamma);
            ce = ce + (0.25 * g.hx * g.hy * dc.qw[k] * dc.qw[l]) * ent_of(x[q], pq, g.gamma);
          }
      }
      cell_ent_FV[e] = (den >= PP_EPS && prs >= PP_EPS) ? ent_of(den, prs, g.gamma) : 0.0;
      cell_ent_DG[e] = flag ? ce : 0.0;
      cell_ent_nan[e] = flag ? 0 : 1;
    }
  }

  __syncthreads();

  // LDF projection of (Bx - avg, By - avg) with the dense nodal operator
  if (apply_ldf) {
    for (int it = tid; it < TE * N2; it += PP_NT) {
      const int e = it / N2, o = it - e * N2;
      if (!s_valid[e]) continue;
      const double* xb = s_u + e * EB + 4 * NN;  // Bx then By, contiguous (vars 4 and 5)
      const double ax = s_avg[e * 8 + 4], ay = s_avg[e * 8 + 5];
      double acc = 0.0;
#pragma unroll 8
      for (int m = 0; m < N2; ++m) acc += s_A[o + N2 * m] * (xb[m] - (m < NN ? ax : ay));
      s_out[it] = acc + (o < NN ? ax : ay);
    }
    __syncthreads();
    for (int it = tid; it < TE * N2; it += PP_NT) {
      const int e = it / N2, o = it - e * N2;
      if (!s_valid[e]) continue;
      s_u[e * EB + 4 * NN + o] = s_out[it];
    }
  }
  __syncthreads();
  if (limit)  // loop 3 on the interior elements (DG_solver.f90:526-633)
    limit_elements<P>(s_u, s_avg, s_inner, ne, e0, g, ctrl, ent_offset, 0, cell_ent_DG, cell_ent_FV, cell_ent_nan,
                      nullptr);

  // write back state and averages
  for (int it = tid; it < ne * EB / 2; it += PP_NT) {
    const int e = (2 * it) / EB;
    if (!s_valid[e]) continue;
    reinterpret_cast<double2*>(u + e0 * EB)[it] = reinterpret_cast<const double2*>(s_u)[it];
  }
  for (int it = tid; it < ne * 8; it += PP_NT) {
    if (!s_valid[it >> 3]) continue;
    u_avg[e0 * 8 + it] = s_avg[it];
  }

  if (need_global) {
    // per-block sum of (hx*hy)*avg over interior elements in element order (DG_solver.f90:227-229)
    if (tid < 8) {
      double sacc = 0.0;
      for (int e = 0; e < ne; ++e)
        if (s_inner[e]) sacc = sacc + (g.hx * g.hy) * s_avg[e * 8 + tid];
      partial_out[tid] = sacc;
    }
    // per-variable max and min of the post-LDF interior node values
    double vmax[8], vmin[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      vmax[v] = -1.0e308;
      vmin[v] = 1.0e308;
    }
    for (int it = tid; it < ne * NN; it += PP_NT) {
      const int e = it / NN, q = it - e * NN;
      if (!s_inner[e]) continue;
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const double x = s_u[e * EB + v * NN + q];
        vmax[v] = fmax(vmax[v], x);
        vmin[v] = fmin(vmin[v], x);
      }
    }
#pragma unroll
    for (int v = 0; v < 8; ++v) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        vmax[v] = fmax(vmax[v], __shfl_xor_sync(0xffffffffu, vmax[v], o));
        vmin[v] = fmin(vmin[v], __shfl_xor_sync(0xffffffffu, vmin[v], o));
      }
    }
    if ((tid & 31) == 0)
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        s_mx[v * (PP_NT / 32) + (tid >> 5)] = vmax[v];
        s_mn[v * (PP_NT / 32) + (tid >> 5)] = vmin[v];
      }
    __syncthreads();
    if (tid < 8) {
      double a = s_mx[tid * (PP_NT / 32)], b = s_mn[tid * (PP_NT / 32)];
      for (int w = 1; w < PP_NT / 32; ++w) {
        a = fmax(a, s_mx[tid * (PP_NT / 32) + w]);
        b = fmin(b, s_mn[tid * (PP_NT / 32) + w]);
      }
      atomicMax(&ctrl->umax_bits[tid], ord_enc(a));
      atomicMin(&ctrl->umin_bits[tid], ord_enc(b));
    }
  }
}

template <int P>
__global__ void __launch_bounds__(PP_NT)
    pp_avg_ldf_kernel(double* __restrict__ u, double* __restrict__ u_avg, Geo g, Ctrl* ctrl,
                      int gate, int apply_ldf, int need_global, int ent_offset,
                      double* __restrict__ partial_sum,  // [gridDim.x][8]
                      double* __restrict__ cell_ent_DG, double* __restrict__ cell_ent_FV,
                      unsigned char* __restrict__ cell_ent_nan, int limit) {
  if (!gate_open(ctrl, gate)) return;
  pp_avg_ldf_chunk<P>(u, u_avg, g, ctrl, blockIdx.x, apply_ldf, need_global, ent_offset,
                      partial_sum + (long long)blockIdx.x * 8, cell_ent_DG, cell_ent_FV, cell_ent_nan, limit);
}

// many instances: items = every member's chunks; slot = the stage state; `final` selects the
// final-stage form (OEDG global reductions for instances that use OEDG); the other stages fuse
// loop 3 (limit)
template <int P>
__global__ void __launch_bounds__(PP_NT)
    pp_avg_ldf_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                       const int* __restrict__ nwork, const int* __restrict__ ninst, int slot, int final, int gate) {
  const int nw = *nwork, n = *ninst;
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int m = batch_member(pref, n, w), chunk = w - __ldg(pref + m);
    const InstDesc& d = insts[m];
    if (!gate_open(d.ctrl, gate)) continue;
    pp_avg_ldf_chunk<P>(d.u[slot], d.u_avg, d.g, d.ctrl, chunk, d.use_ldf, d.use_oedg && final,
                        d.ent_offset, d.partial + (long long)chunk * 8, d.cell_ent_DG, d.cell_ent_FV,
                        d.cell_ent_nan, !final);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// global average (fixed-order sum of block partials) and u_vari_global.  One CTA.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void pp_reduce_body(const double* __restrict__ partial, int nblk, Ctrl* ctrl) {
  __shared__ double s[8][256];
  const int tid = threadIdx.x;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = tid; b < nblk; b += 256)
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[v] = acc[v] + partial[b * 8 + v];
#pragma unroll
  for (int v = 0; v < 8; ++v) s[v][tid] = acc[v];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w)
#pragma unroll
      for (int v = 0; v < 8; ++v) s[v][tid] = s[v][tid] + s[v][tid + w];
    __syncthreads();
  }
  if (tid < 8) {
    const double gsum = s[tid][0];
    ctrl->u_avg_global[tid] = gsum;
    const double umax = ord_dec(ctrl->umax_bits[tid]), umin = ord_dec(ctrl->umin_bits[tid]);
    ctrl->u_vari[tid] = fmax(0.0, fmax(umax - gsum, gsum - umin));
  }
}

__global__ void __launch_bounds__(256) pp_reduce_kernel(const double* __restrict__ partial, int nblk,
                                                        Ctrl* ctrl, int gate) {
  if (!gate_open(ctrl, gate)) return;
  pp_reduce_body(partial, nblk, ctrl);
}

// many instances: CTA per instance (persistent over the instance list)
__global__ void __launch_bounds__(256) pp_reduce_batched(const InstDesc* __restrict__ insts,
                                                         const int* __restrict__ ninst, int final, int gate) {
  const int n = *ninst;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const InstDesc& d = insts[i];
    if (!gate_open(d.ctrl, gate) || !(d.use_oedg && final)) continue;
    pp_reduce_body(d.partial, d.nblk_avg, d.ctrl);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// OEDG face jump indicators (DG_solver.f90:295-422), one value per (face, variable):
//   sigsum = sum_{kk,ll} (2m+1) h^m / (2 max(2p-1,1) kk! ll!) * <0.5 w, |d^kk_x d^ll_y jump|>
// A CTA owns a TX x TY tile of interior elements and computes the left x face and the bottom y
// face of each (plus the right/top boundary faces on the last tile of a row/column).  The tile
// and its left/bottom neighbours (and the ghost column/row on the last tiles) are staged in
// shared memory with coalesced loads; each (face, variable) item then reads two variable blocks.
// Shared records are padded (NN+1 doubles per variable) against bank conflicts.
// ---------------------------------------------------------------------------------------------
// x face: L, R = the variable's nodes [k + N*l] of the left and right element
template <int P>
__device__ __forceinline__ double sigsum_x_face(const double* R, const double* Lf, double hx, double hy) {
  constexpr int N = P + 1;
  const DegConst& dc = c_deg[P];
  const int denom_base = 2 * max(2 * P - 1, 1);
  const double sx = 2.0 / hx, sy = 2.0 / hy;
  double total = 0.0;
  double sxk = 1.0, hx_pow_kk = 1.0;
  int fac_kk = 1;
#pragma unroll 1
  for (int kk = 0; kk <= P; ++kk) {
    double jump[N];
#pragma unroll
    for (int l = 0; l < N; ++l) {
      double tr = 0.0, tl = 0.0;
#pragma unroll
      for (int k = 0; k < N; ++k) {
        tr += dc.R0[kk][k] * R[k + N * l];
        tl += dc.RN[kk][k] * Lf[k + N * l];
      }
      jump[l] = sxk * tr - sxk * tl;
    }
    int fac_ll = 1;
    double h_pow = hx_pow_kk;
#pragma unroll
    for (int ll = 0; ll <= P - kk; ++ll) {
      double L1 = 0.0;
#pragma unroll
      for (int l = 0; l < N; ++l) L1 += (0.5 * dc.qw[l]) * fabs(jump[l]);
      const double coef = ((2 * (kk + ll) + 1) * h_pow) / (double)(denom_base * fac_kk * fac_ll);
      total = total + coef * L1;
      if (ll < P) {
        double nj[N];
#pragma unroll
        for (int a = 0; a < N; ++a) {
          double acc = 0.0;
#pragma unroll
          for (int b = 0; b < N; ++b) acc += (sy * dc.D[a + N * b]) * jump[b];
          nj[a] = acc;
        }
#pragma unroll
        for (int a = 0; a < N; ++a) jump[a] = nj[a];
        fac_ll *= (ll + 1);
        h_pow *= hx;
      }
    }
    if (kk < P) {
      fac_kk *= (kk + 1);
      hx_pow_kk *= hx;
      sxk *= sx;
    }
  }
  return total;
}

// y face: B, T = the variable's nodes of the bottom and top element
template <int P>
__device__ __forceinline__ double sigsum_y_face(const double* T, const double* B, double hx, double hy) {
  constexpr int N = P + 1;
  const DegConst& dc = c_deg[P];
  const int denom_base = 2 * max(2 * P - 1, 1);
  const double sx = 2.0 / hx, sy = 2.0 / hy;
  double total = 0.0;
  double syl = 1.0, hy_pow_ll = 1.0;
  int fac_ll = 1;
#pragma unroll 1
  for (int ll = 0; ll <= P; ++ll) {
    double jump[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double tt = 0.0, tb = 0.0;
#pragma unroll
      for (int l = 0; l < N; ++l) {
        tt += dc.R0[ll][l] * T[k + N * l];
        tb += dc.RN[ll][l] * B[k + N * l];
      }
      jump[k] = syl * tt - syl * tb;
    }
    int fac_kk = 1;
    double h_pow = hy_pow_ll;
#pragma unroll
    for (int kk = 0; kk <= P - ll; ++kk) {
      double L1 = 0.0;
#pragma unroll
      for (int k = 0; k < N; ++k) L1 += (0.5 * dc.qw[k]) * fabs(jump[k]);
      const double coef = ((2 * (kk + ll) + 1) * h_pow) / (double)(denom_base * fac_kk * fac_ll);
      total = total + coef * L1;
      if (kk < P) {
        double nj[N];
#pragma unroll
        for (int a = 0; a < N; ++a) {
          double acc = 0.0;
#pragma unroll
          for (int b = 0; b < N; ++b) acc += (sx * dc.D[a + N * b]) * jump[b];
          nj[a] = acc;
        }
#pragma unroll
        for (int a = 0; a < N; ++a) jump[a] = nj[a];
        fac_kk *= (kk + 1);
        h_pow *= hy;
      }
    }
    if (ll < P) {
      fac_ll *= (ll + 1);
      hy_pow_ll *= hy;
      syl *= sy;
    }
  }
  return total;
}

template <int P>
struct SigCfg;
template <>
struct SigCfg<1> { static constexpr int TX = 8, TY = 8; };
template <>
struct SigCfg<2> { static constexpr int TX = 8, TY = 4; };
template <>
struct SigCfg<3> { static constexpr int TX = 4, TY = 4; };

template <int P>
struct SigLayout {
  static constexpr int N = P + 1, NN = N * N, EB = 8 * NN;
  static constexpr int TX = SigCfg<P>::TX, TY = SigCfg<P>::TY;
  static constexpr int VS = NN + 1, ES = 8 * VS;   // padded variable / element record
  static constexpr int RW = TX + 2, RH = TY + 2;   // staged rectangle (max)
  static constexpr int DOUBLES = RW * RH * ES;
};

template <int P>
__device__ __forceinline__ void pp_sigsum_tile(const double* __restrict__ u, const Geo& g, int tile_x, int tile_y,
                                               double* __restrict__ sig_x, double* __restrict__ sig_y) {
  using L = SigLayout<P>;
  constexpr int NN = L::NN, EB = L::EB, VS = L::VS, ES = L::ES, TX = L::TX, TY = L::TY, RW = L::RW;
  constexpr int NT = 256;
  __shared__ double s_e[L::DOUBLES];  // face math reads its two variable blocks from here
  const int tid = threadIdx.x;
  const int nx = g.nx, ny = g.ny, NXG = nx + 2;
  const int i0 = 1 + tile_x * TX, j0 = 1 + tile_y * TY;
  const int W = min(TX, nx - i0 + 1), H = min(TY, ny - j0 + 1);
  const int right = (i0 + W - 1 == nx), top = (j0 + H - 1 == ny);
  const int cw = W + 1 + right, rh = H + 1 + top;  // staged columns i0-1 .., rows j0-1 ..
  // stage: rect row rr = grid row j0-1+rr, rect column cc = grid column i0-1+cc
  for (int it = tid; it < rh * cw * EB; it += NT) {
    const int rr = it / (cw * EB), rem = it - rr * cw * EB;  // rem indexes a contiguous run of cw elements
    const int cc = rem / EB, w = rem - cc * EB, v = w / NN, q = w - v * NN;
    s_e[(rr * RW + cc) * ES + v * VS + q] = __ldg(u + ((long long)(j0 - 1 + rr) * NXG + (i0 - 1)) * EB + rem);
  }
  __syncthreads();
  const int nfx = H * (W + right), nfy = W * (H + top);
  for (int it = tid; it < 8 * (nfx + nfy); it += NT) {
    const int v = it & 7, f = it >> 3;
    if (f < nfx) {  // x face: row r, face c between columns c-1 and c of the tile
      const int r = f / (W + right), c = f - r * (W + right);
      const double* pl = s_e + ((r + 1) * RW + c) * ES + v * VS;
      const int i = i0 + c, j = j0 + r;
      sig_x[(((long long)(j - 1) * (nx + 1)) + (i - 1)) * 8 + v] = sigsum_x_face<P>(pl + ES, pl, g.hx, g.hy);
    } else {  // y face: column c, face r between rows r-1 and r of the tile
      const int f2 = f - nfx;
      const int c = f2 / (H + top), r = f2 - c * (H + top);
      const double* pb = s_e + (r * RW + c + 1) * ES + v * VS;
      const int i = i0 + c, j = j0 + r;
      sig_y[(((long long)(j - 1) * nx) + (i - 1)) * 8 + v] = sigsum_y_face<P>(pb + RW * ES, pb, g.hx, g.hy);
    }
  }
}

template <int P>
__global__ void __launch_bounds__(256, 2)
    pp_sigsum_kernel(const double* __restrict__ u, Geo g, Ctrl* ctrl, int gate,
                     double* __restrict__ sig_x, double* __restrict__ sig_y) {
  if (!gate_open(ctrl, gate)) return;
  pp_sigsum_tile<P>(u, g, blockIdx.x, blockIdx.y, sig_x, sig_y);
}

// many instances: items = every member's tiles (row-major)
template <int P>
__global__ void __launch_bounds__(256, 2)
    pp_sigsum_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                      const int* __restrict__ nwork, const int* __restrict__ ninst, int slot, int final, int gate) {
  const int nw = *nwork, n = *ninst;
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int m = batch_member(pref, n, w), local = w - __ldg(pref + m);
    const InstDesc& d = insts[m];
    if (!gate_open(d.ctrl, gate) || !(d.use_oedg && final)) continue;
    const int ntx = (d.g.nx + SigCfg<P>::TX - 1) / SigCfg<P>::TX;
    pp_sigsum_tile<P>(d.u[slot], d.g, local % ntx, local / ntx, d.sig_x, d.sig_y);
    __syncthreads();  // the next tile reuses shared memory
  }
}

// ---------------------------------------------------------------------------------------------
// loop 3: OEDG damping, positivity, entropy offset, entropy.  A CTA owns TE consecutive
// interior elements of one row j (a contiguous run of memory).
// ---------------------------------------------------------------------------------------------
template <int P>
__device__ __forceinline__ void pp_limit_segment(
    double* __restrict__ u, const double* __restrict__ u_avg, const Geo& g, Ctrl* ctrl, int seg, int jrow,
    int apply_oedg, double oedg_dt, int ent_offset, int comput_ent, const double* __restrict__ sig_x,
    const double* __restrict__ sig_y, const double* __restrict__ cell_ent_DG,
    const double* __restrict__ cell_ent_FV, const unsigned char* __restrict__ cell_ent_nan,
    double* __restrict__ ent_out, double* __restrict__ accept_dst) {
  using C = PPCfg<P>;
  constexpr int NN = C::NN, EB = C::EB, TE = C::TE;
  if (ctrl->neg_avg) return;  // the reference skips loop 3 once neg_avg is set (DG_solver.f90:431)
  __shared__ __align__(16) double s_u[TE * EB];
  __shared__ double s_avg[TE * 8];
  __shared__ double s_nd[TE * NN * 2];  // per-node scratch (wave speeds, pressures, entropies)
  __shared__ double s_theta[TE];
  const int tid = threadIdx.x;
  const int nx = g.nx, NXG = nx + 2;
  const int j = 1 + jrow;
  const int i0 = 1 + seg * TE;
  const int ne = min(TE, nx - i0 + 1);
  const long long ebase = (long long)j * NXG + i0;
  const double gamma = g.gamma;
  for (int it = tid; it < ne * EB / 2; it += PP_NT)
    reinterpret_cast<double2*>(s_u)[it] = reinterpret_cast<const double2*>(u + ebase * EB)[it];
  for (int it = tid; it < ne * 8; it += PP_NT) s_avg[it] = u_avg[ebase * 8 + it];
  __syncthreads();

  if (apply_oedg) {  // DG_solver.f90:448-524
    for (int it = tid; it < ne * NN; it += PP_NT) {
      const int e = it / NN, q = it - e * NN;
      const double* x = s_u + e * EB + q;
      const double rho = fmax(x[0], PP_EPS);
      const double ir = 1.0 / rho;
      const double vx = ir * x[NN], vy = ir * x[2 * NN];
      const double ek = 0.5 * ir * (x[NN] * x[NN] + x[2 * NN] * x[2 * NN] + x[3 * NN] * x[3 * NN]);
      const double bx = x[4 * NN], by = x[5 * NN], bz = x[6 * NN];
      const double bsq = bx * bx + by * by + bz * bz;
      const double pf = fmax((gamma - 1.0) * (x[7 * NN] - (ek + 0.5 * bsq)), PP_EPS);
      const double cs = gamma * pf * ir, ss = cs + bsq * ir, sqsq = ss * ss, coef = 4.0 * cs * ir;
      s_nd[e * 2 * NN + q] = fabs(vx) + sqrt(0.5 * fmax(ss + sqrt(fmax(sqsq - coef * (bx * bx), 0.0)), 0.0));
      s_nd[e * 2 * NN + NN + q] = fabs(vy) + sqrt(0.5 * fmax(ss + sqrt(fmax(sqsq - coef * (by * by), 0.0)), 0.0));
    }
    __syncthreads();
    if (tid < ne) {
      const int e = tid, i = i0 + e;
      double mx = 0.0, my = 0.0;
      for (int q = 0; q < NN; ++q) {
        mx = fmax(mx, s_nd[e * 2 * NN + q]);
        my = fmax(my, s_nd[e * 2 * NN + NN + q]);
      }
      const long long fxl = ((long long)(j - 1) * (nx + 1) + (i - 1)) * 8;
      const long long fyb = ((long long)(j - 1) * nx + (i - 1)) * 8;
      const long long fyt = ((long long)j * nx + (i - 1)) * 8;
      double dmaxv = -1.0e308;
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const double uv = ctrl->u_vari[v];
        double d = 0.0;
        if (uv > OEDG_EPS)
          d = ((mx / g.hx) * (sig_x[fxl + v] + sig_x[fxl + 8 + v]) + (my / g.hy) * (sig_y[fyb + v] + sig_y[fyt + v])) / uv;
        dmaxv = fmax(dmaxv, d);
      }
      s_theta[e] = exp(-oedg_dt * dmaxv);
    }
    __syncthreads();
    for (int it = tid; it < ne * EB; it += PP_NT) {
      const int e = it / EB, v = (it - e * EB) / NN;
      const double a = s_avg[e * 8 + v];
      s_u[it] = a + s_theta[e] * (s_u[it] - a);
    }
    __syncthreads();
  }

  limit_elements<P>(s_u, s_avg, nullptr, ne, ebase, g, ctrl, ent_offset, comput_ent, cell_ent_DG, cell_ent_FV,
                    cell_ent_nan, ent_out);

  for (int it = tid; it < ne * EB / 2; it += PP_NT) {
    const double2 val = reinterpret_cast<const double2*>(s_u)[it];
    reinterpret_cast<double2*>(u + ebase * EB)[it] = val;
    if (accept_dst) reinterpret_cast<double2*>(accept_dst + ebase * EB)[it] = val;
  }
}

template <int P>
__global__ void __launch_bounds__(PP_NT)
    pp_limit_kernel(double* __restrict__ u, const double* __restrict__ u_avg, Geo g, Ctrl* ctrl,
                    int gate, int apply_oedg, const double* __restrict__ dt_ptr, double oedg_dt_arg,
                    int ent_offset, int comput_ent, const double* __restrict__ sig_x,
                    const double* __restrict__ sig_y, const double* __restrict__ cell_ent_DG,
                    const double* __restrict__ cell_ent_FV, const unsigned char* __restrict__ cell_ent_nan,
                    double* __restrict__ ent_partial, double* __restrict__ accept_dst) {
  if (!gate_open(ctrl, gate)) return;
  const double oedg_dt = dt_ptr ? *dt_ptr : oedg_dt_arg;
  pp_limit_segment<P>(u, u_avg, g, ctrl, blockIdx.x, blockIdx.y, apply_oedg, oedg_dt, ent_offset, comput_ent,
                      sig_x, sig_y, cell_ent_DG, cell_ent_FV, cell_ent_nan,
                      ent_partial + (long long)blockIdx.y * gridDim.x + blockIdx.x, accept_dst);
}

// many instances: items = every member's row segments (row-major); the final stage applies OEDG
// (if the instance uses it), computes the entropy and writes the accepted interior into slot 0
template <int P>
__global__ void __launch_bounds__(PP_NT)
    pp_limit_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                     const int* __restrict__ nwork, const int* __restrict__ ninst, int slot, int final, int gate) {
  const int nw = *nwork, n = *ninst;
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int m = batch_member(pref, n, w), local = w - __ldg(pref + m);
    const InstDesc& d = insts[m];
    if (!gate_open(d.ctrl, gate)) continue;
    const int nseg = (d.g.nx + PPCfg<P>::TE - 1) / PPCfg<P>::TE;
    const int seg = local % nseg, row = local / nseg;
    pp_limit_segment<P>(d.u[slot], d.u_avg, d.g, d.ctrl, seg, row, d.use_oedg && final, d.ctrl->dt,
                        d.ent_offset, final, d.sig_x, d.sig_y, d.cell_ent_DG, d.cell_ent_FV, d.cell_ent_nan,
                        d.ent_partial + local, final ? d.u[0] : nullptr);
    __syncthreads();
  }
}

// total entropy = fixed-order sum of the per-CTA partials.  One CTA.
__device__ __forceinline__ void pp_entsum_body(const double* __restrict__ partial, int nblk, Ctrl* ctrl) {
  __shared__ double s[256];
  const int tid = threadIdx.x;
  double acc = 0.0;
  for (int b = tid; b < nblk; b += 256) acc = acc + partial[b];
  s[tid] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) s[tid] = s[tid] + s[tid + w];
    __syncthreads();
  }
  if (tid == 0) ctrl->tot_ent = s[0];
}

__global__ void __launch_bounds__(256) pp_entsum_kernel(const double* __restrict__ partial, int nblk,
                                                        Ctrl* ctrl, int gate) {
  if (!gate_open(ctrl, gate)) return;
  if (ctrl->neg_avg) return;
  pp_entsum_body(partial, nblk, ctrl);
}

__global__ void __launch_bounds__(256) pp_entsum_batched(const InstDesc* __restrict__ insts,
                                                         const int* __restrict__ ninst, int gate) {
  const int n = *ninst;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const InstDesc& d = insts[i];
    if (!gate_open(d.ctrl, gate) || d.ctrl->neg_avg) continue;
    pp_entsum_body(d.ent_partial, d.nseg_limit, d.ctrl);
    __syncthreads();
  }
}

}  // namespace mhd
