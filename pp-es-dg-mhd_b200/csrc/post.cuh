// post.cuh -- post_process (DG_solver.f90:128-661) as sm_100a kernels.
//
//   pp_avg_ldf_kernel   loop 1 (DG_solver.f90:161-277): cell averages of every interior and
//                       non-corner ghost element, admissibility of the average, the LDF projection
//                       of (Bx,By) as one dense nodal operator, and (for OEDG) per-chunk partial
//                       sums of the average.  In the time-step pipeline a stage without OEDG also
//                       runs loop 3 here (fused).
//   pp_reduce_kernel    the global average sum in a fixed order (DG_solver.f90:282-286).
//   pp_sigsum_kernel    the OEDG face jump indicators OEDG_sigsum_x/y (DG_solver.f90:295-422), and
//                       the max and min of the post-LDF interior node values (read from the tile
//                       it stages anyway).
//   pp_limit_kernel     loop 3 (DG_solver.f90:428-656): OEDG damping, with u_vari_global
//                       (DG_solver.f90:287-294) = max|u - g| = max(umax - g, g - umin) (rounding
//                       is monotone), Zhang-Shu positivity
//                       scaling with its bounded re-limit loop, entropy-offset limiting, cell
//                       entropy (segment partials, fixed order); in the time-step pipeline the
//                       final stage's result goes to u_con only (the accepted state).
//   pp_entsum_kernel    total entropy from the partials (fixed order).
//   stage_end_bc_kernel the end of a stage of the time-step pipeline in one launch: the entropy sum
//                       (final stage), the stage-end decision, the next stage's pseudo-time and
//                       the ghost fill of the stage state.
//
// Loops 1 and 3 work element-locally, so they map one element to a group of lanes of a warp (GS
// in loop 1, GSL in the limiter kernel; PPCfg), one lane per GLL node, each lane holding its node's
// 8 variables in registers.  Loads and stores of a variable are then 8*NN-byte runs per group
// (coalesced), per-element sums, minima and maxima are reductions inside the group (butterflies for
// power-of-two groups, a fold plus a butterfly for the 9-lane groups; every lane ends with the same
// value), and no CTA-wide barrier sits between the steps of one element.  A CTA of NT threads handles a chunk of TE = (NT/32) * (32/GS) consecutive
// elements; per-chunk partial sums are formed in element order.  The single-instance loop-1
// kernel is a persistent grid over the chunks in which each warp copies its elements of the next
// chunk into shared memory (cp.async) while it works on the current one.  In the first stage of
// a time step loop 1 also forms the stage state from u_con and k1 (Stage1Src).  The indicator
// kernel stages each tile of elements in shared memory with cp.async, row by row.
#pragma once
#include "common.cuh"
#include "misc.cuh"

namespace mhd {

constexpr unsigned FULL_MASK = 0xffffffffu;

// Per degree: threads per CTA and CTAs per SM (the register budget) of the loop-1 and loop-3
// kernels (MHD_PP_CFG<p> = NT, MINB), and the element tile and CTAs per SM of the OEDG indicator
// kernel (MHD_SIG_CFG<p> = TX, TY, MINB).  autotune.py times candidates on the GPU at hand and
// writes post_tuned.h, which takes precedence when present.
#if __has_include("post_tuned.h")
#include "post_tuned.h"
#endif
#ifndef MHD_PP_CFG1
#define MHD_PP_CFG1 256, 4
#endif
#ifndef MHD_PP_CFG2
#define MHD_PP_CFG2 256, 4
#endif
#ifndef MHD_PP_CFG3
#define MHD_PP_CFG3 256, 4
#endif
#ifndef MHD_SIG_CFG1
#define MHD_SIG_CFG1 8, 8, 3
#endif
#ifndef MHD_SIG_CFG2
#define MHD_SIG_CFG2 8, 4, 3
#endif
#ifndef MHD_SIG_CFG3
#define MHD_SIG_CFG3 4, 4, 2
#endif
struct PPParams {
  int NT, MINB;
};
struct SigParams {
  int TX, TY, MINB;
};
template <int P>
struct PPTune;
template <>
struct PPTune<1> {
  static constexpr PPParams pp{MHD_PP_CFG1};
  static constexpr SigParams sig{MHD_SIG_CFG1};
};
template <>
struct PPTune<2> {
  static constexpr PPParams pp{MHD_PP_CFG2};
  static constexpr SigParams sig{MHD_SIG_CFG2};
};
template <>
struct PPTune<3> {
  static constexpr PPParams pp{MHD_PP_CFG3};
  static constexpr SigParams sig{MHD_SIG_CFG3};
};

// Lanes per element: loop 1 takes a power-of-two group of GS lanes (16 for the 9 nodes of p = 2);
// the final stage's limiter kernel takes GSL lanes, 9 at p = 2 (three elements per warp, lanes
// 27-31 idle), where its per-node work outweighs the dearer reductions of a 9-lane group (measured
// on the 400x400 p = 2 blast: limiter 0.115 -> 0.088 ms; loop 1 with 9-lane groups and its cell
// sums through shared memory was 3 % slower and stays at 16 lanes).
template <int P>
struct PPCfg {
  static constexpr int N = P + 1, NN = N * N, EB = 8 * NN, N2 = 2 * NN;
  static constexpr int NT = PPTune<P>::pp.NT, MINB = PPTune<P>::pp.MINB;
  static constexpr int GS = NN <= 4 ? 4 : (NN <= 8 ? 8 : (NN <= 16 ? 16 : 32));  // loop 1: lanes per element
  static constexpr int G = 32 / GS;                                               // elements per warp
  static constexpr int TE = (NT / 32) * G;                                        // elements per CTA chunk
  static constexpr int GSL = NN == 9 ? 9 : GS;                                    // limiter kernel: lanes per element
  static constexpr int GL = 32 / GSL;
  static constexpr int TEL = (NT / 32) * GL;                                      // elements per limiter CTA
  static_assert(NT % 32 == 0 && NT <= 1024, "whole warps");
};

// This lane's group and node for groups of GS lanes.  Where GS does not divide 32 the lanes past
// the last group are idle: they take group 0's lanes as partners in the group reductions (their
// results are unused) and a node number beyond every element (node >= NN).
template <int GS>
struct GrpLane {
  int grp, node;
  bool idle;
};
template <int GS>
__device__ __forceinline__ GrpLane<GS> grp_lane() {
  const int lane = threadIdx.x & 31, g = lane / GS;
  const bool idle = g >= 32 / GS;
  return GrpLane<GS>{idle ? 0 : g, idle ? lane : lane - g * GS, idle};
}
// the smallest chunk of any degree: per-chunk partial buffers are sized by it
constexpr int pp_min_chunk() {
  return PPCfg<1>::TE < PPCfg<2>::TE ? (PPCfg<1>::TE < PPCfg<3>::TE ? PPCfg<1>::TE : PPCfg<3>::TE)
                                     : (PPCfg<2>::TE < PPCfg<3>::TE ? PPCfg<2>::TE : PPCfg<3>::TE);
}

// global -> shared copies that do not pass through registers (cp.async, sm_80 and later): 8 bytes,
// or 16 bytes with both addresses 16-byte aligned
__device__ __forceinline__ void cp_async8(double* dst_shared, const double* src_global) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst_shared);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src_global) : "memory");
}
__device__ __forceinline__ void cp_async16(double* dst_shared, const double* src_global) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst_shared);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src_global) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Reduction over a group of GS lanes, the result in every lane of the group.  A power-of-two group
// uses the xor butterfly.  Otherwise (GS = 9) the lanes past the largest power of two P2 are
// folded onto the group's first lanes, the P2 lanes reduce by a butterfly with partners inside the
// group (explicit lane indices), and every lane takes the group's first lane's result: a fixed
// order, and one value for the whole group.
template <int GS, class Op>
__device__ __forceinline__ double grp_reduce(double v, Op op) {
  if constexpr ((GS & (GS - 1)) == 0) {
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
  } else {
    constexpr int P2 = GS >= 16 ? 16 : (GS >= 8 ? 8 : (GS >= 4 ? 4 : 2));
    static_assert(GS - P2 <= P2, "one fold");
    const GrpLane<GS> gl = grp_lane<GS>();
    const int gb = gl.grp * GS, node = gl.node;
    const double hi = __shfl_sync(FULL_MASK, v, gb + (node + P2 < GS ? node + P2 : 0));
    if (node + P2 < GS) v = op(v, hi);
#pragma unroll
    for (int o = P2 / 2; o > 0; o >>= 1) v = op(v, __shfl_sync(FULL_MASK, v, gb + ((node ^ o) & (P2 - 1))));
    return __shfl_sync(FULL_MASK, v, gb);
  }
}
struct OpAdd {
  __device__ __forceinline__ double operator()(double a, double b) const { return a + b; }
};
struct OpMin {
  __device__ __forceinline__ double operator()(double a, double b) const { return fmin(a, b); }
};
struct OpMax {
  __device__ __forceinline__ double operator()(double a, double b) const { return fmax(a, b); }
};
template <int GS>
__device__ __forceinline__ double grp_sum(double v) { return grp_reduce<GS>(v, OpAdd{}); }
template <int GS>
__device__ __forceinline__ double grp_min(double v) { return grp_reduce<GS>(v, OpMin{}); }
template <int GS>
__device__ __forceinline__ double grp_max(double v) { return grp_reduce<GS>(v, OpMax{}); }

// All eight sums of a[0..7] over each group of GS lanes, in every lane of the group, by a
// reduce-scatter (each exchange halves the values a lane carries, one lane bit per level: 8
// exchanges at GS = 16 instead of 8 butterflies of 4) and an all-gather through the group's
// shared row `row` (8 doubles).  Deterministic, and every lane of a group ends with the same sums
// (each final sum is formed in one lane pair as x + y and y + x, which IEEE addition makes equal,
// and read from the one copy in `row`).
template <int GS>
__device__ __forceinline__ void grp_sum8(double* a, double* row) {
  static_assert((GS & (GS - 1)) == 0, "power-of-two groups");
  constexpr int LV = GS >= 8 ? 3 : (GS == 4 ? 2 : 1);  // halving levels
  const int lane = threadIdx.x & 31;
  constexpr int CNT = 8 >> LV;                          // values a lane keeps after them
#pragma unroll
  for (int j = 0; j < LV; ++j) {
    const int o = GS >> (j + 1);
    const int half = 4 >> j;
    const bool hi = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < half; ++i) {
      const double send = hi ? a[i] : a[i + half];
      const double recv = __shfl_xor_sync(FULL_MASK, send, o);
      a[i] = (hi ? a[i + half] : a[i]) + recv;
    }
  }
#pragma unroll
  for (int o = GS >> (LV + 1); o > 0; o >>= 1)
#pragma unroll
    for (int i = 0; i < CNT; ++i) a[i] = a[i] + __shfl_xor_sync(FULL_MASK, a[i], o);
  // all-gather through the group's shared row: the lane that holds variables vb..vb+CNT-1 (and
  // whose low bits are zero) writes them, every lane reads all 8
  int vb = 0;
#pragma unroll
  for (int j = 0; j < LV; ++j)
    if (lane & (GS >> (j + 1))) vb += 4 >> j;
  if ((lane & ((GS >> LV) - 1)) == 0)
#pragma unroll
    for (int i = 0; i < CNT; ++i) row[vb + i] = a[i];
  __syncwarp();
#pragma unroll
  for (int v = 0; v < 8; ++v) a[v] = row[v];
  __syncwarp();  // the row is rewritten next
}

// a[v] for a lane-dependent v in 0..7, by selects (an indexed read would put a[] in local memory)
__device__ __forceinline__ double pick8(const double* a, int v) {
  double r = a[0];
#pragma unroll
  for (int q = 1; q < 8; ++q) r = (v == q) ? a[q] : r;
  return r;
}

__device__ __forceinline__ double node_prs(const double* x, double gamma) {
  return prs_of(x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], gamma);
}

// ---------------------------------------------------------------------------------------------
// Loop 3 for the element of this lane's group (DG_solver.f90:526-649): Zhang-Shu positivity with
// its bounded re-limit loop, entropy-offset limiting, and the cell entropy.  x = this lane's node,
// avg = the element average (all lanes of the group), node = lane's node (active = node < NN and
// the group's element is limited).  Every lane of the warp calls this (the group reductions need
// the whole warp); returns the cell entropy (0 where not computed) and sets *negcell.  GS: lanes
// per element of the caller's layout.
// ---------------------------------------------------------------------------------------------
template <int P, int GS = PPCfg<P>::GS>
__device__ __forceinline__ double limit_group(double* x, const double* avg, bool active, bool lead, int node,
                                              long long ce, const Geo& g, Ctrl* ctrl, int ent_offset,
                                              int comput_ent, const double* __restrict__ cell_ent_DG,
                                              const double* __restrict__ cell_ent_FV,
                                              const unsigned char* __restrict__ cell_ent_nan, bool* negcell,
                                              bool* scaled = nullptr) {
  using C = PPCfg<P>;
  constexpr int N = C::N;
  constexpr double BIG = 1.7976931348623157e308;
  const double gamma = g.gamma;
  const DegConst& dc = c_deg[P];
  // density: theta from the minimum nodal density (DG_solver.f90:538-553).  The minimum only
  // matters below PP_EPS, so the reduction runs only when some lane of the warp is below it.
  double thd = -1.0;
  if (__any_sync(FULL_MASK, active && x[0] < PP_EPS)) {
    const double den_min = grp_min<GS>(active ? x[0] : BIG);
    if (den_min < PP_EPS) thd = fmax(fmin((avg[0] - PP_EPS) / (avg[0] - den_min), 1.0), 0.0);
  }
  if (active && thd >= 0.0) x[0] = fmax(avg[0] + thd * (x[0] - avg[0]), PP_EPS);
  // pressure: theta from the minimum nodal pressure (DG_solver.f90:556-571), likewise
  const double pq = active ? node_prs(x, gamma) : BIG;
  double pmin = BIG;
  if (__any_sync(FULL_MASK, pq < PP_EPS)) pmin = grp_min<GS>(pq);
  double thp = -1.0;
  if (pmin < PP_EPS) {
    const double pa = prs_of(avg[0], avg[1], avg[2], avg[3], avg[4], avg[5], avg[6], avg[7], gamma);
    thp = fmax(fmin((pa - PP_EPS) / (pa - pmin), 1.0), 0.0);
  }
  *negcell = lead && active && (thd >= 0.0 || thp >= 0.0);  // neg_node (DG_solver.f90:602)
  if (scaled) *scaled = active && (thd >= 0.0 || thp >= 0.0);  // this lane's node values changed
  if (active && thp >= 0.0)
#pragma unroll
    for (int v = 0; v < 8; ++v) x[v] = avg[v] + thp * (x[v] - avg[v]);
  // re-check after the FP-inexact theta (DG_solver.f90:573-599): at most two extra shrinks; the
  // loop runs while any group of the warp still checks, so that the reductions see the whole warp
  bool pending = active && thp >= 0.0;
  double theta = thp;
  for (int it_count = 0; __any_sync(FULL_MASK, pending); ++it_count) {
    const double pm = grp_min<GS>(pending ? node_prs(x, gamma) : BIG);
    if (pending) {
      if (!(pm < 0.99 * PP_EPS)) {
        pending = false;
      } else if (it_count > 1) {
        if (lead) atomicOr(&ctrl->pp_relimit, 1);
        pending = false;
      } else {
        theta = 0.6 * theta;
#pragma unroll
        for (int v = 0; v < 8; ++v) x[v] = avg[v] + theta * (x[v] - avg[v]);
      }
    }
  }
  const int k = node % N, l = node / N;
  const double wq = (node < C::NN) ? 0.25 * g.hx * g.hy * dc.qw[k] * dc.qw[l] : 0.0;
  // entropy-offset limiter (DG_solver.f90:606-633)
  if (ent_offset) {
    const bool use = active && !cell_ent_nan[ce];
    const double nw = grp_sum<GS>(use ? wq * ent_of(x[0], fmax(node_prs(x, gamma), PP_EPS), gamma) : 0.0);
    if (use) {
      const double old = cell_ent_DG[ce], eavg = cell_ent_FV[ce];
      if (nw > old) {
        const double th = fmax(fmin((old - eavg) / (nw - eavg), 1.0), 0.0);
#pragma unroll
        for (int v = 0; v < 8; ++v) x[v] = avg[v] + th * (x[v] - avg[v]);
        if (scaled) *scaled = true;
      }
    }
  }
  // cell entropy (DG_solver.f90:635-649)
  if (comput_ent) return grp_sum<GS>(active ? wq * ent_of(x[0], fmax(node_prs(x, gamma), PP_EPS), gamma) : 0.0);
  return 0.0;
}

// ---------------------------------------------------------------------------------------------
// loop 1 for one chunk of TE consecutive element blocks of the ghosted grid (one contiguous run of
// memory).  s_A = the LDF operator in shared memory, in output-row pairs (load_ldf); s_red = CTA
// scratch of TE * 8 doubles for the chunk sums, which a caller either alternates between two such
// buffers from chunk to chunk or protects with a barrier after the call (one barrier per chunk
// here, between the writes of s_red and the reads).
//
// limit = 1 fuses loop 3 for a stage without OEDG and without the entropy sum: the interior
// elements are limited in registers before the one write-back.  The reference skips loop 3
// altogether when any element has an inadmissible average (neg_avg); here other CTAs may already
// have limited their elements by then.  That is only allowed where the stage result is discarded
// on neg_avg (the time-step pipeline re-tries the step from u_con), so the stand-alone
// post_process never fuses.
// ---------------------------------------------------------------------------------------------
// Stage-1 source of loop 1 (time-step pipeline only).  With u0 set, the stage state is formed
// here instead of being read from u: u0 + (coef*dt)*k1 on interior elements, rounded as
// combine_value rounds stage 1, and the ghost ring from those values by bc_source, as the boundary
// fill would leave it.  Every element is then written back, the inadmissible ones unchanged.
struct Stage1Src {
  const double* u0;  // state at the start of the step (ghosted layout)
  const double* k1;  // stage-1 residual (interior layout)
  const double* dt;
  double coef;       // 1 for SSP-RK(1,1), (2,2), (3,3); the first stage weight of SSP-RK(5,4)
};

template <int P>
__device__ __forceinline__ double stage1_node(const Stage1Src& s1, const Geo& g, int i, int j, bool inner, int v,
                                              int q, double dts) {
  constexpr int NN = (P + 1) * (P + 1), EB = 8 * NN;
  int si = i, sj = j, sq = q;
  bool neg = false;
  if (!inner) {
    const BcSrc b = bc_source<P>(g, i, j, v, q);
    if (b.fixed) return g.bc_state[v];
    si = b.si;
    sj = b.sj;
    sq = b.sq;
    neg = b.neg;
  }
  const long long gi = ((long long)sj * (g.nx + 2) + si) * EB + v * NN + sq;
  const long long ki = ((long long)(sj - 1) * g.nx + (si - 1)) * EB + v * NN + sq;
  const double x = __dadd_rn(s1.u0[gi], __dmul_rn(dts, s1.k1[ki]));
  return neg ? -x : x;
}

// Row and column of element e of the ghosted grid (rows of nxg elements) by one 32-bit division
// (the element count of any mesh that fits on the device is below 2^32; a 64-bit division by a
// run-time divisor is a long software sequence), and a position advanced along the rows.
struct GridRC {
  int j, i;
};
__device__ __forceinline__ GridRC grid_rc(long long e, int nxg) {
  const unsigned q = (unsigned)e / (unsigned)nxg;
  return GridRC{(int)q, (int)((unsigned)e - q * (unsigned)nxg)};
}
__device__ __forceinline__ GridRC grid_adv(GridRC p, int d, int nxg) {  // d >= 0 elements further
  p.i += d;
  while (p.i >= nxg) {
    p.i -= nxg;
    ++p.j;
  }
  return p;
}

// Queues this warp's elements of `chunk` into its shared buffers as one cp.async group (16-byte
// pieces; element blocks are multiples of 16 bytes): the blocks of u, or, with a stage-1 source,
// the blocks of u_con (bu) and k1 (bk) of the interior elements (ghost elements are formed from
// direct loads).  bu, bk: G * EB doubles each, 16-byte aligned.
template <int P>
__device__ __forceinline__ void pp_prefetch(const double* __restrict__ u, const Geo& g, long long chunk,
                                            GridRC cpos, const Stage1Src& s1, double* bu, double* bk) {
  using C = PPCfg<P>;
  constexpr int EB = C::EB, G = C::G, TE = C::TE, H2 = EB / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nx = g.nx, NXG = nx + 2;
  const long long total = (long long)NXG * (g.ny + 2);
  const long long ef = chunk * TE + warp * G;  // the warp's first element (cpos: the chunk's first)
  const GridRC fp = grid_adv(cpos, warp * G, NXG);
  const int jf = fp.j, if_ = fp.i;
#pragma unroll
  for (int it = lane; it < G * H2; it += 32) {
    const int k = it / H2, o = 2 * (it - k * H2);
    const long long e = ef + k;
    if (e >= total) continue;
    if (!s1.u0) {
      cp_async16(bu + k * EB + o, u + e * EB + o);
    } else {
      int i = if_ + k, j = jf;
      while (i >= NXG) {
        i -= NXG;
        ++j;
      }
      if (i >= 1 && i <= nx && j >= 1 && j <= g.ny) {
        cp_async16(bu + k * EB + o, s1.u0 + e * EB + o);
        cp_async16(bk + k * EB + o, s1.k1 + ((long long)(j - 1) * nx + (i - 1)) * EB + o);
      }
    }
  }
  cp_async_commit();
}

template <int P, bool NEEDG, bool PF>
__device__ __forceinline__ void pp_avg_ldf_chunk(double* __restrict__ u, double* __restrict__ u_avg, const Geo& g,
                                                 Ctrl* ctrl, long long chunk, GridRC cpos, int apply_ldf, int need_global,
                                                 int ent_offset, double* __restrict__ partial_out,  // 8 doubles
                                                 double* __restrict__ cell_ent_DG, double* __restrict__ cell_ent_FV,
                                                 unsigned char* __restrict__ cell_ent_nan, int limit,
                                                 const double* s_A, double* s_ldf, double* s_red, int* s_cnt,
                                                 const Stage1Src& s1,
                                                 double* bu, double* bk, long long next_chunk, GridRC npos) {
  using C = PPCfg<P>;
  constexpr int N = C::N, NN = C::NN, EB = C::EB, N2 = C::N2, GS = C::GS, G = C::G, TE = C::TE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const GrpLane<GS> gl = grp_lane<GS>();
  const int grp = gl.grp, node = gl.node;
  const int nx = g.nx, ny = g.ny, NXG = nx + 2;
  const long long total = (long long)NXG * (ny + 2);
  const long long e0 = chunk * TE;
  const int ne = (int)min((long long)TE, total - e0);
  const int el = warp * G + grp;  // element of this group within the chunk
  const long long e = e0 + el;
  const DegConst& dc = c_deg[P];
  const double gamma = g.gamma;
  bool valid = false, inner = false;
  int i = 0, j = 0;
  if (el < ne && !gl.idle) {
    const GridRC me = grid_adv(cpos, el, NXG);  // cpos: the chunk's first element
    j = me.j;
    i = me.i;
    const bool ii = (i >= 1 && i <= nx), jj = (j >= 1 && j <= ny);
    valid = ii || jj;  // DG_solver.f90:165 (corners are skipped)
    inner = ii && jj;
  }
  const bool nd = node < NN;
  const bool act = valid && nd;
  double x[8];
  if (PF) {  // this chunk's blocks are in the warp's buffers (pp_prefetch)
    const double* pu = bu + grp * EB + node;
    const double* pk = bk + grp * EB + node;
    if (s1.u0) {
      const double dts = __dmul_rn(s1.coef, *s1.dt);
      if (inner && nd) {  // the common case, one branch for all eight variables
#pragma unroll
        for (int v = 0; v < 8; ++v) x[v] = __dadd_rn(pu[v * NN], __dmul_rn(dts, pk[v * NN]));
      } else if (act) {  // a ghost element
#pragma unroll
        for (int v = 0; v < 8; ++v) x[v] = stage1_node<P>(s1, g, i, j, false, v, node, dts);
      } else {
#pragma unroll
        for (int v = 0; v < 8; ++v) x[v] = 0.0;
      }
    } else {
#pragma unroll
      for (int v = 0; v < 8; ++v) x[v] = act ? pu[v * NN] : 0.0;
    }
    __syncwarp();  // every lane has read the buffers: queue the next chunk into them
    if (next_chunk >= 0) pp_prefetch<P>(u, g, next_chunk, npos, s1, bu, bk);
  } else if (s1.u0) {
    const double dts = __dmul_rn(s1.coef, *s1.dt);
    if (inner && nd) {  // an interior node: u_con and k1 at this node (stage1_node's interior case)
      const double* pu = s1.u0 + e * EB + node;
      const double* pk = s1.k1 + ((long long)(j - 1) * nx + (i - 1)) * EB + node;
#pragma unroll
      for (int v = 0; v < 8; ++v) x[v] = __dadd_rn(pu[v * NN], __dmul_rn(dts, pk[v * NN]));
    } else if (act) {  // a ghost element
#pragma unroll
      for (int v = 0; v < 8; ++v) x[v] = stage1_node<P>(s1, g, i, j, false, v, node, dts);
    } else {
#pragma unroll
      for (int v = 0; v < 8; ++v) x[v] = 0.0;
    }
  } else {
#pragma unroll
    for (int v = 0; v < 8; ++v) x[v] = act ? u[e * EB + v * NN + node] : 0.0;
  }
  // cell averages (DG_solver.f90:177-184)
  const int k = node % N, l = node / N;
  const double w = nd ? 0.25 * dc.qw[k] * dc.qw[l] : 0.0;
  double avg[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) avg[v] = w * x[v];
  grp_sum8<GS>(avg, s_ldf + (warp * G + grp) * (N2 + 2));
  // admissibility of the average (DG_solver.f90:186-193): an inadmissible element is left unwritten
  if (valid) {
    const double prs = prs_of(avg[0], avg[1], avg[2], avg[3], avg[4], avg[5], avg[6], avg[7], gamma);
    if (avg[0] < PP_EPS || prs < PP_EPS) {
      if (node == 0) atomicOr(&ctrl->neg_avg, 1);
      valid = inner = false;
    }
  }
  // cell entropies for the entropy-offset limiter (DG_solver.f90:195-224)
  if (ent_offset) {
    const double pq = act ? node_prs(x, gamma) : 0.0;
    const bool okq = !act || (x[0] >= PP_EPS && pq >= PP_EPS);
    const double okall = grp_min<GS>(okq ? 1.0 : 0.0);
    const double ce = grp_sum<GS>((act && okall > 0.5) ? 0.25 * g.hx * g.hy * dc.qw[k] * dc.qw[l] * ent_of(x[0], pq, gamma) : 0.0);
    if (valid && node == 0) {
      const double prs = prs_of(avg[0], avg[1], avg[2], avg[3], avg[4], avg[5], avg[6], avg[7], gamma);
      cell_ent_FV[e] = ent_of(avg[0], prs, gamma);
      cell_ent_DG[e] = okall > 0.5 ? ce : 0.0;
      cell_ent_nan[e] = okall > 0.5 ? 0 : 1;
    }
  }
  // LDF projection of (Bx - avg, By - avg) with the dense nodal operator: this lane forms the
  // outputs at its node (rows `node` and NN + node); the inputs come from the group's lanes
  if (apply_ldf) {  // the group's (Bx, By) - avg pass through a padded per-group shared row
    double* sb = s_ldf + (warp * G + grp) * (N2 + 2);
    if (nd) {
      sb[node] = x[4] - avg[4];
      sb[NN + node] = x[5] - avg[5];
    }
    __syncwarp();
    double ox = 0.0, oy = 0.0;
    if (nd) {
      // s_A holds (row node, row NN + node) of column m as one pair at m * NN + node (load_ldf),
      // and the input row is read two entries at a time; the sums run over m in order
      const double2* a2 = reinterpret_cast<const double2*>(s_A) + node;
      const double2* b2 = reinterpret_cast<const double2*>(sb);
#pragma unroll
      for (int m = 0; m < N2; m += 2) {
        const double2 b = b2[m >> 1];
        const double2 a0 = a2[m * NN], a1 = a2[(m + 1) * NN];
        ox += a0.x * b.x;
        oy += a0.y * b.x;
        ox += a1.x * b.y;
        oy += a1.y * b.y;
      }
    }
    __syncwarp();  // the row is rewritten by the next chunk
    if (valid) {
      x[4] = ox + avg[4];
      x[5] = oy + avg[5];
    }
  }
  if (NEEDG && need_global) {
    // chunk sum of (hx*hy)*avg over interior elements in element order (DG_solver.f90:227-229)
    if (el < TE)
#pragma unroll
      for (int v0 = 0; v0 < 8; v0 += GS)
        if (node + v0 < 8) s_red[el * 8 + node + v0] = inner ? (g.hx * g.hy) * pick8(avg, node + v0) : 0.0;
  }
  bool neg = false, scaled = false;
  if (limit) {
    __syncwarp();  // the group's lane 0 wrote the cell entropies limit_group reads
    limit_group<P>(x, avg, inner && nd, inner && node == 0, node, e, g, ctrl, ent_offset, 0, cell_ent_DG, cell_ent_FV,
                   cell_ent_nan, &neg, &scaled);
    const unsigned cnt = __popc(__ballot_sync(FULL_MASK, neg));
    if (lane == 0 && cnt) atomicAdd(s_cnt, (int)cnt);
  }
  // write back the state of every element formed here, and of an admissible element what changed
  // in place: (Bx, By) after the LDF, all eight variables where the limiter scaled the element
  // (the positivity and entropy-offset scalings are conditional, so most elements keep six of
  // their eight variables bit for bit and need not store them)
  if (act) {
    if (s1.u0 || scaled) {
#pragma unroll
      for (int v = 0; v < 8; ++v) u[e * EB + v * NN + node] = x[v];
    } else if (valid && apply_ldf) {
      u[e * EB + 4 * NN + node] = x[4];
      u[e * EB + 5 * NN + node] = x[5];
    }
  }
  if (valid)
#pragma unroll
    for (int v0 = 0; v0 < 8; v0 += GS)
      if (node + v0 < 8) u_avg[e * 8 + node + v0] = pick8(avg, node + v0);
  if (NEEDG && need_global) {
    __syncthreads();
    if (tid < 8) {
      double sacc = 0.0;
      for (int q = 0; q < ne; ++q) sacc = sacc + s_red[q * 8 + tid];
      partial_out[tid] = sacc;
    }
  }
}


template <int P>
__device__ __forceinline__ void load_ldf(const double* __restrict__ A, double* s_A) {
  constexpr int N2 = PPCfg<P>::N2;
  constexpr int NN = PPCfg<P>::NN;
  // pair (A[node][m], A[NN + node][m]) at m * NN + node; A is stored column-major (row + N2 * m)
  for (int it = threadIdx.x; it < N2 * NN; it += PPCfg<P>::NT) {
    const int m = it / NN, node = it - m * NN;
    s_A[2 * it] = __ldg(A + node + N2 * m);
    s_A[2 * it + 1] = __ldg(A + NN + node + N2 * m);
  }
}

// one CTA walks chunks blockIdx.x, blockIdx.x + gridDim.x, ... (the LDF operator is loaded once).
// NEEDG: the OEDG form (need_global), with the per-chunk partial sums of the averages.
template <int P, bool NEEDG>
__global__ void __launch_bounds__(PPCfg<P>::NT, PPCfg<P>::MINB)
    pp_avg_ldf_kernel(double* __restrict__ u, double* __restrict__ u_avg, Geo g, Ctrl* ctrl,
                      int gate, int apply_ldf, int need_global, int ent_offset,
                      double* __restrict__ partial_sum,  // [chunks][8]
                      double* __restrict__ cell_ent_DG, double* __restrict__ cell_ent_FV,
                      unsigned char* __restrict__ cell_ent_nan, int limit, int nchunks, Stage1Src s1) {
  using C = PPCfg<P>;
  __shared__ __align__(16) double s_A[C::N2 * C::N2];
  __shared__ __align__(16) double s_ldf[C::TE * (C::N2 + 2)];
  __shared__ double s_red[2 * C::TE * 8];  // chunk sums, two buffers used in turn
  __shared__ __align__(16) double s_pf[(C::NT / 32) * 2 * C::G * C::EB];  // per warp: u (or u_con), k1
  __shared__ int s_cnt;
  if (!gate_open(ctrl, gate)) return;
  if (threadIdx.x == 0) s_cnt = 0;
  if (apply_ldf) load_ldf<P>(g.ldfA, s_A);
  __syncthreads();
  // the copies of a warp's next chunk are in flight while it works on this one
  double* bu = s_pf + (threadIdx.x >> 5) * 2 * C::G * C::EB;
  double* bk = bu + C::G * C::EB;
  // grid positions of the chunks' first elements, advanced by the CTA's stride (no division in
  // the loop)
  const int NXG = g.nx + 2;
  const GridRC stride = grid_rc((long long)gridDim.x * C::TE, NXG);
  GridRC pos = grid_rc((long long)blockIdx.x * C::TE, NXG);
  if (blockIdx.x < nchunks) pp_prefetch<P>(u, g, blockIdx.x, pos, s1, bu, bk);
  // the chunk sums of consecutive chunks go to alternate halves of s_red: the barrier of chunk
  // k + 1 orders the reads of chunk k before the writes of chunk k + 2
  int half = 0;
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x, half ^= 1) {
    cp_async_wait_all();
    __syncwarp();
    const long long nxt = c + gridDim.x < nchunks ? (long long)c + gridDim.x : -1;
    GridRC npos{pos.j + stride.j, pos.i + stride.i};
    if (npos.i >= NXG) {
      npos.i -= NXG;
      ++npos.j;
    }
    pp_avg_ldf_chunk<P, NEEDG, true>(u, u_avg, g, ctrl, c, pos, apply_ldf, need_global, ent_offset,
                                     partial_sum + (long long)c * 8, cell_ent_DG, cell_ent_FV, cell_ent_nan, limit,
                                     s_A, s_ldf, s_red + half * C::TE * 8, &s_cnt, s1, bu, bk, nxt, npos);
    pos = npos;
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_cnt) atomicAdd(&ctrl->num_negcell, s_cnt);
}

// many instances: items = every member's chunks; slot = the stage state; `final` selects the
// final-stage form (OEDG global reductions for instances that use OEDG); the other stages fuse
// loop 3 (limit)
template <int P, bool FINAL>
__global__ void __launch_bounds__(PPCfg<P>::NT, PPCfg<P>::MINB > 3 ? 3 : PPCfg<P>::MINB)
    pp_avg_ldf_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                       const int* __restrict__ nwork, const int* __restrict__ ninst, int slot, int gate,
                       int stage1) {
  using C = PPCfg<P>;
  __shared__ __align__(16) double s_A[C::N2 * C::N2];
  __shared__ __align__(16) double s_ldf[C::TE * (C::N2 + 2)];
  __shared__ double s_red[C::TE * 8];  // chunk sums (the loop's barriers protect it)
  __shared__ int s_cnt;
  __shared__ SharedWalk s_walk;  // the walker's state, out of the registers the chunk needs
  if (threadIdx.x == 0) s_walk.start(pref, *ninst, *nwork);
  __syncthreads();
  int loaded = -1;  // member whose LDF operator s_A holds
  while (s_walk.w < s_walk.last) {
    const int m = s_walk.m, chunk = s_walk.w - s_walk.mstart;
    const InstDesc& d = insts[m];
    const bool open = gate_open(d.ctrl, gate);
    if (open) {
      if (d.use_ldf && loaded != m) {  // (the previous item ended with a barrier)
        load_ldf<P>(d.g.ldfA, s_A);
        loaded = m;
      }
      if (threadIdx.x == 0) s_cnt = 0;
    }
    __syncthreads();  // every thread has read the walker; s_A and s_cnt are in place
    if (threadIdx.x == 0) s_walk.advance(pref);
    if (open) {
      const Stage1Src s1 = stage1 ? Stage1Src{d.u[0], d.ut[1], &d.ctrl->dt, stage1_coef(d.R)} : Stage1Src{};
      pp_avg_ldf_chunk<P, FINAL, false>(d.u[slot], d.u_avg, d.g, d.ctrl, chunk,
                                        grid_rc((long long)chunk * C::TE, d.g.nx + 2), d.use_ldf, FINAL && d.use_oedg,
                                        d.ent_offset, d.partial + (long long)chunk * 8, d.cell_ent_DG, d.cell_ent_FV,
                                        d.cell_ent_nan, !FINAL, s_A, s_ldf, s_red, &s_cnt, s1,
                                        nullptr, nullptr, -1, GridRC{0, 0});
    }
    __syncthreads();  // the item is done; the walker has advanced
    if (open && threadIdx.x == 0 && s_cnt) atomicAdd(&d.ctrl->num_negcell, s_cnt);
  }
}

// ---------------------------------------------------------------------------------------------
// global average (fixed-order sum of block partials).  One CTA.
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
  if (tid < 8) ctrl->u_avg_global[tid] = s[tid][0];
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
// One face, either direction.  Rp, Lm = the variable's nodes of the element after and before the
// face (its first trace, R0, and last trace, RN, along the normal); node (a along the normal, b
// along the face) sits at a*sn + b*st (x face: sn = 1, st = N; y face: sn = N, st = 1).  sn_h,
// st_h = 2/h along the normal and along the face; coef[n][t] = (2(n+t)+1) h^(n+t) / (2 max(2p-1,1)
// n! t!) with h the element size along the normal.  The x face of the reference (DG_solver.f90:
// 296-343) is this with (R, L, hx, hy); its y face (:360-407) with (T, B, hy, hx): the two loops
// are the same arithmetic with the roles of the directions exchanged.
template <int P>
__device__ __forceinline__ double sigsum_face(const double* Rp, const double* Lm, int sn, int st, double sn_h,
                                              double st_h, const double* coef) {
  constexpr int N = P + 1;
  const DegConst& dc = c_deg[P];
  // J[kk][b] = the jump of the kk-th normal derivative at face node b, formed column by column
  // (each column of the two variable blocks is read from shared memory once)
  double sk[N], J[N][N];
  double snk = 1.0;
#pragma unroll
  for (int kk = 0; kk <= P; ++kk) {
    sk[kk] = snk;
    snk *= sn_h;
  }
#pragma unroll
  for (int b = 0; b < N; ++b) {
    double cr[N], cl[N];
#pragma unroll
    for (int a = 0; a < N; ++a) {
      cr[a] = Rp[a * sn + b * st];
      cl[a] = Lm[a * sn + b * st];
    }
    // order 0: the rows of D^0 = I pick the end nodes (the sums below give exactly these values)
    J[0][b] = cr[0] - cl[N - 1];
#pragma unroll
    for (int kk = 1; kk <= P; ++kk) {
      double tr = 0.0, tl = 0.0;
#pragma unroll
      for (int a = 0; a < N; ++a) {
        tr += dc.R0[kk][a] * cr[a];
        tl += dc.RN[kk][a] * cl[a];
      }
      J[kk][b] = sk[kk] * tr - sk[kk] * tl;
    }
  }
  double total = 0.0;
#pragma unroll
  for (int kk = 0; kk <= P; ++kk) {
    double jump[N];
#pragma unroll
    for (int b = 0; b < N; ++b) jump[b] = J[kk][b];
#pragma unroll
    for (int ll = 0; ll <= P; ++ll) {
      if (ll > P - kk) break;
      double L1 = 0.0;
#pragma unroll
      for (int b = 0; b < N; ++b) L1 += (0.5 * dc.qw[b]) * fabs(jump[b]);
      total = total + coef[kk * N + ll] * L1;
      if (ll < P - kk) {  // tangential derivative for the next order
        double nj[N];
#pragma unroll
        for (int a = 0; a < N; ++a) {
          double acc = 0.0;
#pragma unroll
          for (int b = 0; b < N; ++b) acc += (st_h * dc.D[a + N * b]) * jump[b];
          nj[a] = acc;
        }
#pragma unroll
        for (int a = 0; a < N; ++a) jump[a] = nj[a];
      }
    }
  }
  return total;
}

// The part of sigsum_face from the normal-derivative orders KA and KB only (in that order): the two
// halves {0, P} and {1, P-1} of a face at P = 3, each computed by its own warp (fewer registers,
// half the dependent chain); the face's value is the sum of the two halves.
template <int P, int KA, int KB>
__device__ __forceinline__ double sigsum_face_pair(const double* Rp, const double* Lm, int sn, int st, double sn_h,
                                                   double st_h, const double* coef) {
  constexpr int N = P + 1;
  const DegConst& dc = c_deg[P];
  constexpr int KS[2] = {KA, KB};
  double sk[2], J[2][N];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    double snk = 1.0;
#pragma unroll
    for (int i = 0; i < KS[h]; ++i) snk *= sn_h;  // sn_h^kk, the running product of sigsum_face
    sk[h] = snk;
  }
#pragma unroll
  for (int b = 0; b < N; ++b) {
    double cr[N], cl[N];
#pragma unroll
    for (int a = 0; a < N; ++a) {
      cr[a] = Rp[a * sn + b * st];
      cl[a] = Lm[a * sn + b * st];
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int kk = KS[h];
      if (kk == 0) {
        J[h][b] = cr[0] - cl[N - 1];
      } else {
        double tr = 0.0, tl = 0.0;
#pragma unroll
        for (int a = 0; a < N; ++a) {
          tr += dc.R0[kk][a] * cr[a];
          tl += dc.RN[kk][a] * cl[a];
        }
        J[h][b] = sk[h] * tr - sk[h] * tl;
      }
    }
  }
  double total = 0.0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int kk = KS[h];
    double jump[N];
#pragma unroll
    for (int b = 0; b < N; ++b) jump[b] = J[h][b];
#pragma unroll
    for (int ll = 0; ll <= P; ++ll) {
      if (ll > P - kk) break;
      double L1 = 0.0;
#pragma unroll
      for (int b = 0; b < N; ++b) L1 += (0.5 * dc.qw[b]) * fabs(jump[b]);
      total = total + coef[kk * N + ll] * L1;
      if (ll < P - kk) {  // tangential derivative for the next order (D from the constant bank,
        double nj[N];     // the scale applied after the sum: no scaled copy of D held in registers)
#pragma unroll
        for (int a = 0; a < N; ++a) {
          double acc = 0.0;
#pragma unroll
          for (int b = 0; b < N; ++b) acc += dc.D[a + N * b] * jump[b];
          nj[a] = st_h * acc;
        }
#pragma unroll
        for (int a = 0; a < N; ++a) jump[a] = nj[a];
      }
    }
  }
  return total;
}

// coef[n][t] of sigsum_face for element size h (the reference's running products h^(n+t), n! t!)
template <int P>
__device__ __forceinline__ double sigsum_coef(int n, int t, double h) {
  const int denom_base = 2 * max(2 * P - 1, 1);
  double hp = 1.0;
  int fn = 1, ft = 1;
  for (int i = 0; i < n; ++i) {
    hp *= h;
    fn *= (i + 1);
  }
  for (int i = 0; i < t; ++i) {
    hp *= h;
    ft *= (i + 1);
  }
  return ((2 * (n + t) + 1) * hp) / (double)(denom_base * fn * ft);
}

template <int P>
struct SigCfg {
  static constexpr int TX = PPTune<P>::sig.TX, TY = PPTune<P>::sig.TY, MINB = PPTune<P>::sig.MINB;
};

template <int P>
struct SigLayout {
  static constexpr int N = P + 1, NN = N * N, EB = 8 * NN;
  static constexpr int TX = SigCfg<P>::TX, TY = SigCfg<P>::TY;
  static constexpr int VS = NN + 1, ES = 8 * VS;   // padded variable / element record
  static constexpr int RW = TX + 2, RH = TY + 2;   // staged rectangle (max)
  static constexpr int DOUBLES = RW * RH * ES;
  static constexpr int NQ = 8 * ((TX + 1) * TY + TX * (TY + 1));  // face-variable items of a tile, at most
};


// The tile's own elements also give the max and min of every variable over their nodes, merged
// into ctrl->umax_bits / umin_bits (order-preserving encodings; max and min are exact, so neither
// the order of the merge nor the tiling changes the result).  The atomic is skipped when the value
// already there is not exceeded, so that most tiles issue none.
// Where the indicator tile's results go.  Taken by reference, so that the batched kernel can keep
// it in shared memory instead of in registers for the whole tile.
struct SigOut {
  double* sig_x;
  double* sig_y;
  Ctrl* ctrl;
};

template <int P>
__device__ __forceinline__ void pp_sigsum_tile(const double* __restrict__ u, const Geo& g, const SigOut& so,
                                               int tile_x, int tile_y) {
  using L = SigLayout<P>;
  constexpr int NN = L::NN, EB = L::EB, VS = L::VS, ES = L::ES, TX = L::TX, TY = L::TY, RW = L::RW;
  constexpr int NT = 256;
  __shared__ double s_e[L::DOUBLES];  // face math reads its two variable blocks from here
  __shared__ double s_coef[2 * (P + 1) * (P + 1)];  // x faces (h = hx), then y faces (h = hy)
  __shared__ double s_mm[2][NT / 32][8];              // per warp: max, min of each variable
  __shared__ double s_part[P == 3 ? 2 * L::NQ : 1];   // P = 3: the two halves of every item
  const int tid = threadIdx.x;
  const int nx = g.nx, ny = g.ny;
  const int i0 = 1 + tile_x * TX, j0 = 1 + tile_y * TY;
  const int W = min(TX, nx - i0 + 1), H = min(TY, ny - j0 + 1);
  const int right = (i0 + W - 1 == nx), top = (j0 + H - 1 == ny);
  const int cw = W + 1 + right, rh = H + 1 + top;  // staged columns i0-1 .., rows j0-1 ..
  // stage: rect row rr = grid row j0-1+rr (a contiguous run of cw elements in u), rect column
  // cc = grid column i0-1+cc.  The copies go straight to shared memory; the divisions are by
  // compile-time constants.
  {
    const int run = cw * EB;
    const long long row = (long long)(nx + 2) * EB;
    const double* src = u + ((long long)(j0 - 1) * (nx + 2) + (i0 - 1)) * EB;
    for (int rr = 0; rr < rh; ++rr, src += row) {
      double* dst = s_e + rr * RW * ES;
      for (int rem = tid; rem < run; rem += NT) {
        const int cc = rem / EB, w = rem - cc * EB, v = w / NN, q = w - v * NN;
        cp_async8(dst + cc * ES + v * VS + q, src + rem);
      }
    }
    cp_async_commit();
  }
  if (tid < 2 * (P + 1) * (P + 1)) {
    const int d = tid / ((P + 1) * (P + 1)), r = tid - d * (P + 1) * (P + 1), n = r / (P + 1), t = r - n * (P + 1);
    s_coef[tid] = (n + t <= P) ? sigsum_coef<P>(n, t, d == 0 ? g.hx : g.hy) : 0.0;
  }
  cp_async_wait_all();
  __syncthreads();
  {  // extrema of the own elements: thread tid takes variable tid & 7 of elements tid/8, tid/8 + NT/8, ...
    const int v = tid & 7;
    double mx = -1.0e308, mn = 1.0e308;
    for (int e = tid >> 3; e < W * H; e += NT / 8) {
      const int r = e / W, c = e - r * W;
      const double* src = s_e + ((r + 1) * RW + c + 1) * ES + v * VS;
#pragma unroll
      for (int q = 0; q < NN; ++q) {
        mx = fmax(mx, src[q]);
        mn = fmin(mn, src[q]);
      }
    }
#pragma unroll
    for (int o = 8; o < 32; o <<= 1) {
      mx = fmax(mx, __shfl_xor_sync(FULL_MASK, mx, o));
      mn = fmin(mn, __shfl_xor_sync(FULL_MASK, mn, o));
    }
    if ((tid & 31) < 8) {
      s_mm[0][tid >> 5][v] = mx;
      s_mm[1][tid >> 5][v] = mn;
    }
  }
  const double sxh = 2.0 / g.hx, syh = 2.0 / g.hy;
  const int wr = W + right, ht = H + top;  // TX and TY on interior tiles
  const int nfx = H * wr, nfy = W * ht;
  // face-variable item q: the variable's block of the element before the face, and the output
  auto item = [&](int q, bool& xf, const double*& lo, double*& dst) {
    const int v = q & 7, f = q >> 3;
    xf = f < nfx;
    if (xf) {  // x face: row r, face c between columns c-1 and c of the tile
      const int r = (wr == TX) ? f / TX : f / wr, c = f - r * wr;
      lo = s_e + ((r + 1) * RW + c) * ES + v * VS;
      dst = so.sig_x + (((long long)(j0 + r - 1) * (nx + 1)) + (i0 + c - 1)) * 8 + v;
    } else {  // y face: column c, face r between rows r-1 and r of the tile
      const int f2 = f - nfx;
      const int c = (ht == TY) ? f2 / TY : f2 / ht, r = f2 - c * ht;
      lo = s_e + (r * RW + c + 1) * ES + v * VS;
      dst = so.sig_y + (((long long)(j0 + r - 1) * nx) + (i0 + c - 1)) * 8 + v;
    }
  };
  const int nq = 8 * (nfx + nfy);
  if constexpr (P == 3) {
    // two warps per 32 items: the even warps take the orders {0, 3}, the odd ones {1, 2}
    // (sigsum_face_pair; the warp's half is uniform, so neither diverges); the halves meet in
    // shared memory and are added in that order
    static_assert(((NT / 32) & 1) == 0, "warps pair up");
    for (int it = tid; it < 2 * ((nq + 31) & ~31); it += NT) {
      const int half = (it >> 5) & 1, q = ((it >> 6) << 5) + (it & 31);
      if (q < nq) {
        bool xf;
        const double* lo;
        double* dst;
        item(q, xf, lo, dst);
        const double* rp = lo + (xf ? ES : RW * ES);
        const int sn = xf ? 1 : P + 1, st = xf ? P + 1 : 1;
        const double snh = xf ? sxh : syh, sth = xf ? syh : sxh;
        const double* cf = s_coef + (xf ? 0 : (P + 1) * (P + 1));
        s_part[half * L::NQ + q] = half == 0 ? sigsum_face_pair<P, 0, 3>(rp, lo, sn, st, snh, sth, cf)
                                             : sigsum_face_pair<P, 1, 2>(rp, lo, sn, st, snh, sth, cf);
      }
    }
    __syncthreads();
    for (int q = tid; q < nq; q += NT) {
      bool xf;
      const double* lo;
      double* dst;
      item(q, xf, lo, dst);
      *dst = s_part[q] + s_part[L::NQ + q];
    }
  } else {
    for (int q = tid; q < nq; q += NT) {
      bool xf;
      const double* lo;
      double* dst;
      item(q, xf, lo, dst);
      // one call site for both directions (the strides and scales select the direction)
      *dst = sigsum_face<P>(lo + (xf ? ES : RW * ES), lo, xf ? 1 : P + 1, xf ? P + 1 : 1, xf ? sxh : syh,
                            xf ? syh : sxh, s_coef + (xf ? 0 : (P + 1) * (P + 1)));
    }
  }
  __syncthreads();
  if (tid < 16) {  // threads 0-7: max of variable tid; 8-15: min of variable tid - 8
    const int v = tid & 7, lo = tid >> 3;
    double m = s_mm[lo][0][v];
    for (int w = 1; w < NT / 32; ++w) m = lo ? fmin(m, s_mm[1][w][v]) : fmax(m, s_mm[0][w][v]);
    unsigned long long* dst = lo ? &so.ctrl->umin_bits[v] : &so.ctrl->umax_bits[v];
    const unsigned long long enc = ord_enc(m), cur = *reinterpret_cast<volatile unsigned long long*>(dst);
    if (lo ? (m < 1.0e308 && enc < cur) : (m > -1.0e308 && enc > cur)) {
      if (lo) atomicMin(dst, enc);
      else atomicMax(dst, enc);
    }
  }
}

template <int P>
__global__ void __launch_bounds__(256, SigCfg<P>::MINB)
    pp_sigsum_kernel(const double* __restrict__ u, Geo g, Ctrl* ctrl, int gate,
                     double* __restrict__ sig_x, double* __restrict__ sig_y) {
  if (!gate_open(ctrl, gate)) return;
  pp_sigsum_tile<P>(u, g, SigOut{sig_x, sig_y, ctrl}, blockIdx.x, blockIdx.y);
}

// many instances: items = every member's tiles (row-major)
template <int P>
__global__ void __launch_bounds__(256, SigCfg<P>::MINB)
    pp_sigsum_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                      const int* __restrict__ nwork, const int* __restrict__ ninst, int slot, int final, int gate) {
  __shared__ Geo s_g;  // the member's geometry and outputs, per tile (see SigOut)
  __shared__ SigOut s_so;
  __shared__ SharedWalk s_walk;
  if (threadIdx.x == 0) s_walk.start(pref, *ninst, *nwork);
  __syncthreads();
  while (s_walk.w < s_walk.last) {
    const int m = s_walk.m, local = s_walk.w - s_walk.mstart;
    const InstDesc& d = insts[m];
    const bool open = gate_open(d.ctrl, gate) && d.use_oedg && final;
    if (open && threadIdx.x == 0) {
      s_g = d.g;
      s_so = SigOut{d.sig_x, d.sig_y, d.ctrl};
    }
    __syncthreads();  // every thread has read the walker; the item's arguments are in place
    if (threadIdx.x == 0) s_walk.advance(pref);
    if (open) {
      const int ntx = (d.g.nx + SigCfg<P>::TX - 1) / SigCfg<P>::TX;
      pp_sigsum_tile<P>(d.u[slot], s_g, s_so, local % ntx, local / ntx);
    }
    __syncthreads();  // the item is done (the next one reuses shared memory); the walker has advanced
  }
}

// ---------------------------------------------------------------------------------------------
// loop 3: OEDG damping, positivity, entropy offset, entropy.  A CTA owns TE consecutive
// interior elements of one row j (a contiguous run of memory).
// ---------------------------------------------------------------------------------------------
// The arrays and switches of one limiter segment.  Taken by reference, so that the batched kernel
// can keep them in shared memory (read where used) instead of in registers for the whole segment.
struct LimitIO {
  double* u;                  // the stage state (interior updated in place unless accept_only)
  const double* u_avg;        // cell averages (loop 1)
  Ctrl* ctrl;
  const double* sig_x;        // OEDG face indicators (x faces, y faces)
  const double* sig_y;
  const double* cell_ent_DG;  // entropy-offset inputs of loop 1
  const double* cell_ent_FV;
  const unsigned char* cell_ent_nan;
  double* ent_out;            // the segment's entropy partial (comput_ent)
  double* accept_dst;         // the accepted state (u_con) or nullptr
  double oedg_dt;
  int apply_oedg, ent_offset, comput_ent, accept_only;
};

template <int P>
__device__ __forceinline__ void pp_limit_segment(const LimitIO& io, const Geo& g, int seg, int jrow, double* s_ent,
                                                 int* s_cnt) {
  using C = PPCfg<P>;
  constexpr int NN = C::NN, EB = C::EB, GS = C::GSL, G = C::GL, TE = C::TEL;  // the limiter's groups
  if (io.ctrl->neg_avg) return;  // the reference skips loop 3 once neg_avg is set (DG_solver.f90:431)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const GrpLane<GS> gl = grp_lane<GS>();
  const int grp = gl.grp, node = gl.node;
  const int nx = g.nx, NXG = nx + 2;
  const int j = 1 + jrow;
  const int i0 = 1 + seg * TE;
  const int ne = min(TE, nx - i0 + 1);
  const int el = warp * G + grp;
  const bool inside = el < ne && !gl.idle, nd = node < NN;
  const bool act = inside && nd;
  const long long e = (long long)j * NXG + i0 + el;
  const double gamma = g.gamma;
  double x[8], avg[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    x[v] = act ? io.u[e * EB + v * NN + node] : 0.0;
    avg[v] = inside ? io.u_avg[e * 8 + v] : 1.0;
  }
  if (io.apply_oedg) {  // DG_solver.f90:448-524
    double sx = 0.0, sy = 0.0;
    if (act) {
      const double rho = fmax(x[0], PP_EPS);
      const double ir = 1.0 / rho;
      const double vx = ir * x[1], vy = ir * x[2];
      const double ek = 0.5 * ir * (x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
      const double bx = x[4], by = x[5], bz = x[6];
      const double bsq = bx * bx + by * by + bz * bz;
      const double pf = fmax((gamma - 1.0) * (x[7] - (ek + 0.5 * bsq)), PP_EPS);
      const double cs = gamma * pf * ir, ss = cs + bsq * ir, sqsq = ss * ss, coef = 4.0 * cs * ir;
      sx = fabs(vx) + sqrt(0.5 * fmax(ss + sqrt(fmax(sqsq - coef * (bx * bx), 0.0)), 0.0));
      sy = fabs(vy) + sqrt(0.5 * fmax(ss + sqrt(fmax(sqsq - coef * (by * by), 0.0)), 0.0));
    }
    const double mx = grp_max<GS>(sx), my = grp_max<GS>(sy);
    // lane `node` of the group forms delta_v for v = node, node + GS, ... from the element's four faces
    double d = -1.0e308;
    if (inside) {
      const int i = i0 + el;
      const long long fxl = ((long long)(j - 1) * (nx + 1) + (i - 1)) * 8;
      const long long fyb = ((long long)(j - 1) * nx + (i - 1)) * 8;
      const long long fyt = ((long long)j * nx + (i - 1)) * 8;
      const Ctrl* ctrl = io.ctrl;
      const double* sig_x = io.sig_x;
      const double* sig_y = io.sig_y;
      for (int v = node; v < 8; v += GS) {
        const double gs = ctrl->u_avg_global[v];
        const double uv = fmax(0.0, fmax(ord_dec(ctrl->umax_bits[v]) - gs, gs - ord_dec(ctrl->umin_bits[v])));
        double dv = 0.0;
        if (uv > OEDG_EPS)
          dv = ((mx / g.hx) * (sig_x[fxl + v] + sig_x[fxl + 8 + v]) + (my / g.hy) * (sig_y[fyb + v] + sig_y[fyt + v])) / uv;
        d = fmax(d, dv);
      }
    }
    const double dmax = grp_max<GS>(d);
    const double theta = exp(-io.oedg_dt * dmax);
    if (act)
#pragma unroll
      for (int v = 0; v < 8; ++v) x[v] = avg[v] + theta * (x[v] - avg[v]);
  }
  bool neg = false;
  const double ce = limit_group<P, GS>(x, avg, act, inside && node == 0, node, e, g, io.ctrl, io.ent_offset,
                                       io.comput_ent, io.cell_ent_DG, io.cell_ent_FV, io.cell_ent_nan, &neg);
  const unsigned cnt = __popc(__ballot_sync(FULL_MASK, neg));
  if (lane == 0 && cnt) atomicAdd(s_cnt, (int)cnt);
  if (act)
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      if (!io.accept_only) io.u[e * EB + v * NN + node] = x[v];
      if (io.accept_dst) io.accept_dst[e * EB + v * NN + node] = x[v];
    }
  if (io.comput_ent) {  // chunk partial in element order
    if (inside && node == 0) s_ent[el] = ce;
    __syncthreads();
    if (tid == 0) {
      double tot = 0.0;
      for (int q = 0; q < ne; ++q) tot = tot + s_ent[q];
      *io.ent_out = tot;
    }
  }
}

template <int P>
__global__ void __launch_bounds__(PPCfg<P>::NT, PPCfg<P>::MINB)
    pp_limit_kernel(double* __restrict__ u, const double* __restrict__ u_avg, Geo g, Ctrl* ctrl,
                    int gate, int apply_oedg, const double* __restrict__ dt_ptr, double oedg_dt_arg,
                    int ent_offset, int comput_ent, const double* __restrict__ sig_x,
                    const double* __restrict__ sig_y, const double* __restrict__ cell_ent_DG,
                    const double* __restrict__ cell_ent_FV, const unsigned char* __restrict__ cell_ent_nan,
                    double* __restrict__ ent_partial, double* __restrict__ accept_dst, int accept_only) {
  __shared__ double s_ent[PPCfg<P>::TEL];
  __shared__ int s_cnt;
  if (!gate_open(ctrl, gate)) return;
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  const LimitIO io{u, u_avg, ctrl, sig_x, sig_y, cell_ent_DG, cell_ent_FV, cell_ent_nan,
                   ent_partial + (long long)blockIdx.y * gridDim.x + blockIdx.x, accept_dst,
                   dt_ptr ? *dt_ptr : oedg_dt_arg, apply_oedg, ent_offset, comput_ent, accept_only};
  pp_limit_segment<P>(io, g, blockIdx.x, blockIdx.y, s_ent, &s_cnt);
  __syncthreads();
  if (threadIdx.x == 0 && s_cnt) atomicAdd(&ctrl->num_negcell, s_cnt);
}

// many instances: items = every member's row segments (row-major); the final stage applies OEDG
// (if the instance uses it), computes the entropy and writes the accepted interior into slot 0
// only, as the single-instance pipeline does
template <int P>
__global__ void __launch_bounds__(PPCfg<P>::NT, PPCfg<P>::MINB > 3 ? 3 : PPCfg<P>::MINB)
    pp_limit_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                     const int* __restrict__ nwork, const int* __restrict__ ninst, int slot, int final, int gate) {
  __shared__ double s_ent[PPCfg<P>::TEL];
  __shared__ int s_cnt;
  __shared__ Geo s_g;      // the member's geometry and arrays, per item (see LimitIO)
  __shared__ LimitIO s_io;
  __shared__ SharedWalk s_walk;
  if (threadIdx.x == 0) s_walk.start(pref, *ninst, *nwork);
  __syncthreads();
  while (s_walk.w < s_walk.last) {
    const int m = s_walk.m, local = s_walk.w - s_walk.mstart;
    const InstDesc& d = insts[m];
    const bool open = gate_open(d.ctrl, gate);
    if (open && threadIdx.x == 0) {
      s_cnt = 0;
      s_g = d.g;
      s_io = LimitIO{d.u[slot], d.u_avg, d.ctrl, d.sig_x, d.sig_y, d.cell_ent_DG, d.cell_ent_FV, d.cell_ent_nan,
                     d.ent_partial + local, final ? d.u[0] : nullptr, d.ctrl->dt, d.use_oedg && final,
                     d.ent_offset, final, final};
    }
    __syncthreads();  // every thread has read the walker; the item's arguments are in place
    if (threadIdx.x == 0) s_walk.advance(pref);
    if (open) {
      const int nseg = (d.g.nx + PPCfg<P>::TEL - 1) / PPCfg<P>::TEL;
      pp_limit_segment<P>(s_io, s_g, local % nseg, local / nseg, s_ent, &s_cnt);
    }
    __syncthreads();  // the item is done; the walker has advanced
    if (open && threadIdx.x == 0 && s_cnt) atomicAdd(&s_io.ctrl->num_negcell, s_cnt);
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

// The end of a stage of the time-step pipeline in one launch over the ghost values of the stage
// state u: block 0 forms the total entropy from the limiter's partials (final stage only:
// ent_partial != NULL) and then, in one thread, the stage-end decision (ctl_stage_end_body) and the
// pseudo-time of the next stage (next_stage > 0); every block fills the ghost ring of u if the
// stage was still running when the launch began.  A block that already sees the stage abandoned
// skips its fill, and a fill of an abandoned stage only writes scratch ghosts, so the result is
// that of the separate launches in sequence.
// The stage's record goes to the driver log (log may be nullptr).
// src: the array whose interior the ghost ring is filled from (u itself, or u_con after the final
// stage, whose limiter writes the accepted interior to u_con only).
template <int P>
__global__ void __launch_bounds__(256) stage_end_bc_kernel(const double* src, double* u, Geo g, Ctrl* ctrl, int R,
                                                          int stage, int next_stage,
                                                          const double* __restrict__ ent_partial, int ent_nblk,
                                                          LogEntry* log, int log_cap) {
  __shared__ int s_run, s_ent;
  bool run;
  if (blockIdx.x == 0) {  // one read of the state for the whole block, before thread 0 updates it
    if (threadIdx.x == 0) {
      s_run = ctrl->state == ST_RUN;
      s_ent = s_run && ent_partial && !ctrl->neg_avg;
    }
    __syncthreads();
    run = s_run;
    if (s_ent) pp_entsum_body(ent_partial, ent_nblk, ctrl);  // whole block
    if (threadIdx.x == 0) {
      ctl_stage_end_body(ctrl);
      if (run) ctl_log_stage(ctrl, stage, log, log_cap);
      if (next_stage > 0) ctl_stage_time_body(ctrl, R, next_stage);
    }
  } else {
    run = *reinterpret_cast<volatile const int*>(&ctrl->state) == ST_RUN;
  }
  if (run) bc_value<P>(src, u, g, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(256) pp_entsum_kernel(const double* __restrict__ partial, int nblk,
                                                        Ctrl* ctrl, int gate) {
  if (!gate_open(ctrl, gate)) return;
  if (ctrl->neg_avg) return;
  pp_entsum_body(partial, nblk, ctrl);
}

// many instances: stage_end_bc_kernel for every member of a batch -- the ghost fills of all
// members (items = every member's blocks of 256 ghost values) and, one CTA per member, the entropy
// sum (final stage), the stage-end decision and the next stage's pseudo-time.  A fill that runs
// after its member's decision abandoned the stage is skipped, which changes nothing (the stage's
// state is scratch then).
template <int P>
__global__ void __launch_bounds__(256) stage_end_bc_batched(const InstDesc* __restrict__ insts,
                                                           const int* __restrict__ pref, const int* __restrict__ nwork,
                                                           const int* __restrict__ ninst, int slot, int R,
                                                           int next_stage, int final) {
  __shared__ int s_run, s_ent;
  const int nw = *nwork, n = *ninst;
  for (BatchWalk it(pref, n, nw); it.more(); it.next()) {
    const InstDesc& d = insts[it.m];
    if (*reinterpret_cast<volatile const int*>(&d.ctrl->state) != ST_RUN) continue;
    // after the final stage the ring is filled from u_con, which alone holds the accepted interior
    bc_value<P>(final ? d.u[0] : d.u[slot], d.u[slot], d.g, (long long)it.local() * 256 + threadIdx.x);
  }
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const InstDesc& d = insts[i];
    __syncthreads();  // s_run and s_ent of the previous member are read
    if (threadIdx.x == 0) {
      s_run = d.ctrl->state == ST_RUN;
      s_ent = s_run && final && !d.ctrl->neg_avg;
    }
    __syncthreads();
    if (s_ent) pp_entsum_body(d.ent_partial, d.nseg_limit, d.ctrl);  // whole block
    if (threadIdx.x == 0) {
      ctl_stage_end_body(d.ctrl);
      if (s_run) ctl_log_stage(d.ctrl, slot, d.log, d.log_cap);
      if (next_stage > 0) ctl_stage_time_body(d.ctrl, R, next_stage);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Stage diagnostics (optional, for checking the invariants the method promises): over the interior
// nodes of a state, the minimum density, the minimum pressure (_macro_prs_, DG_solver.f90:125) and
// the domain integrals of the eight conserved variables by the GLL rule the cell averages use
// (sum of (hx hy / 4) w_k w_l u, DG_solver.f90:177-184,227-229).  Block b takes a fixed contiguous
// range of elements and reduces in a fixed order; the last block to finish (a ticket counter, no
// waiting) combines the block partials in block order and writes the newest log record.  The
// result is therefore independent of timing.  `part` holds DIAG_MAX_BLOCKS x 10 doubles and the
// ticket; the ticket is left at zero.
// ---------------------------------------------------------------------------------------------
constexpr int DIAG_MAX_BLOCKS = 592;  // 4 x 148 SMs
constexpr int DIAG_VALS = 18;          // per block: min rho, min p, 8 sums and their 8 compensations

// Neumaier's compensated summation (a running sum s and the sum c of its rounding errors): the
// domain integrals are checked against conservation at the 1e-13 level, below the rounding error of
// a plain sum of 10^5-10^7 terms.
__device__ __forceinline__ void neu_add(double& s, double& c, double x) {
  const double t = __dadd_rn(s, x);
  c = __dadd_rn(c, fabs(s) >= fabs(x) ? __dadd_rn(__dadd_rn(s, -t), x) : __dadd_rn(__dadd_rn(x, -t), s));
  s = t;
}

template <int P>
__global__ void __launch_bounds__(256) stage_diag_kernel(const double* __restrict__ u, Geo g, Ctrl* ctrl, int gate,
                                                        double* __restrict__ part, unsigned int* ticket,
                                                        LogEntry* log, int log_cap) {
  constexpr int N = P + 1, NN = N * N, EB = 8 * NN;
  __shared__ double s[DIAG_VALS][256];
  __shared__ bool s_last;
  if (!gate_open(ctrl, gate) || !log || log_cap <= 0 || ctrl->log_seq <= 0) return;
  const int tid = threadIdx.x;
  const int nx = g.nx, ny = g.ny;
  const long long E = (long long)nx * ny;
  const long long e0 = E * blockIdx.x / gridDim.x, e1 = E * (blockIdx.x + 1) / gridDim.x;
  const DegConst& dc = c_deg[P];
  const double gamma = g.gamma, q4 = __dmul_rn(__dmul_rn(0.25, g.hx), g.hy);
  double rmin = 1.0e308, pmin = 1.0e308, sum[8], cmp[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) sum[v] = cmp[v] = 0.0;
  for (long long it = e0 * NN + tid; it < e1 * NN; it += 256) {
    const long long e = it / NN;
    const int q = (int)(it - e * NN), k = q % N, l = q / N;
    const int j = 1 + (int)(e / nx), i = 1 + (int)(e - (long long)(j - 1) * nx);
    const double* x = u + ((long long)j * (nx + 2) + i) * EB + q;
    double w[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) w[v] = x[v * NN];
    rmin = fmin(rmin, w[0]);
    pmin = fmin(pmin, prs_of(w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], gamma));
    const double wq = __dmul_rn(__dmul_rn(q4, dc.qw[k]), dc.qw[l]);
#pragma unroll
    for (int v = 0; v < 8; ++v) neu_add(sum[v], cmp[v], __dmul_rn(wq, w[v]));
  }
  s[0][tid] = rmin;
  s[1][tid] = pmin;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    s[2 + v][tid] = sum[v];
    s[10 + v][tid] = cmp[v];
  }
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) {
      s[0][tid] = fmin(s[0][tid], s[0][tid + w]);
      s[1][tid] = fmin(s[1][tid], s[1][tid + w]);
#pragma unroll
      for (int v = 0; v < 8; ++v) {  // (s, c) + (s', c'): the sums by Neumaier, the compensations plainly
        double a = s[2 + v][tid], c = __dadd_rn(s[10 + v][tid], s[10 + v][tid + w]);
        neu_add(a, c, s[2 + v][tid + w]);
        s[2 + v][tid] = a;
        s[10 + v][tid] = c;
      }
    }
    __syncthreads();
  }
  if (tid < DIAG_VALS) part[blockIdx.x * DIAG_VALS + tid] = s[tid][0];
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const volatile double* vp = part;
  LogEntry* e = log + ((ctrl->log_seq - 1) % log_cap);
  if (tid < 2) {
    double r = vp[tid];
    for (unsigned b = 1; b < gridDim.x; ++b) r = fmin(r, vp[b * DIAG_VALS + tid]);
    if (tid == 0) e->rho_min = r;
    else e->p_min = r;
  } else if (tid < 10) {  // the blocks' (sum, compensation) pairs in block order
    double a = vp[tid], c = vp[tid + 8];
    for (unsigned b = 1; b < gridDim.x; ++b) {
      c = __dadd_rn(c, vp[b * DIAG_VALS + tid + 8]);
      neu_add(a, c, vp[b * DIAG_VALS + tid]);
    }
    e->total[tid - 2] = __dadd_rn(a, c);
  }
  if (tid == 0) *ticket = 0u;
}

}  // namespace mhd
