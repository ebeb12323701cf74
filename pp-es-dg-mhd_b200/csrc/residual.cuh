// residual.cuh -- DG_semidiscretize (DG_solver.f90:663-892) as one sm_100a kernel.
//
// ut = L(u): the entropy-conservative two-point flux differencing over the GLL nodes of each
// element, the ESPP-HLL interface flux, the Godunov-Powell source and the surface terms, and
// dt_lim.  One CTA owns a tile of elements; one lane owns one node (see residual_tile2 below).
// Sums are formed in a fixed order, so the kernel is deterministic.
#pragma once
#include "common.cuh"

namespace mhd {

// swap_xy (DG_solver.f90:1556-1568) as a variable permutation: 1 <-> 2, 4 <-> 5
__host__ __device__ constexpr int swap_xy_var(int v) { return v == 1 ? 2 : v == 2 ? 1 : v == 4 ? 5 : v == 5 ? 4 : v; }

// The next stage's SSP-RK combination folded into the residual (drive.f90:185-241 for SSP-RK3,
// :148-183 for SSP-RK(2,2)): out = ca*u0 + cb*(u + dt*L(u)), rounded exactly as combine_value
// forms it, written to the interior of the next stage's state instead of storing L(u).  Only
// where that combination uses no other stage's L (u0 == nullptr: plain residual into ut).
struct StageCombine {
  const double* u0;     // u_con (ghosted layout)
  double* out;          // the next stage's state (ghosted layout)
  double ca, cb;
  const double* dt;     // the try's dt (device control block)
};

// =============================================================================================
// Node-per-lane form of the residual.
//
// A lane owns one GLL node of one element (p = 3: two elements per warp, p = 2: three, p = 1:
// eight) and keeps the node's state and primitives in registers.  The entropy-conservative flux of
// each node pair of a line is computed once, by one of the pair's two lanes, from the partner's
// primitives fetched with a warp shuffle; the other lane receives the flux by a shuffle.  Rounds
// per degree (k along x, l along y; every round gives each lane exactly one flux to compute):
//   p = 1  one round: lanes with k == l take their x pair, the others their y pair
//   p = 2  a ring along x (partner k+1 mod 3, received from k+2 mod 3), then the same along y:
//          the three pairs of a line are the ring's three edges
//   p = 3  rings along x and y (four of the six pairs of a line), then a round for the pairs
//          (k, k^2) / (l, l^2): lanes with (k>>1)^(l>>1) == 0 take the x pair, the others the y
//          pair (each such pair has exactly one endpoint of each kind)
// so no pair flux goes through shared memory.  The tile's element blocks arrive in shared memory by
// bulk asynchronous copies (one per contiguous run) completed on an mbarrier; the interface fluxes
// are computed from there as in the shared-memory form (every face node once, y faces through
// swap_xy), spread evenly over the warps.  Each lane then forms its node's residual and stores it
// directly (a variable's nodes of one element are contiguous, so the stores coalesce).
// =============================================================================================
#if __has_include("residual2_tuned.h")
#include "residual2_tuned.h"
#endif
#ifndef MHD_RES2_CFG1
#define MHD_RES2_CFG1 8, 8, 256, 2
#endif
#ifndef MHD_RES2_CFG2
#define MHD_RES2_CFG2 6, 4, 256, 2
#endif
#ifndef MHD_RES2_CFG3
#define MHD_RES2_CFG3 4, 4, 256, 2
#endif
struct Res2Params {
  int TX, TY, NT, MINB;
};
template <int P>
struct Res2Cfg;
template <>
struct Res2Cfg<1> {
  static constexpr Res2Params c{MHD_RES2_CFG1};
  static constexpr int TX = c.TX, TY = c.TY, NT = c.NT, MINB = c.MINB;
};
template <>
struct Res2Cfg<2> {
  static constexpr Res2Params c{MHD_RES2_CFG2};
  static constexpr int TX = c.TX, TY = c.TY, NT = c.NT, MINB = c.MINB;
};
template <>
struct Res2Cfg<3> {
  static constexpr Res2Params c{MHD_RES2_CFG3};
  static constexpr int TX = c.TX, TY = c.TY, NT = c.NT, MINB = c.MINB;
};

template <int P>
struct Res2Layout {
  static constexpr int N = P + 1, NN = N * N, EB = 8 * NN;
  static constexpr int G = 32 / NN;  // elements per warp
  static constexpr int ES = EB + (P == 2 ? 0 : 2);  // padded records as in the shared-memory form
  static constexpr int TX = Res2Cfg<P>::TX, TY = Res2Cfg<P>::TY, TE = TX * TY;
  static constexpr int NT = Res2Cfg<P>::NT, NW = NT / 32;
  static constexpr int NFX = (TX + 1) * TY * N;
  static constexpr int NFY = TX * (TY + 1) * N;
  static constexpr int FW = 11;
  static_assert(TE <= NW * G, "every element of the tile needs a lane group");
  static_assert(NT % 32 == 0 && NT <= 1024, "whole warps");
  static_assert((ES * 8) % 16 == 0, "bulk copies land on 16-byte boundaries");
  static constexpr int O_CONS = 0;
  static constexpr int O_U0 = O_CONS + TE * ES;  // u_con's tile when the next stage is formed here
  static constexpr int O_HXL = O_U0 + TE * ES;
  static constexpr int O_HXR = O_HXL + TY * 8 * N;
  static constexpr int O_HYB = O_HXR + TY * 8 * N;
  static constexpr int O_HYT = O_HYB + TX * 8 * N;
  static constexpr int O_FX = O_HYT + TX * 8 * N;
  static constexpr int O_FY = O_FX + NFX * FW;
  static constexpr int O_DM = O_FY + NFY * FW;  // D (N x N) and 1/w_k
  static constexpr int O_RED = O_DM + NN + N;   // NW doubles of the block minimum; [31] = the try's dt
  static constexpr int O_BAR = O_RED + 32;      // the tile's mbarrier (8 bytes)
  static constexpr int TOTAL = O_BAR + 2;
  static constexpr size_t BYTES = sizeof(double) * TOTAL;
  static_assert(BYTES <= 227 * 1024, "residual tile does not fit the shared memory of one CTA");
};

// Once per CTA before its first tile: the copy barrier and the degree's D and 1/w in shared memory.
template <int P>
__device__ __forceinline__ void res2_prologue(double* sm) {
  using L = Res2Layout<P>;
  const DegConst& dc = c_deg[P];
  if (threadIdx.x == 0) mbar_init(reinterpret_cast<unsigned long long*>(sm + L::O_BAR), 1);
  if (threadIdx.x < L::NN) sm[L::O_DM + threadIdx.x] = dc.D[threadIdx.x];
  if (threadIdx.x < L::N) sm[L::O_DM + L::NN + threadIdx.x] = dc.iqw[threadIdx.x];
  __syncthreads();
}

// max over the NN lanes of this lane's element group (every lane of the group gets it); gbase =
// the group's first lane
template <int NN>
__device__ __forceinline__ double group_max(double v, int gbase) {
  if constexpr ((NN & (NN - 1)) == 0) {
#pragma unroll
    for (int o = NN / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
  } else {
    double m = __shfl_sync(0xffffffffu, v, gbase);
#pragma unroll
    for (int r = 1; r < NN; ++r) m = fmax(m, __shfl_sync(0xffffffffu, v, gbase + r));
    return m;
  }
}

// Where a tile's results go: the L(u) array and the control block (dt_lim, flags).  Taken by
// reference, so that the batched kernel can keep it in shared memory, out of the registers.
struct TileOut {
  double* ut;
  Ctrl* ctrl;
};

// One tile (elements tile_x*TX + 1 .., tile_y*TY + 1 ..).  `phase` = the parity of the tile
// barrier's next phase (flipped here).  Returns false if the wait for the tile's copies ran out
// (FLAG_DEVICE_WAIT is then set): the caller must stop.  ug = the array whose ghost ring the
// boundary halos come from (u itself, or the last stage array whose ring was filled from u's
// interior after the final stage; the interior always comes from u).
template <int P>
__device__ __forceinline__ bool residual_tile2(const double* __restrict__ u, const double* __restrict__ ug,
                                               const TileOut& to, const Geo& g, int tile_x,
                                               int tile_y, double* sm, unsigned& phase,
                                               const StageCombine& sc = StageCombine{}) {
  using L = Res2Layout<P>;
  constexpr int N = L::N, NN = L::NN, EB = L::EB, ES = L::ES, TX = L::TX, TY = L::TY, TE = L::TE;
  constexpr int NT = L::NT, NW = L::NW, G = L::G;
  constexpr unsigned FULL = 0xffffffffu;
  double* s_cons = sm + L::O_CONS;
  double* s_u0 = sm + L::O_U0;
  double* s_hxl = sm + L::O_HXL;
  double* s_hxr = sm + L::O_HXR;
  double* s_hyb = sm + L::O_HYB;
  double* s_hyt = sm + L::O_HYT;
  double* s_fx = sm + L::O_FX;
  double* s_fy = sm + L::O_FY;
  const double* s_dm = sm + L::O_DM;
  double* s_red = sm + L::O_RED;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + L::O_BAR);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nx = g.nx, ny = g.ny;
  const int i0 = 1 + tile_x * TX, j0 = 1 + tile_y * TY;
  const int W = min(TX, nx - i0 + 1), H = min(TY, ny - j0 + 1);
  const long long rowstride = (long long)(nx + 2) * EB;
  const double gamma = g.gamma;

  // ---- phase 0: the tile's element blocks by bulk copies (warp 0), halo traces by loads ----
  // (with a next-stage combination, u_con's blocks of the tile come the same way)
  const int ncopy = sc.u0 ? 2 : 1;
  if (warp == 0) {
    if (lane == 0) {
      fence_proxy_async_smem();  // the previous tile's reads of s_cons come before these writes
      mbar_arrive_expect_tx(bar, (unsigned)(ncopy * H * W * EB * 8));
      if (sc.u0) s_red[31] = *sc.dt;
    }
    __syncwarp();
    for (int which = 0; which < ncopy; ++which) {
      const double* src = which ? sc.u0 : u;
      double* dst = which ? s_u0 : s_cons;
      if (ES == EB) {  // unpadded records: one copy per tile row
        for (int r = lane; r < H; r += 32)
          bulk_copy_g2s(dst + r * TX * ES, src + (long long)(j0 + r) * rowstride + (long long)i0 * EB,
                        (unsigned)(W * EB * 8), bar);
      } else {  // padded records: one copy per element block
        for (int it = lane; it < H * W; it += 32) {
          const int r = it / W, c = it - r * W;
          bulk_copy_g2s(dst + (r * TX + c) * ES, src + (long long)(j0 + r) * rowstride + (long long)(i0 + c) * EB,
                        (unsigned)(EB * 8), bar);
        }
      }
    }
  }
  // a halo side on the domain boundary reads the ghost ring (of ug)
  const double* uxl = i0 == 1 ? ug : u;
  const double* uxr = i0 + W == nx + 1 ? ug : u;
  const double* uyb = j0 == 1 ? ug : u;
  const double* uyt = j0 + H == ny + 1 ? ug : u;
  for (int it = tid; it < TY * 8 * N; it += NT) {  // x halos: traces k = n-1 (left) / 0 (right)
    const int r = it / (8 * N), rem = it - r * 8 * N, v = rem / N, l = rem - v * N;
    if (r < H) {
      const long long row = (long long)(j0 + r) * rowstride;
      s_hxl[it] = __ldg(uxl + row + (long long)(i0 - 1) * EB + v * NN + (N - 1) + N * l);
      s_hxr[it] = __ldg(uxr + row + (long long)(i0 + W) * EB + v * NN + 0 + N * l);
    }
  }
  for (int it = tid; it < TX * 8 * N; it += NT) {  // y halos: traces l = n-1 (bottom) / 0 (top)
    const int c = it / (8 * N), rem = it - c * 8 * N, v = rem / N, k = rem - v * N;
    if (c < W) {
      s_hyb[it] = __ldg(uyb + (long long)(j0 - 1) * rowstride + (long long)(i0 + c) * EB + v * NN + k + N * (N - 1));
      s_hyt[it] = __ldg(uyt + (long long)(j0 + H) * rowstride + (long long)(i0 + c) * EB + v * NN + k);
    }
  }
  {
    const bool ok = mbar_wait_bounded(bar, phase & 1u);
    if (__syncthreads_or(!ok)) {  // the copies did not arrive: flag it, give them one more bound, stop
      if (tid == 0) atomicOr(&to.ctrl->flags, FLAG_DEVICE_WAIT);
      mbar_wait_bounded(bar, phase & 1u);
      __syncthreads();
      return false;
    }
    phase ^= 1u;
  }

  const double igm1 = 1.0 / (gamma - 1.0);
  // ---- phase 1: interface fluxes, every face node of the tile once ----
  // Thread-major: the items fill whole warps first, so the fewest warps run this code (a warp
  // pays its issue slots whether or not all its lanes have an item); the others go on to phase 2.
  {
    constexpr int NH = L::NFX + L::NFY;
    for (int f = tid; f < NH; f += NT) {
      const bool ydir = f >= L::NFX;
      const double *pl, *pr;
      int sl, sr;
      double* dst;
      int ostride;
      bool live = true;
      if (!ydir) {
        const int fi = f / (TY * N), rem = f - fi * TY * N, r = rem / N, l = rem - r * N;
        live = r < H && fi <= W;
        if (fi == 0) { pl = s_hxl + r * 8 * N + l; sl = N; }
        else { pl = s_cons + (r * TX + fi - 1) * ES + (N - 1) + N * l; sl = NN; }
        if (fi == W) { pr = s_hxr + r * 8 * N + l; sr = N; }
        else { pr = s_cons + (r * TX + fi) * ES + N * l; sr = NN; }
        dst = s_fx + f;
        ostride = L::NFX;
      } else {
        const int q = f - L::NFX;
        const int fj = q / (TX * N), rem = q - fj * TX * N, c = rem / N, k = rem - c * N;
        live = c < W && fj <= H;
        if (fj == 0) { pl = s_hyb + c * 8 * N + k; sl = N; }
        else { pl = s_cons + ((fj - 1) * TX + c) * ES + k + N * (N - 1); sl = NN; }
        if (fj == H) { pr = s_hyt + c * 8 * N + k; sr = N; }
        else { pr = s_cons + (fj * TX + c) * ES + k; sr = NN; }
        dst = s_fy + q;
        ostride = L::NFY;
      }
      if (!live) continue;
      double wl[8], wr[8], o[11];
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const int sv = ydir ? swap_xy_var(v) : v;
        wl[v] = pl[sv * sl];
        wr[v] = pr[sv * sr];
      }
      espp_hll(wl, wr, gamma, igm1, o);
#pragma unroll
      for (int c = 0; c < L::FW; ++c) dst[(ydir && c < 8 ? swap_xy_var(c) : c) * ostride] = o[c];
    }
  }

  // ---- phase 2: node per lane: primitives, node-pair fluxes by rounds, local div B ----
  const int grp = lane / NN, node = lane - grp * NN;
  const int el = warp * G + grp;
  const int er = el / TX, ec = el - er * TX;
  const bool act = grp < G && el < TE && er < H && ec < W;
  const int gbase = (grp < G ? grp : 0) * NN;  // lanes beyond the groups mirror group 0
  const int k = node % N, l = node / N;
  const double sxh = 2.0 / g.hx, syh = 2.0 / g.hy;
  double w[8];
  {
    const double* cw = s_cons + (act ? el : 0) * ES + node;
#pragma unroll
    for (int v = 0; v < 8; ++v) w[v] = cw[v * NN];
  }
  // (all arithmetic of the tile is exactly rounded as written: dmul/dadd/dsub/dfma of common.cuh)
  const double ir = 1.0 / w[0];
  const double vx = dmul(ir, w[1]), vy = dmul(ir, w[2]), vz = dmul(ir, w[3]);
  double pt, sgx, sgy, pp[8];  // pp: (rho, vx, vy, vz, Bx, By, Bz, beta), the EC flux's inputs
  {
    const double ek = dmul(dmul(0.5, ir), dsq3(w[1], w[2], w[3]));
    const double bsq = dsq3(w[4], w[5], w[6]);
    const double pf = fmax(dmul(dsub(gamma, 1.0), dsub(w[7], dfma(0.5, bsq, ek))), PP_EPS);
    pp[0] = w[0];
    pp[1] = vx;
    pp[2] = vy;
    pp[3] = vz;
    pp[4] = w[4];
    pp[5] = w[5];
    pp[6] = w[6];
    pp[7] = dmul(0.5, w[0]) / pf;
    const double cs = dmul(dmul(gamma, pf), ir), ss = dfma(bsq, ir, cs), coef = dmul(dmul(4.0, cs), ir);
    pt = dfma(0.5, bsq, pf);
    sgx = dadd(fabs(vx), sqrt(dmul(0.5, fmax(dadd(ss, sqrt(fmax(dfma(ss, ss, -dmul(coef, dmul(w[4], w[4]))), 0.0))), 0.0))));
    sgy = dadd(fabs(vy), sqrt(dmul(0.5, fmax(dadd(ss, sqrt(fmax(dfma(ss, ss, -dmul(coef, dmul(w[5], w[5]))), 0.0))), 0.0))));
  }
  auto Dm = [&](int i) { return s_dm[i]; };
  // the partner lane of node (kk, ll) of this lane's element
  auto lane_of = [&](int kk, int ll) { return gbase + kk + N * ll; };
  // local div B (DG_solver.f90:813), the sums in node order
  // (every product-sum of the accumulation below is an explicit fused multiply-add, so that each
  // kernel this tile is inlined into rounds it the same way: a batch member equals its solo run)
  double dbx = 0.0, dby = 0.0;
#pragma unroll
  for (int r = 0; r < N; ++r) dbx = __fma_rn(Dm(k + N * r), __shfl_sync(FULL, w[4], lane_of(r, l)), dbx);
#pragma unroll
  for (int m = 0; m < N; ++m) dby = __fma_rn(__shfl_sync(FULL, w[5], lane_of(k, m)), Dm(l + N * m), dby);
  // node flux F, G and Godunov-Powell coefficients (DG_solver.f90:749-799), formed again for the
  // surface terms after the barrier; the accumulation starts, as the reference's does
  // (DG_solver.f90:833), with the diagonal and Godunov-Powell terms
  auto node_fluxes = [&](double* F, double* Gf, double* GP) {
    const double bx = w[4], by = w[5], bz = w[6];
    const double bu = ddot3(bx, vx, by, vy, bz, vz);
    const double ex = dfma(by, vz, -dmul(bz, vy)), ey = dfma(bz, vx, -dmul(bx, vz)), ez = dfma(bx, vy, -dmul(by, vx));
    F[0] = w[1];
    F[1] = dadd(dfma(vx, w[1], -dmul(bx, bx)), pt);
    F[2] = dfma(vx, w[2], -dmul(by, bx));
    F[3] = dfma(vx, w[3], -dmul(bz, bx));
    F[4] = 0.0;
    F[5] = -ez;
    F[6] = ey;
    F[7] = dfma(vx, dadd(w[7], pt), -dmul(bx, bu));
    Gf[0] = w[2];
    Gf[1] = dfma(vy, w[1], -dmul(bx, by));
    Gf[2] = dadd(dfma(vy, w[2], -dmul(by, by)), pt);
    Gf[3] = dfma(vy, w[3], -dmul(bz, by));
    Gf[4] = ez;
    Gf[5] = 0.0;
    Gf[6] = -ex;
    Gf[7] = dfma(vy, dadd(w[7], pt), -dmul(by, bu));
    GP[0] = 0.0;
    GP[1] = bx;
    GP[2] = by;
    GP[3] = bz;
    GP[4] = vx;
    GP[5] = vy;
    GP[6] = vz;
    GP[7] = bu;
  };
  double acc[8];
  {
    double F[8], Gf[8], GP[8];
    node_fluxes(F, Gf, GP);
    const double divB = dfma(syh, dby, dmul(sxh, dbx));
    const double ckk = 2.0 * sxh * Dm(k + N * k), cll = 2.0 * syh * Dm(l + N * l);
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[v] = __fma_rn(-divB, GP[v], __fma_rn(-cll, Gf[v], -__dmul_rn(ckk, F[v])));
  }
  // This lane's flux with the node in lane `src` (x frame, or y through swap_xy); the result F is
  // in the global frame.  Every lane of the warp calls it (the shuffles need the full warp).
  auto pair_flux = [&](int src, bool ydir, double* F) {
    double A[8], B[8], Fx[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) B[v] = __shfl_sync(FULL, pp[v], src);
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const int sv = swap_xy_var(v);
      A[v] = ydir ? pp[sv] : pp[v];
      const double b = ydir ? B[sv] : B[v];
      Fx[v] = b;  // reuse as the rotated partner
    }
    ec_flux<0>(A, Fx, igm1, B);
#pragma unroll
    for (int v = 0; v < 8; ++v) F[v] = ydir ? B[swap_xy_var(v)] : B[v];
  };
  if constexpr (P == 1) {
    const bool xb = (k == l);
    double F[8];
    pair_flux(xb ? lane_of(1 - k, l) : lane_of(k, 1 - l), !xb, F);
    const double c1 = xb ? 2.0 * sxh * Dm(k + N * (1 - k)) : 2.0 * syh * Dm(l + N * (1 - l));
    const int src2 = xb ? lane_of(k, 1 - l) : lane_of(1 - k, l);
    const double c2 = xb ? 2.0 * syh * Dm(l + N * (1 - l)) : 2.0 * sxh * Dm(k + N * (1 - k));
    // the reference's order: x partner below, y partner below, x above, y above
    const int rx = (1 - k) < k ? 0 : 2, ry = (1 - l) < l ? 1 : 3;
    const bool own_first = xb ? rx < ry : ry < rx;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const double fr = __shfl_sync(FULL, F[v], src2);
      acc[v] = __fma_rn(-(own_first ? c1 : c2), own_first ? F[v] : fr, acc[v]);
      acc[v] = __fma_rn(-(own_first ? c2 : c1), own_first ? fr : F[v], acc[v]);
    }
  } else {
    // rings along x and y: compute with the next node, receive from the previous one
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const int a = dir == 0 ? k : l;
      const int an = (a + 1) % N, ap = (a + N - 1) % N;
      const double h2 = dir == 0 ? 2.0 * sxh : 2.0 * syh;
      double F[8];
      pair_flux(dir == 0 ? lane_of(an, l) : lane_of(k, an), dir == 1, F);
      const double c1 = h2 * Dm(a + N * an), c2 = h2 * Dm(a + N * ap);
      const int src2 = dir == 0 ? lane_of(ap, l) : lane_of(k, ap);
      const bool next_first = an < ap;  // the two contributions in ascending partner order
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        if (v == (dir == 0 ? 4 : 5)) continue;  // that component of the flux is identically zero
        const double fr = __shfl_sync(FULL, F[v], src2);
        acc[v] = __fma_rn(-(next_first ? c1 : c2), next_first ? F[v] : fr, acc[v]);
        acc[v] = __fma_rn(-(next_first ? c2 : c1), next_first ? fr : F[v], acc[v]);
      }
    }
    if constexpr (P == 3) {  // the pairs (k, k^2) along x and (l, l^2) along y
      const bool xb = ((k >> 1) ^ (l >> 1)) == 0;
      double F[8];
      pair_flux(xb ? lane_of(k ^ 2, l) : lane_of(k, l ^ 2), !xb, F);
      const double cx = 2.0 * sxh * Dm(k + N * (k ^ 2)), cy = 2.0 * syh * Dm(l + N * (l ^ 2));
      const int src2 = xb ? lane_of(k, l ^ 2) : lane_of(k ^ 2, l);
      // the reference's order: x partner below, y partner below, x above, y above
      const int rx = (k ^ 2) < k ? 0 : 2, ry = (l ^ 2) < l ? 1 : 3;
      const bool own_first = xb ? rx < ry : ry < rx;
      const double c1 = xb ? cx : cy, c2 = xb ? cy : cx;
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const double fr = __shfl_sync(FULL, F[v], src2);
        acc[v] = __fma_rn(-(own_first ? c1 : c2), own_first ? F[v] : fr, acc[v]);
        acc[v] = __fma_rn(-(own_first ? c2 : c1), own_first ? fr : F[v], acc[v]);
      }
    }
  }
  __syncthreads();  // the interface fluxes of phase 1 are complete

  // ---- phase 3: surface terms; dt_lim; store ----
  {
    const double bx = w[4], by = w[5];
    double F[8], Gf[8], GP[8];
    node_fluxes(F, Gf, GP);
    // surface terms (DG_solver.f90:872-882): left face (k = 0) with -, right face (k = N-1) with +;
    // likewise bottom/top in y
    if (k == 0 || k == N - 1) {
      const bool right = (k == N - 1);
      const double* fr = s_fx + (((ec + (right ? 1 : 0)) * TY + er) * N + l);
      const double c = (right ? sxh : -sxh) * s_dm[NN + k];
      const double jb = __dadd_rn(bx, -fr[8 * L::NFX]);
#pragma unroll
      for (int v = 0; v < 8; ++v) acc[v] = __fma_rn(c, __fma_rn(GP[v], jb, __dadd_rn(F[v], -fr[v * L::NFX])), acc[v]);
    }
    if (l == 0 || l == N - 1) {
      const bool top = (l == N - 1);
      const double* fr = s_fy + (((er + (top ? 1 : 0)) * TX + ec) * N + k);
      const double c = (top ? syh : -syh) * s_dm[NN + l];
      const double jb = __dadd_rn(by, -fr[8 * L::NFY]);
#pragma unroll
      for (int v = 0; v < 8; ++v) acc[v] = __fma_rn(c, __fma_rn(GP[v], jb, __dadd_rn(Gf[v], -fr[v * L::NFY])), acc[v]);
    }
  }
  // dt_lim of the element: the largest node speed and interface speed per direction
  double my_dt = 1.0e300;
  {
    double ax = sgx, ay = sgy;
    if (act) {
      if (k == 0) ax = fmax(ax, s_fx[10 * L::NFX + (ec * TY + er) * N + l]);
      if (k == N - 1) ax = fmax(ax, -s_fx[9 * L::NFX + ((ec + 1) * TY + er) * N + l]);
      if (l == 0) ay = fmax(ay, s_fy[10 * L::NFY + (er * TX + ec) * N + k]);
      if (l == N - 1) ay = fmax(ay, -s_fy[9 * L::NFY + ((er + 1) * TX + ec) * N + k]);
    }
    ax = group_max<NN>(ax, gbase);
    ay = group_max<NN>(ay, gbase);
    if (act && node == 0) my_dt = 1.0 / ((2 * P + 1) * ax / g.hx + (2 * P + 1) * ay / g.hy);
  }
  if (act) {
    if (sc.u0) {  // the next stage's state instead of L(u)
      const long long e = ((long long)(j0 + er) * (nx + 2) + (i0 + ec)) * EB + node;
      const double dt = s_red[31];
      const double* u0n = s_u0 + el * ES + node;
#pragma unroll
      for (int v = 0; v < 8; ++v)
        sc.out[e + v * NN] = __dadd_rn(__dmul_rn(sc.ca, u0n[v * NN]),
                                       __dmul_rn(sc.cb, __dadd_rn(w[v], __dmul_rn(dt, acc[v]))));
    } else {
      double* o = to.ut + ((long long)(j0 + er - 1) * nx + (i0 + ec - 1)) * EB + node;
#pragma unroll
      for (int v = 0; v < 8; ++v) o[v * NN] = acc[v];
    }
  }
  // block minimum of dt_lim -> one atomicMin
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_dt = fmin(my_dt, __shfl_xor_sync(FULL, my_dt, o));
  static_assert(L::NW <= 31, "s_red[31] holds dt");
  if (lane == 0) s_red[warp] = my_dt;
  __syncthreads();
  if (tid == 0) {
    double m = s_red[0];
    for (int q = 1; q < NW; ++q) m = fmin(m, s_red[q]);
    atomicMin(&to.ctrl->dt_lim_bits, (unsigned long long)__double_as_longlong(m));
  }
  return true;
}

// single instance: one CTA per tile (ug: the ghost-ring source, see residual_tile2)
template <int P>
__global__ void __launch_bounds__(Res2Cfg<P>::NT, Res2Cfg<P>::MINB)
    residual2_kernel(const double* __restrict__ u, const double* __restrict__ ug, double* __restrict__ ut, Geo g,
                     Ctrl* ctrl, int gate, StageCombine sc) {
  if (!gate_open(ctrl, gate)) return;
  extern __shared__ __align__(16) double sm[];
  res2_prologue<P>(sm);
  unsigned phase = 0;
  residual_tile2<P>(u, ug, TileOut{ut, ctrl}, g, blockIdx.x, blockIdx.y, sm, phase, sc);
}

// single instance, persistent: CTA b computes tiles b, b + gridDim.x, ... (row-major, ntx per row).
// For a launch that is usually gated off (the re-try residual of every try): a grid of resident
// CTAs that return at once costs far less than one CTA per tile.
template <int P>
__global__ void __launch_bounds__(Res2Cfg<P>::NT, Res2Cfg<P>::MINB)
    residual2_persistent(const double* __restrict__ u, double* __restrict__ ut, Geo g, Ctrl* ctrl, int gate,
                         int ntx, int ntiles) {
  if (!gate_open(ctrl, gate)) return;
  extern __shared__ __align__(16) double sm[];
  res2_prologue<P>(sm);
  unsigned phase = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    if (!residual_tile2<P>(u, u, TileOut{ut, ctrl}, g, t % ntx, t / ntx, sm, phase, StageCombine{})) return;
    __syncthreads();  // the next tile reuses shared memory
  }
}

// many instances of degree P: a persistent grid walks every member's tiles (row-major per member);
// the state is slot `src`, the result goes to ut[dst], or (next_stage > 0) the combination of
// stage next_stage goes to slot next_stage.  The tile's arithmetic is fully rounded as written
// (explicit fused multiply-adds, see common.cuh), so a member is bitwise equal to its solo run
// although this is a different kernel.
template <int P>
__global__ void __launch_bounds__(Res2Cfg<P>::NT, Res2Cfg<P>::MINB)
    residual2_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                      const int* __restrict__ nwork, const int* __restrict__ ninst, int src, int dst, int gate,
                      int next_stage, double ca, double cb) {
  extern __shared__ __align__(16) double sm[];
  // the member's geometry, stage combination and outputs, copied per tile into shared memory: the
  // tile reads them there after each barrier instead of holding them in registers from the table
  // entry (the single-instance kernel reads them from its parameters in the same way)
  __shared__ Geo s_g;
  __shared__ StageCombine s_sc;
  __shared__ TileOut s_to;
  __shared__ SharedWalk s_walk;  // the walker's state, out of the registers the tile needs
  if (threadIdx.x == 0) s_walk.start(pref, *ninst, *nwork);
  res2_prologue<P>(sm);  // (ends with a barrier)
  unsigned phase = 0;
  while (s_walk.w < s_walk.last) {
    const int m = s_walk.m, local = s_walk.w - s_walk.mstart;
    const InstDesc& d = insts[m];
    const bool open = gate_open(d.ctrl, gate);
    if (open && threadIdx.x == 0) {
      s_g = d.g;
      s_sc = next_stage > 0 ? StageCombine{d.u[0], d.u[next_stage], ca, cb, &d.ctrl->dt} : StageCombine{};
      s_to = TileOut{d.ut[dst], d.ctrl};
    }
    __syncthreads();  // every thread has read the walker; the item's arguments are in place
    if (threadIdx.x == 0) s_walk.advance(pref);
    if (open) {
      const int ntx = (d.g.nx + Res2Cfg<P>::TX - 1) / Res2Cfg<P>::TX;
      // the state after the final stage: u_con's interior with the last stage array's ghost ring
      const int srci = (src == d.R) ? 0 : src;
      if (!residual_tile2<P>(d.u[srci], d.u[src], s_to, s_g, local % ntx, local / ntx, sm, phase, s_sc))
        return;
    }
    __syncthreads();  // the item is done (the next one reuses shared memory); the walker has advanced
  }
}

}  // namespace mhd
