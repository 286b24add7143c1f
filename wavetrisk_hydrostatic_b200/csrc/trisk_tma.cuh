// Trend + RK sub-step kernel with its stencil inputs staged in shared memory by
// the tensor memory accelerator (TMA).
//
// A block owns a TT_X x TT_Y tile of padded nodes of one lozenge and one layer.
// One thread issues S_NPLANE tiled bulk-tensor copies (cp.async.bulk.tensor,
// no multicast) of the tile plus its halo into shared memory: the mass and
// Theta fluxes and qe (3 edge planes each), theta, Bernoulli, Phi, the six
// hexagon area parts and hex_inv.  The copies complete on one mbarrier, which
// every thread waits on for at most one second; meanwhile the threads fetch
// their base state and edge lengths.  Flux entries of nodes in the border band
// of the lozenge are then overwritten with the value of the edge their ghost
// copies (the remap table), and the arithmetic of k_trend runs on shared
// memory, expression for expression.
//
// Box geometry: x starts at x0-2 (x0 a multiple of TT_X, so the start is even
// and x*8 bytes is a multiple of 16) and spans TT_X+4 nodes (288 bytes); y
// starts at y0-1 and spans TT_Y+2 rows.  Boxes that reach outside the padded
// array are filled with zeros by the copy engine; no thread that reads such a
// slot uses it.
#pragma once
#include <cuda.h>

#include "trisk_kernels.cuh"

namespace wtk {

constexpr int TT_X = 32, TT_Y = 8;
constexpr int TB_X = TT_X + 4, TB_Y = TT_Y + 2;
constexpr int TB_N = TB_X * TB_Y;                       // 360 slots per plane
constexpr int PLANE_BYTES = 2944;                       // 360*8 = 2880, rounded up to 128
constexpr int PLANE_STRIDE = PLANE_BYTES / 8;           // in doubles
enum { S_HFM = 0, S_HFT = 3, S_QE = 6, S_TH = 9, S_B = 10, S_F = 11, S_PART = 12, S_HINV = 18, S_NPLANE = 19 };
constexpr int TREND_TMA_SMEM = S_NPLANE * PLANE_BYTES + 64;  // planes + mbarrier
constexpr unsigned TREND_TMA_TX = S_NPLANE * TB_N * 8;       // bytes the copies deliver
constexpr unsigned long long TMA_WAIT_NS = 1000000000ull;  // a block gives up on its copies after 1 s
// Test-only injection (wt_tune WT_TUNE_TEST_TMA_TIMEOUT): the block declares
// TMA_INJECT_TX bytes more than its copies deliver, so its phase cannot
// complete, and gives up after TMA_INJECT_WAIT_NS; on the failure path it
// then retires the extra bytes itself (complete_tx) and waits, bounded, for
// its real copies, so no copy is in flight when it exits.
constexpr unsigned TMA_INJECT_TX = 16;
constexpr unsigned long long TMA_INJECT_WAIT_NS = 20000ull;

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_complete_tx(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Polls the mbarrier until its phase completes or limit_ns have passed.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, unsigned parity,
                                                  unsigned long long limit_ns = TMA_WAIT_NS) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (global_ns() - t0 < limit_ns)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

// get_weights (src/ops.f90:1006-1021) from the staged area parts.
__device__ __forceinline__ void weights5_s(const double* __restrict__ S, int q, int offs, double w[5]) {
  double acc = S[(S_PART + offs) * PLANE_STRIDE + q];
  const double hinv = S[S_HINV * PLANE_STRIDE + q];
  double wgt[5];
  wgt[0] = acc;
#pragma unroll
  for (int r = 2; r <= 5; ++r) {
    acc = acc + S[(S_PART + (r + offs - 1) % 6) * PLANE_STRIDE + q];
    wgt[r - 1] = acc;
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) wgt[r] = 0.5 - wgt[r] * hinv;
  w[0] = wgt[0]; w[1] = -wgt[1]; w[2] = wgt[2]; w[3] = -wgt[3]; w[4] = wgt[4];
}

// Same trends and sub-step as k_trend (scalar_trend, du_source/Qperp, du_grad,
// RK_sub_step; src/ops.f90:739-901, src/time_integr.f90:206-225).
// MODE_ML is k_trend_ml of the finest level of a hierarchy (src/multi_level.f90:
// 5-188): trends only where mask_n >= TRSK, dmass and dTheta written on
// [0, n]^2, the velocity source on [0, n)^2, the sub-step on every padded node;
// with a needed-node map, tiles with no needed node are left out before any
// copy is issued and nodes that are not needed write nothing.
// Block b: layer b % nz, then tile x, tile y, lozenge.  err receives 1 when a
// block's copies did not complete within the wait limit; inject != 0 forces
// that path (test only, see TMA_INJECT_TX).
template <int MODE>
__global__ void __launch_bounds__(TT_X * TT_Y, 3)
    k_trend_tma(LevelDev L, int nz, int nbx, int nby, TrendIO io, int* __restrict__ err, int inject,
                const __grid_constant__ TrendMaps M) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* __restrict__ S = reinterpret_cast<double*>(smem_raw);
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t bar = s_base + S_NPLANE * PLANE_BYTES;

  int b = blockIdx.x;
  const int k = b % nz;
  b /= nz;
  const int bx = b % nbx;
  b /= nbx;
  const int by = b % nby;
  const int d = b / nby;
  const int x0 = bx * TT_X, y0 = by * TT_Y;
  const int tid = threadIdx.x;
  if (MODE == MODE_ML && io.need) {
    const int pi = x0 + tid % TT_X, pj = y0 + tid / TT_X;
    int v = 0;
    if (pi < L.P && pj < L.P) v = io.need[__ldg(L.nsrc + (d * L.P + pj) * L.P + pi)];
    if (!__syncthreads_or(v)) return;
  }

  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(bar, TREND_TMA_TX + (inject ? TMA_INJECT_TX : 0u));
    const int cx = x0 - 2, cy = y0 - 1;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      tma_load_4d(s_base + (S_HFM + e) * PLANE_BYTES, &M.hfm, cx, cy, d, 3 * k + e, bar);
      tma_load_4d(s_base + (S_HFT + e) * PLANE_BYTES, &M.hft, cx, cy, d, 3 * k + e, bar);
      tma_load_4d(s_base + (S_QE + e) * PLANE_BYTES, &M.qe, cx, cy, d, 3 * k + e, bar);
    }
    tma_load_4d(s_base + S_TH * PLANE_BYTES, &M.theta, cx, cy, d, k, bar);
    tma_load_4d(s_base + S_B * PLANE_BYTES, &M.bern, cx, cy, d, k, bar);
    tma_load_4d(s_base + S_F * PLANE_BYTES, &M.phik, cx, cy, d, k, bar);
#pragma unroll
    for (int r = 0; r < 6; ++r) tma_load_4d(s_base + (S_PART + r) * PLANE_BYTES, &M.part, cx, cy, d, r, bar);
    tma_load_4d(s_base + S_HINV * PLANE_BYTES, &M.hinv, cx, cy, d, 0, bar);
  }

  // Work that does not need the tile, overlapping the copies.
  const int P = L.P, NN = L.NN, n = L.n;
  const int tx = tid % TT_X, ty = tid / TT_X;
  const int ip = x0 + tx, jp = y0 + ty;
  const bool inside = ip < P && jp < P;
  const int i = ip - 2, j = jp - 2;
  const int id = (d * P + jp) * P + ip;
  const int64_t ko = (int64_t)k * NN;
  const bool scal = inside && i >= 0 && j >= 0 && i <= n && j <= n;
  const bool own = inside && i >= 0 && j >= 0 && i < n && j < n;
  const int64_t vo = 3 * ko + id;
  double bm = 0.0, bt = 0.0, bv0 = 0.0, bv1 = 0.0, bv2 = 0.0;
  if ((MODE == MODE_RK || MODE == MODE_ML) && inside) {
    bm = io.base_m[ko + id];
    bt = io.base_t[ko + id];
    bv0 = io.base_v[vo];
    bv1 = io.base_v[vo + NN];
    bv2 = io.base_v[vo + 2 * NN];
  }
  double lRT = 1.0, lDG = 1.0, lUP = 1.0;
  if (own) {
    lRT = L.len[RT * NN + id];
    lDG = L.len[DG * NN + id];
    lUP = L.len[UP * NN + id];
  }

  const bool ok = mbar_wait_bounded(bar, 0, inject ? TMA_INJECT_WAIT_NS : TMA_WAIT_NS);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicCAS(err, 0, 1);
      if (inject) mbar_complete_tx(bar, TMA_INJECT_TX);
    }
    if (!ok) mbar_wait_bounded(bar, 0);  // copies still in flight target this block's shared memory
    return;
  }

  // Ghost fluxes: slots whose node lies outside [1, n-2]^2 take the signed
  // value of the edge named by the remap (update_bdry of horiz_flux).
  const int sx0 = x0 - 4, sy0 = y0 - 3;  // node coordinates (i, j) of slot (0, 0)
  if (sx0 < 1 || sy0 < 1 || sx0 + TB_X - 1 > n - 2 || sy0 + TB_Y - 1 > n - 2) {
    const double* __restrict__ gm = io.hfm + 3 * ko;
    const double* __restrict__ gt = io.hft + 3 * ko;
    for (int q = tid; q < TB_N; q += TT_X * TT_Y) {
      const int sx = q % TB_X, sy = q / TB_X;
      const int pi = x0 - 2 + sx, pj = y0 - 1 + sy;
      if (pi < 0 || pj < 0 || pi >= P || pj >= P) continue;
      const int si = pi - 2, sj = pj - 2;
      if (si >= 1 && sj >= 1 && si <= n - 2 && sj <= n - 2) continue;
      const int x = (d * P + pj) * P + pi;
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        const int c = __ldg(L.esrc + e * NN + x);
        const double vm = gm[c >> 1], vt = gt[c >> 1];
        S[(S_HFM + e) * PLANE_STRIDE + q] = (c & 1) ? -vm : vm;
        S[(S_HFT + e) * PLANE_STRIDE + q] = (c & 1) ? -vt : vt;
      }
    }
  }
  __syncthreads();

  if (!inside) return;
  bool on = true;
  if (MODE == MODE_ML) {
    if (io.need && !io.need[__ldg(L.nsrc + id)]) return;
    on = io.mask_n[id] >= 2;  // TRSK
  }
  const int q0 = (ty + 1) * TB_X + (tx + 2);
  constexpr int oE = 1, oW = -1, oN = TB_X, oS = -TB_X, oNE = TB_X + 1, oSW = -TB_X - 1, oSE = 1 - TB_X,
                oNW = TB_X - 1;
#define SM(pl, o) S[(pl) * PLANE_STRIDE + q0 + (o)]
  double dms = 0.0, dts = 0.0, dv0 = 0.0, dv1 = 0.0, dv2 = 0.0;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;  // velocity source -Qperp
  if (scal && on) {
    const double hinv = SM(S_HINV, 0);
    const double divm = (SM(S_HFM + RT, 0) - SM(S_HFM + RT, oW) + SM(S_HFM + DG, oSW) - SM(S_HFM + DG, 0) +
                         SM(S_HFM + UP, 0) - SM(S_HFM + UP, oS)) * hinv;
    const double divt = (SM(S_HFT + RT, 0) - SM(S_HFT + RT, oW) + SM(S_HFT + DG, oSW) - SM(S_HFT + DG, 0) +
                         SM(S_HFT + UP, 0) - SM(S_HFT + UP, oS)) * hinv;
    dms = -divm;
    dts = -divt;
  }
  if (own && on) {
#define TQ(e1, o1, q0v, w) (SM(S_HFM + (e1), o1) * interp(SM(S_QE + (e1), o1), (q0v)) * (w))
    double w1[5], w2[5];
    double qv = SM(S_QE + RT, 0);
    weights5_s(S, q0, 0, w1);
    weights5_s(S, q0 + oE, 3, w2);
    const double Q0 = TQ(DG, 0, qv, w1[0]) + TQ(UP, 0, qv, w1[1]) + TQ(RT, oW, qv, w1[2]) + TQ(DG, oSW, qv, w1[3]) +
                      TQ(UP, oS, qv, w1[4]) + TQ(DG, oS, qv, w2[0]) + TQ(UP, oSE, qv, w2[1]) + TQ(RT, oE, qv, w2[2]) +
                      TQ(DG, oE, qv, w2[3]) + TQ(UP, oE, qv, w2[4]);
    qv = SM(S_QE + DG, 0);
    weights5_s(S, q0, 1, w1);
    weights5_s(S, q0 + oNE, 4, w2);
    const double Q1 = TQ(UP, 0, qv, w1[0]) + TQ(RT, oW, qv, w1[1]) + TQ(DG, oSW, qv, w1[2]) + TQ(UP, oS, qv, w1[3]) +
                      TQ(RT, 0, qv, w1[4]) + TQ(UP, oE, qv, w2[0]) + TQ(RT, oNE, qv, w2[1]) + TQ(DG, oNE, qv, w2[2]) +
                      TQ(UP, oNE, qv, w2[3]) + TQ(RT, oN, qv, w2[4]);
    qv = SM(S_QE + UP, 0);
    weights5_s(S, q0, 2, w1);
    weights5_s(S, q0 + oN, 5, w2);
    const double Q2 = TQ(RT, oW, qv, w1[0]) + TQ(DG, oSW, qv, w1[1]) + TQ(UP, oS, qv, w1[2]) + TQ(RT, 0, qv, w1[3]) +
                      TQ(DG, 0, qv, w1[4]) + TQ(RT, oN, qv, w2[0]) + TQ(DG, oN, qv, w2[1]) + TQ(UP, oN, qv, w2[2]) +
                      TQ(RT, oNW, qv, w2[3]) + TQ(DG, oW, qv, w2[4]);
#undef TQ
    const double th0 = SM(S_TH, 0), thE = SM(S_TH, oE), thNE = SM(S_TH, oNE), thN = SM(S_TH, oN);
    const double gB0 = (SM(S_B, oE) - SM(S_B, 0)) / lRT, gB1 = (SM(S_B, 0) - SM(S_B, oNE)) / lDG,
                 gB2 = (SM(S_B, oN) - SM(S_B, 0)) / lUP;
    const double xE = -SM(S_F, oE), x0v = -SM(S_F, 0), xNE = -SM(S_F, oNE), xN = -SM(S_F, oN);
    const double gE0 = (xE - x0v) / lRT, gE1 = (x0v - xNE) / lDG, gE2 = (xN - x0v) / lUP;
    s0 = -Q0 + 0.0 * lRT;
    s1 = -Q1 + 0.0 * lDG;
    s2 = -Q2 + 0.0 * lUP;
    dv0 = s0 / lRT - gB0 - interp(th0, thE) * gE0;
    dv1 = s1 / lDG - gB1 - interp(th0, thNE) * gE1;
    dv2 = s2 / lUP - gB2 - interp(th0, thN) * gE2;
  }
#undef SM
  if (MODE == MODE_ML) {
    if (scal) {
      io.dm[ko + id] = dms;
      io.dtt[ko + id] = dts;
    }
    if (own) {
      io.src[vo] = s0;
      io.src[vo + NN] = s1;
      io.src[vo + 2 * NN] = s2;
    }
  }
  if (MODE == MODE_ML && io.grad) {  // u_star
    const double h = io.h, t1 = io.th1;
    io.dst_m[ko + id] = bm + h * dms;
    io.dst_t[ko + id] = bt + h * dts;
    io.dst_v[vo] = bv0 + h * (dv0 + t1 * io.grad[id]);
    io.dst_v[vo + NN] = bv1 + h * (dv1 + t1 * io.grad[NN + id]);
    io.dst_v[vo + 2 * NN] = bv2 + h * (dv2 + t1 * io.grad[2 * NN + id]);
  } else if (MODE == MODE_RK || MODE == MODE_ML) {
    const double h = io.h;
    io.dst_m[ko + id] = bm + h * dms;
    io.dst_t[ko + id] = bt + h * dts;
    io.dst_v[vo] = bv0 + h * dv0;
    io.dst_v[vo + NN] = bv1 + h * dv1;
    io.dst_v[vo + 2 * NN] = bv2 + h * dv2;
  } else {
    io.dm[ko + id] = dms;
    io.dtt[ko + id] = dts;
    io.dv[vo] = dv0;
    io.dv[vo + NN] = dv1;
    io.dv[vo + 2 * NN] = dv2;
  }
}

}  // namespace wtk

namespace wtk {

// --------------------------------------------------------------------------
// step1 (comput/comp_SW/post_step1, src/ops.f90:276-366, 472-522, 526-737)
// with its inputs staged by TMA.  Tiles cover the computed range [0, n]^2:
// tile (bx, by) starts at padded (2 + TT_X*bx, 2 + TT_Y*by), so the box starts
// at x = TT_X*bx (even) and y = 1 + TT_Y*by.
enum {
  P1_M = 0, P1_T = 1, P1_AM = 2, P1_AT = 3, P1_V = 4, P1_LEN = 7, P1_PED = 10, P1_PART = 13, P1_COR = 19,
  P1_NPLANE = 21
};
constexpr int STEP1_TMA_SMEM = P1_NPLANE * PLANE_BYTES + 64;
constexpr unsigned STEP1_TMA_TX = P1_NPLANE * TB_N * 8;

__global__ void __launch_bounds__(TT_X * TT_Y, 3)
    k_step1_tma(LevelDev L, int nz, int nbx, int nby, const double* __restrict__ mass, const double* __restrict__ temp,
                const double* __restrict__ velo, const double* __restrict__ mean_m,
                const double* __restrict__ phik, const double* __restrict__ pterm, Step1Out out,
                int* __restrict__ err, int inject, const __grid_constant__ Step1Maps M,
                const unsigned char* __restrict__ need) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* __restrict__ S = reinterpret_cast<double*>(smem_raw);
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t bar = s_base + P1_NPLANE * PLANE_BYTES;

  int b = blockIdx.x;
  const int k = b % nz;
  b /= nz;
  const int bx = b % nbx;
  b /= nbx;
  const int by = b % nby;
  const int d = b / nby;
  const int cx = TT_X * bx, cy = 1 + TT_Y * by;  // box origin (padded coordinates)
  const int tid = threadIdx.x;
  if (need) {  // a tile none of whose nodes is needed is left out, before any copy is issued
    const int ni = cx + tid % TT_X, nj = cy - 1 + tid / TT_X;
    int v = 0;
    if (ni <= L.n && nj <= L.n) v = need[__ldg(L.nsrc + (d * L.P + nj + 2) * L.P + ni + 2)];
    if (!__syncthreads_or(v)) return;
  }

  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(bar, STEP1_TMA_TX + (inject ? TMA_INJECT_TX : 0u));
    tma_load_4d(s_base + P1_M * PLANE_BYTES, &M.mass, cx, cy, d, k, bar);
    tma_load_4d(s_base + P1_T * PLANE_BYTES, &M.temp, cx, cy, d, k, bar);
    tma_load_4d(s_base + P1_AM * PLANE_BYTES, &M.mean_m, cx, cy, d, k, bar);
    tma_load_4d(s_base + P1_AT * PLANE_BYTES, &M.mean_t, cx, cy, d, k, bar);
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      tma_load_4d(s_base + (P1_V + e) * PLANE_BYTES, &M.velo, cx, cy, d, 3 * k + e, bar);
      tma_load_4d(s_base + (P1_LEN + e) * PLANE_BYTES, &M.len, cx, cy, d, e, bar);
      tma_load_4d(s_base + (P1_PED + e) * PLANE_BYTES, &M.ped, cx, cy, d, e, bar);
    }
#pragma unroll
    for (int r = 0; r < 6; ++r) tma_load_4d(s_base + (P1_PART + r) * PLANE_BYTES, &M.part, cx, cy, d, r, bar);
    tma_load_4d(s_base + (P1_COR + 0) * PLANE_BYTES, &M.cor, cx, cy, d, 0, bar);
    tma_load_4d(s_base + (P1_COR + 1) * PLANE_BYTES, &M.cor, cx, cy, d, 1, bar);
  }

  const int P = L.P, NN = L.NN, n = L.n;
  const int tx = tid % TT_X, ty = tid / TT_X;
  const int i = cx + tx, j = cy - 1 + ty;  // (i, j) = padded - 2
  const bool act = i <= n && j <= n;       // i, j >= 0 by construction
  const int id = (d * P + j + 2) * P + i + 2;
  const int64_t ko = (int64_t)k * NN;
  double ph_k = 0.0, pt_k = 0.0, hinv = 0.0;
  if (act) {
    ph_k = phik[ko + id];
    pt_k = pterm[ko + id];
    hinv = L.hex_inv[id];
  }

  const bool ok = mbar_wait_bounded(bar, 0, inject ? TMA_INJECT_WAIT_NS : TMA_WAIT_NS);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicCAS(err, 0, 1);
      if (inject) mbar_complete_tx(bar, TMA_INJECT_TX);
    }
    if (!ok) mbar_wait_bounded(bar, 0);  // copies still in flight target this block's shared memory
    return;
  }

  // Ghost state: slots outside [1, n-2]^2 take the node / signed edge named by
  // the remap tables (update_bdry of the prognostic variables).
  const int sx0 = cx - 2, sy0 = cy - 2;  // node coordinates of slot (0, 0)
  if (sx0 < 1 || sy0 < 1 || sx0 + TB_X - 1 > n - 2 || sy0 + TB_Y - 1 > n - 2) {
    const double* __restrict__ Mm = mass + ko;
    const double* __restrict__ Mt = temp + ko;
    const double* __restrict__ V = velo + 3 * ko;
    for (int q = tid; q < TB_N; q += TT_X * TT_Y) {
      const int sx = q % TB_X, sy = q / TB_X;
      const int pi = cx + sx, pj = cy + sy;
      if (pi < 0 || pj < 0 || pi >= P || pj >= P) continue;
      const int si = pi - 2, sj = pj - 2;
      if (si >= 1 && sj >= 1 && si <= n - 2 && sj <= n - 2) continue;
      const int x = (d * P + pj) * P + pi;
      const int src = __ldg(L.nsrc + x);
      S[P1_M * PLANE_STRIDE + q] = Mm[src];
      S[P1_T * PLANE_STRIDE + q] = Mt[src];
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        const int c = __ldg(L.esrc + e * NN + x);
        const double v = V[c >> 1];
        S[(P1_V + e) * PLANE_STRIDE + q] = (c & 1) ? -v : v;
      }
    }
  }
  __syncthreads();
  if (!act) return;

  const int q0 = (ty + 1) * TB_X + (tx + 2);
  constexpr int oE = 1, oW = -1, oN = TB_X, oS = -TB_X, oNE = TB_X + 1, oSW = -TB_X - 1;
  const int idW = id - 1, idS = id - P, idSW = id - P - 1;
#define SM(pl, o) S[(pl) * PLANE_STRIDE + q0 + (o)]
#define RHO(o) (SM(P1_M, o) + SM(P1_AM, o))
#define THT(o) (SM(P1_T, o) + SM(P1_AT, o))
#define VEL(e, o) SM(P1_V + (e), o)
#define LEN(e, o) SM(P1_LEN + (e), o)
#define PED(e, o) SM(P1_PED + (e), o)
#define PART(o, kk) SM(P1_PART + (kk) - 1, o)
#define COR(t, o) SM(P1_COR + (t), o)
  double* __restrict__ qe = out.qe + 3 * ko;
  double* __restrict__ hfm = out.hfm + 3 * ko;
  double* __restrict__ hft = out.hft + 3 * ko;

  const double r0 = RHO(0), rN = RHO(oN), rE = RHO(oE), rS = RHO(oS), rW = RHO(oW), rNE = RHO(oNE);
  const double t0 = THT(0);
  out.theta[ko + id] = t0 / r0;
  const double vRT = VEL(RT, 0), vDG = VEL(DG, 0), vUP = VEL(UP, 0);
  const double vRT_W = VEL(RT, oW), vDG_SW = VEL(DG, oSW), vUP_S = VEL(UP, oS);
  const double u_dual_RT = vRT * PED(RT, 0);
  const double u_dual_DG = vDG * PED(DG, 0);
  const double u_dual_UP = vUP * PED(UP, 0);
  const double u_dual_RT_W = vRT_W * PED(RT, oW);
  const double u_dual_DG_SW = vDG_SW * PED(DG, oSW);
  const double u_dual_UP_S = vUP_S * PED(UP, oS);

  const double u_prim_RT = vRT * LEN(RT, 0);
  const double u_prim_RT_W = vRT_W * LEN(RT, oW);
  const double u_prim_DG = vDG * LEN(DG, 0);
  const double u_prim_DG_SW = vDG_SW * LEN(DG, oSW);
  const double u_prim_UP = vUP * LEN(UP, 0);
  const double u_prim_UP_S = vUP_S * LEN(UP, oS);
  const double u_prim_DG_W = VEL(DG, oW) * LEN(DG, oW);
  const double u_prim_UP_E = VEL(UP, oE) * LEN(UP, oE);

  const double circ_LORT = u_prim_RT + u_prim_UP_E + u_prim_DG;
  const double circ_W_LORT = u_prim_RT_W + u_prim_UP + u_prim_DG_W;
  const double pv_LORT = (COR(LORT, 0) + circ_LORT) / (r0 * PART(0, 1) + rE * PART(oE, 3) + rNE * PART(oNE, 5));
  const double pv_W_LORT = (COR(LORT, oW) + circ_W_LORT) / (rW * PART(oW, 1) + r0 * PART(0, 3) + rN * PART(oN, 5));
  const double u_prim_RT_N = VEL(RT, oN) * LEN(RT, oN);
  const double circ_UPLT = -(u_prim_DG + u_prim_UP + u_prim_RT_N);
  const double pv_UPLT = (COR(UPLT, 0) + circ_UPLT) / (r0 * PART(0, 2) + rNE * PART(oNE, 4) + rN * PART(oN, 6));
  const double u_prim_DG_S = VEL(DG, oS) * LEN(DG, oS);
  const double circ_S_UPLT = -(u_prim_RT + u_prim_DG_S + u_prim_UP_S);
  const double pv_S_UPLT = (COR(UPLT, oS) + circ_S_UPLT) / (rS * PART(oS, 2) + rE * PART(oE, 4) + r0 * PART(0, 6));

  qe[RT * NN + id] = interp(pv_S_UPLT, pv_LORT);
  qe[DG * NN + id] = interp(pv_UPLT, pv_LORT);
  // comp_SW at (0, j+1) rewrites qe(UP) of (0, j) after comput; that value is
  // written by comp_SW below.
  if (!(i == 0 && j < n)) qe[UP * NN + id] = interp(pv_UPLT, pv_W_LORT);

  const double ke = (u_prim_UP * u_dual_UP + u_prim_DG * u_dual_DG + u_prim_RT * u_dual_RT + u_prim_UP_S * u_dual_UP_S +
                     u_prim_DG_SW * u_dual_DG_SW + u_prim_RT_W * u_dual_RT_W) *
                    hinv / 4.0;
  out.bern[ko + id] = ke + ph_k + pt_k;

  hfm[RT * NN + id] = u_dual_RT * interp(r0, rE) + 0.0;
  hfm[DG * NN + id] = u_dual_DG * interp(r0, rNE) + 0.0;
  hfm[UP * NN + id] = u_dual_UP * interp(r0, rN) + 0.0;
  hft[RT * NN + id] = u_dual_RT * interp(t0, THT(oE)) + 0.0;
  hft[DG * NN + id] = u_dual_DG * interp(t0, THT(oNE)) + 0.0;
  hft[UP * NN + id] = u_dual_UP * interp(t0, THT(oN)) + 0.0;

  if (i == 0 || j == 0) {  // comp_SW
    const double rSW = RHO(oSW);
    const double tS = THT(oS), tW = THT(oW), tSW = THT(oSW);
    const double u_prim_RT_SW = VEL(RT, oSW) * LEN(RT, oSW);
    const double u_prim_UP_SW = VEL(UP, oSW) * LEN(UP, oSW);
    const double circ_SW_LORT = u_prim_RT_SW + u_prim_UP_S + u_prim_DG_SW;
    const double circ_SW_UPLT = -(u_prim_RT_W + u_prim_DG_SW + u_prim_UP_SW);
    const double qm1 = rSW * PART(oSW, 1) + rS * PART(oS, 3) + r0 * PART(0, 5);
    const double qm2 = rSW * PART(oSW, 2) + r0 * PART(0, 4) + rW * PART(oW, 6);
    const double pv_SW_LORT = (COR(LORT, oSW) + circ_SW_LORT) / qm1;
    const double pv_SW_UPLT = (COR(UPLT, oSW) + circ_SW_UPLT) / qm2;
    if (i == 0) {
      qe[RT * NN + idW] = interp(pv_W_LORT, pv_SW_UPLT);
      hfm[RT * NN + idW] = u_dual_RT_W * interp(r0, rW) + 0.0;
      hft[RT * NN + idW] = u_dual_RT_W * interp(t0, tW) + 0.0;
    }
    qe[DG * NN + idSW] = interp(pv_SW_LORT, pv_SW_UPLT);
    qe[UP * NN + idS] = interp(pv_SW_LORT, pv_S_UPLT);
    hfm[DG * NN + idSW] = u_dual_DG_SW * interp(r0, rSW) + 0.0;
    hfm[UP * NN + idS] = u_dual_UP_S * interp(r0, rS) + 0.0;
    hft[DG * NN + idSW] = u_dual_DG_SW * interp(t0, tSW) + 0.0;
    hft[UP * NN + idS] = u_dual_UP_S * interp(t0, tS) + 0.0;
  }
#undef SM
#undef RHO
#undef THT
#undef VEL
#undef LEN
#undef PED
#undef PART
#undef COR
  if ((i == 0 || i == n) && (j == 0 || j == n)) {
    const int c = (i == n) ? (j == n ? 0 : 1) : (j == 0 ? 2 : 3);
    post_corner(L, c, d, ko, mass, velo, mean_m, out.qe);
  }
}

}  // namespace wtk
