// Trend of one level of the multi-level trend_ml (src/multi_level.f90:5-188):
// scalar_trend with its mask, the velocity source computed (du_source) or
// restricted from the child level (u_source_cpt_restr, src/multi_level.f90:
// 365-392), and du_grad with its mask (src/ops.f90:739-832), in one pass per
// (layer, node).  The Bernoulli function, Phi_k and the mass and Theta fluxes
// it reads are those of the level after their compute-or-restrict step.
#pragma once
#include "trisk_read.cuh"

namespace wtk {

struct TrendML {
  const double* __restrict__ theta;  // Theta/rho of the level's state (k_step1)
  const double* __restrict__ qe;
  const double* __restrict__ hfm;
  const double* __restrict__ hft;
  const double* __restrict__ bern;
  const double* __restrict__ phik;    // exner = -Phi_k
  const int* __restrict__ mask_n;     // [NN] of the level
  const int* __restrict__ mask_e_chd; // [3*NN_chd] of level+1; null on level_end
  const double* __restrict__ src_chd; // [nz][3][NN_chd] velocity sources of level+1; null on level_end
  int P_chd, NN_chd;
  double* dm;
  double* dtt;
  double* dv;                         // may be null when the RK sub-step is fused (dst_* set)
  double* src;                        // [nz][3][NN] velocity sources of this level (for level-1)
  // RK_sub_step fused (src/time_integr.f90:206-225): dst = base + h * trend on
  // every padded node of the level, the trend being 0 where it is not computed.
  const double* base_m; const double* base_t; const double* base_v;
  double* dst_m; double* dst_t; double* dst_v;
  double h;
  // needed-node map (need_map.cuh) of the finest level, or null: nodes with
  // need[nsrc[id]] == 0 write nothing
  const unsigned char* need;
  // u_star (src/barotropic_2d.f90:29-50) when grad is set: the velocity sub-step
  // is base + h * (trend + th1 * grad), grad the level's external pressure
  // gradient [3][NN] (grad_eta)
  const double* grad;
  double th1;
};

constexpr int ML_TRSK = 2, ML_ADJZONE = 8;

__device__ __forceinline__ void trend_ml_node(const LevelDev& L, int nz, const TrendML& io, int k, int id, int i,
                                              int j);

__global__ void __launch_bounds__(NODE_TILE, 4) k_trend_ml(LevelDev L, int nz, TrendML io) {
  int k, id, i, j;
  if (!layer_node(L, nz, k, id, i, j)) return;
  if (io.need && !io.need[__ldg(L.nsrc + id)]) return;
  trend_ml_node(L, nz, io, k, id, i, j);
}

// The same over a work list (persistent blocks): the list holds the padded
// slots of the needed-node map.
#ifndef WT_ML_LIST_MINB
#define WT_ML_LIST_MINB 3
#endif
__global__ void __launch_bounds__(NODE_TILE, WT_ML_LIST_MINB)
    k_trend_ml_list(LevelDev L, int nz, TrendML io, NodeList W) {
  const int cnt = __ldg(W.count);
  for (int64_t w = blockIdx.x; w < list_items(cnt, nz); w += gridDim.x) {
    int k, id, i, j;
    if (list_entry(L, nz, W, cnt, w, k, id, i, j)) trend_ml_node(L, nz, io, k, id, i, j);
  }
}

__device__ __forceinline__ void trend_ml_node(const LevelDev& L, int nz, const TrendML& io, int k, int id, int i,
                                              int j) {
  const int P = L.P;
  const int NN = L.NN;
  const int n = L.n;
  const int64_t ko = (int64_t)k * NN;
  const int64_t vo = 3 * ko + id;
  const bool rk = io.dst_m != nullptr;
  const Rd R(L, i >= 1 && j >= 1 && i <= n - 2 && j <= n - 2);
  const bool on = io.mask_n[id] >= ML_TRSK;
  double dms = 0.0, dts = 0.0;
  if (i >= 0 && j >= 0 && i <= n && j <= n) {
    if (on) {
      const int idW = id - 1, idS = id - P, idSW = id - P - 1;
      const double* __restrict__ fm = io.hfm + 3 * ko;
      const double* __restrict__ ft = io.hft + 3 * ko;
      const double hinv = L.hex_inv[id];
      const double divm = (R.e(fm, RT * NN + id) - R.e(fm, RT * NN + idW) + R.e(fm, DG * NN + idSW) -
                           R.e(fm, DG * NN + id) + R.e(fm, UP * NN + id) - R.e(fm, UP * NN + idS)) * hinv;
      const double divt = (R.e(ft, RT * NN + id) - R.e(ft, RT * NN + idW) + R.e(ft, DG * NN + idSW) -
                           R.e(ft, DG * NN + id) + R.e(ft, UP * NN + id) - R.e(ft, UP * NN + idS)) * hinv;
      dms = -divm;
      dts = -divt;
    }
    io.dm[ko + id] = dms;
    io.dtt[ko + id] = dts;
  }
  double dv3[3] = {0.0, 0.0, 0.0};
  if (i >= 0 && j >= 0 && i < n && j < n) {
    const double len3[3] = {L.len[RT * NN + id], L.len[DG * NN + id], L.len[UP * NN + id]};
    double s[3];
    bool restr[3] = {false, false, false};
    if (io.src_chd) {
      const int d = id / (P * P);
      const int Pc = io.P_chd, NC = io.NN_chd;
      const int idc = (d * Pc + 2 * j + 2) * Pc + 2 * i + 2;
      const int nbc[3] = {1, Pc + 1, Pc};  // E, NE, N child of the edge
      const double* __restrict__ sc = io.src_chd + (int64_t)3 * k * NC;
#pragma unroll
      for (int e = 0; e < 3; ++e)
        if (io.mask_e_chd[e * NC + idc] >= ML_ADJZONE) {
          restr[e] = true;
          s[e] = sc[e * NC + idc] + sc[e * NC + idc + nbc[e]];
        }
    }
    if (!(restr[0] && restr[1] && restr[2])) {
      double Q[3] = {0.0, 0.0, 0.0};
      if (on) qperp(L, R, io.hfm + 3 * ko, io.qe + 3 * ko, id, Q);
#pragma unroll
      for (int e = 0; e < 3; ++e)
        if (!restr[e]) s[e] = on ? -Q[e] + 0.0 * len3[e] : 0.0;
    }
#pragma unroll
    for (int e = 0; e < 3; ++e) io.src[vo + e * NN] = s[e];
    if (on) {
      const int idN = id + P, idNE = id + P + 1, idE = id + 1;
      const double* __restrict__ th = io.theta + ko;
      const double th0 = th[id], thE = th[idE], thNE = th[idNE], thN = th[idN];
      const double* __restrict__ B = io.bern + ko;
      const double* __restrict__ F = io.phik + ko;
      const double gB0 = (B[idE] - B[id]) / len3[0], gB1 = (B[id] - B[idNE]) / len3[1],
                   gB2 = (B[idN] - B[id]) / len3[2];
      const double xE = -F[idE], x0 = -F[id], xNE = -F[idNE], xN = -F[idN];
      const double gE0 = (xE - x0) / len3[0], gE1 = (x0 - xNE) / len3[1], gE2 = (xN - x0) / len3[2];
      dv3[0] = s[0] / len3[0] - gB0 - interp(th0, thE) * gE0;
      dv3[1] = s[1] / len3[1] - gB1 - interp(th0, thNE) * gE1;
      dv3[2] = s[2] / len3[2] - gB2 - interp(th0, thN) * gE2;
    }
    if (io.dv) {
#pragma unroll
      for (int e = 0; e < 3; ++e) io.dv[vo + e * NN] = dv3[e];
    }
  }
  if (rk) {
    const double h = io.h;
    io.dst_m[ko + id] = io.base_m[ko + id] + h * dms;
    io.dst_t[ko + id] = io.base_t[ko + id] + h * dts;
#pragma unroll
    for (int e = 0; e < 3; ++e)
      io.dst_v[vo + e * NN] = io.grad ? io.base_v[vo + e * NN] + h * (dv3[e] + io.th1 * io.grad[e * NN + id])
                                      : io.base_v[vo + e * NN] + h * dv3[e];
  }
}

}  // namespace wtk
