// Mixed-precision TRiSK: the flux stencils of step1 in FP32 inside the FP64
// step (the reduced-precision pattern of the single-level stepper).
//
// k_step1_f32 evaluates comput/comp_SW (src/ops.f90:276-366, 472-522) and
// post_step1 (:526-737) with FP32 arithmetic and FP32 results: the potential
// vorticity qe, the mass and Theta fluxes, the kinetic energy and Theta/rho.
// Its inputs are the FP64 state (rho dz = mean + perturbation is formed in
// FP64 and then rounded) and the FP64 geometry (rounded on load).  The
// Bernoulli function is not formed in FP32: its geopotential and pressure
// parts are four orders of magnitude larger than the kinetic energy, and their
// gradient would lose most of its digits; k_trend_mixed forms
// B = ke + Phi_k + p/rho0 in FP64 from the FP32 kinetic energy and the FP64
// column results.
//
// k_trend_mixed evaluates scalar_trend, du_source/Qperp and du_grad in FP64
// arithmetic on the FP32 inputs (each widened exactly), and the RK sub-step
// in FP64: every flux is one value shared by the two cells it joins, so the
// FP64 divergence conserves mass and Theta to FP64 rounding, and the stage
// accumulation stays FP64.  Per node-layer and stage the pair moves 256
// algorithmic bytes where the FP64 pair moves 336 (step1 writes 11 FP32 words
// instead of 11 FP64 words; the trend reads them and two FP64 words instead
// of 12 FP64 words).
#pragma once
#include <cstdint>

#include "trisk_read.cuh"
#include "trisk_types.cuh"

namespace wtk {

struct Step1OutF {
  float* __restrict__ qe;     // [nz][3][NN]
  float* __restrict__ hfm;    // [nz][3][NN]
  float* __restrict__ hft;    // [nz][3][NN]
  float* __restrict__ ke;     // [nz][NN]
  float* __restrict__ theta;  // [nz][NN]
};

struct TrendIOF {
  const float* __restrict__ theta;
  const float* __restrict__ qe;
  const float* __restrict__ hfm;
  const float* __restrict__ hft;
  const float* __restrict__ ke;
  const double* __restrict__ phik;
  const double* __restrict__ pterm;
  const double* base_m; const double* base_t; const double* base_v;
  double* dst_m; double* dst_t; double* dst_v;
  double h;
  double* dm; double* dtt; double* dv;
};

__device__ __forceinline__ float interpf(float a, float b) { return 0.5f * (a + b); }

// Reads through the ghost remap, FP32 results.
struct RdF {
  const int* __restrict__ nsrc;
  const int* __restrict__ esrc;
  bool direct;
  __device__ __forceinline__ RdF(const LevelDev& L, bool dir) : nsrc(L.nsrc), esrc(L.esrc), direct(dir) {}
  __device__ __forceinline__ int nx(int x) const { return direct ? x : __ldg(nsrc + x); }
  __device__ __forceinline__ float ed(const double* __restrict__ f, int slot) const {
    if (direct) return (float)f[slot];
    const int c = __ldg(esrc + slot);
    const double v = f[c >> 1];
    return (float)((c & 1) ? -v : v);
  }
  __device__ __forceinline__ double ef(const float* __restrict__ f, int slot) const {  // widened
    if (direct) return (double)f[slot];
    const int c = __ldg(esrc + slot);
    const double v = (double)f[c >> 1];
    return (c & 1) ? -v : v;
  }
};

// post_step1 at a pentagon corner (FP32 twin of post_corner).
__device__ __noinline__ void post_corner_f32(const LevelDev L, int c, int d, int64_t ko, const double* __restrict__ mass,
                                             const double* __restrict__ velo, const double* __restrict__ mean_m,
                                             float* __restrict__ qe) {
  const int n = L.n;
  const int64_t NN = L.NN;
  const RdF R(L, false);
  const double* v = velo + 3 * ko;
  auto rho = [&](int64_t x) { return (float)(mass[ko + R.nx((int)x)] + mean_m[ko + x]); };
  auto pr = [&](int e, int64_t x) { return R.ed(v, (int)(e * NN + x)) * (float)L.len[e * NN + x]; };
  auto part = [&](int64_t x, int kk) { return (float)L.part[(int64_t)(kk - 1) * NN + x]; };
  auto tri = [&](int tt, int64_t x) { return (float)L.triarea[(int64_t)tt * NN + x]; };
  auto cor = [&](int tt, int64_t x) { return (float)L.coriolis[(int64_t)tt * NN + x]; };
  auto I = [&](int i, int j) { return nid(L, d, i, j); };
  float* q = qe + 3 * ko;
  if (c == 0) {  // north-east corner
    int64_t id = I(n, n), idN = I(n, n + 1), idE = I(n + 1, n), idS = I(n, n - 1), idW = I(n - 1, n);
    float r0 = rho(id), rN = rho(idN), rE = rho(idE), rS = rho(idS), rW = rho(idW);
    float circ_LORT = pr(RT, id) - pr(RT, idN) - pr(UP, id);
    float vW = (pr(RT, idW) + pr(UP, id) + pr(DG, idW)) / tri(LORT, idW);
    float vS = -(pr(DG, idS) + pr(UP, idS) + pr(RT, id)) / tri(UPLT, idS);
    float pm1 = rE * part(idE, 3) + r0 * (part(id, 1) + part(id, 2)) + rN * part(idN, 6);
    float pm2 = rW * part(idW, 1) + r0 * part(id, 3) + rN * part(idN, 5);
    float pm3 = rS * part(idS, 2) + rE * part(idE, 4) + r0 * part(id, 6);
    float pv_LORT = (cor(LORT, id) + circ_LORT) / pm1;
    float pv_W_LORT = (cor(LORT, idW) + vW * tri(LORT, idW)) / pm2;
    float pv_S_UPLT = (cor(UPLT, idS) + vS * tri(UPLT, idS)) / pm3;
    q[(int64_t)RT * NN + id] = interpf(pv_LORT, pv_S_UPLT);
    q[(int64_t)UP * NN + id] = interpf(pv_LORT, pv_W_LORT);
  } else if (c == 1) {  // south-east corner
    int64_t id = I(n, 0), idE = I(n + 1, 0), idS = I(n, -1), idW = I(n - 1, 0), idNE = I(n + 1, 1), idSW = I(n - 1, -1);
    float r0 = rho(id), rE = rho(idE), rS = rho(idS), rW = rho(idW), rNE = rho(idNE), rSW = rho(idSW);
    float circ_SW_LORT = -pr(RT, id) + pr(RT, idSW) + pr(DG, idSW);
    float vL = (pr(RT, id) + pr(UP, idE) + pr(DG, id)) / tri(LORT, id);
    float vU = -(pr(RT, idW) + pr(DG, idSW) + pr(UP, idSW)) / tri(UPLT, idSW);
    float pm1 = rSW * part(idSW, 1) + rS * part(idS, 3) + r0 * (part(id, 5) + part(id, 6));
    float pm2 = r0 * part(id, 1) + rE * part(idE, 3) + rNE * part(idNE, 5);
    float pm3 = rSW * part(idSW, 2) + r0 * part(id, 4) + rW * part(idW, 6);
    float pv_SW_LORT = (cor(LORT, idSW) + circ_SW_LORT) / pm1;
    float pv_LORT = (cor(LORT, id) + vL * tri(LORT, id)) / pm2;
    float pv_SW_UPLT = (cor(UPLT, idSW) + vU * tri(UPLT, idSW)) / pm3;
    q[(int64_t)RT * NN + id] = interpf(pv_SW_LORT, pv_LORT);
    q[(int64_t)DG * NN + idSW] = interpf(pv_SW_LORT, pv_SW_UPLT);
  } else if (c == 2) {  // south-west corner
    int64_t id = I(0, 0), idN = I(0, 1), idE = I(1, 0), idS = I(0, -1), idW = I(-1, 0), idSW = I(-1, -1);
    float r0 = rho(id), rN = rho(idN), rE = rho(idE), rS = rho(idS), rW = rho(idW);
    float circ_SW_LORT = pr(UP, idS) - pr(RT, idW) + pr(RT, idSW);
    float vW = (pr(RT, idW) + pr(UP, id) + pr(DG, idW)) / tri(LORT, idW);
    float vS = -(pr(RT, id) + pr(DG, idS) + pr(UP, idS)) / tri(UPLT, idS);
    float pm1 = rW * part(idW, 6) + r0 * (part(id, 4) + part(id, 5)) + rS * part(idS, 3);
    float pm2 = rW * part(idW, 1) + r0 * part(id, 3) + rN * part(idN, 5);
    float pm3 = rS * part(idS, 2) + rE * part(idE, 4) + r0 * part(id, 6);
    float pv_W_LORT = (cor(LORT, idW) + vW * tri(LORT, idW)) / pm1;
    float pv_SW_LORT = (cor(LORT, idSW) + circ_SW_LORT) / pm2;
    float pv_S_UPLT = (cor(UPLT, idS) + vS * tri(UPLT, idS)) / pm3;
    q[(int64_t)RT * NN + idW] = interpf(pv_W_LORT, pv_SW_LORT);
    q[(int64_t)UP * NN + idS] = interpf(pv_S_UPLT, pv_SW_LORT);
  } else {  // north-west corner
    int64_t id = I(0, n), idN = I(0, n + 1), idS = I(0, n - 1), idW = I(-1, n), idNE = I(1, n + 1), idSW = I(-1, n - 1);
    float r0 = rho(id), rN = rho(idN), rS = rho(idS), rW = rho(idW), rNE = rho(idNE), rSW = rho(idSW);
    float circ_SW_UPLT = pr(UP, id) - pr(DG, idSW) - pr(UP, idSW);
    float vU = -(pr(DG, id) + pr(UP, id) + pr(RT, idN)) / tri(UPLT, id);
    float vL = (pr(RT, idSW) + pr(UP, idS) + pr(DG, idSW)) / tri(LORT, idSW);
    float pm1 = rSW * part(idSW, 2) + r0 * (part(id, 3) + part(id, 4)) + rW * part(idW, 6);
    float pm2 = r0 * part(id, 2) + rNE * part(idNE, 4) + rN * part(idN, 6);
    float pm3 = rSW * part(idSW, 1) + rS * part(idS, 3) + r0 * part(id, 5);
    float pv_SW_UPLT = (cor(UPLT, idSW) + circ_SW_UPLT) / pm1;
    float pv_UPLT = (cor(UPLT, id) + vU * tri(UPLT, id)) / pm2;
    float pv_SW_LORT = (cor(LORT, idSW) + vL * tri(LORT, idSW)) / pm3;
    q[(int64_t)UP * NN + id] = interpf(pv_SW_UPLT, pv_UPLT);
    q[(int64_t)DG * NN + idSW] = interpf(pv_SW_LORT, pv_SW_UPLT);
  }
}

// step1 itype 0 in FP32 on [0, n]^2, with the edge ownership of k_step1.
__global__ void __launch_bounds__(NODE_TILE, 4)
    k_step1_f32(LevelDev L, int nz, const double* __restrict__ mass, const double* __restrict__ temp,
                const double* __restrict__ velo, const double* __restrict__ mean_m, const double* __restrict__ mean_t,
                Step1OutF out) {
  int k, id, i, j;
  if (!layer_node(L, nz, k, id, i, j)) return;
  if (i < 0 || j < 0 || i > L.n || j > L.n) return;
  const int NN = L.NN;
  const int P = L.P;
  const int idN = id + P, idE = id + 1, idS = id - P, idW = id - 1, idNE = id + P + 1, idSW = id - P - 1;
  const int64_t ko = (int64_t)k * NN;
  const RdF R(L, i >= 1 && j >= 1 && i <= L.n - 2 && j <= L.n - 2);
  const double* __restrict__ Mm = mass + ko;
  const double* __restrict__ Mt = temp + ko;
  const double* __restrict__ Am = mean_m + ko;
  const double* __restrict__ At = mean_t + ko;
  const double* __restrict__ v = velo + 3 * ko;
  float* __restrict__ qe = out.qe + 3 * ko;
  float* __restrict__ hfm = out.hfm + 3 * ko;
  float* __restrict__ hft = out.hft + 3 * ko;
  const double* __restrict__ len = L.len;
  const double* __restrict__ ped = L.pedlen;
  const double* __restrict__ part = L.part;
  const double* __restrict__ cor = L.coriolis;
#define E3(e, x) ((e) * NN + (x))
#define PART(x, kk) ((float)part[((kk) - 1) * NN + (x)])
#define RHO(F, A, x) ((float)(F[R.nx(x)] + A[x]))
  const float r0 = RHO(Mm, Am, id), rN = RHO(Mm, Am, idN), rE = RHO(Mm, Am, idE), rS = RHO(Mm, Am, idS),
              rW = RHO(Mm, Am, idW), rNE = RHO(Mm, Am, idNE);
  const float t0 = RHO(Mt, At, id);
  out.theta[ko + id] = t0 / r0;
  const float vRT = R.ed(v, E3(RT, id)), vDG = R.ed(v, E3(DG, id)), vUP = R.ed(v, E3(UP, id));
  const float vRT_W = R.ed(v, E3(RT, idW)), vDG_SW = R.ed(v, E3(DG, idSW)), vUP_S = R.ed(v, E3(UP, idS));
  const float u_dual_RT = vRT * (float)ped[E3(RT, id)];
  const float u_dual_DG = vDG * (float)ped[E3(DG, id)];
  const float u_dual_UP = vUP * (float)ped[E3(UP, id)];
  const float u_dual_RT_W = vRT_W * (float)ped[E3(RT, idW)];
  const float u_dual_DG_SW = vDG_SW * (float)ped[E3(DG, idSW)];
  const float u_dual_UP_S = vUP_S * (float)ped[E3(UP, idS)];
  const float u_prim_RT = vRT * (float)len[E3(RT, id)];
  const float u_prim_RT_W = vRT_W * (float)len[E3(RT, idW)];
  const float u_prim_DG = vDG * (float)len[E3(DG, id)];
  const float u_prim_DG_SW = vDG_SW * (float)len[E3(DG, idSW)];
  const float u_prim_UP = vUP * (float)len[E3(UP, id)];
  const float u_prim_UP_S = vUP_S * (float)len[E3(UP, idS)];
  const float u_prim_DG_W = R.ed(v, E3(DG, idW)) * (float)len[E3(DG, idW)];
  const float u_prim_UP_E = R.ed(v, E3(UP, idE)) * (float)len[E3(UP, idE)];

  const float circ_LORT = u_prim_RT + u_prim_UP_E + u_prim_DG;
  const float circ_W_LORT = u_prim_RT_W + u_prim_UP + u_prim_DG_W;
  const float pv_LORT =
      ((float)cor[E3(LORT, id)] + circ_LORT) / (r0 * PART(id, 1) + rE * PART(idE, 3) + rNE * PART(idNE, 5));
  const float pv_W_LORT =
      ((float)cor[E3(LORT, idW)] + circ_W_LORT) / (rW * PART(idW, 1) + r0 * PART(id, 3) + rN * PART(idN, 5));
  const float u_prim_RT_N = R.ed(v, E3(RT, idN)) * (float)len[E3(RT, idN)];
  const float circ_UPLT = -(u_prim_DG + u_prim_UP + u_prim_RT_N);
  const float pv_UPLT =
      ((float)cor[E3(UPLT, id)] + circ_UPLT) / (r0 * PART(id, 2) + rNE * PART(idNE, 4) + rN * PART(idN, 6));
  const float u_prim_DG_S = R.ed(v, E3(DG, idS)) * (float)len[E3(DG, idS)];
  const float circ_S_UPLT = -(u_prim_RT + u_prim_DG_S + u_prim_UP_S);
  const float pv_S_UPLT =
      ((float)cor[E3(UPLT, idS)] + circ_S_UPLT) / (rS * PART(idS, 2) + rE * PART(idE, 4) + r0 * PART(id, 6));

  qe[E3(RT, id)] = interpf(pv_S_UPLT, pv_LORT);
  qe[E3(DG, id)] = interpf(pv_UPLT, pv_LORT);
  if (!(i == 0 && j < L.n)) qe[E3(UP, id)] = interpf(pv_UPLT, pv_W_LORT);

  out.ke[ko + id] = (u_prim_UP * u_dual_UP + u_prim_DG * u_dual_DG + u_prim_RT * u_dual_RT +
                     u_prim_UP_S * u_dual_UP_S + u_prim_DG_SW * u_dual_DG_SW + u_prim_RT_W * u_dual_RT_W) *
                    (float)L.hex_inv[id] / 4.0f;

  hfm[E3(RT, id)] = u_dual_RT * interpf(r0, rE);
  hfm[E3(DG, id)] = u_dual_DG * interpf(r0, rNE);
  hfm[E3(UP, id)] = u_dual_UP * interpf(r0, rN);
  hft[E3(RT, id)] = u_dual_RT * interpf(t0, RHO(Mt, At, idE));
  hft[E3(DG, id)] = u_dual_DG * interpf(t0, RHO(Mt, At, idNE));
  hft[E3(UP, id)] = u_dual_UP * interpf(t0, RHO(Mt, At, idN));

  if (i == 0 || j == 0) {  // comp_SW
    const float rSW = RHO(Mm, Am, idSW);
    const float tS = RHO(Mt, At, idS), tW = RHO(Mt, At, idW), tSW = RHO(Mt, At, idSW);
    const float u_prim_RT_SW = R.ed(v, E3(RT, idSW)) * (float)len[E3(RT, idSW)];
    const float u_prim_UP_SW = R.ed(v, E3(UP, idSW)) * (float)len[E3(UP, idSW)];
    const float circ_SW_LORT = u_prim_RT_SW + u_prim_UP_S + u_prim_DG_SW;
    const float circ_SW_UPLT = -(u_prim_RT_W + u_prim_DG_SW + u_prim_UP_SW);
    const float qm1 = rSW * PART(idSW, 1) + rS * PART(idS, 3) + r0 * PART(id, 5);
    const float qm2 = rSW * PART(idSW, 2) + r0 * PART(id, 4) + rW * PART(idW, 6);
    const float pv_SW_LORT = ((float)cor[E3(LORT, idSW)] + circ_SW_LORT) / qm1;
    const float pv_SW_UPLT = ((float)cor[E3(UPLT, idSW)] + circ_SW_UPLT) / qm2;
    if (i == 0) {
      qe[E3(RT, idW)] = interpf(pv_W_LORT, pv_SW_UPLT);
      hfm[E3(RT, idW)] = u_dual_RT_W * interpf(r0, rW);
      hft[E3(RT, idW)] = u_dual_RT_W * interpf(t0, tW);
    }
    qe[E3(DG, idSW)] = interpf(pv_SW_LORT, pv_SW_UPLT);
    qe[E3(UP, idS)] = interpf(pv_SW_LORT, pv_S_UPLT);
    hfm[E3(DG, idSW)] = u_dual_DG_SW * interpf(r0, rSW);
    hfm[E3(UP, idS)] = u_dual_UP_S * interpf(r0, rS);
    hft[E3(DG, idSW)] = u_dual_DG_SW * interpf(t0, tSW);
    hft[E3(UP, idS)] = u_dual_UP_S * interpf(t0, tS);
  }
#undef E3
#undef PART
#undef RHO
  if ((i == 0 || i == L.n) && (j == 0 || j == L.n)) {
    const int d = id / (P * P);
    const int c = (i == L.n) ? (j == L.n ? 0 : 1) : (j == 0 ? 2 : 3);
    post_corner_f32(L, c, d, ko, mass, velo, mean_m, out.qe);
  }
}

// Qperp (src/ops.f90:834-901) in FP64 on FP32 mass fluxes and qe.
__device__ __forceinline__ void qperp_f32in(const LevelDev& L, const RdF& R, const float* __restrict__ hm,
                                            const float* __restrict__ qe, int id, double Q[3]) {
  const int P = L.P, NN = L.NN;
  const int idNW = id + P - 1, idN = id + P, idNE = id + P + 1, idW = id - 1, idE = id + 1, idSW = id - P - 1,
            idS = id - P, idSE = id - P + 1;
#define TQ(e1, n1, q0, w) (R.ef(hm, (e1) * NN + (n1)) * interp((double)qe[(e1) * NN + (n1)], (q0)) * (w))
  double w1[5], w2[5];
  double q0 = qe[RT * NN + id];
  weights5(L, id, 0, w1);
  weights5(L, idE, 3, w2);
  Q[0] = TQ(DG, id, q0, w1[0]) + TQ(UP, id, q0, w1[1]) + TQ(RT, idW, q0, w1[2]) + TQ(DG, idSW, q0, w1[3]) +
         TQ(UP, idS, q0, w1[4]) + TQ(DG, idS, q0, w2[0]) + TQ(UP, idSE, q0, w2[1]) + TQ(RT, idE, q0, w2[2]) +
         TQ(DG, idE, q0, w2[3]) + TQ(UP, idE, q0, w2[4]);
  q0 = qe[DG * NN + id];
  weights5(L, id, 1, w1);
  weights5(L, idNE, 4, w2);
  Q[1] = TQ(UP, id, q0, w1[0]) + TQ(RT, idW, q0, w1[1]) + TQ(DG, idSW, q0, w1[2]) + TQ(UP, idS, q0, w1[3]) +
         TQ(RT, id, q0, w1[4]) + TQ(UP, idE, q0, w2[0]) + TQ(RT, idNE, q0, w2[1]) + TQ(DG, idNE, q0, w2[2]) +
         TQ(UP, idNE, q0, w2[3]) + TQ(RT, idN, q0, w2[4]);
  q0 = qe[UP * NN + id];
  weights5(L, id, 2, w1);
  weights5(L, idN, 5, w2);
  Q[2] = TQ(RT, idW, q0, w1[0]) + TQ(DG, idSW, q0, w1[1]) + TQ(UP, idS, q0, w1[2]) + TQ(RT, id, q0, w1[3]) +
         TQ(DG, id, q0, w1[4]) + TQ(RT, idN, q0, w2[0]) + TQ(DG, idN, q0, w2[1]) + TQ(UP, idN, q0, w2[2]) +
         TQ(RT, idNW, q0, w2[3]) + TQ(DG, idW, q0, w2[4]);
#undef TQ
}

// Trends (FP64 arithmetic on the FP32 step1 results) and the FP64 RK sub-step,
// on the same node sets as k_trend.
template <int MODE>
__global__ void __launch_bounds__(NODE_TILE, 3) k_trend_mixed(LevelDev L, int nz, TrendIOF io) {
  int k, id, i, j;
  if (!layer_node(L, nz, k, id, i, j)) return;
  const int P = L.P;
  const int NN = L.NN;
  const int n = L.n;
  const int64_t ko = (int64_t)k * NN;
  const RdF R(L, i >= 1 && j >= 1 && i <= n - 2 && j <= n - 2);
  double dms = 0.0, dts = 0.0, dv0 = 0.0, dv1 = 0.0, dv2 = 0.0;
  const bool scal = (i >= 0 && j >= 0 && i <= n && j <= n);
  const bool own = (i >= 0 && j >= 0 && i < n && j < n);
  if (scal) {
    const int idW = id - 1, idS = id - P, idSW = id - P - 1;
    const float* __restrict__ fm = io.hfm + 3 * ko;
    const float* __restrict__ ft = io.hft + 3 * ko;
    const double hinv = L.hex_inv[id];
    const double divm = (R.ef(fm, RT * NN + id) - R.ef(fm, RT * NN + idW) + R.ef(fm, DG * NN + idSW) -
                         R.ef(fm, DG * NN + id) + R.ef(fm, UP * NN + id) - R.ef(fm, UP * NN + idS)) * hinv;
    const double divt = (R.ef(ft, RT * NN + id) - R.ef(ft, RT * NN + idW) + R.ef(ft, DG * NN + idSW) -
                         R.ef(ft, DG * NN + id) + R.ef(ft, UP * NN + id) - R.ef(ft, UP * NN + idS)) * hinv;
    dms = -divm;
    dts = -divt;
  }
  if (own) {
    const float* __restrict__ hm = io.hfm + 3 * ko;
    const float* __restrict__ qe = io.qe + 3 * ko;
    const int idN = id + P, idNE = id + P + 1, idE = id + 1;
    double Q[3];
    qperp_f32in(L, R, hm, qe, id, Q);
    const float* __restrict__ th = io.theta + ko;
    const double th0 = th[id], thE = th[idE], thNE = th[idNE], thN = th[idN];
    const float* __restrict__ K = io.ke + ko;
    const double* __restrict__ F = io.phik + ko;
    const double* __restrict__ Pt = io.pterm + ko;
    auto B = [&](int x) { return (double)K[x] + F[x] + Pt[x]; };   // bernoulli (src/ops.f90:355)
    const double lRT = L.len[RT * NN + id], lDG = L.len[DG * NN + id], lUP = L.len[UP * NN + id];
    const double B0 = B(id), BE = B(idE), BNE = B(idNE), BN = B(idN);
    const double gB0 = (BE - B0) / lRT, gB1 = (B0 - BNE) / lDG, gB2 = (BN - B0) / lUP;
    const double xE = -F[idE], x0 = -F[id], xNE = -F[idNE], xN = -F[idN];
    const double gE0 = (xE - x0) / lRT, gE1 = (x0 - xNE) / lDG, gE2 = (xN - x0) / lUP;
    dv0 = -Q[0] / lRT - gB0 - interp(th0, thE) * gE0;
    dv1 = -Q[1] / lDG - gB1 - interp(th0, thNE) * gE1;
    dv2 = -Q[2] / lUP - gB2 - interp(th0, thN) * gE2;
  }
  const int64_t vo = 3 * ko + id;
  if (MODE == MODE_RK) {
    const double h = io.h;
    io.dst_m[ko + id] = io.base_m[ko + id] + h * dms;
    io.dst_t[ko + id] = io.base_t[ko + id] + h * dts;
    io.dst_v[vo] = io.base_v[vo] + h * dv0;
    io.dst_v[vo + NN] = io.base_v[vo + NN] + h * dv1;
    io.dst_v[vo + 2 * NN] = io.base_v[vo + 2 * NN] + h * dv2;
  } else {
    io.dm[ko + id] = dms;
    io.dtt[ko + id] = dts;
    io.dv[vo] = dv0;
    io.dv[vo + NN] = dv1;
    io.dv[vo + 2 * NN] = dv2;
  }
}

}  // namespace wtk
