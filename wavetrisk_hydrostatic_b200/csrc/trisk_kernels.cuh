// TRiSK operator kernels for one uniform level of the padded lozenge layout.
//
// Node (d, i, j) lives at (d*P + j+2)*P + i+2, so every neighbour of the
// reference's idx() (src/domain.f90:757-812) is a constant offset
// (E = +1, N = +P, NE = P+1, W = -1, S = -P, SW = -P-1, SE = 1-P, NW = P-1):
// the kernels never branch on patch or boundary-patch membership.
//
// Ghost cells of the prognostic state and of the mass flux are not copied:
// threads near a lozenge border read them through the level's remap tables
// (nsrc, esrc), which name the node or signed edge the reference's
// update_bdry copies there.  Threads in the interior read directly.
//
// Floating point follows the reference expression by expression (operand order
// and parenthesisation of src/ops.f90); the file is compiled with --fmad=false
// so that no multiply-add is contracted, which keeps every result bit-identical
// to the CPU restatement.
#pragma once
#include <cstdint>

#include "trisk_read.cuh"
#include "trisk_types.cuh"

namespace wtk {

// --------------------------------------------------------------------------
// Ghost copy (cp_bdry_inside, src/comm.f90:785-808) of the layered state:
// node entries for mass and temp, signed edge entries for velocity.  Used to
// hand the host a state whose ghosts hold their copies.
__global__ void k_halo_state(int nz, int64_t NN, const int2* __restrict__ hn, int n_hn, const int3* __restrict__ he,
                             int n_he, double* __restrict__ mass, double* __restrict__ temp, double* __restrict__ velo) {
  const int per_layer = 2 * n_hn + n_he;
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)per_layer * nz) return;
  int k = (int)(t / per_layer);
  int r = (int)(t - (int64_t)k * per_layer);
  if (r < 2 * n_hn) {
    int2 e = hn[r % n_hn];
    double* f = (r < n_hn ? mass : temp) + (int64_t)k * NN;
    f[e.x] = f[e.y];
  } else {
    int3 e = he[r - 2 * n_hn];
    double* f = velo + (int64_t)k * 3 * NN;
    double v = f[e.y];
    f[e.x] = e.z < 0 ? -v : v;
  }
}

// --------------------------------------------------------------------------
// Column pass: cal_surf_press/column_mass (src/ops.f90:1023-1072) and
// integrate_pressure_up (src/ops.f90:1094-1131), incompressible case, for every
// node (i, j) in [0, n]^2 of every lozenge.  Writes the layer geopotential
// Phi_k = interp(geopot, geopot_lower) and press/(rho0*phi).
__device__ __forceinline__ void column_node(const LevelDev& L, const Phys& ph, int nz, const double* __restrict__ mass,
                                            const double* __restrict__ temp, const double* __restrict__ mean_m,
                                            const double* __restrict__ mean_t, double* __restrict__ phik,
                                            double* __restrict__ pterm, int id, int i, int j);

__global__ void __launch_bounds__(NODE_TILE) k_column(LevelDev L, Phys ph, int nz, const double* __restrict__ mass,
                                                      const double* __restrict__ temp, const double* __restrict__ mean_m,
                                                      const double* __restrict__ mean_t, double* __restrict__ phik,
                                                      double* __restrict__ pterm,
                                                      const unsigned char* __restrict__ need) {
  // one thread per padded node, all layers; with a needed-node map (need[nsrc])
  // only the nodes it marks
  int k0, id, i, j;
  if (!layer_node(L, 1, k0, id, i, j)) return;
  if (i < 0 || j < 0 || i > L.n || j > L.n) return;
  if (need && !need[__ldg(L.nsrc + id)]) return;
  column_node(L, ph, nz, mass, temp, mean_m, mean_t, phik, pterm, id, i, j);
}

// The same over a work list (persistent blocks).
__global__ void __launch_bounds__(NODE_TILE) k_column_list(LevelDev L, Phys ph, int nz, const double* __restrict__ mass,
                                                           const double* __restrict__ temp,
                                                           const double* __restrict__ mean_m,
                                                           const double* __restrict__ mean_t, double* __restrict__ phik,
                                                           double* __restrict__ pterm, NodeList W) {
  const int cnt = __ldg(W.count);
  for (int64_t w = blockIdx.x; w < list_items(cnt, 1); w += gridDim.x) {
    int k, id, i, j;
    if (!list_entry(L, 1, W, cnt, w, k, id, i, j) || i < 0 || j < 0 || i > L.n || j > L.n) continue;
    column_node(L, ph, nz, mass, temp, mean_m, mean_t, phik, pterm, id, i, j);
  }
}

__device__ __forceinline__ void column_node(const LevelDev& L, const Phys& ph, int nz, const double* __restrict__ mass,
                                            const double* __restrict__ temp, const double* __restrict__ mean_m,
                                            const double* __restrict__ mean_t, double* __restrict__ phik,
                                            double* __restrict__ pterm, int id, int i, int j) {
  const int src = (i < L.n && j < L.n) ? id : L.nsrc[id];
  double sp = 0.0;
  for (int k = 0; k < nz; ++k) {
    const int64_t o = (int64_t)k * L.NN;
    double rho_dz = mean_m[o + id] + mass[o + src];
    double rho_dz_theta = mean_t[o + id] + temp[o + src];
    sp = sp + (rho_dz - rho_dz_theta);
  }
  double p_lower = ph.grav * sp + ph.p_top;
  double geopot = ph.grav * L.topo[id];
  for (int k = 0; k < nz; ++k) {
    const int64_t o = (int64_t)k * L.NN;
    double rho_dz = mean_m[o + id] + mass[o + src];
    double rho_dz_theta = mean_t[o + id] + temp[o + src];
    double geopot_lower = geopot;
    double p_upper = p_lower - ph.grav * (rho_dz - rho_dz_theta);
    double press = interp(p_lower, p_upper);
    geopot = geopot_lower + ph.grav * rho_dz / (ph.ref_density * 1.0);
    p_lower = p_upper;
    phik[o + id] = interp(geopot, geopot_lower);
    pterm[o + id] = press / (ph.ref_density * 1.0);
  }
}

struct Step1Out {
  double* __restrict__ qe;    // [nz][3][NN]
  double* __restrict__ hfm;   // [nz][3][NN]
  double* __restrict__ hft;   // [nz][3][NN]
  double* __restrict__ bern;  // [nz][NN]
  double* __restrict__ theta; // [nz][NN]
};

// post_step1 (src/ops.f90:526-737): PV of the merged triangle at a pentagon
// corner.  Run by the thread that owns the corrected edges; the vorticity the
// reference reads back from its vort array is re-formed from the same
// circulation sum its last writer used, divided by the same triangle area.
__device__ __noinline__ void post_corner(const LevelDev L, int c, int d, int64_t ko, const double* __restrict__ mass,
                                         const double* __restrict__ velo, const double* __restrict__ mean_m,
                                         double* __restrict__ qe) {
  const int n = L.n;
  const int64_t NN = L.NN;
  const Rd R(L, false);
  const double* v = velo + 3 * ko;
  auto rho = [&](int64_t x) { return R.n(mass + ko, x) + mean_m[ko + x]; };
  auto pr = [&](int e, int64_t x) { return R.e(v, (int64_t)e * NN + x) * L.len[(int64_t)e * NN + x]; };
  auto part = [&](int64_t x, int kk) { return L.part[(int64_t)(kk - 1) * NN + x]; };
  auto tri = [&](int tt, int64_t x) { return L.triarea[(int64_t)tt * NN + x]; };
  auto cor = [&](int tt, int64_t x) { return L.coriolis[(int64_t)tt * NN + x]; };
  auto I = [&](int i, int j) { return nid(L, d, i, j); };
  double* q = qe + 3 * ko;
  if (c == 0) {  // IJPLUS (north-east corner)
    int64_t id = I(n, n), idN = I(n, n + 1), idE = I(n + 1, n), idS = I(n, n - 1), idW = I(n - 1, n);
    double r0 = rho(id), rN = rho(idN), rE = rho(idE), rS = rho(idS), rW = rho(idW);
    double circ_LORT = pr(RT, id) - pr(RT, idN) - pr(UP, id);
    double vW = (pr(RT, idW) + pr(UP, id) + pr(DG, idW)) / tri(LORT, idW);
    double vS = -(pr(DG, idS) + pr(UP, idS) + pr(RT, id)) / tri(UPLT, idS);
    double circ_W_LORT = vW * tri(LORT, idW);
    double circ_S_UPLT = vS * tri(UPLT, idS);
    double pm1 = rE * part(idE, 3) + r0 * (part(id, 1) + part(id, 2)) + rN * part(idN, 6);
    double pm2 = rW * part(idW, 1) + r0 * part(id, 3) + rN * part(idN, 5);
    double pm3 = rS * part(idS, 2) + rE * part(idE, 4) + r0 * part(id, 6);
    double pv_LORT = (cor(LORT, id) + circ_LORT) / pm1;
    double pv_W_LORT = (cor(LORT, idW) + circ_W_LORT) / pm2;
    double pv_S_UPLT = (cor(UPLT, idS) + circ_S_UPLT) / pm3;
    double pv_UPLT = pv_LORT;
    q[(int64_t)RT * NN + id] = interp(pv_LORT, pv_S_UPLT);
    q[(int64_t)UP * NN + id] = interp(pv_UPLT, pv_W_LORT);
  } else if (c == 1) {  // IPLUSJMINUS (south-east corner)
    int64_t id = I(n, 0), idE = I(n + 1, 0), idS = I(n, -1), idW = I(n - 1, 0), idNE = I(n + 1, 1), idSW = I(n - 1, -1);
    double r0 = rho(id), rE = rho(idE), rS = rho(idS), rW = rho(idW), rNE = rho(idNE), rSW = rho(idSW);
    double circ_SW_LORT = -pr(RT, id) + pr(RT, idSW) + pr(DG, idSW);
    double vL = (pr(RT, id) + pr(UP, idE) + pr(DG, id)) / tri(LORT, id);
    double vU = -(pr(RT, idW) + pr(DG, idSW) + pr(UP, idSW)) / tri(UPLT, idSW);
    double circ_LORT = vL * tri(LORT, id);
    double circ_SW_UPLT = vU * tri(UPLT, idSW);
    double pm1 = rSW * part(idSW, 1) + rS * part(idS, 3) + r0 * (part(id, 5) + part(id, 6));
    double pm2 = r0 * part(id, 1) + rE * part(idE, 3) + rNE * part(idNE, 5);
    double pm3 = rSW * part(idSW, 2) + r0 * part(id, 4) + rW * part(idW, 6);
    double pv_SW_LORT = (cor(LORT, idSW) + circ_SW_LORT) / pm1;
    double pv_LORT = (cor(LORT, id) + circ_LORT) / pm2;
    double pv_SW_UPLT = (cor(UPLT, idSW) + circ_SW_UPLT) / pm3;
    double pv_S_UPLT = pv_SW_LORT;
    q[(int64_t)RT * NN + id] = interp(pv_S_UPLT, pv_LORT);
    q[(int64_t)DG * NN + idSW] = interp(pv_SW_LORT, pv_SW_UPLT);
  } else if (c == 2) {  // IJMINUS (south-west corner)
    int64_t id = I(0, 0), idN = I(0, 1), idE = I(1, 0), idS = I(0, -1), idW = I(-1, 0), idSW = I(-1, -1);
    double r0 = rho(id), rN = rho(idN), rE = rho(idE), rS = rho(idS), rW = rho(idW);
    double circ_SW_LORT = pr(UP, idS) - pr(RT, idW) + pr(RT, idSW);
    double vW = (pr(RT, idW) + pr(UP, id) + pr(DG, idW)) / tri(LORT, idW);
    double vS = -(pr(RT, id) + pr(DG, idS) + pr(UP, idS)) / tri(UPLT, idS);
    double circ_W_LORT = vW * tri(LORT, idW);
    double circ_S_UPLT = vS * tri(UPLT, idS);
    double pm1 = rW * part(idW, 6) + r0 * (part(id, 4) + part(id, 5)) + rS * part(idS, 3);
    double pm2 = rW * part(idW, 1) + r0 * part(id, 3) + rN * part(idN, 5);
    double pm3 = rS * part(idS, 2) + rE * part(idE, 4) + r0 * part(id, 6);
    double pv_W_LORT = (cor(LORT, idW) + circ_W_LORT) / pm1;
    double pv_SW_LORT = (cor(LORT, idSW) + circ_SW_LORT) / pm2;
    double pv_S_UPLT = (cor(UPLT, idS) + circ_S_UPLT) / pm3;
    double pv_SW_UPLT = pv_SW_LORT;
    q[(int64_t)RT * NN + idW] = interp(pv_W_LORT, pv_SW_UPLT);
    q[(int64_t)UP * NN + idS] = interp(pv_S_UPLT, pv_SW_LORT);
  } else {  // IMINUSJPLUS (north-west corner)
    int64_t id = I(0, n), idN = I(0, n + 1), idS = I(0, n - 1), idW = I(-1, n), idNE = I(1, n + 1), idSW = I(-1, n - 1);
    double r0 = rho(id), rN = rho(idN), rS = rho(idS), rW = rho(idW), rNE = rho(idNE), rSW = rho(idSW);
    double circ_SW_UPLT = pr(UP, id) - pr(DG, idSW) - pr(UP, idSW);
    double vU = -(pr(DG, id) + pr(UP, id) + pr(RT, idN)) / tri(UPLT, id);
    double vL = (pr(RT, idSW) + pr(UP, idS) + pr(DG, idSW)) / tri(LORT, idSW);
    double circ_UPLT = vU * tri(UPLT, id);
    double circ_SW_LORT = vL * tri(LORT, idSW);
    double pm1 = rSW * part(idSW, 2) + r0 * (part(id, 3) + part(id, 4)) + rW * part(idW, 6);
    double pm2 = r0 * part(id, 2) + rNE * part(idNE, 4) + rN * part(idN, 6);
    double pm3 = rSW * part(idSW, 1) + rS * part(idS, 3) + r0 * part(id, 5);
    double pv_SW_UPLT = (cor(UPLT, idSW) + circ_SW_UPLT) / pm1;
    double pv_UPLT = (cor(UPLT, id) + circ_UPLT) / pm2;
    double pv_SW_LORT = (cor(LORT, idSW) + circ_SW_LORT) / pm3;
    double pv_W_LORT = pv_SW_UPLT;
    q[(int64_t)UP * NN + id] = interp(pv_W_LORT, pv_UPLT);
    q[(int64_t)DG * NN + idSW] = interp(pv_SW_LORT, pv_SW_UPLT);
  }
}

// --------------------------------------------------------------------------
// step1 itype 0 (src/ops.f90:276-366 comput, :472-522 comp_SW) at every node
// (i, j) in [0, n]^2 and layer k: potential vorticity qe, mass and Theta fluxes,
// kinetic energy and the Bernoulli function.  comp_SW runs where i == 0 or
// j == 0, as at the reference's south and west domain boundaries.  Each edge
// has exactly one writer, chosen so that the stored value is the one the
// reference's sequential sweep leaves behind; the four corner threads then
// apply post_step1.  The node's potential temperature Theta/rho
// (src/ops.f90:798, theta_e's node factor) is stored for the velocity trend.
__device__ __forceinline__ void step1_node(const LevelDev& L, int nz, const double* __restrict__ mass,
                                           const double* __restrict__ temp, const double* __restrict__ velo,
                                           const double* __restrict__ mean_m, const double* __restrict__ mean_t,
                                           const double* __restrict__ phik, const double* __restrict__ pterm,
                                           const Step1Out& out, int k, int id, int i, int j);

__global__ void __launch_bounds__(NODE_TILE, 3)
    k_step1(LevelDev L, int nz, const double* __restrict__ mass, const double* __restrict__ temp,
            const double* __restrict__ velo, const double* __restrict__ mean_m, const double* __restrict__ mean_t,
            const double* __restrict__ phik, const double* __restrict__ pterm, Step1Out out,
            const unsigned char* __restrict__ need) {
  int k, id, i, j;
  if (!layer_node(L, nz, k, id, i, j)) return;
  if (i < 0 || j < 0 || i > L.n || j > L.n) return;
  if (need && !need[__ldg(L.nsrc + id)]) return;  // needed-node map (need_map.cuh)
  step1_node(L, nz, mass, temp, velo, mean_m, mean_t, phik, pterm, out, k, id, i, j);
}

// The same over a work list (persistent blocks).
#ifndef WT_STEP1_LIST_MINB
#define WT_STEP1_LIST_MINB 4
#endif
__global__ void __launch_bounds__(NODE_TILE, WT_STEP1_LIST_MINB)
    k_step1_list(LevelDev L, int nz, const double* __restrict__ mass, const double* __restrict__ temp,
                 const double* __restrict__ velo, const double* __restrict__ mean_m,
                 const double* __restrict__ mean_t, const double* __restrict__ phik,
                 const double* __restrict__ pterm, Step1Out out, NodeList W) {
  const int cnt = __ldg(W.count);
  for (int64_t w = blockIdx.x; w < list_items(cnt, nz); w += gridDim.x) {
    int k, id, i, j;
    if (!list_entry(L, nz, W, cnt, w, k, id, i, j) || i < 0 || j < 0 || i > L.n || j > L.n) continue;
    step1_node(L, nz, mass, temp, velo, mean_m, mean_t, phik, pterm, out, k, id, i, j);
  }
}

__device__ __forceinline__ void step1_node(const LevelDev& L, int nz, const double* __restrict__ mass,
                                           const double* __restrict__ temp, const double* __restrict__ velo,
                                           const double* __restrict__ mean_m, const double* __restrict__ mean_t,
                                           const double* __restrict__ phik, const double* __restrict__ pterm,
                                           const Step1Out& out, int k, int id, int i, int j) {
  const int NN = L.NN;
  const int P = L.P;
  const int idN = id + P, idE = id + 1, idS = id - P, idW = id - 1, idNE = id + P + 1, idSW = id - P - 1;
  const int64_t ko = (int64_t)k * NN;
  const Rd R(L, i >= 1 && j >= 1 && i <= L.n - 2 && j <= L.n - 2);
  const double* __restrict__ Mm = mass + ko;
  const double* __restrict__ Mt = temp + ko;
  const double* __restrict__ Am = mean_m + ko;
  const double* __restrict__ At = mean_t + ko;
  const double* __restrict__ v = velo + 3 * ko;
  double* __restrict__ qe = out.qe + 3 * ko;
  double* __restrict__ hfm = out.hfm + 3 * ko;
  double* __restrict__ hft = out.hft + 3 * ko;
  const double* __restrict__ len = L.len;
  const double* __restrict__ ped = L.pedlen;
  const double* __restrict__ part = L.part;
  const double* __restrict__ cor = L.coriolis;
#define E3(e, x) ((e) * NN + (x))
#define PART(x, kk) part[((kk) - 1) * NN + (x)]

  const double r0 = R.n(Mm, id) + Am[id], rN = R.n(Mm, idN) + Am[idN], rE = R.n(Mm, idE) + Am[idE],
               rS = R.n(Mm, idS) + Am[idS], rW = R.n(Mm, idW) + Am[idW], rNE = R.n(Mm, idNE) + Am[idNE];
  const double t0 = R.n(Mt, id) + At[id];
  out.theta[ko + id] = t0 / r0;
  const double vRT = R.e(v, E3(RT, id)), vDG = R.e(v, E3(DG, id)), vUP = R.e(v, E3(UP, id));
  const double vRT_W = R.e(v, E3(RT, idW)), vDG_SW = R.e(v, E3(DG, idSW)), vUP_S = R.e(v, E3(UP, idS));
  const double u_dual_RT = vRT * ped[E3(RT, id)];
  const double u_dual_DG = vDG * ped[E3(DG, id)];
  const double u_dual_UP = vUP * ped[E3(UP, id)];
  const double u_dual_RT_W = vRT_W * ped[E3(RT, idW)];
  const double u_dual_DG_SW = vDG_SW * ped[E3(DG, idSW)];
  const double u_dual_UP_S = vUP_S * ped[E3(UP, idS)];

  const double u_prim_RT = vRT * len[E3(RT, id)];
  const double u_prim_RT_W = vRT_W * len[E3(RT, idW)];
  const double u_prim_DG = vDG * len[E3(DG, id)];
  const double u_prim_DG_SW = vDG_SW * len[E3(DG, idSW)];
  const double u_prim_UP = vUP * len[E3(UP, id)];
  const double u_prim_UP_S = vUP_S * len[E3(UP, idS)];
  const double u_prim_DG_W = R.e(v, E3(DG, idW)) * len[E3(DG, idW)];
  const double u_prim_UP_E = R.e(v, E3(UP, idE)) * len[E3(UP, idE)];

  const double circ_LORT = u_prim_RT + u_prim_UP_E + u_prim_DG;
  const double circ_W_LORT = u_prim_RT_W + u_prim_UP + u_prim_DG_W;
  const double pv_LORT = (cor[E3(LORT, id)] + circ_LORT) / (r0 * PART(id, 1) + rE * PART(idE, 3) + rNE * PART(idNE, 5));
  const double pv_W_LORT =
      (cor[E3(LORT, idW)] + circ_W_LORT) / (rW * PART(idW, 1) + r0 * PART(id, 3) + rN * PART(idN, 5));
  const double u_prim_RT_N = R.e(v, E3(RT, idN)) * len[E3(RT, idN)];
  const double circ_UPLT = -(u_prim_DG + u_prim_UP + u_prim_RT_N);
  const double pv_UPLT = (cor[E3(UPLT, id)] + circ_UPLT) / (r0 * PART(id, 2) + rNE * PART(idNE, 4) + rN * PART(idN, 6));
  const double u_prim_DG_S = R.e(v, E3(DG, idS)) * len[E3(DG, idS)];
  const double circ_S_UPLT = -(u_prim_RT + u_prim_DG_S + u_prim_UP_S);
  const double pv_S_UPLT =
      (cor[E3(UPLT, idS)] + circ_S_UPLT) / (rS * PART(idS, 2) + rE * PART(idE, 4) + r0 * PART(id, 6));

  qe[E3(RT, id)] = interp(pv_S_UPLT, pv_LORT);
  qe[E3(DG, id)] = interp(pv_UPLT, pv_LORT);
  // On the west column the reference's comp_SW at (0, j+1) rewrites qe(UP) of
  // (0, j) after comput; that later value is written by comp_SW below.
  if (!(i == 0 && j < L.n)) qe[E3(UP, id)] = interp(pv_UPLT, pv_W_LORT);

  const double ke = (u_prim_UP * u_dual_UP + u_prim_DG * u_dual_DG + u_prim_RT * u_dual_RT + u_prim_UP_S * u_dual_UP_S +
                     u_prim_DG_SW * u_dual_DG_SW + u_prim_RT_W * u_dual_RT_W) *
                    L.hex_inv[id] / 4.0;
  out.bern[ko + id] = ke + phik[ko + id] + pterm[ko + id];

  hfm[E3(RT, id)] = u_dual_RT * interp(r0, rE) + 0.0;
  hfm[E3(DG, id)] = u_dual_DG * interp(r0, rNE) + 0.0;
  hfm[E3(UP, id)] = u_dual_UP * interp(r0, rN) + 0.0;
  hft[E3(RT, id)] = u_dual_RT * interp(t0, R.n(Mt, idE) + At[idE]) + 0.0;
  hft[E3(DG, id)] = u_dual_DG * interp(t0, R.n(Mt, idNE) + At[idNE]) + 0.0;
  hft[E3(UP, id)] = u_dual_UP * interp(t0, R.n(Mt, idN) + At[idN]) + 0.0;

  if (i == 0 || j == 0) {  // comp_SW
    const double rSW = R.n(Mm, idSW) + Am[idSW];
    const double tS = R.n(Mt, idS) + At[idS], tW = R.n(Mt, idW) + At[idW], tSW = R.n(Mt, idSW) + At[idSW];
    const double u_prim_RT_SW = R.e(v, E3(RT, idSW)) * len[E3(RT, idSW)];
    const double u_prim_UP_SW = R.e(v, E3(UP, idSW)) * len[E3(UP, idSW)];
    const double circ_SW_LORT = u_prim_RT_SW + u_prim_UP_S + u_prim_DG_SW;
    const double circ_SW_UPLT = -(u_prim_RT_W + u_prim_DG_SW + u_prim_UP_SW);
    const double qm1 = rSW * PART(idSW, 1) + rS * PART(idS, 3) + r0 * PART(id, 5);
    const double qm2 = rSW * PART(idSW, 2) + r0 * PART(id, 4) + rW * PART(idW, 6);
    const double pv_SW_LORT = (cor[E3(LORT, idSW)] + circ_SW_LORT) / qm1;
    const double pv_SW_UPLT = (cor[E3(UPLT, idSW)] + circ_SW_UPLT) / qm2;
    // RT of the west neighbour is also produced, bit-identically, by comput at
    // (i-1, 0) when i > 0; only the ghost edge (i == 0) is written here.
    if (i == 0) {
      qe[E3(RT, idW)] = interp(pv_W_LORT, pv_SW_UPLT);
      hfm[E3(RT, idW)] = u_dual_RT_W * interp(r0, rW) + 0.0;
      hft[E3(RT, idW)] = u_dual_RT_W * interp(t0, tW) + 0.0;
    }
    qe[E3(DG, idSW)] = interp(pv_SW_LORT, pv_SW_UPLT);
    qe[E3(UP, idS)] = interp(pv_SW_LORT, pv_S_UPLT);
    hfm[E3(DG, idSW)] = u_dual_DG_SW * interp(r0, rSW) + 0.0;
    hfm[E3(UP, idS)] = u_dual_UP_S * interp(r0, rS) + 0.0;
    hft[E3(DG, idSW)] = u_dual_DG_SW * interp(t0, tSW) + 0.0;
    hft[E3(UP, idS)] = u_dual_UP_S * interp(t0, tS) + 0.0;
  }
#undef E3
#undef PART
  // post_step1 at the pentagon corners, by the thread that wrote those edges
  if ((i == 0 || i == L.n) && (j == 0 || j == L.n)) {
    const int d = id / (P * P);
    const int c = (i == L.n) ? (j == L.n ? 0 : 1) : (j == 0 ? 2 : 3);
    post_corner(L, c, d, ko, mass, velo, mean_m, out.qe);
  }
}

// --------------------------------------------------------------------------
// Trends and the RK sub-step (src/time_integr.f90:206-225) fused:
//   scalar_trend  dscalar = -div(h_flux) on [0, n]^2          (src/ops.f90:739)
//   du_source     dvelo   = -Qperp on owned nodes [0, n)^2    (src/ops.f90:757,834)
//   du_grad       dvelo   = dvelo/len - grad B - theta_e grad Exner  (src/ops.f90:787)
// Mass fluxes at ghost edges are read from their source edges (the
// reference's update_bdry(horiz_flux)).  For MODE_RK every node of the padded
// level (all layers) is written as dest = base + h * trend (trend = 0 where
// the reference leaves it zero); MODE_TREND writes the trends themselves.
// MODE_ML: one level of the multi-level trend_ml at the finest level (no
// restricted source), with the RK sub-step (trisk_tma.cuh only).
enum { MODE_TREND = 0, MODE_RK = 1, MODE_ML = 2 };


template <int MODE>
__global__ void __launch_bounds__(NODE_TILE, 3) k_trend(LevelDev L, int nz, TrendIO io) {
  int k, id, i, j;
  if (!layer_node(L, nz, k, id, i, j)) return;
  const int P = L.P;
  const int NN = L.NN;
  const int n = L.n;
  const int64_t ko = (int64_t)k * NN;
  const Rd R(L, i >= 1 && j >= 1 && i <= n - 2 && j <= n - 2);
  double dms = 0.0, dts = 0.0, dv0 = 0.0, dv1 = 0.0, dv2 = 0.0;
  const bool scal = (i >= 0 && j >= 0 && i <= n && j <= n);
  const bool own = (i >= 0 && j >= 0 && i < n && j < n);
  if (scal) {
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
  if (own) {
    const double* __restrict__ hm = io.hfm + 3 * ko;
    const double* __restrict__ qe = io.qe + 3 * ko;
    const int idN = id + P, idNE = id + P + 1, idE = id + 1;
    double Q[3];
    qperp(L, R, hm, qe, id, Q);
    const double Q0 = Q[0], Q1 = Q[1], Q2 = Q[2];
    // du_grad
    const double* __restrict__ th = io.theta + ko;
    const double th0 = th[id], thE = th[idE], thNE = th[idNE], thN = th[idN];
    const double* __restrict__ B = io.bern + ko;
    const double* __restrict__ F = io.phik + ko;  // exner = -Phi_k (src/ops.f90:358)
    const double lRT = L.len[RT * NN + id], lDG = L.len[DG * NN + id], lUP = L.len[UP * NN + id];
    const double gB0 = (B[idE] - B[id]) / lRT, gB1 = (B[id] - B[idNE]) / lDG, gB2 = (B[idN] - B[id]) / lUP;
    const double xE = -F[idE], x0 = -F[id], xNE = -F[idNE], xN = -F[idN];
    const double gE0 = (xE - x0) / lRT, gE1 = (x0 - xNE) / lDG, gE2 = (xN - x0) / lUP;
    dv0 = (-Q0 + 0.0 * lRT) / lRT - gB0 - interp(th0, thE) * gE0;
    dv1 = (-Q1 + 0.0 * lDG) / lDG - gB1 - interp(th0, thNE) * gE1;
    dv2 = (-Q2 + 0.0 * lUP) / lUP - gB2 - interp(th0, thN) * gE2;
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
