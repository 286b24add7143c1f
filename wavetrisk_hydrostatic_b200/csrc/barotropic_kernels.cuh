// Barotropic pieces of the mode-split step on one uniform level
// (src/barotropic_2d.f90): the vertically summed mass flux and its divergence
// (flux_divergence, step1 itype 4), the right-hand side of the free-surface
// equation (rhs_elliptic), the external pressure gradient (grad_eta, step1
// itype 3) and the velocity update with it (u_update).
//
// Every edge flux is a function of the edge alone, so the south/west-border
// formulas of comp_SW (src/ops.f90:420-445) are written to the ghost edges
// they own, every edge is written by exactly one thread (the reference's
// repeated writes carry identical bits), and every other ghost edge is read
// through the level's remap.
// Operand order follows the reference; compiled with --fmad=false.
#pragma once
#include <cstdint>

#include "trisk_read.cuh"

namespace wtb {

using wtk::DG;
using wtk::LORT;
using wtk::UPLT;
using wtk::interp;
using wtk::LevelDev;
using wtk::Rd;
using wtk::RT;
using wtk::UP;

// step1 itype 4 (src/ops.f90:229-244, comp_SW :420-437): h_flux = pedlen *
// sum_k u_k interp(rho dz_k) at the edges of nodes [0, n]^2 and, on the
// south/west borders, at the ghost edges comp_SW writes.
__global__ void k_flux_sum(LevelDev L, int nz, const double* __restrict__ mass, const double* __restrict__ mean_m,
                           const double* __restrict__ velo, double* __restrict__ hflux) {
  const int m = L.n + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  const int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
  const int P = L.P, NN = L.NN;
  const int id = (d * P + j + 2) * P + i + 2;
  const int idE = id + 1, idN = id + P, idNE = id + P + 1, idW = id - 1, idS = id - P, idSW = id - P - 1;
  const Rd R(L, i >= 1 && j >= 1 && i <= L.n - 2 && j <= L.n - 2);
  double fRT = 0.0, fDG = 0.0, fUP = 0.0;
  for (int k = 0; k < nz; ++k) {
    const int64_t ko = (int64_t)k * NN;
    const double* Mm = mass + ko;
    const double* Am = mean_m + ko;
    const double* v = velo + 3 * ko;
    const double dz0 = R.n(Mm, id) + Am[id];
    double dz = interp(dz0, R.n(Mm, idE) + Am[idE]);
    fRT = fRT + R.e(v, RT * NN + id) * dz;
    dz = interp(dz0, R.n(Mm, idNE) + Am[idNE]);
    fDG = fDG + R.e(v, DG * NN + id) * dz;
    dz = interp(dz0, R.n(Mm, idN) + Am[idN]);
    fUP = fUP + R.e(v, UP * NN + id) * dz;
  }
  hflux[RT * NN + id] = fRT * L.pedlen[RT * NN + id];
  hflux[DG * NN + id] = fDG * L.pedlen[DG * NN + id];
  hflux[UP * NN + id] = fUP * L.pedlen[UP * NN + id];
  if (i == 0 || j == 0) {  // comp_SW
    double gW = 0.0, gSW = 0.0, gS = 0.0;
    for (int k = 0; k < nz; ++k) {
      const int64_t ko = (int64_t)k * NN;
      const double* Mm = mass + ko;
      const double* Am = mean_m + ko;
      const double* v = velo + 3 * ko;
      const double dz0 = R.n(Mm, id) + Am[id];
      double dz = interp(dz0, R.n(Mm, idW) + Am[idW]);
      gW = gW + R.e(v, RT * NN + idW) * dz;
      dz = interp(dz0, R.n(Mm, idSW) + Am[idSW]);
      gSW = gSW + R.e(v, DG * NN + idSW) * dz;
      dz = interp(dz0, R.n(Mm, idS) + Am[idS]);
      gS = gS + R.e(v, UP * NN + idS) * dz;
    }
    // Edges an interior node also produces, bit-identically, are left to it:
    // RT of (i-1, 0) when i > 0 and UP of (0, j-1) when j > 0.
    if (i == 0) hflux[RT * NN + idW] = gW * L.pedlen[RT * NN + idW];
    hflux[DG * NN + idSW] = gSW * L.pedlen[DG * NN + idSW];
    if (!(i == 0 && j > 0)) hflux[UP * NN + idS] = gS * L.pedlen[UP * NN + idS];
  }
}

// Ghost copy of one node field of a level (update_bdry): dst = src per entry.
__global__ void k_halo_nodes(const int2* __restrict__ hn, int n_hn, double* f) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n_hn) f[hn[q].x] = f[hn[q].y];
}

// cal_div (src/ops.f90:1325-1355) at nodes [0, n]^2:
//   div = hex_inv * (F_RT - F_RT,W + F_DG,SW - F_DG + F_UP - F_UP,S)
__global__ void k_div(LevelDev L, const double* __restrict__ hflux, double* __restrict__ div) {
  const int m = L.n + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  const int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
  const int P = L.P, NN = L.NN;
  const int id = (d * P + j + 2) * P + i + 2;
  const Rd R(L, i >= 1 && j >= 1 && i <= L.n - 2 && j <= L.n - 2);
  div[id] = (R.e(hflux, RT * NN + id) - R.e(hflux, RT * NN + id - 1) + R.e(hflux, DG * NN + id - P - 1) -
             R.e(hflux, DG * NN + id) + R.e(hflux, UP * NN + id) - R.e(hflux, UP * NN + id - P)) *
            L.hex_inv[id];
}

// cal_rhs_elliptic (src/barotropic_2d.f90:167-184) at nodes [0, n]^2, after
// flux_divergence's ghost copy of div (read through the remap):
//   rhs = -eta + dt (theta2 div + (1 - theta2) div_old) / rho0
__global__ void k_rhs(LevelDev L, const double* __restrict__ div, const double* __restrict__ eta,
                      const double* __restrict__ div_old, double dt, double theta2, double rho0,
                      double* __restrict__ rhs) {
  const int m = L.n + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  const int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
  const int id = (d * L.P + j + 2) * L.P + i + 2;
  const Rd R(L, i >= 1 && j >= 1 && i <= L.n - 2 && j <= L.n - 2);
  rhs[id] = -R.n(eta, id) + dt * (theta2 * R.n(div, id) + (1.0 - theta2) * R.n(div_old, id)) / rho0;
}

// step1 itype 3 (src/ops.f90:225-228, comp_SW :416-419) with porosity 1,
// h_flux = g (eta_far - eta_near) / len, and u_update
// (src/barotropic_2d.f90:131-149): velo_k -= theta1 dt h_flux on every layer.
// With DIRECT, eta is read where it is stored (ghosts included): the copy that
// grad_eta restricts on coarser levels is not ghost-copied again.
template <bool DIRECT = false>
__global__ void k_grad_eta_update(LevelDev L, int nz, double grav, const double* __restrict__ eta, double scale,
                                  double* __restrict__ grad, double* __restrict__ velo) {
  const int m = L.n + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  const int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
  const int P = L.P, NN = L.NN;
  const int id = (d * P + j + 2) * P + i + 2;
  const Rd R(L, DIRECT || (i >= 1 && j >= 1 && i <= L.n - 2 && j <= L.n - 2));
  const double e0 = R.n(eta, id) / 1.0;
  int slot[6];
  double g[6];
  int ne = 3;
  slot[0] = RT * NN + id;
  g[0] = grav * (R.n(eta, id + 1) / 1.0 - e0) / L.len[slot[0]];
  slot[1] = DG * NN + id;
  g[1] = grav * (e0 - R.n(eta, id + P + 1) / 1.0) / L.len[slot[1]];
  slot[2] = UP * NN + id;
  g[2] = grav * (R.n(eta, id + P) / 1.0 - e0) / L.len[slot[2]];
  if (i == 0 || j == 0) {  // comp_SW
    if (i == 0) {
      slot[ne] = RT * NN + id - 1;
      g[ne] = -grav * (R.n(eta, id - 1) / 1.0 - e0) / L.len[slot[ne]];
      ++ne;
    }
    slot[ne] = DG * NN + id - P - 1;
    g[ne] = -grav * (e0 - R.n(eta, id - P - 1) / 1.0) / L.len[slot[ne]];
    ++ne;
    // UP of (0, j-1) is the own edge of that node (same value): updated once, there
    if (!(i == 0 && j > 0)) {
      slot[ne] = UP * NN + id - P;
      g[ne] = -grav * (R.n(eta, id - P) / 1.0 - e0) / L.len[slot[ne]];
      ++ne;
    }
  }
  for (int q = 0; q < ne; ++q) {
    grad[slot[q]] = g[q];
    for (int k = 0; k < nz; ++k) {
      double* v = velo + (int64_t)k * 3 * NN;
      v[slot[q]] = v[slot[q]] - scale * g[q];
    }
  }
}

// barotropic_correction (src/barotropic_2d.f90:52-116) on one level: the total
// height of the column (total_height/cal_height, :368-412: the layers' rho dz /
// (rho0 phi) summed bottom-up from 0) and the layer-dilation correction of
// every layer's mass and mass-weighted buoyancy from the free surface eta:
//   theta = (mean_t + temp) / (mean_m + mass)
//   mass  = (eta/phi - topo) / height * (mean_m + mass) - mean_m
//   temp  = (mean_m + mass) * theta - mean_t
// with porosity phi = 1.  One thread per node of [0, n]^2 that is its own
// source: owned nodes, and the slots of row n near the pentagon corners that no
// ghost copy fills (stencils read them as stored).  Ghost copies of row n are
// left alone: every kernel reads them through the remaps.
__global__ void k_barotropic_correction(LevelDev L, int nz, double rho0, const double* __restrict__ eta,
                                        const double* __restrict__ mean_m, const double* __restrict__ mean_t,
                                        double* __restrict__ mass, double* __restrict__ temp) {
  const int m = L.n + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  const int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
  const int64_t NN = L.NN;
  const int id = (d * L.P + j + 2) * L.P + i + 2;
  if (__ldg(L.nsrc + id) != id) return;
  double height = 0.0;
  for (int k = 0; k < nz; ++k) {
    const double rho_dz = mean_m[k * NN + id] + mass[k * NN + id];
    height = height + rho_dz / (rho0 * 1.0);
  }
  const double e = eta[id] / 1.0;
  for (int k = 0; k < nz; ++k) {
    const int64_t x = k * NN + id;
    double rho_dz = mean_m[x] + mass[x];
    const double rho_dz_theta = mean_t[x] + temp[x];
    const double theta = rho_dz_theta / rho_dz;
    mass[x] = (e - L.topo[id]) / height * rho_dz - mean_m[x];
    rho_dz = mean_m[x] + mass[x];
    temp[x] = rho_dz * theta - mean_t[x];
  }
}

}  // namespace wtb

namespace wtb {

// step1 itypes 1, 5, 6, 7 (src/ops.f90:198-201, 245-262; comp_SW :396-401,
// 438-455) on one layer, at the edges of nodes [0, n]^2 and at the
// south/west ghost edges comp_SW owns (once each, as in k_flux_sum):
//   1  scalar gradient flux   (s_far - s_near) / len * pedlen
//   5  divu flux              u * pedlen
//   6  surface pressure flux  (s_far - s_near) * u * pedlen / 4
//   7  mass flux              u * pedlen * interp(rho dz)
template <int ITYPE>
__global__ void k_step1_flux(LevelDev L, const double* __restrict__ s, const double* __restrict__ v,
                             const double* __restrict__ mass, const double* __restrict__ mean_m,
                             double* __restrict__ hflux) {
  const int m = L.n + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  const int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
  const int P = L.P, NN = L.NN;
  const int id = (d * P + j + 2) * P + i + 2;
  const Rd R(L, i >= 1 && j >= 1 && i <= L.n - 2 && j <= L.n - 2);
  // comput: edge e of node id towards node nb; the scalar difference is
  // s(nb) - s(id) for RT and UP, s(id) - s(nb) for DG
  auto comput = [&](int e, int nb) {
    const int slot = e * NN + id;
    if (ITYPE == 1) {
      const double dsc = (e == DG) ? R.n(s, id) - R.n(s, nb) : R.n(s, nb) - R.n(s, id);
      hflux[slot] = dsc / L.len[slot] * L.pedlen[slot];
    } else if (ITYPE == 5) {
      hflux[slot] = R.e(v, slot) * L.pedlen[slot];
    } else if (ITYPE == 6) {
      const double dsc = (e == DG) ? R.n(s, id) - R.n(s, nb) : R.n(s, nb) - R.n(s, id);
      hflux[slot] = dsc * R.e(v, slot) * L.pedlen[slot] / 4.0;
    } else {
      const double dz0 = R.n(mass, id) + mean_m[id];
      const double dz = interp(dz0, R.n(mass, nb) + mean_m[nb]);
      hflux[slot] = R.e(v, slot) * L.pedlen[slot] * dz;
    }
  };
  comput(RT, id + 1);
  comput(DG, id + P + 1);
  comput(UP, id + P);
  if (!(i == 0 || j == 0)) return;
  // comp_SW: edge e of the ghost node g, which joins g and id; the scalar
  // difference is -(s(g) - s(id)) for RT and UP, -(s(id) - s(g)) for DG
  auto comp_sw = [&](int e, int g) {
    const int slot = e * NN + g;
    if (ITYPE == 1) {
      const double dsc = (e == DG) ? R.n(s, id) - R.n(s, g) : R.n(s, g) - R.n(s, id);
      hflux[slot] = -(dsc / L.len[slot] * L.pedlen[slot]);
    } else if (ITYPE == 5) {
      hflux[slot] = R.e(v, slot) * L.pedlen[slot];
    } else if (ITYPE == 6) {
      const double dsc = (e == DG) ? R.n(s, id) - R.n(s, g) : R.n(s, g) - R.n(s, id);
      hflux[slot] = -(dsc * R.e(v, slot) * L.pedlen[slot] / 4.0);
    } else {
      const double dz0 = R.n(mass, id) + mean_m[id];
      const double dz = interp(dz0, R.n(mass, g) + mean_m[g]);
      hflux[slot] = R.e(v, slot) * L.pedlen[slot] * dz;
    }
  };
  if (i == 0) comp_sw(RT, id - 1);
  comp_sw(DG, id - P - 1);
  if (!(i == 0 && j > 0)) comp_sw(UP, id - P);
}

// step1 itype 8, vorticity of one layer's velocity (src/ops.f90:256-271,
// comp_SW :460-471), with post_vort's pentagon values (src/ops.f90:1159-1228).
// The reference's loop writes most triangles twice; the two LORT expressions
// are the same sum, the two UPLT ones are not (own: -(DG + UP + RT_N), from
// the node above: -(RT_N + DG + UP)).  The reference visits the nodes
// [0, n)^2 row by row, then the north row (i < n, n) and (n, n), then the
// east column (n, j < n), so the node-above form lands last except on the top
// row and at (n, n-1).  Here each triangle has one writer that evaluates the
// expression that lands last: thread (i, j) in [0, n]^2 writes LORT(i, j) and
// UPLT(i, j); thread (0, j) also writes
// LORT(-1, j) and UPLT(-1, j-1), thread (i, 0) LORT(i-1, -1) and UPLT(i, -1);
// the four lozenge-corner threads write the pentagon values instead.
__global__ void k_step1_vort(LevelDev L, const double* __restrict__ v, double* __restrict__ vort) {
  const int n = L.n, m = n + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  const int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
  const int P = L.P, NN = L.NN;
  const int id = (d * P + j + 2) * P + i + 2;
  const Rd R(L, i >= 1 && j >= 1 && i <= n - 2 && j <= n - 2);
  auto up = [&](int e, int x) { const int slot = e * NN + x; return R.e(v, slot) * L.len[slot]; };
  auto lort = [&](int x) { return up(RT, x) + up(UP, x + 1) + up(DG, x); };
  auto uplt_n = [&](int x) { return -(up(RT, x + P) + up(DG, x) + up(UP, x)); };  // written from the node above
  auto put = [&](int tri, int x, double c) { vort[tri * NN + x] = c / L.triarea[tri * NN + x]; };
  const int idW = id - 1, idS = id - P, idSW = id - P - 1;
  if (i == n && j == n) {  // IJPLUS
    const double c = up(RT, id) - up(RT, id + P) - up(UP, id);
    put(LORT, id, c);
    vort[UPLT * NN + id] = vort[LORT * NN + id];
    return;
  }
  put(LORT, id, lort(id));
  if (j < n && !(i == n && j == n - 1)) put(UPLT, id, uplt_n(id));
  else put(UPLT, id, -(up(DG, id) + up(UP, id) + up(RT, id + P)));
  if (i == 0 && j == 0) {  // IJMINUS
    const double c = up(UP, idS) - up(RT, idW) + up(RT, idSW);
    put(LORT, idSW, c);
    vort[UPLT * NN + idSW] = vort[LORT * NN + idSW];
    put(LORT, idW, lort(idW));
    put(UPLT, idS, uplt_n(idS));
    return;
  }
  if (i == 0 && j == n) {  // IMINUSJPLUS
    const double c = up(UP, id) - up(DG, idSW) - up(UP, idSW);
    put(UPLT, idSW, c);
    vort[LORT * NN + idW] = vort[UPLT * NN + idSW];
    return;
  }
  if (i == n && j == 0) {  // IPLUSJMINUS
    const double c = -up(RT, id) + up(RT, idSW) + up(DG, idSW);
    put(LORT, idSW, c);
    vort[UPLT * NN + idS] = vort[LORT * NN + idSW];
    return;
  }
  if (i == 0) {
    put(LORT, idW, lort(idW));
    put(UPLT, idSW, uplt_n(idSW));
  }
  if (j == 0) {
    put(LORT, idSW, lort(idSW));
    put(UPLT, idS, uplt_n(idS));
  }
}

}  // namespace wtb
