// Vertical remap of the Lagrangian layers back to the hybrid sigma grid
// (remap_vertical_coordinates / remap_incompressible, src/remap.f90:18-76,
// 147-216): one thread per node column.  The node's old interfaces come from
// its layer masses (find_coordinates_incompressible, :235-257, porosity 1),
// the new ones from z_new = a_vert eta_surf + b_vert z_s; the buoyancy is
// remapped on the node's column and each of its three edge velocities on the
// column averaged with the neighbour at the edge's far end.  The column
// routines follow remap0 (:259-285), remap1 (:287-380) and remap2PPM
// (:382-495) with the reference's operand order; FP64, no FMA contraction.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace wtr {

constexpr int kRemapMaxNz = 64;
enum { REMAP_0 = 0, REMAP_1 = 1, REMAP_2PPM = 2 };

// remap0: piecewise constant (donor cell).
__device__ inline void remap0(int N, double* vnew, const double* znew, const double* vold, const double* zold) {
  double FC[kRemapMaxNz + 1];
  for (int k = 1; k <= N - 1; ++k) {
    const double dz = znew[k] - zold[k];
    FC[k] = fmin(dz, 0.0) * vold[k] + fmax(dz, 0.0) * vold[k + 1];
  }
  FC[0] = 0.0;
  FC[N] = 0.0;
  for (int k = 1; k <= N; ++k)
    vnew[k] = ((zold[k] - zold[k - 1]) * vold[k] + FC[k] - FC[k - 1]) / (znew[k] - znew[k - 1]);
}

// remap1: piecewise linear with the harmonic-mean slope and ten rounds of
// interface reconciliation under a minmod limiter (ENHANCE), Dirichlet ends.
__device__ inline void remap1(int N, double* vnew, const double* znew, const double* vold, const double* zold) {
  double Hz[kRemapMaxNz + 1], FC[kRemapMaxNz + 1], aL[kRemapMaxNz + 1], aR[kRemapMaxNz + 1];
  for (int k = 1; k <= N; ++k) Hz[k] = zold[k] - zold[k - 1];
  for (int k = N - 1; k >= 1; --k) FC[k] = (vold[k + 1] - vold[k]) / (Hz[k + 1] + Hz[k]);
  FC[0] = FC[1];
  FC[N] = FC[N - 1];
  for (int k = 1; k <= N; ++k) {
    double cff;
    if (FC[k] * FC[k - 1] < 0.0)
      cff = 0.0;
    else
      cff = 2 * FC[k] * FC[k - 1] / (FC[k] + FC[k - 1]);
    aR[k] = vold[k] + cff * Hz[k];
    aL[k] = vold[k] - cff * Hz[k];
  }
  for (int iter = 1; iter <= 10; ++iter) {
    for (int k = 1; k <= N - 1; ++k) FC[k] = 0.5 * (aR[k] + aL[k + 1]);
    FC[N] = aR[N];
    FC[0] = aL[1];
    for (int k = 1; k <= N; ++k) {
      const double dR = FC[k] - vold[k], dL = vold[k] - FC[k - 1];
      double cff;
      if (dR * dL < 0.0)
        cff = 0.0;
      else if (fabs(dR) > fabs(dL))
        cff = dL;
      else
        cff = dR;
      aR[k] = vold[k] + cff;
      aL[k] = vold[k] - cff;
    }
  }
  for (int k = 1; k <= N - 1; ++k) {
    const double dz = znew[k] - zold[k];
    double cff, cff1, dh;
    if (dz > 0.0) {
      cff = aL[k + 1];
      cff1 = aR[k + 1] - aL[k + 1];
      dh = Hz[k + 1];
    } else {
      cff = aR[k];
      cff1 = aR[k] - aL[k];
      dh = Hz[k];
    }
    FC[k] = dz * (cff + 0.5 * cff1 * dz / dh);
  }
  FC[0] = 0.0;
  FC[N] = 0.0;
  for (int k = 1; k <= N; ++k) vnew[k] = (Hz[k] * vold[k] + FC[k] - FC[k - 1]) / (znew[k] - znew[k - 1]);
}

// remap2PPM: Colella-Woodward PPM with limited slopes, Dirichlet ends, no
// interior limiting.
__device__ inline void remap2ppm(int N, double* vnew, const double* znew, const double* vold,
                                 const double* zold) {
  double Hz[kRemapMaxNz + 1], aL[kRemapMaxNz + 1], aR[kRemapMaxNz + 1], CF[kRemapMaxNz + 1],
      FC[kRemapMaxNz + 1], FC1[kRemapMaxNz + 1];
  for (int k = 1; k <= N; ++k) Hz[k] = zold[k] - zold[k - 1];
  for (int k = 1; k <= N - 1; ++k) {
    const double cff = 1.0 / (Hz[k] + Hz[k + 1]);
    CF[k] = cff * (vold[k + 1] * Hz[k] + vold[k] * Hz[k + 1]);
    FC[k] = cff * (vold[k + 1] - vold[k]);
  }
  for (int k = 2; k <= N - 1; ++k) {
    double cff = Hz[k] * ((2.0 * Hz[k - 1] + Hz[k]) * FC[k] + (2.0 * Hz[k + 1] + Hz[k]) * FC[k - 1]) /
                 (Hz[k - 1] + Hz[k] + Hz[k + 1]);
    const double cffR = 2.0 * (vold[k + 1] - vold[k]);
    const double cffL = 2.0 * (vold[k] - vold[k - 1]);
    if (cffR * cffL > 0.0) {
      if (fabs(cffL) < fabs(cff)) cff = cffL;
      if (fabs(cffR) < fabs(cff)) cff = cffR;
    } else {
      cff = 0.0;
    }
    FC1[k] = cff;
  }
  FC1[N] = Hz[N] * FC[N - 1];
  FC1[1] = Hz[1] * FC[1];
  for (int k = 1; k <= N - 1; ++k) {
    const int k1 = k - 1 > 1 ? k - 1 : 1;
    const int k2 = k + 2 < N ? k + 2 : N;
    const double cff = Hz[k1] + Hz[k] + Hz[k + 1] + Hz[k2];
    const double cffL = (Hz[k1] + Hz[k]) / (cff * (2.0 * Hz[k] + Hz[k + 1]));
    const double cffR = (Hz[k + 1] + Hz[k2]) / (cff * (Hz[k] + 2.0 * Hz[k + 1]));
    aR[k] = CF[k] + 2.0 * Hz[k] * Hz[k + 1] * (cffL - cffR) * FC[k] - cffL * Hz[k] * FC1[k + 1] +
            cffR * Hz[k + 1] * FC1[k];
    aL[k + 1] = aR[k];
  }
  aR[N] = 2.0 * vold[N] - aL[N];
  aL[1] = 2.0 * vold[1] - aR[1];
  for (int k = 1; k <= N; ++k) {
    CF[k] = 0.5 * (aR[k] - aL[k]);
    FC[k] = 0.5 * (aR[k] + aL[k]) - vold[k];
  }
  for (int k = 1; k <= N - 1; ++k) {
    const double dz = znew[k] - zold[k];
    double alpha, cff, cffR, cffL;
    if (dz > 0.0) {
      alpha = Hz[k + 1];
      cff = aL[k + 1];
      cffR = CF[k + 1];
      cffL = FC[k + 1];
    } else {
      alpha = -Hz[k];
      cff = aR[k];
      cffR = -CF[k];
      cffL = FC[k];
    }
    alpha = dz / alpha;
    FC[k] = dz * (cff + alpha * (cffR - cffL * (3.0 - 2.0 * alpha)));
  }
  FC[0] = 0.0;
  FC[N] = 0.0;
  for (int k = 1; k <= N; ++k) vnew[k] = (Hz[k] * vold[k] + FC[k] - FC[k - 1]) / (znew[k] - znew[k - 1]);
}

__device__ inline void remap_column(int type, int N, double* vnew, const double* znew, const double* vold,
                                    const double* zold) {
  if (type == REMAP_0)
    remap0(N, vnew, znew, vold, zold);
  else if (type == REMAP_1)
    remap1(N, vnew, znew, vold, zold);
  else
    remap2ppm(N, vnew, znew, vold, zold);
}

}  // namespace wtr

namespace wtr {

struct RemapLevel {
  int n, P;
  int64_t NN;
  const int* nsrc;
  const double* topo;
  const double* mean_m;
  const double* mean_t;
  const double* mold;  // the layer masses before the remap (every slot)
  double* mass;
  double* temp;
  double* velo;
};

// find_coordinates_incompressible (src/remap.f90:235-257) at slot x: old
// interfaces from the old masses, new ones a_vert eta_surf + b_vert z_s.
__device__ inline void column_coords(const RemapLevel& L, int nz, int x, const double* __restrict__ av,
                                     const double* __restrict__ bv, double rho0, double* zn, double* zo) {
  const double zs = L.topo[x];
  zo[0] = zs;
  for (int k = 1; k <= nz; ++k) {
    const int64_t o = (int64_t)(k - 1) * L.NN + x;
    const double rho_dz = L.mean_m[o] + L.mold[o];
    zo[k] = zo[k - 1] + rho_dz / (rho0 * 1.0);
  }
  const double eta = zo[nz];
  for (int k = 0; k <= nz; ++k) zn[k] = av[k] * eta + bv[k] * zs;
}

// remap_incompressible (src/remap.f90:147-216) of every own-source node of
// [0, n]^2 (the pole slots: masses only).  a_vert, b_vert: nz + 1 values,
// index 0 at the bottom.
__global__ void __launch_bounds__(128) k_remap_incompressible(RemapLevel L, int nz, int type,
                                                              const double* __restrict__ av,
                                                              const double* __restrict__ bv, double rho0) {
  const int m = L.n + 1;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)10 * m * m) return;
  const int d = (int)(t / ((int64_t)m * m));
  const int r = (int)(t - (int64_t)d * m * m);
  const int j = r / m, i = r - j * m;
  const int x = (d * L.P + j + 2) * L.P + i + 2;
  if (L.nsrc[x] != x) return;
  const bool pole = i == L.n || j == L.n;
  double zn[kRemapMaxNz + 1], zo[kRemapMaxNz + 1], vo[kRemapMaxNz + 1], vn[kRemapMaxNz + 1];
  column_coords(L, nz, x, av, bv, rho0, zn, zo);
  double dz[kRemapMaxNz + 1];
  for (int k = 1; k <= nz; ++k) dz[k] = zn[k] - zn[k - 1];
  if (!pole) {
    // edge velocities RT, DG, UP on the columns averaged with the node at the edge's far end
    const int xr[3] = {x + 1, x + L.P + 1, x + L.P};
    for (int e = 0; e < 3; ++e) {
      double zen[kRemapMaxNz + 1], zeo[kRemapMaxNz + 1];
      column_coords(L, nz, L.nsrc[xr[e]], av, bv, rho0, zen, zeo);
      for (int k = 0; k <= nz; ++k) {
        zen[k] = 0.5 * (zn[k] + zen[k]);
        zeo[k] = 0.5 * (zo[k] + zeo[k]);
      }
      for (int k = 1; k <= nz; ++k) vo[k] = L.velo[(int64_t)(k - 1) * 3 * L.NN + e * L.NN + x];
      remap_column(type, nz, vn, zen, vo, zeo);
      for (int k = 1; k <= nz; ++k) L.velo[(int64_t)(k - 1) * 3 * L.NN + e * L.NN + x] = vn[k];
    }
  }
  // buoyancy of the old state, remapped; new masses from the new thicknesses
  for (int k = 1; k <= nz; ++k) {
    const int64_t o = (int64_t)(k - 1) * L.NN + x;
    vo[k] = (L.mean_t[o] + L.temp[o]) / (L.mean_m[o] + L.mass[o]);
  }
  remap_column(type, nz, vn, zn, vo, zo);
  for (int k = 1; k <= nz; ++k) {
    const int64_t o = (int64_t)(k - 1) * L.NN + x;
    const double rho = rho0 * 1.0;
    const double rho_dz = rho * dz[k];
    L.mass[o] = rho_dz - L.mean_m[o];
    L.temp[o] = rho_dz * vn[k] - L.mean_t[o];
  }
}

// cal_min_mass (src/main.f90:642-693), incompressible case on the A/B hybrid
// grid with porosity 1: the smallest rho_dz_k / (rho0 dz_k) over the layers of
// the level's own nodes in [0, n]^2 (the owned nodes and the pole slots) whose
// node mask is at least ADJZONE (8; every such node when mask_n is null), with
// dz_k = (b_vert[k+1] - b_vert[k]) z_s the layer of the zero-perturbation grid
// and rho_dz_k = mean_m + mass.  A layer mass that is not positive or not a
// number counts as 0 (where the reference aborts: "A layer has collapsed").
// The minimum is kept as the bits of a non-negative double, which atomicMin
// orders as the values.
__global__ void __launch_bounds__(128) k_min_mass(RemapLevel L, int nz, const double* __restrict__ bv, double rho0,
                                                  const int* __restrict__ mask_n,
                                                  unsigned long long* __restrict__ out) {
  const int m = L.n + 1;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long key = ~0ull;
  if (t < (int64_t)10 * m * m) {
    const int d = (int)(t / ((int64_t)m * m));
    const int r = (int)(t - (int64_t)d * m * m);
    const int j = r / m, i = r - j * m;
    const int x = (d * L.P + j + 2) * L.P + i + 2;
    if (L.nsrc[x] == x && (!mask_n || mask_n[x] >= 8)) {
      const double zs = L.topo[x];
      double mn = 1e16;
      for (int k = 0; k < nz; ++k) {
        const double rho_dz = L.mass[(int64_t)k * L.NN + x] + L.mean_m[(int64_t)k * L.NN + x];
        const double rel = rho_dz / (rho0 * (bv[k + 1] * zs - bv[k] * zs));
        if (!(rho_dz > 0.0) || !(rel > 0.0)) {  // collapsed, or not a number
          mn = 0.0;
          break;
        }
        mn = fmin(mn, rel);
      }
      key = (unsigned long long)__double_as_longlong(mn);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_down_sync(0xffffffffu, key, o);
    key = v < key ? v : key;
  }
  if ((threadIdx.x & 31) == 0 && key != ~0ull) atomicMin(out, key);
}

}  // namespace wtr
