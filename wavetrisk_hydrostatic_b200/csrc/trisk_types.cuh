// Plain data types shared by the TRiSK kernels and the device context.
#pragma once
#include <cuda.h>

#include <cstdint>

namespace wtk {

enum { RT = 0, DG = 1, UP = 2 };
enum { LORT = 0, UPLT = 1 };

// A level's work list: the padded slots a kernel computes (those of the
// needed-node map), their count on the device, built inside the step's graph
// (need_map.cuh: k_list_count, k_list_scan, k_list_write).
struct NodeList {
  const int* ids;
  const int* count;
};

struct LevelDev {
  int n, P;
  int NN;  // 10*P*P; 6*NN < 2^31, so offsets inside one layer fit an int
  const double* __restrict__ len;      // 3*NN
  const double* __restrict__ pedlen;   // 3*NN
  const double* __restrict__ part;     // 6*NN
  const double* __restrict__ hex_inv;  // NN
  const double* __restrict__ triarea;  // 2*NN
  const double* __restrict__ coriolis; // 2*NN
  const double* __restrict__ topo;     // NN
  // Ghost remaps (cp_bdry_inside, src/comm.f90:785): node x reads x' = nsrc[x];
  // edge slot e reads slot esrc[e] >> 1, negated when esrc[e] & 1.
  const int* __restrict__ nsrc;        // NN
  const int* __restrict__ esrc;        // 3*NN
};

// Tensor maps of one handle's trend inputs, dims (x = P, y = P, lozenge = 10,
// plane); consumed by the TMA-staged trend kernel.
struct TrendMaps {
  CUtensorMap hfm, hft, qe;       // plane = 3*layer + edge orientation
  CUtensorMap theta, bern, phik;  // plane = layer
  CUtensorMap part;               // plane = area part 0..5
  CUtensorMap hinv;               // one plane
};

// Tensor maps of the step1 inputs for one stage state buffer.
struct Step1Maps {
  CUtensorMap mass, temp, velo;  // plane = layer (velo: 3*layer + edge orientation)
  CUtensorMap mean_m, mean_t;    // plane = layer
  CUtensorMap len, ped, part, cor;  // plane = edge orientation / area part / triangle
};

// Inputs and outputs of the trend kernels (trisk_kernels.cuh, trisk_tma.cuh).
struct TrendIO {
  const double* __restrict__ theta;  // Theta/rho of the stage state at [0, n]^2 (k_step1)
  const double* __restrict__ qe;
  const double* __restrict__ hfm;
  const double* __restrict__ hft;
  const double* __restrict__ bern;
  const double* __restrict__ phik;
  // MODE_RK
  const double* base_m; const double* base_t; const double* base_v;
  double* dst_m; double* dst_t; double* dst_v;
  double h;
  // MODE_TREND (and dm, dtt in MODE_ML)
  double* dm; double* dtt; double* dv;
  // MODE_ML: the level's node masks, the velocity source it writes on
  // [0, n)^2, and the needed-node map (need_map.cuh) or null
  const int* mask_n; double* src; const unsigned char* need;
  // MODE_ML with u_star: velocity sub-step base + h * (trend + th1 * grad)
  const double* grad; double th1;
};

struct Phys {
  double grav, ref_density, p_top;
};

}  // namespace wtk
