// Plain data types shared by the TRiSK kernels and the device context.
#pragma once
#include <cstdint>

namespace wtk {

enum { RT = 0, DG = 1, UP = 2 };
enum { LORT = 0, UPLT = 1 };

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

struct Phys {
  double grav, ref_density, p_top;
};

}  // namespace wtk
