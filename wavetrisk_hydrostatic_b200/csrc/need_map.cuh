// Nodes of the finest level whose step1 and trend results can reach the state
// after WT_after_step.  After every RK stage the finest level is rebuilt by
// the inverse transform from the next coarser level and the wavelets kept by
// compress_wavelets, so its stage results are read only
//   * by the trend where mask_n >= TRSK (stencils of radius 2),
//   * by the forward wavelets of slots with mask >= ADJZONE (radius 2),
//   * by the restriction into parents with mask >= RESTRCT (radius 3 around the
//     parent's child node), and by the coarser trend's restricted velocity
//     source (child edges with mask >= ADJZONE).
// The map seeds those nodes and dilates them NEED_R hex steps through the ghost
// remaps; the lozenge corners (pentagons, poles), whose neighbourhoods the
// remaps describe only for the stencils that use them, are always in the map.
// Values of the map are read through nsrc: need[nsrc[x]].
#pragma once
#include "wavelet_kernels.cuh"

namespace wtw {

#ifndef WT_NEED_R
#define WT_NEED_R 6
#endif
constexpr int NEED_R = WT_NEED_R;

// seed of every padded slot of level C (parent level P)
__global__ void k_need_seed(WLev C, WLev P, unsigned char* __restrict__ out) {
  const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= C.NN) return;
  const int PP = C.P * C.P;
  const int d = (int)(x / PP), r = (int)(x - (int64_t)d * PP);
  const int i = r % C.P - 2, j = r / C.P - 2, n = C.n;
  int v;
  if (i >= 0 && j >= 0 && i < n && j < n) {
    v = C.mask_n[x] >= TRSK || C.mask_e[x] >= TRSK || C.mask_e[C.NN + x] >= TRSK || C.mask_e[2 * C.NN + x] >= TRSK;
    if (!v && !(i & 1) && !(j & 1)) {
      const int p = nid(P, d, i / 2, j / 2);
      v = P.mask_n[p] >= RESTRCT || P.mask_e[p] >= RESTRCT || P.mask_e[P.NN + p] >= RESTRCT ||
          P.mask_e[2 * P.NN + p] >= RESTRCT;
    }
    const int c = NEED_R + 1;
    if ((i <= c || i >= n - 1 - c) && (j <= c || j >= n - 1 - c)) v = 1;
  } else {
    v = __ldg(C.nsrc + x) == (int)x;  // a slot outside [0, n)^2 that is its own source
  }
  out[x] = (unsigned char)v;
}

// one hex step: a slot is needed if it or one of its six neighbours is
__global__ void k_need_dilate(WLev C, const unsigned char* __restrict__ in, unsigned char* __restrict__ out) {
  const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= C.NN) return;
  const int PP = C.P * C.P;
  const int d = (int)(x / PP), r = (int)(x - (int64_t)d * PP);
  const int i = r % C.P - 2, j = r / C.P - 2;
  int v = in[__ldg(C.nsrc + x)];
  const int di[6] = {1, -1, 0, 0, 1, -1}, dj[6] = {0, 0, 1, -1, 1, -1};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int a = i + di[q], b = j + dj[q];
    if (inr(C, a, b)) v |= in[__ldg(C.nsrc + nid(C, d, a, b))];
  }
  out[x] = (unsigned char)v;
}

}  // namespace wtw
