// Interscale wavelet kernels with the layer loop inside the thread: one thread
// per (lozenge, parent node) resolves its ghost remaps, masks, overlap areas
// and interpolation weights once, then runs every layer (and both scalars)
// with the same expressions, in the same operand order, as the reference's
// per-node routines (src/wavelet.f90).  A warp still covers consecutive
// parents, so each layer's loads and stores stay coalesced along rows.
#pragma once
#include "wavelet_kernels.cuh"

// Minimum resident blocks per SM of the layer-group kernels, i.e. register
// caps.  Measured on B200 (WT_after_step, J5..J7 x 16 / J6..J8 x 32): no caps
// 0.80 / 4.92 ms; scalar and outer 6, inner 4 (the inner kernels spill about
// 60 bytes) 0.66 / 3.83 ms; 8, 8, 4 0.67 / 3.76 ms.
#ifndef WL_MINB_SCALAR
#define WL_MINB_SCALAR 6
#endif
#ifndef WL_MINB_OUTER
#define WL_MINB_OUTER 6
#endif
#ifndef WL_MINB_INNER
#define WL_MINB_INNER 4
#endif

namespace wtw {

// Codes of the remapped readers: node code = source node, edge code = source
// slot * 2 + negate; -1 outside the padded level (the reader returns 0).
__device__ __forceinline__ int wn_code(const WLev& L, int d, int i, int j) {
  return inr(L, i, j) ? __ldg(L.nsrc + nid(L, d, i, j)) : -1;
}
__device__ __forceinline__ int we_code(const WLev& L, int e, int d, int i, int j) {
  return inr(L, i, j) ? __ldg(L.esrc + e * L.NN + nid(L, d, i, j)) : -1;
}
__device__ __forceinline__ double wn(const double* __restrict__ f, int c) { return c < 0 ? 0.0 : f[c]; }
__device__ __forceinline__ double we(const double* __restrict__ f, int c) {
  if (c < 0) return 0.0;
  const double v = f[c >> 1];
  return (c & 1) ? -v : v;
}

// Parent (d, ip, jp) of [0, m)^2 and layer range [k0, k1) of this thread: the
// layers are split into groups of lpt (grid: 10 m^2 threads per group, group
// slowest), trading the once-per-thread setup against the number of threads.
__device__ __forceinline__ bool parent_of(int m, int nz, int lpt, int& d, int& ip, int& jp, int& k0, int& k1) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)10 * m * m;
  const int ng = (nz + lpt - 1) / lpt;
  if (t >= per * ng) return false;
  const int g = (int)(t / per);
  const int r0 = (int)(t - (int64_t)g * per);
  d = r0 / (m * m);
  const int r = r0 - d * m * m;
  jp = r / m;
  ip = r - jp * m;
  k0 = g * lpt;
  k1 = min(nz, k0 + lpt);
  return true;
}

// Whether the inverse transform rebuilds parent (d, ip, jp) of level Pa: every
// parent when rec is null, else where the parent map rec (need_map.cuh) says so.
__device__ __forceinline__ bool rebuilt(const unsigned char* __restrict__ rec, const WLev& Pa, int d, int ip, int jp) {
  return !rec || rec[__ldg(Pa.nsrc + nid(Pa, d, ip, jp))];
}

// Interp_node's four weights and hex_inv at child node (i, j) with its four
// neighbours' codes.
struct NodeInterp {
  double o[4], h;
  int c[4];
};
__device__ __forceinline__ void node_interp(NodeInterp& N, const WLev& C, int d, int i, int j, int i1, int j1,
                                            int i2, int j2, int i3, int j3, int i4, int j4) {
#pragma unroll
  for (int q = 0; q < 4; ++q) N.o[q] = oa(C, d, i, j, q + 1);
  N.h = hv(C, d, i, j);
  N.c[0] = wn_code(C, d, i1, j1);
  N.c[1] = wn_code(C, d, i2, j2);
  N.c[2] = wn_code(C, d, i3, j3);
  N.c[3] = wn_code(C, d, i4, j4);
}
__device__ __forceinline__ double node_eval(const NodeInterp& N, const double* __restrict__ s) {
  return (N.o[0] * wn(s, N.c[0]) + N.o[1] * wn(s, N.c[1]) + N.o[2] * wn(s, N.c[2]) + N.o[3] * wn(s, N.c[3])) * N.h;
}
// The three new child nodes of parent (ip, jp): E (i+1, j), NE (i+1, j+1), N (i, j+1).
__device__ __forceinline__ void child_interps(NodeInterp N[3], const WLev& C, int d, int i, int j) {
  node_interp(N[0], C, d, i + 1, j, i, j, i + 2, j, i + 2, j + 2, i, j - 2);
  node_interp(N[1], C, d, i + 1, j + 1, i + 2, j + 2, i, j, i + 2, j, i, j + 2);
  node_interp(N[2], C, d, i, j + 1, i, j, i, j + 2, i - 2, j, i + 2, j + 2);
}

// Compute_scalar_wavelets (src/wavelet.f90:642-670), parents [0, np)^2.
// CMP 1: the wavelets are not zeroed beforehand and compress_wavelets follows
// (WT_after_step), so each of the three child slots is written, with 0 where
// the child's mask is below ADJZONE; the other slots of the level (parent-
// coincident nodes, ghost rows) hold 0 from the last zeroing.  CMP 2: the same
// when the slots below ADJZONE already hold 0 (compress_wavelets ran under the
// current masks), so only the kept slots are written.  CMP 0: the forward
// transform (wavelets zeroed beforehand, no compression).
template <int CMP>
__global__ void __launch_bounds__(128, WL_MINB_SCALAR) k_scalar_wc_l(WLev C, int np, int nz, int lpt, ParentList PL) {
  auto body = [&](int d, int ip, int jp, int k0, int k1) {
    const int i = 2 * ip, j = 2 * jp;
    const int ci[3] = {i + 1, i + 1, i}, cj[3] = {j, j + 1, j + 1};
    bool on[3];
    int self[3], at[3];
  #pragma unroll
    for (int q = 0; q < 3; ++q) {
      on[q] = mn(C, d, ci[q], cj[q]) >= ADJZONE;
      self[q] = wn_code(C, d, ci[q], cj[q]);
      at[q] = nid(C, d, ci[q], cj[q]);
    }
    if (!(on[0] || on[1] || on[2])) {
      if (CMP == 1)
        for (int k = k0; k < k1; ++k)
  #pragma unroll
          for (int q = 0; q < 3; ++q) {
            C.wm[(int64_t)k * C.NN + at[q]] = 0.0;
            C.wt[(int64_t)k * C.NN + at[q]] = 0.0;
          }
      return;
    }
    NodeInterp N[3];
    child_interps(N, C, d, i, j);
    for (int k = k0; k < k1; ++k)
  #pragma unroll
      for (int v = 0; v < 2; ++v) {
        const double* s = (v == 0 ? C.sm : C.st) + (int64_t)k * C.NN;
        double* wc = (v == 0 ? C.wm : C.wt) + (int64_t)k * C.NN;
  #pragma unroll
        for (int q = 0; q < 3; ++q)
          if (on[q])
            wc[at[q]] = wn(s, self[q]) - node_eval(N[q], s);
          else if (CMP == 1)
            wc[at[q]] = 0.0;
      }
  };
  if (PL.ids) {
    for_parents(np, np, nz, lpt, PL, body);
    return;
  }
  int d, ip, jp, k0, k1;
  if (!parent_of(np, nz, lpt, d, ip, jp, k0, k1)) return;
  body(d, ip, jp, k0, k1);
}

// Reconstruct_scalar (src/wavelet.f90:614-640), parents [0, np)^2.
__global__ void __launch_bounds__(128, WL_MINB_SCALAR) k_recon_scalar_l(WLev Pa, WLev C, int np, int nz, int lpt,
                                                                         const unsigned char* __restrict__ rec,
                                                                         ParentList PL) {
  auto body = [&](int d, int ip, int jp, int k0, int k1) {
    if (!rebuilt(rec, Pa, d, ip, jp)) return;
    const int i = 2 * ip, j = 2 * jp;
    const int ci[3] = {i + 1, i + 1, i}, cj[3] = {j, j + 1, j + 1};
    int self[3], at[3];
  #pragma unroll
    for (int q = 0; q < 3; ++q) {
      self[q] = wn_code(C, d, ci[q], cj[q]);
      at[q] = nid(C, d, ci[q], cj[q]);
    }
    NodeInterp N[3];
    child_interps(N, C, d, i, j);
    for (int k = k0; k < k1; ++k)
  #pragma unroll
      for (int v = 0; v < 2; ++v) {
        const double* wc = (v == 0 ? C.wm : C.wt) + (int64_t)k * C.NN;
        double* s = (v == 0 ? C.sm : C.st) + (int64_t)k * C.NN;
        double r[3];
  #pragma unroll
        for (int q = 0; q < 3; ++q) r[q] = node_eval(N[q], s) + wn(wc, self[q]);
  #pragma unroll
        for (int q = 0; q < 3; ++q) s[at[q]] = r[q];
      }
  };
  if (PL.ids) {
    for_parents(np, np, nz, lpt, PL, body);
    return;
  }
  int d, ip, jp, k0, k1;
  if (!parent_of(np, nz, lpt, d, ip, jp, k0, k1)) return;
  body(d, ip, jp, k0, k1);
}

// Prolong_scalar (src/wavelet.f90:571-612), parents [0, np]^2: the eleven
// lifting terms the reference sums.
__global__ void __launch_bounds__(128, WL_MINB_SCALAR) k_prolong_l(WLev Pa, WLev C, int nz, int lpt,
                                                                    const unsigned char* __restrict__ rec,
                                                                    ParentList PL) {
  const int np = Pa.n;
  auto body = [&](int d, int ip, int jp, int k0, int k1) {
    if (!rebuilt(rec, Pa, d, ip, jp)) return;
    const int i = 2 * ip, j = 2 * jp;
    if (mn(C, d, i, j) == FROZEN) return;
    const int ti[11] = {i + 1, i + 1, i + 2, i, i - 1, i - 1, i - 2, i - 1, i, i - 1, i + 1};
    const int tj[11] = {j, j + 1, j + 1, j + 1, j, j + 1, j - 1, j - 1, j - 1, j - 2, j - 1};
    const int tk[11] = {1, 2, 3, 1, 2, 3, 4, 1, 2, 3, 4};
    double w[11];
    int c[11];
  #pragma unroll
    for (int q = 0; q < 11; ++q) {
      w[q] = oa(C, d, ti[q], tj[q], tk[q]);
      c[q] = wn_code(C, d, ti[q], tj[q]);
    }
    const double hp = hv(Pa, d, ip, jp);
    const int cp = wn_code(Pa, d, ip, jp);
    const int at = nid(C, d, i, j);
    for (int k = k0; k < k1; ++k)
  #pragma unroll
      for (int v = 0; v < 2; ++v) {
        const double* wc = (v == 0 ? C.wm : C.wt) + (int64_t)k * C.NN;
        const double* sp = (v == 0 ? Pa.sm : Pa.st) + (int64_t)k * Pa.NN;
        double* s = (v == 0 ? C.sm : C.st) + (int64_t)k * C.NN;
        double sum = wn(wc, c[0]) * w[0];
  #pragma unroll
        for (int q = 1; q < 11; ++q) sum = sum + wn(wc, c[q]) * w[q];
        s[at] = wn(sp, cp) - sum * hp;
      }
  };
  if (PL.ids) {
    for_parents(np, np + 1, nz, lpt, PL, body);
    return;
  }
  int d, ip, jp, k0, k1;
  if (!parent_of(np + 1, nz, lpt, d, ip, jp, k0, k1)) return;
  body(d, ip, jp, k0, k1);
}

// Interp_outer_velo (src/wavelet.f90:1064-1094) of the outer child edge e of
// parent (ip, jp): the nine weights and the parent edge codes of its terms.
struct OuterInterp {
  double w[9];
  int c[13];  // t0, t1..t4, then the pairs of t5..t8
};
__device__ __forceinline__ void outer_interp(OuterInterp& O, const WLev& Pa, const WLev& C, int d, int ip, int jp,
                                             int ic, int jc, int e) {
  const int hs = c_hex_s_offs[e];
  auto code = [&](const int* off, int col) {
    return we_code(Pa, c_hex_sides[col][2], d, ip + off[0] + c_hex_sides[col][0], jp + off[1] + c_hex_sides[col][1]);
  };
  const int* e1 = c_end_pt[e][0];
  const int* e2 = c_end_pt[e][1];
  const int* o1 = c_opp_no[e][0];
  const int* o2 = c_opp_no[e][1];
  O.c[0] = we_code(Pa, e, d, ip, jp);
  O.c[1] = code(e2, hs + 2);
  O.c[2] = code(e1, hs + 3);
  O.c[3] = code(e1, hs + 5);
  O.c[4] = code(e2, hs + 0);
  O.c[5] = code(o1, hs + 1);
  O.c[6] = code(e1, hs + 2);
  O.c[7] = code(e2, hs + 3);
  O.c[8] = code(o1, hs + 4);
  O.c[9] = code(o2, hs + 4);
  O.c[10] = code(e2, hs + 5);
  O.c[11] = code(e1, hs + 0);
  O.c[12] = code(o2, hs + 1);
#pragma unroll
  for (int q = 0; q < 9; ++q) O.w[q] = c_iu_base[q] + iw(C, q, d, ic, jc);
}
__device__ __forceinline__ double outer_eval(const OuterInterp& O, const double* __restrict__ vp, double& t0) {
  double t[9];
  t[0] = we(vp, O.c[0]);
  t[1] = we(vp, O.c[1]);
  t[2] = we(vp, O.c[2]);
  t[3] = we(vp, O.c[3]);
  t[4] = we(vp, O.c[4]);
  t[5] = we(vp, O.c[5]) - we(vp, O.c[6]);
  t[6] = we(vp, O.c[7]) - we(vp, O.c[8]);
  t[7] = we(vp, O.c[9]) - we(vp, O.c[10]);
  t[8] = we(vp, O.c[11]) - we(vp, O.c[12]);
  t0 = t[0];
  double sum = 0.0;
#pragma unroll
  for (int q = 0; q < 9; ++q) sum = sum + O.w[q] * t[q];
  return sum;
}

// Compute_velo_wavelets' outer edges (src/wavelet.f90:672-710), parents
// [0, np)^2, with the pentagon corrections of the corner parents.  CMP as for
// k_scalar_wc_l: both child slots of each parent edge are written (CMP 1; CMP 2
// leaves out the pairs whose slots hold 0 already) and compress_vector's rule
// (0 where the slot's own mask is below ADJZONE) is applied to them, after the
// pentagon corrections in the corner parents.
template <int CMP>
__global__ void __launch_bounds__(128, WL_MINB_OUTER) k_velo_wc_outer_l(WLev Pa, WLev C, int nz, int lpt, ParentList PL) {
  auto body = [&](int d, int ip, int jp, int k0, int k1) {
    const int i = 2 * ip, j = 2 * jp;
    const bool corner = (ip == 0 || ip == Pa.n - 1) && (jp == 0 || jp == Pa.n - 1);
    for (int e = 0; e < 3; ++e) {
      const int a1 = i + c_end_pt[e][0][0], b1 = j + c_end_pt[e][0][1];
      const int a2 = i + c_end_pt[e][1][0], b2 = j + c_end_pt[e][1][1];
      const int x2 = e * C.NN + nid(C, d, a2, b2), x1 = e * C.NN + nid(C, d, a1, b1);
      if (me(C, e, d, a2, b2) < ADJZONE) {
        if (CMP == 1)
          for (int k = k0; k < k1; ++k) {
            C.wv[(int64_t)k * 3 * C.NN + x2] = 0.0;
            C.wv[(int64_t)k * 3 * C.NN + x1] = 0.0;
          }
        else if (CMP == 2 && me(C, e, d, a1, b1) >= ADJZONE)  // a kept slot that the pair leaves at 0
          for (int k = k0; k < k1; ++k) C.wv[(int64_t)k * 3 * C.NN + x1] = 0.0;
        continue;
      }
      const bool keep1 = CMP == 0 || corner || me(C, e, d, a1, b1) >= ADJZONE;
      OuterInterp O;
      outer_interp(O, Pa, C, d, ip, jp, a2, b2, e);
      const int cv = we_code(C, e, d, a2, b2);
      for (int k = k0; k < k1; ++k) {
        const double* vp = Pa.sv + (int64_t)k * 3 * Pa.NN;
        const double* v = C.sv + (int64_t)k * 3 * C.NN;
        double* wc = C.wv + (int64_t)k * 3 * C.NN;
        double t0;
        const double u = outer_eval(O, vp, t0);
        const double w = we(v, cv) - u;
        wc[x2] = w;
        wc[x1] = keep1 ? -w : 0.0;
      }
    }
    if (corner) {
      for (int k = k0; k < k1; ++k)
        penta_compute(Pa, C, Pa.sv + (int64_t)k * 3 * Pa.NN, C.wv + (int64_t)k * 3 * C.NN, d, ip, jp);
      if (CMP)
        for (int e = 0; e < 3; ++e)
  #pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int a = i + c_end_pt[e][h][0], b = j + c_end_pt[e][h][1];
            if (me(C, e, d, a, b) >= ADJZONE) continue;
            const int x = e * C.NN + nid(C, d, a, b);
            for (int k = k0; k < k1; ++k) C.wv[(int64_t)k * 3 * C.NN + x] = 0.0;
          }
    }
  };
  if (PL.ids) {
    for_parents(Pa.n, Pa.n, nz, lpt, PL, body);
    return;
  }
  int d, ip, jp, k0, k1;
  if (!parent_of(Pa.n, nz, lpt, d, ip, jp, k0, k1)) return;
  body(d, ip, jp, k0, k1);
}

// Interp_inner_velo (src/wavelet.f90:1005-1062) of parent (ip, jp): parent
// circulation terms and the six inner child edges' coefficients.
struct InnerInterp {
  double lp[5], tp[2];     // parent lengths DG(ip,jp), UP(ip+1,jp), RT(ip,jp), UP(ip,jp), RT(ip,jp+1); areas
  int cp[5];               // their codes
  double lc[10];           // child lengths of the ten edges in the circulation terms
  int cc[10];              // their codes
  double tc[6], den[6];    // child triangle areas and the target edges' lengths
  int ct[6], xt[6];        // target edges: codes and slots
};
__device__ __forceinline__ void inner_interp(InnerInterp& I, const WLev& Pa, const WLev& C, int d, int ip, int jp) {
  const int pe[5] = {DG, UP, RT, UP, RT};
  const int pi[5] = {ip, ip + 1, ip, ip, ip};
  const int pj[5] = {jp, jp, jp, jp, jp + 1};
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    I.lp[q] = ln(Pa, pe[q], d, pi[q], pj[q]);
    I.cp[q] = we_code(Pa, pe[q], d, pi[q], pj[q]);
  }
  I.tp[0] = ta(Pa, LORT, d, ip, jp);
  I.tp[1] = ta(Pa, UPLT, d, ip, jp);
  const int i = 2 * ip, j = 2 * jp;
  // RT(i,j) DG(i,j) RT(i+1,j) UP(i+2,j) DG(i+1,j+1) UP(i+2,j+1) UP(i,j) UP(i,j+1) RT(i,j+2) RT(i+1,j+2)
  const int ce[10] = {RT, DG, RT, UP, DG, UP, UP, UP, RT, RT};
  const int ci[10] = {i, i, i + 1, i + 2, i + 1, i + 2, i, i, i, i + 1};
  const int cj[10] = {j, j, j, j, j + 1, j + 1, j, j + 1, j + 2, j + 2};
#pragma unroll
  for (int q = 0; q < 10; ++q) {
    I.lc[q] = ln(C, ce[q], d, ci[q], cj[q]);
    I.cc[q] = we_code(C, ce[q], d, ci[q], cj[q]);
  }
  const int tt[6] = {LORT, LORT, LORT, UPLT, UPLT, UPLT};
  const int ti[6] = {i, i + 1, i + 1, i, i, i + 1};
  const int tj[6] = {j, j, j + 1, j, j + 1, j + 1};
  // target edges UP(i+1,j) DG(i+1,j) RT(i+1,j+1) RT(i,j+1) DG(i,j+1) UP(i+1,j+1)
  const int ge[6] = {UP, DG, RT, RT, DG, UP};
  const int gi[6] = {i + 1, i + 1, i + 1, i, i, i + 1};
  const int gj[6] = {j, j, j + 1, j + 1, j + 1, j + 1};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    I.tc[q] = ta(C, tt[q], d, ti[q], tj[q]);
    I.den[q] = ln(C, ge[q], d, gi[q], gj[q]);
    I.ct[q] = we_code(C, ge[q], d, gi[q], gj[q]);
    I.xt[q] = ge[q] * C.NN + nid(C, d, gi[q], gj[q]);
  }
}
__device__ __forceinline__ void inner_eval(const InnerInterp& I, const double* __restrict__ vp,
                                           const double* __restrict__ v, double u[6]) {
  const double pDG = we(vp, I.cp[0]) * I.lp[0];
  const double curl0 = (pDG + we(vp, I.cp[1]) * I.lp[1] + we(vp, I.cp[2]) * I.lp[2]) / I.tp[0];
  const double curl1 = (pDG + we(vp, I.cp[3]) * I.lp[3] + we(vp, I.cp[4]) * I.lp[4]) / I.tp[1];
  double pr[10];
#pragma unroll
  for (int q = 0; q < 10; ++q) pr[q] = we(v, I.cc[q]) * I.lc[q];
  u[0] = (I.tc[0] * curl0 - pr[0] - pr[1]) / I.den[0];
  u[1] = (I.tc[1] * curl0 - pr[2] - pr[3]) / I.den[1];
  u[2] = (I.tc[2] * curl0 - pr[4] - pr[5]) / I.den[2];
  u[3] = (I.tc[3] * curl1 - pr[6] - pr[1]) / I.den[3];
  u[4] = (I.tc[4] * curl1 - pr[7] - pr[8]) / I.den[4];
  u[5] = (I.tc[5] * curl1 - pr[4] - pr[9]) / I.den[5];
}

// Compute_velo_wavelets' inner edges (src/wavelet.f90:672-710), parents
// [0, np)^2; CMP as for k_scalar_wc_l.
template <int CMP>
__global__ void __launch_bounds__(128, WL_MINB_INNER) k_velo_wc_inner_l(WLev Pa, WLev C, int nz, int lpt, ParentList PL) {
  auto body = [&](int d, int ip, int jp, int k0, int k1) {
    const int i = 2 * ip, j = 2 * jp;
    const int ge[6] = {UP, DG, RT, RT, DG, UP};
    const int gi[6] = {i + 1, i + 1, i + 1, i, i, i + 1};
    const int gj[6] = {j, j, j + 1, j + 1, j + 1, j + 1};
    bool on[6];
    bool any = false;
  #pragma unroll
    for (int q = 0; q < 6; ++q) {
      on[q] = me(C, ge[q], d, gi[q], gj[q]) >= ADJZONE;
      any = any || on[q];
    }
    if (!any) {
      if (CMP == 1)
        for (int k = k0; k < k1; ++k)
  #pragma unroll
          for (int q = 0; q < 6; ++q) C.wv[(int64_t)k * 3 * C.NN + ge[q] * C.NN + nid(C, d, gi[q], gj[q])] = 0.0;
      return;
    }
    InnerInterp I;
    inner_interp(I, Pa, C, d, ip, jp);
    for (int k = k0; k < k1; ++k) {
      const double* vp = Pa.sv + (int64_t)k * 3 * Pa.NN;
      const double* v = C.sv + (int64_t)k * 3 * C.NN;
      double* wc = C.wv + (int64_t)k * 3 * C.NN;
      double u[6];
      inner_eval(I, vp, v, u);
  #pragma unroll
      for (int q = 0; q < 6; ++q)
        if (on[q])
          wc[I.xt[q]] = we(v, I.ct[q]) - u[q];
        else if (CMP == 1)
          wc[I.xt[q]] = 0.0;
    }
  };
  if (PL.ids) {
    for_parents(Pa.n, Pa.n, nz, lpt, PL, body);
    return;
  }
  int d, ip, jp, k0, k1;
  if (!parent_of(Pa.n, nz, lpt, d, ip, jp, k0, k1)) return;
  body(d, ip, jp, k0, k1);
}

// ---------------------------------------------------------------------------
// Velocity reconstruction from per-parent plans.  Everything of
// Interp_outer_velo and Interp_inner_velo that does not depend on the layer
// (remap codes of the parent and child edges, the outer weights Iu_Base_Wgt +
// I_u_wgt, lengths and triangle areas) is geometry: k_outer_plan and
// k_inner_plan store it once per hierarchy (structure of arrays over the
// parents), and the reconstruction kernels stage 32 parents' plans in shared
// memory.  Block (32, ny): 32 consecutive parents, ny threads per parent taking
// layers y, y + ny, ...  Same expression trees and operand order as the
// reference's routines.  Measured on B200 against the per-thread kernels
// (k_*_l): inverse transform J5..J7 x 16 0.247 vs 0.266 ms, J6..J8 x 32 1.62 vs
// 1.81 ms; the same plans in the forward wavelet kernels were slower (J5..J7 x
// 16 forward 0.459 vs 0.429 ms), so those resolve the geometry per thread.
//
// Outer plan, parents [0, np]^2 (u = (d*(np+1) + jp)*(np+1) + ip): per edge e
// int slots e*14 + (0-12: Interp_outer_velo's parent codes, 13: the child edge
// (a2, b2)'s code), double slots e*9 + (0-8: weights).
constexpr int OP_NI = 42, OP_ND = 27;
// Minimum resident blocks per SM of the inner-edge plan kernels (register cap):
// uncapped they take about 148 registers, one block per SM.  Over the parent
// work lists of the adaptive J5..J9 x 32 step, 3 blocks (80 registers, about
// 50 bytes spilled) beat 2 (122 registers): 11.95 vs 12.18 ms a step.
#ifndef WL_PLAN_MINB
#define WL_PLAN_MINB 3
#endif
// Inner plan, parents [0, np)^2 (u = (d*np + jp)*np + ip): int slots parent
// codes (0-4), child circulation codes (5-14), target codes (15-20); double
// slots parent lengths (0-4), parent areas (5-6), child lengths (7-16), child
// areas (17-22), target lengths (23-28).
constexpr int IP_NI = 21, IP_ND = 29;

__global__ void k_outer_plan(WLev Pa, WLev C, int* __restrict__ pi, double* __restrict__ pd) {
  const int m = Pa.n + 1;
  const int64_t ne = (int64_t)10 * m * m;
  const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ne) return;
  const int d = (int)(u / ((int64_t)m * m)), r = (int)(u - (int64_t)d * m * m);
  const int jp = r / m, ip = r - jp * m;
  const int i = 2 * ip, j = 2 * jp;
  for (int e = 0; e < 3; ++e) {
    const int a2 = i + c_end_pt[e][1][0], b2 = j + c_end_pt[e][1][1];
    OuterInterp O;
    outer_interp(O, Pa, C, d, ip, jp, a2, b2, e);
#pragma unroll
    for (int q = 0; q < 13; ++q) pi[(e * 14 + q) * ne + u] = O.c[q];
    pi[(e * 14 + 13) * ne + u] = we_code(C, e, d, a2, b2);
#pragma unroll
    for (int q = 0; q < 9; ++q) pd[(e * 9 + q) * ne + u] = O.w[q];
  }
}

__global__ void k_inner_plan(WLev Pa, WLev C, int* __restrict__ pi, double* __restrict__ pd) {
  const int m = Pa.n;
  const int64_t ne = (int64_t)10 * m * m;
  const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ne) return;
  const int d = (int)(u / ((int64_t)m * m)), r = (int)(u - (int64_t)d * m * m);
  const int jp = r / m, ip = r - jp * m;
  InnerInterp I;
  inner_interp(I, Pa, C, d, ip, jp);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    pi[q * ne + u] = I.cp[q];
    pd[q * ne + u] = I.lp[q];
  }
  pd[5 * ne + u] = I.tp[0];
  pd[6 * ne + u] = I.tp[1];
#pragma unroll
  for (int q = 0; q < 10; ++q) {
    pi[(5 + q) * ne + u] = I.cc[q];
    pd[(7 + q) * ne + u] = I.lc[q];
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    pi[(15 + q) * ne + u] = I.ct[q];
    pd[(17 + q) * ne + u] = I.tc[q];
    pd[(23 + q) * ne + u] = I.den[q];
  }
}

// Stage slots [0, ni) and [0, nd) of the plan rows u0 .. u0+31 (nv valid).
template <int NI, int ND>
__device__ __forceinline__ void stage_plan(int (*si)[32], double (*sd)[32], const int* __restrict__ pi,
                                           const double* __restrict__ pd, int64_t ne, int64_t u0, int nv) {
  const int x = threadIdx.x;
  if (x < nv)
    for (int q = threadIdx.y; q < NI + ND; q += blockDim.y) {
      if (q < NI)
        si[q][x] = pi[q * ne + u0 + x];
      else
        sd[q - NI][x] = pd[(q - NI) * ne + u0 + x];
    }
}

// Interp_outer_velo of edge e of staged parent x (outer_eval's expression).
__device__ __forceinline__ double outer_eval_s(const int (*si)[32], const double (*sd)[32], int e, int x,
                                               const double* __restrict__ vp, double& t0) {
  const int b = e * 14, w = e * 9;
  double t[9];
  t[0] = we(vp, si[b + 0][x]);
  t[1] = we(vp, si[b + 1][x]);
  t[2] = we(vp, si[b + 2][x]);
  t[3] = we(vp, si[b + 3][x]);
  t[4] = we(vp, si[b + 4][x]);
  t[5] = we(vp, si[b + 5][x]) - we(vp, si[b + 6][x]);
  t[6] = we(vp, si[b + 7][x]) - we(vp, si[b + 8][x]);
  t[7] = we(vp, si[b + 9][x]) - we(vp, si[b + 10][x]);
  t[8] = we(vp, si[b + 11][x]) - we(vp, si[b + 12][x]);
  t0 = t[0];
  double sum = 0.0;
#pragma unroll
  for (int q = 0; q < 9; ++q) sum = sum + sd[w + q][x] * t[q];
  return sum;
}

// Interp_inner_velo of staged parent x (inner_eval's expression).
__device__ __forceinline__ void inner_eval_s(const int (*si)[32], const double (*sd)[32], int x,
                                             const double* __restrict__ vp, const double* __restrict__ v,
                                             double u[6]) {
  const double pDG = we(vp, si[0][x]) * sd[0][x];
  const double curl0 = (pDG + we(vp, si[1][x]) * sd[1][x] + we(vp, si[2][x]) * sd[2][x]) / sd[5][x];
  const double curl1 = (pDG + we(vp, si[3][x]) * sd[3][x] + we(vp, si[4][x]) * sd[4][x]) / sd[6][x];
  double pr[10];
#pragma unroll
  for (int q = 0; q < 10; ++q) pr[q] = we(v, si[5 + q][x]) * sd[7 + q][x];
  u[0] = (sd[17][x] * curl0 - pr[0] - pr[1]) / sd[23][x];
  u[1] = (sd[18][x] * curl0 - pr[2] - pr[3]) / sd[24][x];
  u[2] = (sd[19][x] * curl0 - pr[4] - pr[5]) / sd[25][x];
  u[3] = (sd[20][x] * curl1 - pr[6] - pr[1]) / sd[26][x];
  u[4] = (sd[21][x] * curl1 - pr[7] - pr[8]) / sd[27][x];
  u[5] = (sd[22][x] * curl1 - pr[4] - pr[9]) / sd[28][x];
}

// Parent (d, ip, jp) of plan row u over [0, m)^2.
__device__ __forceinline__ void plan_parent(int64_t u, int m, int& d, int& ip, int& jp) {
  d = (int)(u / ((int64_t)m * m));
  const int r = (int)(u - (int64_t)d * m * m);
  jp = r / m;
  ip = r - jp * m;
}

// Plan rows of the block's parents gathered one row per thread (the parents
// of a work list are not consecutive plan rows).
template <int NI, int ND>
__device__ __forceinline__ void gather_plan(int (*si)[32], double (*sd)[32], const int* __restrict__ pi,
                                            const double* __restrict__ pd, int64_t ne, int64_t u, bool live) {
  const int x = threadIdx.x;
  if (live)
    for (int q = threadIdx.y; q < NI + ND; q += blockDim.y) {
      if (q < NI)
        si[q][x] = pi[q * ne + u];
      else
        sd[q - NI][x] = pd[(q - NI) * ne + u];
    }
}

// Reconstruct_outer_velo of the staged parent x of the block (d, ip, jp).
__device__ __forceinline__ void recon_outer_one(const WLev& Pa, const WLev& C, int nz, const int (*si)[32],
                                                const double (*sd)[32], int x, int d, int ip, int jp) {
  const int np = Pa.n, y = threadIdx.y, ny = blockDim.y;
  const int i = 2 * ip, j = 2 * jp;
  for (int e = 0; e < 3; ++e) {
    const int a1 = i + c_end_pt[e][0][0], b1 = j + c_end_pt[e][0][1];
    const int a2 = i + c_end_pt[e][1][0], b2 = j + c_end_pt[e][1][1];
    const int x2 = e * C.NN + nid(C, d, a2, b2), x1 = e * C.NN + nid(C, d, a1, b1);
    const int cw = si[e * 14 + 13][x];
    for (int k = y; k < nz; k += ny) {
      const double* vp = Pa.sv + (int64_t)k * 3 * Pa.NN;
      const double* wc = C.wv + (int64_t)k * 3 * C.NN;
      double* v = C.sv + (int64_t)k * 3 * C.NN;
      double t0;
      const double uu = outer_eval_s(si, sd, e, x, vp, t0);
      const double v2 = uu + we(wc, cw);
      v[x2] = v2;
      v[x1] = 2.0 * t0 - v2;
    }
  }
  if ((ip == 0 || ip == np - 1) && (jp == 0 || jp == np - 1))
    for (int k = y; k < nz; k += ny)
      penta_reconstruct(Pa, C, Pa.sv + (int64_t)k * 3 * Pa.NN, C.sv + (int64_t)k * 3 * C.NN, d, ip, jp);
}

// Reconstruct_outer_velo (src/wavelet.f90:954-976) from the outer plan,
// parents [0, np]^2, then Reconstruct_velo_penta by the corner parents.  With
// a work list (PL), persistent blocks take 32 listed parents at a time.
__global__ void __launch_bounds__(256) k_recon_outer_p(WLev Pa, WLev C, int nz, const int* __restrict__ pi,
                                                       const double* __restrict__ pd,
                                                       const unsigned char* __restrict__ rec, ParentList PL) {
  __shared__ int si[OP_NI][32];
  __shared__ double sd[OP_ND][32];
  const int np = Pa.n, m = np + 1;
  const int64_t ne = (int64_t)10 * m * m;
  const int x = threadIdx.x;
  if (PL.ids) {
    const int cnt = __ldg(PL.count);
    for (int c = blockIdx.x; c < (cnt + 31) / 32; c += gridDim.x) {
      const int e = c * 32 + x;
      int d = 0, ip = 0, jp = 0;
      bool live = e < cnt && list_parent(Pa.n, __ldg(PL.ids + e), m, d, ip, jp) && rebuilt(rec, Pa, d, ip, jp);
      if (__syncthreads_or(live)) {
        gather_plan<OP_NI, OP_ND>(si, sd, pi, pd, ne, ((int64_t)d * m + jp) * m + ip, live);
        __syncthreads();
        if (live) recon_outer_one(Pa, C, nz, si, sd, x, d, ip, jp);
      }
      __syncthreads();
    }
    return;
  }
  const int64_t u0 = (int64_t)blockIdx.x * 32;
  int d = 0, ip = 0, jp = 0;
  bool live = u0 + x < ne;
  if (live) {
    plan_parent(u0 + x, m, d, ip, jp);
    live = rebuilt(rec, Pa, d, ip, jp);
  }
  if (!__syncthreads_or(live)) return;
  stage_plan<OP_NI, OP_ND>(si, sd, pi, pd, ne, u0, (int)min((int64_t)32, ne - u0));
  __syncthreads();
  if (!live) return;
  recon_outer_one(Pa, C, nz, si, sd, x, d, ip, jp);
}

// target edges of the inner plan: UP(i+1,j) DG(i+1,j) RT(i+1,j+1) RT(i,j+1) DG(i,j+1) UP(i+1,j+1)
__device__ __forceinline__ int inner_target(const WLev& C, int q, int d, int i, int j) {
  const int ge[6] = {UP, DG, RT, RT, DG, UP};
  const int gi[6] = {i + 1, i + 1, i + 1, i, i, i + 1};
  const int gj[6] = {j, j, j + 1, j + 1, j + 1, j + 1};
  return ge[q] * C.NN + nid(C, d, gi[q], gj[q]);
}

// Reconstruct_inner_velo of the staged parent x of the block (d, ip, jp).
__device__ __forceinline__ void recon_inner_one(const WLev& Pa, const WLev& C, int nz, const int (*si)[32],
                                                const double (*sd)[32], int x, int d, int ip, int jp) {
  const int y = threadIdx.y, ny = blockDim.y;
  const int i = 2 * ip, j = 2 * jp;
  for (int k = y; k < nz; k += ny) {
    const double* vp = Pa.sv + (int64_t)k * 3 * Pa.NN;
    const double* wc = C.wv + (int64_t)k * 3 * C.NN;
    double* v = C.sv + (int64_t)k * 3 * C.NN;
    double uu[6];
    inner_eval_s(si, sd, x, vp, v, uu);
#pragma unroll
    for (int q = 0; q < 6; ++q) v[inner_target(C, q, d, i, j)] = uu[q] + we(wc, si[15 + q][x]);
  }
}

// Reconstruct_inner_velo (src/wavelet.f90:978-1003) from the inner plan,
// parents [0, np)^2.  With a work list (PL), persistent blocks take 32 listed
// parents at a time.
__global__ void __launch_bounds__(256, WL_PLAN_MINB) k_recon_inner_p(WLev Pa, WLev C, int nz, const int* __restrict__ pi,
                                                       const double* __restrict__ pd,
                                                       const unsigned char* __restrict__ rec, ParentList PL) {
  __shared__ int si[IP_NI][32];
  __shared__ double sd[IP_ND][32];
  const int m = Pa.n;
  const int64_t ne = (int64_t)10 * m * m;
  const int x = threadIdx.x;
  if (PL.ids) {
    const int cnt = __ldg(PL.count);
    for (int c = blockIdx.x; c < (cnt + 31) / 32; c += gridDim.x) {
      const int e = c * 32 + x;
      int d = 0, ip = 0, jp = 0;
      bool live = e < cnt && list_parent(Pa.n, __ldg(PL.ids + e), m, d, ip, jp) && rebuilt(rec, Pa, d, ip, jp);
      if (__syncthreads_or(live)) {
        gather_plan<IP_NI, IP_ND>(si, sd, pi, pd, ne, ((int64_t)d * m + jp) * m + ip, live);
        __syncthreads();
        if (live) recon_inner_one(Pa, C, nz, si, sd, x, d, ip, jp);
      }
      __syncthreads();
    }
    return;
  }
  const int64_t u0 = (int64_t)blockIdx.x * 32;
  int d = 0, ip = 0, jp = 0;
  bool live = u0 + x < ne;
  if (live) {
    plan_parent(u0 + x, m, d, ip, jp);
    live = rebuilt(rec, Pa, d, ip, jp);
  }
  if (!__syncthreads_or(live)) return;
  stage_plan<IP_NI, IP_ND>(si, sd, pi, pd, ne, u0, (int)min((int64_t)32, ne - u0));
  __syncthreads();
  if (!live) return;
  recon_inner_one(Pa, C, nz, si, sd, x, d, ip, jp);
}

}  // namespace wtw
