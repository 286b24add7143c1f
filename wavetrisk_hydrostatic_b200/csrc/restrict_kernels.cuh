// Coarse-level compute-or-restrict kernels of the multi-level trend
// (src/multi_level.f90:311-659): one thread per (layer, lozenge, parent node),
// node index fastest so that a warp reads consecutive parents and the
// stride-2 child rows.  Ghost values of the child flux and dscalar are read
// through the level's remaps (the reference ghost-copies them first);
// R_F_wgt, the overlap areas and the masks are read where they are stored.
// FP64 with the reference's operand order (the build turns FMA contraction off).
#pragma once
#include "wavelet_kernels.cuh"

namespace wtw {

enum { S_UZM = 0, S_UPZ, S_UMZ, S_UZP, S_VMM, S_VPM, S_VMP, S_VPP, S_WMM, S_WPM, S_WMP, S_WPP, S_WMMM, S_WPPP,
       S_VMPP, S_VPMM };
constexpr int M_RESTRCT = 12, M_ADJZONE = 8;

// nghb_pt and bfly_no2 (src/shared.f90:285,330)
__constant__ int c_nghb_pt[10][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 0}, {-1, -1}, {0, -1}, {1, 0}, {1, 1}, {0, 1}, {-1, 0}};
__constant__ int c_bfly_no2[3][4][2] = {{{-3, -2}, {1, -2}, {3, 2}, {-1, 2}},
                                        {{1, 3}, {-3, -1}, {-1, -3}, {3, 1}},
                                        {{2, -1}, {2, 3}, {-2, 1}, {-2, -3}}};

// get_indices (src/multi_level.f90:617-659): the 16 stencil edges as (i, j, e)
// and the diagonal neighbours MP, PP, PM, MM.
struct RInd {
  int ei[16], ej[16], ee[16];
  int ni[4], nj[4];
};

__device__ __forceinline__ void rset(RInd& r, int s, int i, int j, int k) {
  r.ei[s] = i + c_hex_sides[k][0];
  r.ej[s] = j + c_hex_sides[k][1];
  r.ee[s] = c_hex_sides[k][2];
}

__device__ __forceinline__ RInd get_indices(int i, int j, int e) {
  RInd r;
  const int hs = c_hex_s_offs[e];
  rset(r, S_UMZ, i, j, hs + 1);
  rset(r, S_UPZ, i, j, hs + 4);
  rset(r, S_WMP, i, j, hs + 0);
  rset(r, S_VPP, i, j, hs + 5);
  rset(r, S_WPM, i, j, hs + 3);
  rset(r, S_VMM, i, j, hs + 2);
  const int off[4] = {0, 5, 3, 2};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    r.ni[q] = i + c_nghb_pt[hs + off[q]][0];
    r.nj[q] = j + c_nghb_pt[hs + off[q]][1];
  }
  rset(r, S_VMP, r.ni[0], r.nj[0], hs + 2);
  rset(r, S_VMPP, r.ni[0], r.nj[0], hs + 5);
  rset(r, S_UZP, r.ni[0], r.nj[0], hs + 4);
  rset(r, S_WPPP, r.ni[1], r.nj[1], hs + 0);
  rset(r, S_WPP, r.ni[1], r.nj[1], hs + 3);
  rset(r, S_VPM, r.ni[2], r.nj[2], hs + 5);
  rset(r, S_VPMM, r.ni[2], r.nj[2], hs + 2);
  rset(r, S_UZM, r.ni[2], r.nj[2], hs + 1);
  rset(r, S_WMMM, r.ni[3], r.nj[3], hs + 3);
  rset(r, S_WMM, r.ni[3], r.nj[3], hs + 0);
  return r;
}

struct RChild {
  const WLev& C;
  const double* __restrict__ h;   // child flux, one layer
  const double* __restrict__ ds;  // child dscalar, one layer
  int d;

  __device__ __forceinline__ double f(const RInd& r, int s) const { return re(C, h, r.ee[s], d, r.ei[s], r.ej[s]); }
  __device__ __forceinline__ double dsn(int i, int j) const { return rn(C, ds, d, i, j); }
  __device__ __forceinline__ double a(int i, int j, int k) const { return C.oa[k * C.NN + nid(C, d, i, j)]; }
  __device__ __forceinline__ double sp(int i, int j, int k) const { return C.split[k * C.NN + nid(C, d, i, j)]; }
  __device__ __forceinline__ double hi(int i, int j) const { return C.hinv[nid(C, d, i, j)]; }
  __device__ __forceinline__ double rf(int i, int j, int c) const { return C.rf[c * C.NN + nid(C, d, i, j)]; }

  // - sum(f(a) * rf(i0,j0)) - sum((f(p) - f(m)) * rf(i1,j1)), or + ... + when pos
  __device__ __forceinline__ double small(const RInd& r, const int a3[3], const int p3[3], const int m3[3], int i0,
                                          int j0, int i1, int j1, bool pos) const {
    double s1 = f(r, a3[0]) * rf(i0, j0, 0);
    s1 = s1 + f(r, a3[1]) * rf(i0, j0, 1);
    s1 = s1 + f(r, a3[2]) * rf(i0, j0, 2);
    double s2 = (f(r, p3[0]) - f(r, m3[0])) * rf(i1, j1, 0);
    s2 = s2 + (f(r, p3[1]) - f(r, m3[1])) * rf(i1, j1, 1);
    s2 = s2 + (f(r, p3[2]) - f(r, m3[2])) * rf(i1, j1, 2);
    return pos ? s1 + s2 : -s1 - s2;
  }

  // interp_flux (src/multi_level.f90:453-482) at child (i, j)
  __device__ void interp_flux(int i, int j, double sm[4]) const {
    RInd r = get_indices(i + 1, j, RT);
    {
      const int a3[3] = {S_WPM, S_UZM, S_VMM}, p3[3] = {S_VPM, S_WMMM, S_UMZ}, m3[3] = {S_UPZ, S_VPMM, S_WMM};
      sm[0] = small(r, a3, p3, m3, i + 1, j - 2, i + 1, j - 1, false);
    }
    {
      const int a3[3] = {S_WMP, S_UZP, S_VPP}, p3[3] = {S_VMP, S_WPPP, S_UPZ}, m3[3] = {S_UMZ, S_VMPP, S_WPP};
      sm[1] = small(r, a3, p3, m3, i, j, i, j + 1, true);
    }
    r = get_indices(i, j + 1, UP);
    {
      const int a3[3] = {S_UZM, S_VMM, S_WPM}, p3[3] = {S_WMMM, S_UMZ, S_VPM}, m3[3] = {S_VPMM, S_WMM, S_UPZ};
      sm[2] = small(r, a3, p3, m3, i + 1, j, i + 1, j + 1, false);
    }
    {
      const int a3[3] = {S_UZP, S_VPP, S_WMP}, p3[3] = {S_WPPP, S_UPZ, S_VMP}, m3[3] = {S_VMPP, S_WPP, S_UMZ};
      sm[3] = small(r, a3, p3, m3, i - 2, j, i - 2, j + 1, true);
    }
  }

  // part_coarse_flux (src/multi_level.f90:510-538)
  __device__ double part_coarse_flux(int i, int j, int e) const {
    const RInd r = get_indices(i, j, e);
    double ar0 = a(i, j, 0), ar1 = a(i, j, 1);
    double o0 = sp(i, j, 0), o1 = sp(i, j, 1);
    double o2 = a(i, j, 2) - o0, o3 = a(i, j, 3) - o1;
    ar0 = ar0 + o0 + o3;
    ar1 = ar1 + o1 + o2;
    const double s = ar0 + ar1;
    ar0 = ar0 / s;
    ar1 = ar1 / s;
    const int mpi = r.ni[0], mpj = r.nj[0], ppi = r.ni[1], ppj = r.nj[1];
    const int pmi = r.ni[2], pmj = r.nj[2], mmi = r.ni[3], mmj = r.nj[3];
    o0 = sp(ppi, ppj, 0);
    o1 = sp(mmi, mmj, 1);
    o2 = a(mpi, mpj, 2) - sp(mpi, mpj, 0);
    o3 = a(pmi, pmj, 3) - sp(pmi, pmj, 1);
    double t = f(r, S_UPZ) * ar0;
    t = t + f(r, S_UMZ) * ar1;
    t = t - (f(r, S_VMM) + f(r, S_WMP)) * ar1;
    t = t - (f(r, S_WPM) + f(r, S_VPP)) * ar0;
    t = t + o2 * dsn(mpi, mpj);
    t = t - o3 * dsn(pmi, pmj);
    t = t - o0 * dsn(ppi, ppj);
    return t + o1 * dsn(mmi, mmj);
  }

  // coarse_flux (src/multi_level.f90:540-573); dscalar reads outside the
  // padded level take 0 (their area weights are zero there).
  __device__ double coarse_flux(int i, int j, int e) const {
    const int hs = c_hex_s_offs[e];
#define NB(k, X) const int X##i = i + c_nghb_pt[hs + k][0], X##j = j + c_nghb_pt[hs + k][1];
    NB(1, mz) NB(4, pz) NB(0, mp) NB(5, pp) NB(3, pm) NB(2, mm)
#undef NB
    const double wpp = a(ppi, ppj, 2) * a(ppi, ppj, 3) * hi(ppi, ppj);
    const double wpm = a(pmi, pmj, 2) * a(pmi, pmj, 3) * hi(pmi, pmj);
    const double wmp = a(mpi, mpj, 2) * a(mpi, mpj, 3) * hi(mpi, mpj);
    const double wmm = a(mmi, mmj, 2) * a(mmi, mmj, 3) * hi(mmi, mmj);
    const double d_mm2 = dsn(i + c_bfly_no2[e][0][0], j + c_bfly_no2[e][0][1]);
    const double d_pm2 = dsn(i + c_bfly_no2[e][1][0], j + c_bfly_no2[e][1][1]);
    const double d_pp2 = dsn(i + c_bfly_no2[e][2][0], j + c_bfly_no2[e][2][1]);
    const double d_mp2 = dsn(i + c_bfly_no2[e][3][0], j + c_bfly_no2[e][3][1]);
    const double dmz = dsn(mzi, mzj), dpz = dsn(pzi, pzj);
    double c = a(i, j, 0) * a(i, j, 1) * hi(i, j);
    c = c + a(mpi, mpj, 1) * a(mpi, mpj, 2) * hi(mpi, mpj);
    c = c + a(ppi, ppj, 0) * a(ppi, ppj, 2) * hi(ppi, ppj);
    c = c + a(pmi, pmj, 0) * a(pmi, pmj, 3) * hi(pmi, pmj);
    c = c + a(mmi, mmj, 1) * a(mmi, mmj, 3) * hi(mmi, mmj);
    double t = c * (dpz - dmz);
    t = t + wpp * 0.5 * (d_pp2 - dmz);
    t = t + wpm * 0.5 * (d_pm2 - dmz);
    t = t + wmp * 0.5 * (dpz - d_mp2);
    return t + wmm * 0.5 * (dpz - d_mm2);
  }
};

// flux_cpt_restr, one thread per (group of lpt layers, restricted parent edge)
// (group slowest, then e, node fastest), up to two fluxes (mass, Theta) per
// thread.  The
// ghost remaps, R_F_wgt, the overlap-area factors of part_coarse_flux and
// coarse_flux and the small-flux weights depend only on the grid, so they are
// resolved once per thread; the layer loop then evaluates the same expression
// trees as RChild (the small fluxes sm[e], sm[e+1] of the edge are evaluated by
// each of the two edges that use them, in the same order, so both get the same
// bits).  Edge reads outside the padded child level and node reads outside it
// take 0, as the remapped readers do.
struct SmTerm {  // one interp_flux small flux: +-(sum f(a) w0 + sum (f(p) - f(m)) w1)
  int a[3], p[3], m[3];  // signed edge codes (slot * 2 + negate), -1 outside
  double w0[3], w1[3];
  bool pos;
};

__device__ __forceinline__ int ecode(const WLev& C, int d, int i, int j, int e) {
  if (!inr(C, i, j)) return -1;
  return __ldg(C.esrc + e * C.NN + nid(C, d, i, j));
}
__device__ __forceinline__ int ncode(const WLev& C, int d, int i, int j) {
  if (!inr(C, i, j)) return -1;
  return __ldg(C.nsrc + nid(C, d, i, j));
}
__device__ __forceinline__ double fe(const double* __restrict__ f, int c) {
  if (c < 0) return 0.0;
  const double v = f[c >> 1];
  return (c & 1) ? -v : v;
}
__device__ __forceinline__ double fn(const double* __restrict__ f, int c) { return c < 0 ? 0.0 : f[c]; }

__device__ __forceinline__ void sm_build(SmTerm& t, const WLev& C, int d, const RInd& r, const int a3[3],
                                         const int p3[3], const int m3[3], int i0, int j0, int i1, int j1, bool pos) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    t.a[q] = ecode(C, d, r.ei[a3[q]], r.ej[a3[q]], r.ee[a3[q]]);
    t.p[q] = ecode(C, d, r.ei[p3[q]], r.ej[p3[q]], r.ee[p3[q]]);
    t.m[q] = ecode(C, d, r.ei[m3[q]], r.ej[m3[q]], r.ee[m3[q]]);
    t.w0[q] = C.rf[q * C.NN + nid(C, d, i0, j0)];
    t.w1[q] = C.rf[q * C.NN + nid(C, d, i1, j1)];
  }
  t.pos = pos;
}
__device__ __forceinline__ double sm_eval(const SmTerm& t, const double* __restrict__ h) {
  double s1 = fe(h, t.a[0]) * t.w0[0];
  s1 = s1 + fe(h, t.a[1]) * t.w0[1];
  s1 = s1 + fe(h, t.a[2]) * t.w0[2];
  double s2 = (fe(h, t.p[0]) - fe(h, t.m[0])) * t.w1[0];
  s2 = s2 + (fe(h, t.p[1]) - fe(h, t.m[1])) * t.w1[1];
  s2 = s2 + (fe(h, t.p[2]) - fe(h, t.m[2])) * t.w1[2];
  return t.pos ? s1 + s2 : -s1 - s2;
}
// small flux q of interp_flux at child (i, j) (q = 0..3: UPLT S, LORT, UPLT, LORT W)
__device__ __forceinline__ void sm_make(SmTerm& t, const WLev& C, int d, int i, int j, int q) {
  if (q <= 1) {
    const RInd r = get_indices(i + 1, j, RT);
    if (q == 0) {
      const int a3[3] = {S_WPM, S_UZM, S_VMM}, p3[3] = {S_VPM, S_WMMM, S_UMZ}, m3[3] = {S_UPZ, S_VPMM, S_WMM};
      sm_build(t, C, d, r, a3, p3, m3, i + 1, j - 2, i + 1, j - 1, false);
    } else {
      const int a3[3] = {S_WMP, S_UZP, S_VPP}, p3[3] = {S_VMP, S_WPPP, S_UPZ}, m3[3] = {S_UMZ, S_VMPP, S_WPP};
      sm_build(t, C, d, r, a3, p3, m3, i, j, i, j + 1, true);
    }
  } else {
    const RInd r = get_indices(i, j + 1, UP);
    if (q == 2) {
      const int a3[3] = {S_UZM, S_VMM, S_WPM}, p3[3] = {S_WMMM, S_UMZ, S_VPM}, m3[3] = {S_VPMM, S_WMM, S_UPZ};
      sm_build(t, C, d, r, a3, p3, m3, i + 1, j, i + 1, j + 1, false);
    } else {
      const int a3[3] = {S_UZP, S_VPP, S_WMP}, p3[3] = {S_WPPP, S_UPZ, S_VMP}, m3[3] = {S_VMPP, S_WPP, S_UMZ};
      sm_build(t, C, d, r, a3, p3, m3, i - 2, j, i - 2, j + 1, true);
    }
  }
}

// flux_cpt_restr in two parts.  Everything of a parent edge's restriction that
// does not depend on the layer (remap codes of the child stencil, R_F_wgt, the
// overlap-area factors of part_coarse_flux and coarse_flux) is geometry, so
// k_rf_plan computes it once per hierarchy into a plan (structure of arrays
// over the parent edges u = ((e*10 + d)*m + jp)*m + ip, m = n_par); the
// per-step kernel k_restr_flux3 stages 32 edges' plans in shared memory and
// evaluates the layers with few live registers.
// int slots: the small fluxes sm[e] (0-8: a, p, m) and sm[e+1] (9-17), the six
// edge codes of part_coarse_flux (18-23: UPZ, UMZ, VMM, WMP, WPM, VPP), the node
// codes MP, PP, PM, MM (24-27), MZ, PZ (28-29), MM2, PM2, PP2, MP2 (30-33).
// double slots: w0, w1 of sm[e] (0-5) and sm[e+1] (6-11); ar0, ar1, o0-o3
// (12-17); the coarse_flux weights c, wpp/2, wpm/2, wmp/2, wmm/2 (18-22).
constexpr int RF_NI = 34, RF_ND = 23;

__global__ void k_rf_plan(WLev P, WLev C, int* __restrict__ pi, double* __restrict__ pd) {
  const int m = P.n;
  const int64_t ne = (int64_t)3 * 10 * m * m;
  const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ne) return;
  const int ip = (int)(u % m), jp = (int)((u / m) % m), d = (int)((u / ((int64_t)m * m)) % 10);
  const int e = (int)(u / ((int64_t)10 * m * m));
  const int ic = 2 * ip, jc = 2 * jp;
  int ci_[RF_NI];
  double cd[RF_ND];
  SmTerm sa, sb;
  sm_make(sa, C, d, ic, jc, e);
  sm_make(sb, C, d, ic, jc, e + 1);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    ci_[q] = sa.a[q]; ci_[3 + q] = sa.p[q]; ci_[6 + q] = sa.m[q];
    ci_[9 + q] = sb.a[q]; ci_[12 + q] = sb.p[q]; ci_[15 + q] = sb.m[q];
    cd[q] = sa.w0[q]; cd[3 + q] = sa.w1[q]; cd[6 + q] = sb.w0[q]; cd[9 + q] = sb.w1[q];
  }
  const int ci = (e == UP) ? ic : ic + 1, cj = (e == RT) ? jc : jc + 1;
  const RInd r = get_indices(ci, cj, e);
  // part_coarse_flux
  const RChild G{C, nullptr, nullptr, d};
  double ar0 = G.a(ci, cj, 0), ar1 = G.a(ci, cj, 1);
  double o0 = G.sp(ci, cj, 0), o1 = G.sp(ci, cj, 1);
  double o2 = G.a(ci, cj, 2) - o0, o3 = G.a(ci, cj, 3) - o1;
  ar0 = ar0 + o0 + o3;
  ar1 = ar1 + o1 + o2;
  const double sum = ar0 + ar1;
  ar0 = ar0 / sum;
  ar1 = ar1 / sum;
  const int mpi = r.ni[0], mpj = r.nj[0], ppi = r.ni[1], ppj = r.nj[1];
  const int pmi = r.ni[2], pmj = r.nj[2], mmi = r.ni[3], mmj = r.nj[3];
  o0 = G.sp(ppi, ppj, 0);
  o1 = G.sp(mmi, mmj, 1);
  o2 = G.a(mpi, mpj, 2) - G.sp(mpi, mpj, 0);
  o3 = G.a(pmi, pmj, 3) - G.sp(pmi, pmj, 1);
  const int es[6] = {S_UPZ, S_UMZ, S_VMM, S_WMP, S_WPM, S_VPP};
#pragma unroll
  for (int q = 0; q < 6; ++q) ci_[18 + q] = ecode(C, d, r.ei[es[q]], r.ej[es[q]], r.ee[es[q]]);
  ci_[24] = ncode(C, d, mpi, mpj);
  ci_[25] = ncode(C, d, ppi, ppj);
  ci_[26] = ncode(C, d, pmi, pmj);
  ci_[27] = ncode(C, d, mmi, mmj);
  cd[12] = ar0; cd[13] = ar1; cd[14] = o0; cd[15] = o1; cd[16] = o2; cd[17] = o3;
  // coarse_flux (the neighbours mp, pp, pm, mm are part_coarse_flux's MP, PP, PM, MM)
  const int hs = c_hex_s_offs[e];
  ci_[28] = ncode(C, d, ci + c_nghb_pt[hs + 1][0], cj + c_nghb_pt[hs + 1][1]);
  ci_[29] = ncode(C, d, ci + c_nghb_pt[hs + 4][0], cj + c_nghb_pt[hs + 4][1]);
#pragma unroll
  for (int q = 0; q < 4; ++q) ci_[30 + q] = ncode(C, d, ci + c_bfly_no2[e][q][0], cj + c_bfly_no2[e][q][1]);
  const double wpp = G.a(ppi, ppj, 2) * G.a(ppi, ppj, 3) * G.hi(ppi, ppj);
  const double wpm = G.a(pmi, pmj, 2) * G.a(pmi, pmj, 3) * G.hi(pmi, pmj);
  const double wmp = G.a(mpi, mpj, 2) * G.a(mpi, mpj, 3) * G.hi(mpi, mpj);
  const double wmm = G.a(mmi, mmj, 2) * G.a(mmi, mmj, 3) * G.hi(mmi, mmj);
  double cc = G.a(ci, cj, 0) * G.a(ci, cj, 1) * G.hi(ci, cj);
  cc = cc + G.a(mpi, mpj, 1) * G.a(mpi, mpj, 2) * G.hi(mpi, mpj);
  cc = cc + G.a(ppi, ppj, 0) * G.a(ppi, ppj, 2) * G.hi(ppi, ppj);
  cc = cc + G.a(pmi, pmj, 0) * G.a(pmi, pmj, 3) * G.hi(pmi, pmj);
  cc = cc + G.a(mmi, mmj, 1) * G.a(mmi, mmj, 3) * G.hi(mmi, mmj);
  cd[18] = cc; cd[19] = wpp * 0.5; cd[20] = wpm * 0.5; cd[21] = wmp * 0.5; cd[22] = wmm * 0.5;
#pragma unroll
  for (int q = 0; q < RF_NI; ++q) pi[q * ne + u] = ci_[q];
#pragma unroll
  for (int q = 0; q < RF_ND; ++q) pd[q * ne + u] = cd[q];
}

// One small flux of interp_flux from the staged plan: slots a at ia (9 codes)
// and wd (6 weights) of edge x, sign pos.
__device__ __forceinline__ double sm_eval_s(const int (*si)[32], const double (*sd)[32], int ia, int wd, int x,
                                            bool pos, const double* __restrict__ h) {
  double s1 = fe(h, si[ia + 0][x]) * sd[wd + 0][x];
  s1 = s1 + fe(h, si[ia + 1][x]) * sd[wd + 1][x];
  s1 = s1 + fe(h, si[ia + 2][x]) * sd[wd + 2][x];
  double s2 = (fe(h, si[ia + 3][x]) - fe(h, si[ia + 6][x])) * sd[wd + 3][x];
  s2 = s2 + (fe(h, si[ia + 4][x]) - fe(h, si[ia + 7][x])) * sd[wd + 4][x];
  s2 = s2 + (fe(h, si[ia + 5][x]) - fe(h, si[ia + 8][x])) * sd[wd + 5][x];
  return pos ? s1 + s2 : -s1 - s2;
}

// flux_cpt_restr of up to two fluxes (mass, Theta: fp0/fp1 from the child's
// fc0/fc1 and dscalar dc0/dc1) on the restricted parent edges (mask_e >=
// RESTRCT).  Block (32, ny): 32 consecutive parent edges of the plan, ny
// threads per edge taking layers y, y + ny, ...; blocks without a restricted
// edge return before staging.  With a work list (PL), persistent blocks take
// 32 of the listed parents' edges at a time.  Same expression trees and operand order as
// part_coarse_flux + coarse_flux + interp_flux of the reference.
__device__ __forceinline__ void restr_flux_one(const WLev& P, int nz, const int (*si)[32], const double (*sd)[32],
                                               int x, int d, int ip, int jp, int e, double* __restrict__ fp0,
                                               double* __restrict__ fp1, const double* __restrict__ fc0,
                                               const double* __restrict__ fc1, const double* __restrict__ dc0,
                                               const double* __restrict__ dc1, int NNc) {
  const int y = threadIdx.y, ny = blockDim.y;
  const bool pa = (e & 1) != 0, pb = ((e + 1) & 1) != 0;
  const int64_t so = (int64_t)e * P.NN + nid(P, d, ip, jp);
  const double ar0 = sd[12][x], ar1 = sd[13][x], o0 = sd[14][x], o1 = sd[15][x], o2 = sd[16][x], o3 = sd[17][x];
  for (int k = y; k < nz; k += ny) {
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      double* __restrict__ fp = f == 0 ? fp0 : fp1;
      if (!fp) continue;
      const double* __restrict__ h = (f == 0 ? fc0 : fc1) + (int64_t)3 * k * NNc;
      const double* __restrict__ ds = (f == 0 ? dc0 : dc1) + (int64_t)k * NNc;
      const double sma = sm_eval_s(si, sd, 0, 0, x, pa, h), smb = sm_eval_s(si, sd, 9, 6, x, pb, h);
      double tp = fe(h, si[18][x]) * ar0;
      tp = tp + fe(h, si[19][x]) * ar1;
      tp = tp - (fe(h, si[20][x]) + fe(h, si[21][x])) * ar1;
      tp = tp - (fe(h, si[22][x]) + fe(h, si[23][x])) * ar0;
      tp = tp + o2 * fn(ds, si[24][x]);
      tp = tp - o3 * fn(ds, si[26][x]);
      tp = tp - o0 * fn(ds, si[25][x]);
      tp = tp + o1 * fn(ds, si[27][x]);
      const double dmz = fn(ds, si[28][x]), dpz = fn(ds, si[29][x]);
      double tc = sd[18][x] * (dpz - dmz);
      tc = tc + sd[19][x] * (fn(ds, si[32][x]) - dmz);
      tc = tc + sd[20][x] * (fn(ds, si[31][x]) - dmz);
      tc = tc + sd[21][x] * (dpz - fn(ds, si[33][x]));
      tc = tc + sd[22][x] * (dpz - fn(ds, si[30][x]));
      fp[(int64_t)3 * k * P.NN + so] = tp + tc + sma + smb;
    }
  }
}

__global__ void __launch_bounds__(256) k_restr_flux3(WLev P, int m, int nz, const int* __restrict__ pi,
                                                     const double* __restrict__ pd, double* __restrict__ fp0,
                                                     double* __restrict__ fp1, const double* __restrict__ fc0,
                                                     const double* __restrict__ fc1, const double* __restrict__ dc0,
                                                     const double* __restrict__ dc1, int NNc, ParentList PL) {
  __shared__ int si[RF_NI][32];
  __shared__ double sd[RF_ND][32];
  const int64_t ne = (int64_t)3 * 10 * m * m;
  const int x = threadIdx.x, y = threadIdx.y, ny = blockDim.y;
  if (PL.ids) {
    const int cnt = __ldg(PL.count);
    for (int c = blockIdx.x; c < (3 * cnt + 31) / 32; c += gridDim.x) {
      const int it = c * 32 + x, e = it % 3;
      int d = 0, ip = 0, jp = 0;
      bool on = it < 3 * cnt && list_parent(P.n, __ldg(PL.ids + it / 3), m, d, ip, jp) &&
                P.mask_e[e * P.NN + nid(P, d, ip, jp)] >= M_RESTRCT;
      if (__syncthreads_or(on)) {
        const int64_t u = (((int64_t)e * 10 + d) * m + jp) * m + ip;
        if (on)
          for (int q = y; q < RF_NI + RF_ND; q += ny) {
            if (q < RF_NI)
              si[q][x] = pi[q * ne + u];
            else
              sd[q - RF_NI][x] = pd[(q - RF_NI) * ne + u];
          }
        __syncthreads();
        if (on) restr_flux_one(P, nz, si, sd, x, d, ip, jp, e, fp0, fp1, fc0, fc1, dc0, dc1, NNc);
      }
      __syncthreads();
    }
    return;
  }
  const int64_t u0 = (int64_t)blockIdx.x * 32;
  const int64_t u = u0 + x;
  int ip = 0, jp = 0, d = 0, e = 0;
  bool on = false;
  if (u < ne) {
    ip = (int)(u % m);
    jp = (int)((u / m) % m);
    d = (int)((u / ((int64_t)m * m)) % 10);
    e = (int)(u / ((int64_t)10 * m * m));
    on = P.mask_e[e * P.NN + nid(P, d, ip, jp)] >= M_RESTRCT;
  }
  if (!__syncthreads_or(on)) return;
  const int nv = (int)min((int64_t)32, ne - u0);
  for (int q = y; q < RF_NI + RF_ND; q += ny)
    if (x < nv) {
      if (q < RF_NI)
        si[q][x] = pi[q * ne + u];
      else
        sd[q - RF_NI][x] = pd[(q - RF_NI) * ne + u];
    }
  __syncthreads();
  if (!on) return;
  restr_flux_one(P, nz, si, sd, x, d, ip, jp, e, fp0, fp1, fc0, fc1, dc0, dc1, NNc);
}

// scalar_cpt_restr over parents [0, n]^2, every layer (with a work list, its
// parents only, persistent threads).
__global__ void k_restr_scalar(WLev P, WLev C, int nz, ParentList PL) {
  const int m = P.n + 1;
  if (PL.ids) {
    const int cnt = __ldg(PL.count);
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)cnt * nz;
         t += (int64_t)gridDim.x * blockDim.x) {
      const int k = (int)(t / cnt), e = (int)(t - (int64_t)k * cnt);
      int d, ip, jp;
      if (!list_parent(P.n, __ldg(PL.ids + e), m, d, ip, jp)) continue;
      const int idp = nid(P, d, ip, jp);
      if (P.mask_n[idp] >= M_RESTRCT)
        P.scal[(int64_t)k * P.NN + idp] = C.scal[(int64_t)k * C.NN + nid(C, d, 2 * ip, 2 * jp)];
    }
    return;
  }
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * 10 * m * m) return;
  const int ip = (int)(t % m), jp = (int)((t / m) % m), d = (int)((t / ((int64_t)m * m)) % 10);
  const int k = (int)(t / ((int64_t)10 * m * m));
  const int idp = nid(P, d, ip, jp);
  if (P.mask_n[idp] >= M_RESTRCT)
    P.scal[(int64_t)k * P.NN + idp] = C.scal[(int64_t)k * C.NN + nid(C, d, 2 * ip, 2 * jp)];
}

// flux_cpt_restr over parents [0, n)^2, every layer.
__global__ void k_restr_flux(WLev P, WLev C, int nz) {
  const int m = P.n;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * 10 * m * m) return;
  const int ip = (int)(t % m), jp = (int)((t / m) % m), d = (int)((t / ((int64_t)m * m)) % 10);
  const int k = (int)(t / ((int64_t)10 * m * m));
  const int idp = nid(P, d, ip, jp);
  const int m0 = P.mask_e[idp], m1 = P.mask_e[P.NN + idp], m2 = P.mask_e[2 * P.NN + idp];
  const int mx = max(max(m0, m1), m2);
  if (mx < M_RESTRCT) return;
  const RChild R{C, C.flux + (int64_t)3 * k * C.NN, C.dscal + (int64_t)k * C.NN, d};
  const int ic = 2 * ip, jc = 2 * jp;
  double sm[4];
  R.interp_flux(ic, jc, sm);
  double* fp = P.flux + (int64_t)3 * k * P.NN;
  if (m0 >= M_RESTRCT) {
    const double p = R.part_coarse_flux(ic + 1, jc, RT), c = R.coarse_flux(ic + 1, jc, RT);
    fp[idp] = p + c + sm[0] + sm[1];
  }
  if (m1 >= M_RESTRCT) {
    const double p = R.part_coarse_flux(ic + 1, jc + 1, DG), c = R.coarse_flux(ic + 1, jc + 1, DG);
    fp[P.NN + idp] = p + c + sm[1] + sm[2];
  }
  if (m2 >= M_RESTRCT) {
    const double p = R.part_coarse_flux(ic, jc + 1, UP), c = R.coarse_flux(ic, jc + 1, UP);
    fp[2 * P.NN + idp] = p + c + sm[2] + sm[3];
  }
}

// The restriction of u_source_cpt_restr over parents [0, n)^2, every layer.
__global__ void k_restr_u_source(WLev P, WLev C, int nz) {
  const int m = P.n;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * 10 * m * m) return;
  const int ip = (int)(t % m), jp = (int)((t / m) % m), d = (int)((t / ((int64_t)m * m)) % 10);
  const int k = (int)(t / ((int64_t)10 * m * m));
  const int idp = nid(P, d, ip, jp), idc = nid(C, d, 2 * ip, 2 * jp);
  const double* vc = C.dvelo + (int64_t)3 * k * C.NN;
  double* vp = P.dvelo + (int64_t)3 * k * P.NN;
  if (C.mask_e[idc] >= M_ADJZONE) vp[idp] = vc[idc] + vc[idc + 1];
  if (C.mask_e[C.NN + idc] >= M_ADJZONE) vp[P.NN + idp] = vc[C.NN + idc] + vc[C.NN + idc + C.P + 1];
  if (C.mask_e[2 * C.NN + idc] >= M_ADJZONE) vp[2 * P.NN + idp] = vc[2 * C.NN + idc] + vc[2 * C.NN + idc + C.P];
}

}  // namespace wtw

namespace wtw {

// cal_lnorm (src/lnorms.f90:7-58) partials: block (x, k) reduces layer k of
// nodes x*256 .. of the level into part[k][x] = {mass, Theta, velocity}; node
// scalars over [0, n]^2 and velocities over [0, n)^2 of nodes with mask_n >=
// ADJZONE.  order 0 "inf" (max |.|), 1 "1" (sum |.|), 2 "2" (sum of squares),
// 3 "min" (min).  cnt (k = 0 blocks only) counts nodes [-1, n+1]^2 with mask_n
// >= ADJZONE (count_norm).
__device__ __forceinline__ double lnorm_op(int order, double a, double b) {
  return order == 0 ? fmax(a, b) : order == 3 ? fmin(a, b) : a + b;
}

__global__ void k_lnorm_part(WLev V, const double* __restrict__ mean_m, const double* __restrict__ mean_t,
                             int order, double* part, int* cnt) {
  const int k = blockIdx.y;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const double id0 = order == 3 ? 1e16 : 0.0;
  double r[3] = {id0, id0, id0};
  int c = 0;
  if (x < V.NN) {
    const int pp = V.P * V.P, rr = x % pp, i = rr % V.P - 2, j = rr / V.P - 2;
    const bool act = V.mask_n[x] >= M_ADJZONE;
    if (act && i >= -1 && j >= -1 && i <= V.n + 1 && j <= V.n + 1) c = 1;
    if (act && i >= 0 && j >= 0 && i <= V.n && j <= V.n) {
      const int64_t o = (int64_t)k * V.NN + x;
      const double sm = mean_m[o] + V.sm[o], st = mean_t[o] + V.st[o];
      const double vm = order == 3 ? sm : order == 2 ? sm * sm : fabs(sm);
      const double vt = order == 3 ? st : order == 2 ? st * st : fabs(st);
      r[0] = lnorm_op(order, r[0], vm);
      r[1] = lnorm_op(order, r[1], vt);
      if (i < V.n && j < V.n)
        for (int e = 0; e < 3; ++e) {
          const double u = V.sv[(int64_t)3 * k * V.NN + (int64_t)e * V.NN + x];
          r[2] = lnorm_op(order, r[2], order == 3 ? u : order == 2 ? u * u : fabs(u));
        }
    }
  }
  __shared__ double sh[3][256];
  __shared__ int shc[256];
  for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = r[q];
  shc[threadIdx.x] = c;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = lnorm_op(order, sh[q][threadIdx.x], sh[q][threadIdx.x + s]);
      shc[threadIdx.x] += shc[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int q = 0; q < 3; ++q) part[((int64_t)k * gridDim.x + blockIdx.x) * 3 + q] = sh[q][0];
    if (k == 0) cnt[blockIdx.x] = shc[0];
  }
}

// Final reduction of the partials of every level (one block per layer).
__global__ void k_lnorm_final(const double* __restrict__ part, const int* __restrict__ nparts, int nlev,
                              const int* __restrict__ cnt, int order, int nz, double* out) {
  const int k = blockIdx.x;
  if (threadIdx.x != 0) return;
  const double id0 = order == 3 ? 1e16 : 0.0;
  double r[3] = {id0, id0, id0};
  long long n = 0;
  int64_t base = 0, cbase = 0;
  for (int l = 0; l < nlev; ++l) {
    const int np = nparts[l];
    for (int b = 0; b < np; ++b)
      for (int q = 0; q < 3; ++q) r[q] = lnorm_op(order, r[q], part[base + ((int64_t)k * np + b) * 3 + q]);
    for (int b = 0; b < np; ++b) n += cnt[cbase + b];
    base += (int64_t)nz * np * 3;
    cbase += np;
  }
  for (int q = 0; q < 3; ++q) {
    double v = r[q];
    if (order == 1) v = v / (double)n;
    if (order == 2) v = sqrt(v / (double)n);
    out[q * nz + k] = v;
  }
}

}  // namespace wtw
