// Wavelet transform kernels for the prognostic variables (layer mass,
// potential temperature, velocity) on a uniform hierarchy of padded lozenge
// levels, the threshold mask and compression.
//
// Each kernel is one interscale (parent level l, child level l+1) or onescale
// pass of the reference's drivers (src/wavelet.f90, src/adapt.f90,
// src/mask.f90), one thread per (layer, lozenge, node) of the pass's range;
// the interscale transform kernels that run every layer of a parent per thread
// are in wavelet_layers.cuh, with the pentagon helpers here.
// Ghost values are read through the level's remap tables (the node or signed
// edge that update_bdry copies there); masks and weights are read as stored.
// Floating point keeps the reference's operand order (compiled with
// --fmad=false).
#pragma once
#include <cstdint>

namespace wtw {

enum { RT = 0, DG = 1, UP = 2 };
enum { LORT = 0, UPLT = 1 };
constexpr int FROZEN = 32, TOLRNZ = 16, ADJZONE = 8, ZERO = 0;

// A parent level's work list with a patch tree: the padded parent slots of
// [0, n]^2 that an interscale kernel may have work at (those the inverse after
// adapt rebuilds: the next step's parents and those of the tree's nodes, which
// hold every child slot a mask reaches), their count on the device; built with
// the needed-node maps (need_map.cuh: k_list_count/_scan/_write).  ids null: none.
struct ParentList {
  const int* ids;
  const int* count;
};

// Persistent loop over a parent list for the kernels with one thread per
// (parent, group of lpt layers): items group-major as parent_of's, strided by
// the grid; f(d, ip, jp, k0, k1) for the listed parents of [0, m)^2 (m = n or
// n + 1 of the parent level, whose padded side is np + 4).
template <class F>
__device__ __forceinline__ void for_parents(int np, int m, int nz, int lpt, const ParentList& PL, F f) {
  const int cnt = __ldg(PL.count);
  const int ng = (nz + lpt - 1) / lpt;
  const int P = np + 4, PP = P * P;
  const int64_t tot = (int64_t)cnt * ng;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int g = (int)(t / cnt), e = (int)(t - (int64_t)g * cnt);
    const int x = __ldg(PL.ids + e);
    const int d = x / PP, r = x - d * PP;
    const int ip = r % P - 2, jp = r / P - 2;
    if (ip < 0 || jp < 0 || ip >= m || jp >= m) continue;
    const int k0 = g * lpt;
    f(d, ip, jp, k0, min(nz, k0 + lpt));
  }
}

// The parent (d, ip, jp) of work-list entry x (a padded slot of a parent
// level of side np), or false outside [0, m)^2.
__device__ __forceinline__ bool list_parent(int np, int x, int m, int& d, int& ip, int& jp) {
  const int P = np + 4, PP = P * P;
  d = x / PP;
  const int r = x - d * PP;
  ip = r % P - 2;
  jp = r / P - 2;
  return ip >= 0 && jp >= 0 && ip < m && jp < m;
}

// One level of the hierarchy on the device.
struct WLev {
  int n, P, NN;
  const double* __restrict__ len;   // 3*NN
  const double* __restrict__ tri;   // 2*NN
  const double* __restrict__ hinv;  // NN
  const double* __restrict__ oa;    // 4*NN overlap areas
  const double* __restrict__ iu;    // 9*NN outer velocity weights (null on the coarsest level)
  const int* __restrict__ nsrc;     // node remap
  const int* __restrict__ esrc;     // signed edge remap
  int* mask_n;                      // NN
  int* mask_e;                      // 3*NN
  double *sm, *st, *sv;             // scaling: [nz][NN], [nz][NN], [nz][3*NN]
  double *wm, *wt, *wv;             // wavelets, same shapes
  const double* __restrict__ split; // 2*NN Overl_Area%split (may be null)
  const double* __restrict__ rf;    // 3*NN flux-restriction weights (null on the coarsest level)
  double *scal, *dscal;             // multi-level trend work fields: [nz][NN]
  double *flux, *dvelo;             // [nz][3*NN]
};

__constant__ int c_end_pt[3][2][2] = {{{0, 0}, {1, 0}}, {{1, 1}, {0, 0}}, {{0, 0}, {0, 1}}};
__constant__ int c_opp_no[3][2][2] = {{{0, -1}, {1, 1}}, {{0, 1}, {1, 0}}, {{1, 1}, {-1, 0}}};
__constant__ int c_hex_sides[10][3] = {{0, 0, RT},  {0, 0, DG}, {0, 0, UP}, {-1, 0, RT}, {-1, -1, DG},
                                       {0, -1, UP}, {0, 0, RT}, {0, 0, DG}, {0, 0, UP},  {-1, 0, RT}};
__constant__ int c_hex_s_offs[3] = {2, 0, 4};
// Iu_Base_Wgt (src/wavelet.f90:1764)
__constant__ double c_iu_base[9] = {16.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0, -1.0 / 16.0,
                                    -1.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0};

__device__ __forceinline__ int nid(const WLev& L, int d, int i, int j) { return (d * L.P + j + 2) * L.P + i + 2; }
__device__ __forceinline__ bool inr(const WLev& L, int i, int j) {
  return i >= -2 && j >= -2 && i < L.n + 2 && j < L.n + 2;
}
// node field (one layer) through the ghost remap; 0 outside the padded array
__device__ __forceinline__ double rn(const WLev& L, const double* __restrict__ f, int d, int i, int j) {
  if (!inr(L, i, j)) return 0.0;
  return f[__ldg(L.nsrc + nid(L, d, i, j))];
}
// edge field (one layer, planes of NN) through the signed ghost remap
__device__ __forceinline__ double re(const WLev& L, const double* __restrict__ f, int e, int d, int i, int j) {
  if (!inr(L, i, j)) return 0.0;
  const int c = __ldg(L.esrc + e * L.NN + nid(L, d, i, j));
  const double v = f[c >> 1];
  return (c & 1) ? -v : v;
}
__device__ __forceinline__ double oa(const WLev& L, int d, int i, int j, int k) {
  return inr(L, i, j) ? L.oa[(k - 1) * L.NN + nid(L, d, i, j)] : 0.0;
}
__device__ __forceinline__ double hv(const WLev& L, int d, int i, int j) {
  return inr(L, i, j) ? L.hinv[nid(L, d, i, j)] : 0.0;
}
__device__ __forceinline__ double ln(const WLev& L, int e, int d, int i, int j) {
  return inr(L, i, j) ? L.len[e * L.NN + nid(L, d, i, j)] : 0.0;
}
__device__ __forceinline__ double ta(const WLev& L, int t, int d, int i, int j) {
  return inr(L, i, j) ? L.tri[t * L.NN + nid(L, d, i, j)] : 0.0;
}
__device__ __forceinline__ double iw(const WLev& L, int q, int d, int i, int j) {
  return (L.iu && inr(L, i, j)) ? L.iu[q * L.NN + nid(L, d, i, j)] : 0.0;
}
__device__ __forceinline__ int mn(const WLev& L, int d, int i, int j) {
  return inr(L, i, j) ? L.mask_n[nid(L, d, i, j)] : ZERO;
}
__device__ __forceinline__ int me(const WLev& L, int e, int d, int i, int j) {
  return inr(L, i, j) ? L.mask_e[e * L.NN + nid(L, d, i, j)] : ZERO;
}

// Thread -> (layer k, lozenge d, i, j) over [0, m)^2, layer fastest across blocks.
__device__ __forceinline__ bool decode(int nz, int m, int& k, int& d, int& i, int& j) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)10 * m * m;
  if (t >= per * nz) return false;
  k = (int)(t / per);
  int r = (int)(t - (int64_t)k * per);
  d = r / (m * m);
  r -= d * m * m;
  j = r / m;
  i = r - j * m;
  return true;
}

// Restrict_scalar (parents [0, np]^2, src/wavelet.f90:520-569) and
// Restrict_velo (parents [0, np)^2, :1154-1174).
__global__ void k_restrict(WLev Pa, WLev C, int nz) {
  const int np = Pa.n;
  int k, d, ip, jp;
  if (!decode(nz, np + 1, k, d, ip, jp)) return;
  const int i = 2 * ip, j = 2 * jp;
  if (mn(C, d, i, j) != 0) {
    for (int v = 0; v < 2; ++v) {
      const double* s = (v == 0 ? C.sm : C.st) + (int64_t)k * C.NN;
      const double* wc = (v == 0 ? C.wm : C.wt) + (int64_t)k * C.NN;
      double* sp = (v == 0 ? Pa.sm : Pa.st) + (int64_t)k * Pa.NN;
      const double sum =
          rn(C, wc, d, i + 1, j) * oa(C, d, i + 1, j, 1) + rn(C, wc, d, i + 1, j + 1) * oa(C, d, i + 1, j + 1, 2) +
          rn(C, wc, d, i + 2, j + 1) * oa(C, d, i + 2, j + 1, 3) + rn(C, wc, d, i + 1, j + 2) * oa(C, d, i + 1, j + 2, 4) +
          rn(C, wc, d, i, j + 1) * oa(C, d, i, j + 1, 1) + rn(C, wc, d, i - 1, j) * oa(C, d, i - 1, j, 2) +
          rn(C, wc, d, i - 1, j + 1) * oa(C, d, i - 1, j + 1, 3) + rn(C, wc, d, i - 2, j - 1) * oa(C, d, i - 2, j - 1, 4) +
          rn(C, wc, d, i - 1, j - 1) * oa(C, d, i - 1, j - 1, 1) + rn(C, wc, d, i, j - 1) * oa(C, d, i, j - 1, 2) +
          rn(C, wc, d, i - 1, j - 2) * oa(C, d, i - 1, j - 2, 3) + rn(C, wc, d, i + 1, j - 1) * oa(C, d, i + 1, j - 1, 4);
      sp[nid(Pa, d, ip, jp)] = rn(C, s, d, i, j) + sum * hv(Pa, d, ip, jp);
    }
  }
  if (ip < np && jp < np) {
    const double* v = C.sv + (int64_t)k * 3 * C.NN;
    double* vp = Pa.sv + (int64_t)k * 3 * Pa.NN;
    const int x = nid(Pa, d, ip, jp);
    if (me(C, RT, d, i, j) > 0) vp[RT * Pa.NN + x] = 0.5 * (re(C, v, RT, d, i, j) + re(C, v, RT, d, i + 1, j));
    if (me(C, DG, d, i, j) > 0) vp[DG * Pa.NN + x] = 0.5 * (re(C, v, DG, d, i + 1, j + 1) + re(C, v, DG, d, i, j));
    if (me(C, UP, d, i, j) > 0) vp[UP * Pa.NN + x] = 0.5 * (re(C, v, UP, d, i, j) + re(C, v, UP, d, i, j + 1));
  }
}

__device__ __forceinline__ double& ee(const WLev& L, double* f, int e, int d, int i, int j) {
  return f[e * L.NN + nid(L, d, i, j)];
}

__device__ void penta_compute(const WLev& Pa, const WLev& C, const double* vp, double* wc, int d, int ip, int jp);
__device__ void penta_reconstruct(const WLev& Pa, const WLev& C, const double* vp, double* v, int d, int ip, int jp);

// velo_interp_penta_corr (src/wavelet.f90:927-952) at the south-west corner.
__device__ void penta_corr(const WLev& Pa, const WLev& C, const double* vp, int d, double u[2]) {
  u[0] = (c_iu_base[8] + iw(C, 8, d, 0, 1)) *
         ((-re(Pa, vp, UP, d, 0, -1) - (-re(Pa, vp, RT, d, -1, -1))) - (re(Pa, vp, DG, d, -1, -1) - re(Pa, vp, UP, d, -1, -1)));
  u[1] = (c_iu_base[5] + iw(C, 5, d, 1, 0)) *
         (re(Pa, vp, RT, d, -1, -1) + re(Pa, vp, RT, d, -1, 0) - (re(Pa, vp, RT, d, -1, -1) - re(Pa, vp, DG, d, -1, -1)));
}

// Pentagon corrections at the lozenge corners, in the reference's corner order
// (NE, SE, SW, NW).  Each touches only child edges of one parent's outer pairs,
// so the thread of that parent applies it right after writing them: SE by
// parent (np-1, 0), SW by (0, 0), NW by (0, np-1).
// Compute_velo_wavelets_penta (src/wavelet.f90:712-781), on the wavelets.
__device__ void penta_compute(const WLev& Pa, const WLev& C, const double* vp, double* wc, int d, int ip, int jp) {
  const int np = Pa.n, nc = C.n;
  if (ip == np - 1 && jp == 0) {  // SE (IPLUSJMINUS)
    const double vv = (c_iu_base[6] + iw(C, 6, d, nc - 1, 0)) * (re(Pa, vp, RT, d, np, 0) + re(Pa, vp, UP, d, np, -1));
    if (me(C, RT, d, nc - 2, 0) >= ADJZONE) {
      ee(C, wc, RT, d, nc - 2, 0) = ee(C, wc, RT, d, nc - 2, 0) - vv;
      ee(C, wc, RT, d, nc - 1, 0) = ee(C, wc, RT, d, nc - 1, 0) + vv;
    }
  }
  if (ip == 0 && jp == 0) {  // SW (IJMINUS)
    double u[2];
    penta_corr(Pa, C, vp, d, u);
    if (me(C, UP, d, 0, 0) >= ADJZONE) {
      ee(C, wc, UP, d, 0, 0) = ee(C, wc, UP, d, 0, 0) + u[0];
      ee(C, wc, UP, d, 0, 1) = ee(C, wc, UP, d, 0, 1) - u[0];
    }
    if (me(C, RT, d, 0, 0) >= ADJZONE) {
      ee(C, wc, RT, d, 0, 0) = ee(C, wc, RT, d, 0, 0) + u[1];
      ee(C, wc, RT, d, 1, 0) = ee(C, wc, RT, d, 1, 0) - u[1];
    }
  }
  if (ip == 0 && jp == np - 1) {  // NW (IMINUSJPLUS)
    const double vv = -(c_iu_base[7] + iw(C, 7, d, 0, nc - 1)) * (re(Pa, vp, UP, d, 0, np) + re(Pa, vp, RT, d, -1, np));
    if (me(C, UP, d, 0, nc - 2) >= ADJZONE) {
      ee(C, wc, UP, d, 0, nc - 2) = ee(C, wc, UP, d, 0, nc - 2) - vv;
      ee(C, wc, UP, d, 0, nc - 1) = ee(C, wc, UP, d, 0, nc - 1) + vv;
    }
  }
}

// Reconstruct_velo_penta (src/wavelet.f90:1096-1152), on the child velocity.
__device__ void penta_reconstruct(const WLev& Pa, const WLev& C, const double* vp, double* v, int d, int ip, int jp) {
  const int np = Pa.n, nc = C.n;
  if (ip == np - 1 && jp == 0) {  // SE
    const double vv = -(c_iu_base[6] + iw(C, 6, d, nc - 1, 0)) * (re(Pa, vp, RT, d, np, 0) + re(Pa, vp, UP, d, np, -1));
    ee(C, v, RT, d, nc - 2, 0) = ee(C, v, RT, d, nc - 2, 0) - vv;
    ee(C, v, RT, d, nc - 1, 0) = ee(C, v, RT, d, nc - 1, 0) + vv;
  }
  if (ip == 0 && jp == 0) {  // SW
    double u[2];
    penta_corr(Pa, C, vp, d, u);
    ee(C, v, UP, d, 0, 0) = ee(C, v, UP, d, 0, 0) - u[0];
    ee(C, v, UP, d, 0, 1) = ee(C, v, UP, d, 0, 1) + u[0];
    ee(C, v, RT, d, 0, 0) = ee(C, v, RT, d, 0, 0) - u[1];
    ee(C, v, RT, d, 1, 0) = ee(C, v, RT, d, 1, 0) + u[1];
  }
  if (ip == 0 && jp == np - 1) {  // NW
    const double vv = (c_iu_base[7] + iw(C, 7, d, 0, nc - 1)) * (re(Pa, vp, UP, d, 0, np) + re(Pa, vp, RT, d, -1, np));
    ee(C, v, UP, d, 0, nc - 2) = ee(C, v, UP, d, 0, nc - 2) - vv;
    ee(C, v, UP, d, 0, nc - 1) = ee(C, v, UP, d, 0, nc - 1) + vv;
  }
}

// compress_scalar on nodes [0, n]^2 and compress_vector on [0, n)^2
// (src/adapt.f90:79-232) of one level, one thread per (layer, node).
__global__ void k_compress(WLev L, int nz) {
  int k, d, i, j;
  if (!decode(nz, L.n + 1, k, d, i, j)) return;
  const int x = nid(L, d, i, j);
  if (L.mask_n[x] < ADJZONE) {
    L.wm[(int64_t)k * L.NN + x] = 0.0;
    L.wt[(int64_t)k * L.NN + x] = 0.0;
  }
  if (i < L.n && j < L.n)
    for (int e = 0; e < 3; ++e)
      if (L.mask_e[e * L.NN + x] < ADJZONE) L.wv[(int64_t)k * 3 * L.NN + e * L.NN + x] = 0.0;
}

// compress_wavelets after a mask change whose wavelets were compressed under
// the previous masks (old_n, old_e): the slots kept before and dropped now are
// the only ones not holding 0 already, so only they are zeroed (the result is
// k_compress's).  One thread per node, every layer.
__global__ void k_compress_delta(WLev L, const int* __restrict__ old_n, const int* __restrict__ old_e, int nz) {
  int k, d, i, j;
  if (!decode(1, L.n + 1, k, d, i, j)) return;
  const int x = nid(L, d, i, j);
  const bool zn = old_n[x] >= ADJZONE && L.mask_n[x] < ADJZONE;
  bool ze[3] = {false, false, false};
  if (i < L.n && j < L.n)
    for (int e = 0; e < 3; ++e) ze[e] = old_e[e * L.NN + x] >= ADJZONE && L.mask_e[e * L.NN + x] < ADJZONE;
  if (!(zn || ze[0] || ze[1] || ze[2])) return;
  for (int kk = 0; kk < nz; ++kk) {
    if (zn) {
      L.wm[(int64_t)kk * L.NN + x] = 0.0;
      L.wt[(int64_t)kk * L.NN + x] = 0.0;
    }
    for (int e = 0; e < 3; ++e)
      if (ze[e]) L.wv[(int64_t)kk * 3 * L.NN + e * L.NN + x] = 0.0;
  }
}

// Ghost copy of one level's layered node and edge fields (for host downloads).
__global__ void k_halo_level(int nz, int NN, const int2* __restrict__ hn, int n_hn, const int3* __restrict__ he, int n_he,
                             double* a, double* b, double* v) {
  const int per = 2 * n_hn + n_he;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)per * nz) return;
  const int k = (int)(t / per);
  const int r = (int)(t - (int64_t)k * per);
  if (r < 2 * n_hn) {
    const int2 e = hn[r % n_hn];
    double* f = (r < n_hn ? a : b) + (int64_t)k * NN;
    f[e.x] = f[e.y];
  } else {
    const int3 e = he[r - 2 * n_hn];
    double* f = v + (int64_t)k * 3 * NN;
    const double x = f[e.y];
    f[e.x] = e.z < 0 ? -x : x;
  }
}

}  // namespace wtw

// ---------------------------------------------------------------------------
// adapt's mask sequence (src/adapt.f90:14-65, src/mask.f90) on the dense
// hierarchy.  Each sweep is one kernel over the reference's iteration range;
// set_at_least is an atomic max.  Within every sweep the conditions read
// values the sweep cannot change (they test == TOLRNZ, >= TOLRNZ or
// >= ADJSPACE while the sweep writes lower values, or they read mask classes
// the sweep does not write), so the parallel sweep equals the sequential one.
namespace wtw {

constexpr int ADJSPACE = 14, RESTRCT = 12, TRSK = 2;

__device__ __forceinline__ void sat(int* m, int x, int typ) {
  if (m[x] < typ) atomicMax(m + x, typ);
}
__device__ __forceinline__ void sn(const WLev& g, int d, int i, int j, int typ) {
  if (inr(g, i, j)) sat(g.mask_n, nid(g, d, i, j), typ);
}
__device__ __forceinline__ void se(const WLev& g, int e, int d, int i, int j, int typ) {
  if (inr(g, i, j)) sat(g.mask_e, e * g.NN + nid(g, d, i, j), typ);
}
// thread -> (lozenge, i, j) over [st, m-1+st]^2
__device__ __forceinline__ bool node_of(int m, int st, int& d, int& i, int& j) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return false;
  d = t / (m * m);
  const int r = t - d * m * m;
  j = r / m + st;
  i = r % m + st;
  return true;
}

// serial comm_masks_mpi (src/comm.f90:531-553): node and edge masks to their
// ghost copies (the tables have no chains, so the copy order is immaterial).
// The mask ghost copy of every level in one launch (comm_masks): thread t
// belongs to the level q with start[q] <= t < start[q+1].
constexpr int MH_MAXL = 16;
struct MaskHaloSet {
  int nl;
  int start[MH_MAXL + 1];
  int n_hn[MH_MAXL];
  int* mask_n[MH_MAXL];
  int* mask_e[MH_MAXL];
  const int2* hn[MH_MAXL];
  const int3* he[MH_MAXL];
};
__global__ void k_mask_halo_all(MaskHaloSet S) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.start[S.nl]) return;
  int q = 0;
  while (t >= S.start[q + 1]) ++q;
  const int r = t - S.start[q];
  if (r < S.n_hn[q]) {
    const int2 c = S.hn[q][r];
    S.mask_n[q][c.x] = S.mask_n[q][c.y];
  } else {
    const int3 c = S.he[q][r - S.n_hn[q]];
    S.mask_e[q][c.x] = S.mask_e[q][c.y];
  }
}

// mask_tol_vars (src/mask.f90:102-156) on nodes [st, n-1+en]^2 of one level:
// block (32 nodes, ny), thread y tests layers y, y + ny, ... of the node's two
// scalars and three edges (read through the ghost remaps), and the flags are
// OR-ed in shared memory before the y = 0 thread updates the masks.
// thr[v*nz + k]: v = 0 mass, 1 Theta, 2 velocity.
// Whether padded slot y (its own source) lies in an existing patch of the
// level (exist: [10][n/ps][n/ps] patch bytes); the pole slots count as in.
__device__ __forceinline__ bool slot_in_tree(const WLev& L, const unsigned char* __restrict__ exist, int ps, int y) {
  const int PP = L.P * L.P;
  const int d = y / PP, r = y - d * PP;
  const int i = r % L.P - 2, j = r / L.P - 2;
  if (i < 0 || j < 0 || i >= L.n || j >= L.n) return true;
  const int np = L.n / ps;
  return exist[((int64_t)d * np + j / ps) * np + i / ps] != 0;
}

// With a patch tree (exist non-null), a node whose own wavelets and whose
// edges' wavelets all belong to nodes outside the tree is left out: the
// compression that produced the wavelets kept none there (masks never reach
// outside the tree), and init_masks_zero left its masks ZERO, which a pass
// with zero wavelets keeps.
__global__ void k_mask_tol_y(WLev L, int nz, int st, int en, const double* __restrict__ thr, int below_fill,
                             const unsigned char* __restrict__ exist, int ps) {
  __shared__ int fl[8][32];  // ny <= 8
  __shared__ int s_x[32], s_cn[32], s_ce[3][32];
  __shared__ unsigned char s_in[32], s_go[32];
  const int m = L.n + en - st;
  const int x = threadIdx.x, y = threadIdx.y, ny = blockDim.y;
  if (y == 0) {  // the node of column x, once for the block's layer threads
    const int64_t t = (int64_t)blockIdx.x * 32 + x;
    bool in = t < (int64_t)10 * m * m;
    int d = 0, i = 0, j = 0;
    if (in) {
      d = (int)(t / ((int64_t)m * m));
      const int r = (int)(t - (int64_t)d * m * m);
      j = r / m + st;
      i = r % m + st;
      in = inr(L, i, j);
    }
    int x_ = 0, cn = 0, ce[3] = {0, 0, 0};
    if (in) {
      x_ = nid(L, d, i, j);
      in = L.mask_n[x_] != FROZEN;
    }
    bool read = in;
    if (in) {
      cn = __ldg(L.nsrc + x_);
#pragma unroll
      for (int e = 0; e < 3; ++e) ce[e] = __ldg(L.esrc + e * L.NN + x_);
      if (exist && !below_fill) {
        read = slot_in_tree(L, exist, ps, cn);
#pragma unroll
        for (int e = 0; e < 3; ++e) read = read || slot_in_tree(L, exist, ps, (ce[e] >> 1) % L.NN);
      }
    }
    s_in[x] = in;
    s_go[x] = read;
    s_x[x] = x_;
    s_cn[x] = cn;
#pragma unroll
    for (int e = 0; e < 3; ++e) s_ce[e][x] = ce[e];
  }
  __syncthreads();
  const bool in = s_in[x], go = s_go[x];
  // with a tree, a block none of whose nodes reads a wavelet changes no mask
  if (exist && !below_fill && !__syncthreads_or(go)) return;
  const int x_ = s_x[x], cn = s_cn[x];
  int f = 0;
  if (go) {
    int ce[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) ce[e] = s_ce[e][x];
    for (int k = y; k < nz; k += ny) {
      const double wm = L.wm[(int64_t)k * L.NN + cn], wt = L.wt[(int64_t)k * L.NN + cn];
      if (fabs(wm) >= thr[0 * nz + k] || below_fill) f |= 1;
      if (fabs(wt) >= thr[1 * nz + k] || below_fill) f |= 1;
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        const int c = ce[e];
        const double v = L.wv[(int64_t)k * 3 * L.NN + (c >> 1)];
        if (fabs((c & 1) ? -v : v) >= thr[2 * nz + k] || below_fill) f |= 2 << e;
      }
    }
  }
  fl[y][x] = f;
  __syncthreads();
  if (y != 0 || !in) return;
  for (int q = 1; q < ny; ++q) f |= fl[q][x];
  if (f & 1)
    L.mask_n[x_] = TOLRNZ;
  else if (L.mask_n[x_] > ADJZONE)
    L.mask_n[x_] = ADJZONE;
  for (int e = 0; e < 3; ++e) {
    int& me_ = L.mask_e[e * L.NN + x_];
    if (f & (2 << e))
      me_ = TOLRNZ;
    else if (me_ > ADJZONE)
      me_ = ADJZONE;
  }
}

__global__ void k_mask_zero(WLev g) {  // init_masks_zero on one level
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < g.NN) g.mask_n[t] = ZERO;
  if (t < 3 * g.NN) g.mask_e[t] = ZERO;
}

// mask_parent_nodes (parents [0, np]) and mask_parent_edges (parents [0, np))
__global__ void k_mask_parent(WLev Pa, WLev C) {
  int d, ip, jp;
  if (!node_of(Pa.n + 1, 0, d, ip, jp)) return;
  const int i = 2 * ip, j = 2 * jp;
  if (mn(C, d, i + 1, j) == TOLRNZ || mn(C, d, i + 1, j + 1) == TOLRNZ || mn(C, d, i, j + 1) == TOLRNZ ||
      mn(C, d, i - 1, j) == TOLRNZ || mn(C, d, i - 1, j - 1) == TOLRNZ || mn(C, d, i, j - 1) == TOLRNZ) {
    sn(Pa, d, ip, jp, TOLRNZ);
    sn(C, d, i, j, TOLRNZ);
  }
  if (ip == Pa.n || jp == Pa.n) return;
  auto T = [&](int e, int a, int b) { return me(C, e, d, a, b) == TOLRNZ; };
  if (T(RT, i, j) || T(RT, i + 1, j) || T(DG, i, j - 1) || T(DG, i + 1, j) || T(UP, i + 1, j) || T(UP, i + 1, j - 1))
    se(Pa, RT, d, ip, jp, TOLRNZ);
  if (T(RT, i, j + 1) || T(RT, i + 1, j + 1) || T(DG, i, j) || T(DG, i + 1, j + 1) || T(UP, i + 1, j + 1) || T(UP, i + 1, j))
    se(Pa, DG, d, ip, jp, TOLRNZ);
  if (T(RT, i, j + 1) || T(RT, i - 1, j + 1) || T(DG, i, j + 1) || T(DG, i - 1, j) || T(UP, i, j) || T(UP, i, j + 1))
    se(Pa, UP, d, ip, jp, TOLRNZ);
}

// mask_adj_same_scale_nodes_edges, nodes [0, n]
__global__ void k_mask_adj_same(WLev g) {
  int d, i, j;
  if (!node_of(g.n + 1, 0, d, i, j)) return;
  if (mn(g, d, i + 1, j) == TOLRNZ || mn(g, d, i + 1, j + 1) == TOLRNZ || mn(g, d, i, j + 1) == TOLRNZ ||
      mn(g, d, i - 1, j) == TOLRNZ || mn(g, d, i - 1, j - 1) == TOLRNZ || mn(g, d, i, j - 1) == TOLRNZ)
    sn(g, d, i, j, ADJSPACE);
  auto T = [&](int e, int a, int b) { return me(g, e, d, a, b) == TOLRNZ; };
  if (T(DG, i, j) || T(UP, i, j - 1) || T(DG, i, j - 1) || T(UP, i + 1, j)) se(g, RT, d, i, j, ADJSPACE);
  if (T(UP, i, j) || T(RT, i, j) || T(UP, i + 1, j) || T(RT, i, j + 1)) se(g, DG, d, i, j, ADJSPACE);
  if (T(DG, i, j) || T(RT, i - 1, j) || T(DG, i - 1, j) || T(RT, i, j + 1)) se(g, UP, d, i, j, ADJSPACE);
}

// mask_restrict_flux, nodes [0, n)
__global__ void k_mask_restrict_flux(WLev g) {
  int d, i, j;
  if (!node_of(g.n, 0, d, i, j)) return;
  if (mn(g, d, i, j) >= ADJSPACE) {
    se(g, RT, d, i, j, RESTRCT);
    se(g, DG, d, i, j, RESTRCT);
    se(g, UP, d, i, j, RESTRCT);
  } else {
    if (mn(g, d, i + 1, j) >= ADJSPACE) se(g, RT, d, i, j, RESTRCT);
    if (mn(g, d, i + 1, j + 1) >= ADJSPACE) se(g, DG, d, i, j, RESTRCT);
    if (mn(g, d, i, j + 1) >= ADJSPACE) se(g, UP, d, i, j, RESTRCT);
  }
}

// mask_adj_child, parents [0, np]
__global__ void k_mask_adj_child(WLev Pa, WLev C) {
  int d, ip, jp;
  if (!node_of(Pa.n + 1, 0, d, ip, jp)) return;
  const int i = 2 * ip, j = 2 * jp;
  auto PE = [&](int e, int a, int b, int typ) { return me(Pa, e, d, a, b) >= typ; };
  if (mn(Pa, d, ip, jp) >= TOLRNZ) {
    const int nb[13][2] = {{0, 0},  {1, 0},  {1, 1}, {0, 1}, {-1, 0},  {-1, -1}, {0, -1},
                           {-1, 1}, {1, -1}, {2, 1}, {1, 2}, {-1, -2}, {-2, -1}};
    for (int q = 0; q < 13; ++q) sn(C, d, i + nb[q][0], j + nb[q][1], ADJZONE);
    se(Pa, UP, d, ip, jp, RESTRCT);
    se(Pa, DG, d, ip, jp, RESTRCT);
    se(Pa, RT, d, ip, jp, RESTRCT);
  } else {
    if (mn(Pa, d, ip, jp + 1) >= TOLRNZ) {
      sn(C, d, i, j + 1, ADJZONE);
      se(Pa, UP, d, ip, jp, RESTRCT);
    }
    if (mn(Pa, d, ip + 1, jp + 1) >= TOLRNZ) {
      sn(C, d, i + 1, j + 1, ADJZONE);
      se(Pa, DG, d, ip, jp, RESTRCT);
    }
    if (mn(Pa, d, ip + 1, jp) >= TOLRNZ) {
      sn(C, d, i + 1, j, ADJZONE);
      se(Pa, RT, d, ip, jp, RESTRCT);
    }
  }
  if (PE(UP, ip, jp, TOLRNZ)) {
    sn(C, d, i, j + 1, ADJZONE);
    if (PE(UP, ip, jp - 1, TOLRNZ)) sn(C, d, i, j, ADJZONE);
  }
  if (PE(DG, ip, jp, TOLRNZ)) {
    sn(C, d, i + 1, j + 1, ADJZONE);
    if (PE(DG, ip - 1, jp - 1, TOLRNZ)) sn(C, d, i, j, ADJZONE);
  }
  if (PE(RT, ip, jp, TOLRNZ)) {
    sn(C, d, i + 1, j, ADJZONE);
    if (PE(RT, ip - 1, jp, TOLRNZ)) sn(C, d, i, j, ADJZONE);
  }
  if (PE(UP, ip, jp, TOLRNZ) || PE(DG, ip, jp, TOLRNZ) || PE(RT, ip - 1, jp, TOLRNZ) || PE(DG, ip - 1, jp, TOLRNZ) ||
      PE(RT, ip, jp + 1, TOLRNZ)) {
    se(C, UP, d, i, j, ADJZONE);
    se(C, UP, d, i, j + 1, ADJZONE);
  }
  if (PE(DG, ip, jp, TOLRNZ) || PE(UP, ip, jp, TOLRNZ) || PE(RT, ip, jp, TOLRNZ) || PE(UP, ip + 1, jp, TOLRNZ) ||
      PE(RT, ip, jp + 1, TOLRNZ)) {
    se(C, DG, d, i, j, ADJZONE);
    se(C, DG, d, i + 1, j + 1, ADJZONE);
  }
  if (PE(RT, ip, jp, TOLRNZ) || PE(DG, ip, jp, TOLRNZ) || PE(UP, ip, jp - 1, TOLRNZ) || PE(DG, ip, jp - 1, TOLRNZ) ||
      PE(UP, ip + 1, jp, TOLRNZ)) {
    se(C, RT, d, i, j, ADJZONE);
    se(C, RT, d, i + 1, j, ADJZONE);
  }
  if (PE(UP, ip, jp, TOLRNZ) || PE(DG, ip, jp, TOLRNZ) || PE(RT, ip, jp + 1, TOLRNZ)) {
    se(C, RT, d, i, j + 1, ADJZONE);
    se(C, DG, d, i, j + 1, ADJZONE);
    se(C, UP, d, i + 1, j + 1, ADJZONE);
  }
  if (PE(RT, ip, jp, TOLRNZ) || PE(DG, ip, jp, TOLRNZ) || PE(UP, ip + 1, jp, TOLRNZ)) {
    se(C, UP, d, i + 1, j, ADJZONE);
    se(C, DG, d, i + 1, j, ADJZONE);
    se(C, RT, d, i + 1, j + 1, ADJZONE);
  }
  if (PE(RT, ip, jp, ADJSPACE) || PE(DG, ip, jp, ADJSPACE) || PE(UP, ip, jp, ADJSPACE) || PE(RT, ip - 1, jp, ADJSPACE) ||
      PE(DG, ip - 1, jp - 1, ADJSPACE) || PE(UP, ip, jp - 1, ADJSPACE))
    sn(Pa, d, ip, jp, RESTRCT);
}

// mask_edges_if_both_nodes, nodes [0, n)
__global__ void k_mask_edges_both(WLev g) {
  int d, i, j;
  if (!node_of(g.n, 0, d, i, j)) return;
  if (mn(g, d, i, j) >= ADJZONE) {
    if (mn(g, d, i + 1, j) >= ADJZONE) se(g, RT, d, i, j, ADJZONE);
    if (mn(g, d, i + 1, j + 1) >= ADJZONE) se(g, DG, d, i, j, ADJZONE);
    if (mn(g, d, i, j + 1) >= ADJZONE) se(g, UP, d, i, j, ADJZONE);
  }
}

// mask_edges_consist, parents [0, np]
__global__ void k_mask_edges_consist(WLev Pa, WLev C) {
  int d, ip, jp;
  if (!node_of(Pa.n + 1, 0, d, ip, jp)) return;
  const int i = 2 * ip, j = 2 * jp;
  auto A = [&](int e, int a, int b) { return me(C, e, d, a, b) >= ADJZONE; };
  if (A(RT, i, j) || A(RT, i + 1, j) || A(DG, i, j - 1) || A(DG, i + 1, j) || A(UP, i + 1, j - 1) || A(UP, i + 1, j)) {
    se(C, RT, d, i, j, ADJZONE);
    se(C, RT, d, i + 1, j, ADJZONE);
    se(Pa, RT, d, ip, jp, ADJZONE);
  }
  if (A(RT, i, j + 1) || A(RT, i + 1, j + 1) || A(DG, i, j) || A(DG, i + 1, j + 1) || A(UP, i + 1, j) || A(UP, i + 1, j + 1)) {
    se(C, DG, d, i, j, ADJZONE);
    se(C, DG, d, i + 1, j + 1, ADJZONE);
    se(Pa, DG, d, ip, jp, ADJZONE);
  }
  if (A(RT, i - 1, j + 1) || A(RT, i, j + 1) || A(DG, i - 1, j) || A(DG, i, j + 1) || A(UP, i, j) || A(UP, i, j + 1)) {
    se(C, UP, d, i, j, ADJZONE);
    se(C, UP, d, i, j + 1, ADJZONE);
    se(Pa, UP, d, ip, jp, ADJZONE);
  }
}

// mask_edges_consist2, parents [0, np)
__global__ void k_mask_edges_consist2(WLev Pa, WLev C) {
  int d, ip, jp;
  if (!node_of(Pa.n, 0, d, ip, jp)) return;
  const int i = 2 * ip, j = 2 * jp;
  auto A = [&](int e, int a, int b) { return me(C, e, d, i + a, j + b) >= ADJZONE; };
  if (A(RT, -2, -2) || A(RT, 0, -2) || A(RT, 0, 2) || A(RT, 2, 2) || A(DG, -2, -2) || A(DG, 0, -2) || A(DG, 0, 0) ||
      A(DG, 2, 0) || A(UP, 0, -2) || A(UP, 2, -2) || A(UP, 0, 0) || A(UP, 2, 0))
    se(Pa, RT, d, ip, jp, ADJZONE);
  if (A(RT, -2, 0) || A(RT, 0, 0) || A(RT, 0, 2) || A(RT, 2, 2) || A(DG, 0, -2) || A(DG, -2, 0) || A(DG, 2, 0) ||
      A(DG, 0, 2) || A(UP, 0, -2) || A(UP, 0, 0) || A(UP, 2, 0) || A(UP, 2, 2))
    se(Pa, DG, d, ip, jp, ADJZONE);
  if (A(RT, 0, 0) || A(RT, 0, 2) || A(RT, -2, 0) || A(RT, -2, 2) || A(DG, 0, 2) || A(DG, 0, 0) || A(DG, -2, -2) ||
      A(DG, -2, 0) || A(UP, 2, 0) || A(UP, 2, 2) || A(UP, -2, -2) || A(UP, -2, 0))
    se(Pa, UP, d, ip, jp, ADJZONE);
}

// mask_nodes_if_all_edges, nodes [0, n]
__global__ void k_mask_nodes_all(WLev g) {
  int d, i, j;
  if (!node_of(g.n + 1, 0, d, i, j)) return;
  if (me(g, RT, d, i, j) >= ADJZONE && me(g, DG, d, i, j) >= ADJZONE && me(g, UP, d, i, j) >= ADJZONE &&
      me(g, RT, d, i - 1, j) >= ADJZONE && me(g, DG, d, i - 1, j - 1) >= ADJZONE && me(g, UP, d, i, j - 1) >= ADJZONE)
    sn(g, d, i, j, ADJZONE);
}

// prolong_node_adjzone, parents [0, np]
__global__ void k_mask_prolong_adj(WLev Pa, WLev C) {
  int d, ip, jp;
  if (!node_of(Pa.n + 1, 0, d, ip, jp)) return;
  if (mn(C, d, 2 * ip, 2 * jp) >= ADJZONE) sn(Pa, d, ip, jp, ADJZONE);
}

// mask_node_trsk with div_grad_stencil (no Laplacian diffusion), nodes [-2, n+1]
__global__ void k_mask_trsk(WLev g) {
  int d, i, j;
  if (!node_of(g.n + 4, -2, d, i, j)) return;
  if (mn(g, d, i, j) < ADJZONE) return;
  const int nb[7][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}, {-1, 0}, {-1, -1}, {0, -1}};
  for (int q = 0; q < 7; ++q) sn(g, d, i + nb[q][0], j + nb[q][1], TRSK);
  se(g, RT, d, i, j, TRSK);
  se(g, DG, d, i, j, TRSK);
  se(g, UP, d, i, j, TRSK);
  se(g, RT, d, i - 1, j, TRSK);
  se(g, DG, d, i - 1, j - 1, TRSK);
  se(g, UP, d, i, j - 1, TRSK);
}

// check_child_required (src/refine_patch.f90:289-327): one flag per (lozenge,
// parent patch of side ps, child quadrant c = 0 NE, 1 SE, 2 SW, 3 NW).
__global__ void k_child_required(WLev g, int ps, unsigned char* __restrict__ out) {
  const int np = g.n / ps;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * np * np * 4) return;
  const int c = t % 4, r = t / 4;
  const int pi = r % np, pj = (r / np) % np, d = r / (np * np);
  const int ox = (c == 0 || c == 1) ? ps / 2 : 0, oy = (c == 0 || c == 3) ? ps / 2 : 0;
  bool req = false;
  for (int jj = -2; jj <= ps / 2 + 1 && !req; ++jj)
    for (int ii = -2; ii <= ps / 2 + 1 && !req; ++ii) {
      const int i = pi * ps + ox + ii, j = pj * ps + oy + jj;
      req = mn(g, d, i, j) >= ADJZONE || me(g, RT, d, i, j) >= RESTRCT || me(g, DG, d, i, j) >= RESTRCT ||
            me(g, UP, d, i, j) >= RESTRCT;
    }
  out[t] = req ? 1 : 0;
}

}  // namespace wtw
