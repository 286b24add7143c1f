// Nodes whose step1 and trend results can reach the state after WT_after_step,
// for every level above level_start.  After every RK stage the inverse
// transform rebuilds such a level from the next coarser one and the wavelets
// kept by compress_wavelets, so its stage results are read only
//   * by its trend where mask_n >= TRSK (stencils of hex radius 2),
//   * by the forward wavelets of its slots with mask >= ADJZONE (radius 2),
//   * by the restriction into the parents with mask >= RESTRCT (radius 4 around
//     the parent's node) and by the coarser trend's restricted velocity source
//     (child edges with mask >= ADJZONE),
//   * as the parent velocities of the next finer level's forward wavelets
//     (radius 2 around the parents of that level's slots with mask >= TRSK).
// The map seeds those nodes and dilates them NEED_R hex steps through the ghost
// remaps; the lozenge corners (pentagons, poles), whose neighbourhoods the
// remaps describe only for the stencils that use them, are always in it.
// Values are read through nsrc: need[nsrc[x]].  level_start has no map: the
// inverse transform does not rebuild it.
#pragma once
#include "wavelet_kernels.cuh"

namespace wtw {

#ifndef WT_NEED_R
#define WT_NEED_R 4
#endif
constexpr int NEED_R = WT_NEED_R;
constexpr int NEED_MAXL = 16;

// Entry q is level level_start + q; entry 0 (level_start) only lends its masks.
struct NeedLev {
  int n, P, NN;
  const int* nsrc;
  const int* mask_n;
  const int* mask_e;
  unsigned char* buf[2];  // map and dilation scratch (null on entry 0)
};
struct NeedSet {
  int nl;                      // entries, level_start included
  int start[NEED_MAXL + 1];    // thread offsets of entries 1..nl-1 (start[1] = 0)
  NeedLev L[NEED_MAXL];
};

__device__ __forceinline__ bool need_entry(const NeedSet& S, int64_t t, int& q, int& x) {
  if (t >= S.start[S.nl]) return false;
  q = 1;
  while (t >= S.start[q + 1]) ++q;
  x = (int)(t - S.start[q]);
  return true;
}

__device__ __forceinline__ bool any_mask(const NeedLev& E, int x, int thr) {
  return E.mask_n[x] >= thr || E.mask_e[x] >= thr || E.mask_e[E.NN + x] >= thr || E.mask_e[2 * E.NN + x] >= thr;
}

// seeds of every padded slot of every entry into buf[0]
__global__ void k_need_seed(NeedSet S) {
  int q, x;
  if (!need_entry(S, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, q, x)) return;
  const NeedLev& E = S.L[q];
  const int PP = E.P * E.P;
  const int d = x / PP, r = x - d * PP;
  const int i = r % E.P - 2, j = r / E.P - 2, n = E.n;
  int v;
  if (i >= 0 && j >= 0 && i < n && j < n) {
    v = any_mask(E, x, TRSK);
    if (!v && !(i & 1) && !(j & 1)) {  // parent node with a restricted value or flux
      const NeedLev& Pa = S.L[q - 1];
      v = any_mask(Pa, (d * Pa.P + j / 2 + 2) * Pa.P + i / 2 + 2, RESTRCT);
    }
    if (!v && q + 1 < S.nl) {  // parent of finer slots whose wavelets are computed
      const NeedLev& C = S.L[q + 1];
      for (int c = 0; c < 4 && !v; ++c)
        v = any_mask(C, (d * C.P + 2 * j + (c >> 1) + 2) * C.P + 2 * i + (c & 1) + 2, TRSK);
    }
    const int cr = NEED_R + 1;
    if ((i <= cr || i >= n - 1 - cr) && (j <= cr || j >= n - 1 - cr)) v = 1;
  } else {
    v = __ldg(E.nsrc + x) == x;  // a slot outside [0, n)^2 that is its own source
  }
  E.buf[0][x] = (unsigned char)v;
}

// one hex step from buf[r & 1] into buf[(r + 1) & 1]: a slot is needed if it
// or one of its six neighbours is
__global__ void k_need_dilate(NeedSet S, int r) {
  int q, x;
  if (!need_entry(S, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, q, x)) return;
  const NeedLev& E = S.L[q];
  const unsigned char* __restrict__ in = E.buf[r & 1];
  const int PP = E.P * E.P;
  const int d = x / PP, rr = x - d * PP;
  const int i = rr % E.P - 2, j = rr / E.P - 2;
  int v = in[__ldg(E.nsrc + x)];
  const int di[6] = {1, -1, 0, 0, 1, -1}, dj[6] = {0, 0, 1, -1, 1, -1};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int a = i + di[k], b = j + dj[k];
    if (a >= -2 && b >= -2 && a < E.n + 2 && b < E.n + 2)
      v |= in[__ldg(E.nsrc + (d * E.P + b + 2) * E.P + a + 2)];
  }
  E.buf[(r + 1) & 1][x] = (unsigned char)v;
}

}  // namespace wtw

namespace wtw {

// Parents each inverse transform of an intermediate RK stage rebuilds.  Between
// the stages a level's state is read only by the next stage's step1 (radius 2
// around its needed nodes) and, as the parent of the next finer level, by that
// level's reconstruction (radius 2 around the parents it rebuilds).  From the
// finest level down: rec(c) = dilate(need(c) | recpar(c), 2) on child level c,
// recpar(c-1) = dilate(parents of rec(c), 2) on its parent level; a parent is
// rebuilt where recpar says so (read through nsrc).  The step's last stage and
// the inverse after adapt rebuild every parent.
struct MapLev {
  int n, P, NN;
  const int* nsrc;
};

__global__ void k_map_or(int NN, const unsigned char* __restrict__ a, const unsigned char* __restrict__ b,
                         unsigned char* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < NN) out[x] = (unsigned char)(a[x] | (b ? b[x] : 0));
}

__global__ void k_map_dilate(MapLev L, const unsigned char* __restrict__ in, unsigned char* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= L.NN) return;
  const int PP = L.P * L.P;
  const int d = x / PP, r = x - d * PP;
  const int i = r % L.P - 2, j = r / L.P - 2;
  int v = in[__ldg(L.nsrc + x)];
  const int di[6] = {1, -1, 0, 0, 1, -1}, dj[6] = {0, 0, 1, -1, 1, -1};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int a = i + di[k], b = j + dj[k];
    if (a >= -2 && b >= -2 && a < L.n + 2 && b < L.n + 2)
      v |= in[__ldg(L.nsrc + (d * L.P + b + 2) * L.P + a + 2)];
  }
  out[x] = (unsigned char)v;
}

// parent slot x of level Pa is marked if one of its four children is marked
__global__ void k_map_up(MapLev C, MapLev Pa, const unsigned char* __restrict__ cin, unsigned char* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= Pa.NN) return;
  const int PP = Pa.P * Pa.P;
  const int d = x / PP, r = x - d * PP;
  const int ip = r % Pa.P - 2, jp = r / Pa.P - 2;
  int v = 0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int a = 2 * ip + (c & 1), b = 2 * jp + (c >> 1);
    if (a >= -2 && b >= -2 && a < C.n + 2 && b < C.n + 2)
      v |= cin[__ldg(C.nsrc + (d * C.P + b + 2) * C.P + a + 2)];
  }
  out[x] = (unsigned char)v;
}

}  // namespace wtw

namespace wtw {

// The patch tree's part in the maps (tree_kernels.cuh): the reference
// computes, transforms and keeps values only on the nodes of existing
// patches, and reads the 2-node ring of boundary patches around them.
struct TreeLev {
  int n, P, NN;
  const int* nsrc;
  const unsigned char* exist;  // [10][n/ps][n/ps] patch bytes of this level
};

// Whether padded slot y of a level is a node of an existing patch (through its
// ghost source); the pole slots, which no patch's [0, n)^2 holds, count as
// existing.
__device__ __forceinline__ bool tree_node(const TreeLev& T, int ps, int y) {
  const int s = __ldg(T.nsrc + y);
  const int PP = T.P * T.P;
  const int d = s / PP, r = s - d * PP;
  const int i = r % T.P - 2, j = r / T.P - 2;
  if (i < 0 || j < 0 || i >= T.n || j >= T.n) return true;
  const int np = T.n / ps;
  return T.exist[((int64_t)d * np + j / ps) * np + i / ps] != 0;
}

// Whether a node of an existing patch lies within 2 nodes (i and j each) of
// padded slot (d, i, j), i, j in [0, n): the patch nodes and their 2-node ring.
__device__ __forceinline__ bool tree_near(const TreeLev& T, int ps, int d, int i, int j) {
  for (int b = -2; b <= 2; ++b)
    for (int a = -2; a <= 2; ++a)
      if (tree_node(T, ps, (d * T.P + j + b + 2) * T.P + i + a + 2)) return true;
  return false;
}

// need &= the tree's nodes and their ring, on the owned nodes [0, n)^2 of one
// level (the lozenge-corner regions the seed forces stay in).
__global__ void k_need_tree(TreeLev T, int ps, unsigned char* __restrict__ need) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= T.NN || !need[x]) return;
  const int PP = T.P * T.P;
  const int d = x / PP, r = x - d * PP;
  const int i = r % T.P - 2, j = r / T.P - 2, n = T.n;
  if (i < 0 || j < 0 || i >= n || j >= n) return;
  const int cr = NEED_R + 1;
  if ((i <= cr || i >= n - 1 - cr) && (j <= cr || j >= n - 1 - cr)) return;
  if (!tree_near(T, ps, d, i, j)) need[x] = 0;
}

// The parents the inverse transform after adapt rebuilds with a patch tree:
// those of the next RK stage (recpar, in) and every parent one of whose
// children within 2 nodes of the coincident child is a node of an existing
// patch of the child level, so that the state after the step is complete on
// the tree.  Own-source parent slots only (the kernels read through nsrc).
__global__ void k_map_tree_par(MapLev Lp, TreeLev Tc, int ps, const unsigned char* __restrict__ in,
                               unsigned char* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= Lp.NN) return;
  unsigned char v = in[x];
  if (!v && __ldg(Lp.nsrc + x) == x) {
    const int PP = Lp.P * Lp.P;
    const int d = x / PP, r = x - d * PP;
    const int ip = r % Lp.P - 2, jp = r / Lp.P - 2;
    if (ip >= 0 && jp >= 0 && ip <= Lp.n && jp <= Lp.n) v = tree_near(Tc, ps, d, 2 * ip < Tc.n ? 2 * ip : Tc.n - 1,
                                                                     2 * jp < Tc.n ? 2 * jp : Tc.n - 1);
    else
      v = 1;
  }
  out[x] = v;
}

}  // namespace wtw



namespace wtw {

// Work lists in ascending slot order (so that a warp of a list kernel takes
// neighbouring rows of a patch and their stencils share cache lines), by a
// three-pass compaction over blocks of LIST_B candidates: per-block counts, one
// scan of the counts, then each block writes its entries at its offset.
constexpr int LIST_B = 1024;

// Candidates of a level's node list: every padded slot x, on where
// need[nsrc[x]] is set.
struct NodeCand {
  int NN;
  const int* nsrc;
  const unsigned char* map;
  __device__ __forceinline__ int n() const { return NN; }
  __device__ __forceinline__ bool on(int t, int& x) const {
    x = t;
    return map[__ldg(nsrc + t)] != 0;
  }
};
// Candidates of a parent level's list: the slots of [0, np]^2, on where
// rec[nsrc[x]] is set.
struct ParentCand {
  int np, P;
  const int* nsrc;
  const unsigned char* map;
  __device__ __forceinline__ int n() const { return 10 * (np + 1) * (np + 1); }
  __device__ __forceinline__ bool on(int t, int& x) const {
    const int m = np + 1, d = t / (m * m), r = t - d * m * m;
    const int jp = r / m, ip = r - jp * m;
    x = (d * P + jp + 2) * P + ip + 2;
    return map[__ldg(nsrc + x)] != 0;
  }
};

template <class Cand>
__global__ void __launch_bounds__(LIST_B) k_list_count(Cand c, int* __restrict__ bcnt) {
  const int t = blockIdx.x * LIST_B + threadIdx.x;
  int x;
  const bool on = t < c.n() && c.on(t, x);
  const int k = __syncthreads_count(on);
  if (threadIdx.x == 0) bcnt[blockIdx.x] = k;
}

// Exclusive scan of nb block counts into boff, the total into *count (one block).
__global__ void __launch_bounds__(LIST_B) k_list_scan(int nb, const int* __restrict__ bcnt, int* __restrict__ boff,
                                                      int* __restrict__ count) {
  __shared__ int part[LIST_B];
  const int t = threadIdx.x;
  const int run = (nb + LIST_B - 1) / LIST_B;
  const int a = min(nb, t * run), b = min(nb, a + run);
  int c = 0;
  for (int q = a; q < b; ++q) c += bcnt[q];
  part[t] = c;
  __syncthreads();
  for (int o = 1; o < LIST_B; o <<= 1) {
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int w = part[t] - c;
  for (int q = a; q < b; ++q) {
    boff[q] = w;
    w += bcnt[q];
  }
  if (t == LIST_B - 1) *count = part[t];
}

template <class Cand>
__global__ void __launch_bounds__(LIST_B) k_list_write(Cand c, const int* __restrict__ boff, int* __restrict__ ids) {
  __shared__ int wsum[LIST_B / 32];
  const int t = blockIdx.x * LIST_B + threadIdx.x;
  int x = 0;
  const bool on = t < c.n() && c.on(t, x);
  const unsigned m = __ballot_sync(0xffffffffu, on);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wsum[w] = __popc(m);
  __syncthreads();
  int before = 0;
  for (int q = 0; q < w; ++q) before += wsum[q];
  if (on) ids[boff[blockIdx.x] + before + __popc(m & ((1u << lane) - 1))] = x;
}

}  // namespace wtw
