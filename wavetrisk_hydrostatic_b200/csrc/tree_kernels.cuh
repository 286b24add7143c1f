// The patch tree of a partially refined hierarchy on the device: per level a
// byte per patch of ps x ps owned nodes (ps = PATCH_SIZE, src/patch.f90:6),
// lozenge-major [10][n/ps][n/ps] (row j of patches, then column i).
//
// refine() (src/refine_patch.f90:12-49) creates the child patch of a parent
// patch's quadrant where check_child_required flags it and the parent exists;
// the patches that exist when refine starts are the only parents (its loop
// bound is fixed at entry), which holds here because each parent level's
// launch reads its own existence bytes before any launch of the next coarser
// parent level writes them (the host launches the parent levels top down).
#pragma once
#include <cuda_runtime.h>

#include "wavelet_kernels.cuh"

namespace wtw {

// One thread per (parent patch, quadrant c = 0 NE, 1 SE, 2 SW, 3 NW) of parent
// level l with np patches a side: creates the child patch where the flag is
// set, the parent exists and the child does not, marks it new and raises the
// tree's level_end to l + 1 (refine_patch1: level_end grows when a patch of
// level level_end + 1 is made).
__global__ void k_tree_refine(const unsigned char* __restrict__ req, const unsigned char* __restrict__ par,
                              unsigned char* __restrict__ chd, unsigned char* __restrict__ chd_new, int np, int l,
                              int* __restrict__ level_end) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * np * np * 4) return;
  const int c = t % 4, r = t / 4;
  if (!req[t] || !par[r]) return;
  const int pi = r % np, pj = (r / np) % np, d = r / (np * np);
  const int ox = (c == 0 || c == 1) ? 1 : 0, oy = (c == 0 || c == 3) ? 1 : 0;
  const int nc = 2 * np;
  const int64_t x = ((int64_t)d * nc + 2 * pj + oy) * nc + 2 * pi + ox;
  if (chd[x]) return;
  chd[x] = 1;
  chd_new[x] = 1;
  atomicMax(level_end, l + 1);
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// count_active (src/main.f90:137-172) over the owned nodes of the patches the
// last refine created: node wavelets (mass, Theta) with |w| >= threshold(v, k)
// into cnt[0], the velocity wavelets of the node's three edges into cnt[1].
__global__ void k_tree_count_new(WLev g, const unsigned char* __restrict__ fresh, int ps, int nz,
                                 const double* __restrict__ thr, unsigned long long* __restrict__ cnt) {
  const int n = g.n;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long cn = 0, ce = 0;
  if (t < (int64_t)10 * n * n) {
    const int i = (int)(t % n), j = (int)((t / n) % n), d = (int)(t / ((int64_t)n * n));
    const int np = n / ps;
    if (fresh[((int64_t)d * np + j / ps) * np + i / ps]) {
      const int64_t x = ((int64_t)d * g.P + j + 2) * g.P + i + 2;
      for (int k = 0; k < nz; ++k) {
        const int64_t o = (int64_t)k * g.NN + x;
        cn += fabs(g.wm[o]) >= thr[k] ? 1 : 0;
        cn += fabs(g.wt[o]) >= thr[nz + k] ? 1 : 0;
        for (int e = 0; e < 3; ++e) ce += fabs(g.wv[(int64_t)k * 3 * g.NN + (int64_t)e * g.NN + x]) >= thr[2 * nz + k];
      }
    }
  }
  cn = warp_sum_u64(cn);
  ce = warp_sum_u64(ce);
  if ((threadIdx.x & 31) == 0 && (cn | ce)) {
    atomicAdd(&cnt[0], cn);
    atomicAdd(&cnt[1], ce);
  }
}

// The owned nodes of level g outside the tree whose node mask or one of whose
// three edge masks is not ZERO (cnt[0]); the reference has no such node.
__global__ void k_tree_outside(WLev g, const unsigned char* __restrict__ exist, int ps,
                               unsigned long long* __restrict__ cnt) {
  const int n = g.n;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long c = 0;
  if (t < (int64_t)10 * n * n) {
    const int i = (int)(t % n), j = (int)((t / n) % n), d = (int)(t / ((int64_t)n * n));
    const int np = n / ps;
    if (!exist[((int64_t)d * np + j / ps) * np + i / ps]) {
      const int64_t x = ((int64_t)d * g.P + j + 2) * g.P + i + 2;
      c = (g.mask_n[x] | g.mask_e[x] | g.mask_e[g.NN + x] | g.mask_e[2 * (int64_t)g.NN + x]) != 0 ? 1 : 0;
    }
  }
  c = warp_sum_u64(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

}  // namespace wtw

namespace wtw {

// The existing patches of one level as a list of patch indices in
// lozenge-major order (one block: each thread counts a contiguous run of the
// patch bytes, a block-wide scan gives its offset, then it writes its run),
// so that the host and the device agree on the packed order.  Launch with
// one block of TREE_SCAN threads.
constexpr int TREE_SCAN = 1024;
__global__ void __launch_bounds__(TREE_SCAN) k_patch_list(const unsigned char* __restrict__ exist, int npatch,
                                                          int* __restrict__ ids, int* __restrict__ count) {
  __shared__ int part[TREE_SCAN];
  const int t = threadIdx.x;
  const int run = (npatch + TREE_SCAN - 1) / TREE_SCAN;
  const int a = min(npatch, t * run), b = min(npatch, a + run);
  int c = 0;
  for (int x = a; x < b; ++x) c += exist[x] != 0;
  part[t] = c;
  __syncthreads();
  for (int o = 1; o < TREE_SCAN; o <<= 1) {  // inclusive Hillis-Steele scan
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int w = part[t] - c;
  for (int x = a; x < b; ++x)
    if (exist[x]) ids[w++] = x;
  if (t == TREE_SCAN - 1) *count = part[t];
}

// The level's state on the listed patches, packed patch by patch: mass and
// Theta [patch][layer][ps*ps], velocity [patch][layer][edge][ps*ps], the ps*ps
// owned nodes of a patch row by row.  One thread per (patch, layer, node);
// scatter = false gathers the level into the packed arrays, true scatters them
// back.
template <bool SCATTER>
__global__ void k_tree_pack(int n, int P, int NN, int ps, int nz, const int* __restrict__ ids,
                            const int* __restrict__ count, double* __restrict__ m, double* __restrict__ t,
                            double* __restrict__ v, double* __restrict__ pm, double* __restrict__ pt,
                            double* __restrict__ pv) {
  const int ps2 = ps * ps;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t tot = (int64_t)__ldg(count) * nz * ps2;
  if (g >= tot) return;
  const int s = (int)(g % ps2);
  const int64_t pk = g / ps2;  // patch * nz + layer
  const int k = (int)(pk % nz);
  const int p = __ldg(ids + pk / nz);
  const int np = n / ps;
  const int d = p / (np * np), r = p - d * np * np;
  const int i = (r % np) * ps + s % ps, j = (r / np) * ps + s / ps;
  const int64_t x = ((int64_t)d * P + j + 2) * P + i + 2;
  const int64_t o = (int64_t)k * NN + x;
  if (SCATTER) {
    m[o] = pm[g];
    t[o] = pt[g];
  } else {
    pm[g] = m[o];
    pt[g] = t[o];
  }
  for (int e = 0; e < 3; ++e) {
    const int64_t ov = ((int64_t)k * 3 + e) * NN + x, gv = (pk * 3 + e) * ps2 + s;
    if (SCATTER)
      v[ov] = pv[gv];
    else
      pv[gv] = v[ov];
  }
}

}  // namespace wtw
