// Inline readers shared by the layer kernels: interpolation, node indexing,
// the layer-fastest block mapping and reads of the state through the ghost
// remap tables; device functions and one inline host helper (the grid of a
// persistent kernel), so several translation units may include it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "trisk_types.cuh"


namespace wtk {

__device__ __forceinline__ double interp(double a, double b) { return 0.5 * (a + b); }  // src/utils.f90:528

__device__ __forceinline__ int64_t nid(const LevelDev& L, int d, int i, int j) {
  return ((int64_t)d * L.P + (j + 2)) * L.P + (i + 2);
}

// Block-to-work mapping of the layer kernels: block b covers NODE_TILE
// consecutive padded nodes of layer b % nz, so the nz blocks of one node chunk
// are dispatched back to back and read that chunk's level geometry from L2
// instead of DRAM.  Offsets inside one layer are 32-bit (the context rejects
// levels with 6*NN >= 2^31).
constexpr int NODE_TILE = 256;

__device__ __forceinline__ void node_ij(const LevelDev& L, int id, int& i, int& j) {
  const int pp = L.P * L.P;
  const int r = id - (id / pp) * pp;
  const int jp = r / L.P;
  j = jp - 2;
  i = r - jp * L.P - 2;
}

__device__ __forceinline__ bool layer_node(const LevelDev& L, int nz, int& k, int& id, int& i, int& j) {
  const int chunk = blockIdx.x / nz;
  k = blockIdx.x - chunk * nz;
  id = chunk * NODE_TILE + threadIdx.x;
  if (id >= L.NN) return false;
  node_ij(L, id, i, j);
  return true;
}

// Grid of a persistent kernel: the blocks of NODE_TILE threads the device
// keeps resident at once (never more than `dense`, the blocks of the dense
// launch it replaces).  Host code.
template <class K>
inline unsigned persistent_grid(K kernel, unsigned dense) {
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, NODE_TILE, 0) != cudaSuccess || per < 1)
    return dense;
  const unsigned g = (unsigned)sms * (unsigned)per;
  return g < dense ? g : dense;
}

// Work-list items: (chunk of NODE_TILE entries, layer) layer-fastest as in
// the dense launches; a persistent kernel strides w over [0, list_items) by the
// grid and takes entry (k, id, i, j) of item w where list_entry says so.
__device__ __forceinline__ int64_t list_items(int cnt, int nz) {
  return (int64_t)((cnt + NODE_TILE - 1) / NODE_TILE) * nz;
}
__device__ __forceinline__ bool list_entry(const LevelDev& L, int nz, const NodeList& W, int cnt, int64_t w, int& k,
                                           int& id, int& i, int& j) {
  const int chunk = (int)(w / nz);
  k = (int)(w - (int64_t)chunk * nz);
  const int e = chunk * NODE_TILE + threadIdx.x;
  if (e >= cnt) return false;
  id = __ldg(W.ids + e);
  node_ij(L, id, i, j);
  return true;
}

// Readers of the state through the ghost remap.
struct Rd {
  const int* __restrict__ nsrc;
  const int* __restrict__ esrc;
  bool direct;
  __device__ __forceinline__ Rd(const LevelDev& L, bool dir) : nsrc(L.nsrc), esrc(L.esrc), direct(dir) {}
  __device__ __forceinline__ double n(const double* __restrict__ f, int x) const {
    return f[direct ? x : __ldg(nsrc + x)];
  }
  // edge field with planes of NN: slot = e*NN + x
  __device__ __forceinline__ double e(const double* __restrict__ f, int slot) const {
    if (direct) return f[slot];
    const int c = __ldg(esrc + slot);
    const double v = f[c >> 1];
    return (c & 1) ? -v : v;
  }
};

__device__ __forceinline__ void weights5(const LevelDev& L, int id, int offs, double w[5]) {  // get_weights
  const int NN = L.NN;
  double acc = L.part[offs * NN + id];
  double hinv = L.hex_inv[id];
  double wgt[5];
  wgt[0] = acc;
#pragma unroll
  for (int q = 2; q <= 5; ++q) {
    acc = acc + L.part[((q + offs - 1) % 6) * NN + id];
    wgt[q - 1] = acc;
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) wgt[q] = 0.5 - wgt[q] * hinv;
  w[0] = wgt[0]; w[1] = -wgt[1]; w[2] = wgt[2]; w[3] = -wgt[3]; w[4] = wgt[4];
}

// Qperp (src/ops.f90:834-901): the TRiSK Coriolis term of the three edges of
// node id from the mass flux hm and qe of one layer (ghost edges of hm read
// through the remap).
__device__ __forceinline__ void qperp(const LevelDev& L, const Rd& R, const double* __restrict__ hm,
                                      const double* __restrict__ qe, int id, double Q[3]) {
  const int P = L.P, NN = L.NN;
  const int idNW = id + P - 1, idN = id + P, idNE = id + P + 1, idW = id - 1, idE = id + 1, idSW = id - P - 1,
            idS = id - P, idSE = id - P + 1;
#define TQ(e1, n1, q0, w) (R.e(hm, (e1) * NN + (n1)) * interp(qe[(e1) * NN + (n1)], (q0)) * (w))
  double w1[5], w2[5];
  double q0 = qe[RT * NN + id];
  weights5(L, id, 0, w1);
  weights5(L, idE, 3, w2);
  Q[0] = TQ(DG, id, q0, w1[0]) + TQ(UP, id, q0, w1[1]) + TQ(RT, idW, q0, w1[2]) + TQ(DG, idSW, q0, w1[3]) +
         TQ(UP, idS, q0, w1[4]) + TQ(DG, idS, q0, w2[0]) + TQ(UP, idSE, q0, w2[1]) + TQ(RT, idE, q0, w2[2]) +
         TQ(DG, idE, q0, w2[3]) + TQ(UP, idE, q0, w2[4]);
  q0 = qe[DG * NN + id];
  weights5(L, id, 1, w1);
  weights5(L, idNE, 4, w2);
  Q[1] = TQ(UP, id, q0, w1[0]) + TQ(RT, idW, q0, w1[1]) + TQ(DG, idSW, q0, w1[2]) + TQ(UP, idS, q0, w1[3]) +
         TQ(RT, id, q0, w1[4]) + TQ(UP, idE, q0, w2[0]) + TQ(RT, idNE, q0, w2[1]) + TQ(DG, idNE, q0, w2[2]) +
         TQ(UP, idNE, q0, w2[3]) + TQ(RT, idN, q0, w2[4]);
  q0 = qe[UP * NN + id];
  weights5(L, id, 2, w1);
  weights5(L, idN, 5, w2);
  Q[2] = TQ(RT, idW, q0, w1[0]) + TQ(DG, idSW, q0, w1[1]) + TQ(UP, idS, q0, w1[2]) + TQ(RT, id, q0, w1[3]) +
         TQ(DG, id, q0, w1[4]) + TQ(RT, idN, q0, w2[0]) + TQ(DG, idN, q0, w2[1]) + TQ(UP, idN, q0, w2[2]) +
         TQ(RT, idNW, q0, w2[3]) + TQ(DG, idW, q0, w2[4]);
#undef TQ
}

}  // namespace wtk
