// Inline readers shared by the layer kernels: interpolation, node indexing,
// the layer-fastest block mapping and reads of the state through the ghost
// remap tables.  Device functions only, so several translation units may
// include it.
#pragma once
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

__device__ __forceinline__ bool layer_node(const LevelDev& L, int nz, int& k, int& id, int& i, int& j) {
  const int chunk = blockIdx.x / nz;
  k = blockIdx.x - chunk * nz;
  id = chunk * NODE_TILE + threadIdx.x;
  if (id >= L.NN) return false;
  const int pp = L.P * L.P;
  const int r = id - (id / pp) * pp;
  const int jp = r / L.P;
  j = jp - 2;
  i = r - jp * L.P - 2;
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

}  // namespace wtk
