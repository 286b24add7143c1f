// Vertical remap of every level's layers (remap_vertical_coordinates,
// src/remap.f90:18-76) through the C-ABI.  The host decides when to remap
// (the reference does it when the smallest relative layer mass drops below
// min_mass_remap, src/main.f90:447-454) and which reconstruction to use.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/wavetrisk_gpu.h"
#include "remap_kernels.cuh"
#include "wt_handle.cuh"

int wt_handle_fail(const char* what, cudaError_t e);
int wt_level_mean(wt_handle* h, int level, int field, double** out);
void wt_level_state(wt_handle* h, int level, double** m, double** t, double** v);
void wt_level_masks(wt_handle* h, int level, const int** mask_n, const int** mask_e);

extern "C" {

int wt_remap_vertical(wt_handle* h, int remap_type, const double* a_vert, const double* b_vert) {
  if (!h || !a_vert || !b_vert) return WT_ERR_ARG;
  if (remap_type < WT_REMAP_0 || remap_type > WT_REMAP_2PPM) return WT_ERR_ARG;
  const int nz = h->nz;
  if (nz < 2 || nz > wtr::kRemapMaxNz) return WT_ERR_ARG;
  if (h->flux_bits != 64) return WT_ERR_STATE;
  cudaStream_t s = h->stream;
  const int l0 = h->wav ? h->level_start : h->level_end;
  int64_t maxnn = 0;
  for (int l = l0; l <= h->level_end; ++l) maxnn = std::max<int64_t>(maxnn, h->at(l).NN);
  double *ab = nullptr, *mold = nullptr;
  cudaError_t e = cudaMalloc(&ab, 16 * (size_t)(nz + 1));
  if (e == cudaSuccess) e = cudaMalloc(&mold, 8 * (size_t)nz * maxnn);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ab, a_vert, 8 * (size_t)(nz + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ab + nz + 1, b_vert, 8 * (size_t)(nz + 1), cudaMemcpyHostToDevice, s);
  int rc = WT_OK;
  for (int l = l0; l <= h->level_end && e == cudaSuccess && rc == WT_OK; ++l) {
    const DevLevel& D = h->at(l);
    double *m, *t, *v, *mm, *mt;
    if (l == h->level_end) {
      m = h->mass;
      t = h->temp;
      v = h->velo;
    } else {
      wt_level_state(h, l, &m, &t, &v);
    }
    if ((rc = wt_level_mean(h, l, WT_FIELD_MEAN_MASS, &mm))) break;
    if ((rc = wt_level_mean(h, l, WT_FIELD_MEAN_TEMP, &mt))) break;
    e = cudaMemcpyAsync(mold, m, 8 * (size_t)nz * D.NN, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) break;
    wtr::RemapLevel L{D.n, D.P, D.NN, D.nsrc, D.topo, mm, mt, mold, m, t, v};
    const int64_t cnt = (int64_t)10 * (D.n + 1) * (D.n + 1);
    wtr::k_remap_incompressible<<<(unsigned)((cnt + 127) / 128), 128, 0, s>>>(L, nz, remap_type, ab, ab + nz + 1,
                                                                               h->ph.ref_density);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(ab);
  cudaFree(mold);
  if (rc != WT_OK) return rc;
  if (e != cudaSuccess) return wt_handle_fail("remap", e);
  h->state_halo_done = false;
  return WT_OK;
}

int wt_min_mass(wt_handle* h, const double* b_vert, double* min_mass) {
  if (!h || !b_vert || !min_mass) return WT_ERR_ARG;
  const int nz = h->nz;
  if (nz < 1) return WT_ERR_ARG;
  if (h->flux_bits != 64) return WT_ERR_STATE;
  cudaStream_t s = h->stream;
  const int l0 = h->wav ? h->level_start : h->level_end;
  double* bv = nullptr;
  cudaError_t e = cudaMalloc(&bv, 8 * (size_t)(nz + 2));
  unsigned long long* key = reinterpret_cast<unsigned long long*>(bv + nz + 1);
  if (e == cudaSuccess) e = cudaMemcpyAsync(bv, b_vert, 8 * (size_t)(nz + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(key, 0xff, 8, s);
  int rc = WT_OK;
  for (int l = l0; l <= h->level_end && e == cudaSuccess && rc == WT_OK; ++l) {
    const DevLevel& D = h->at(l);
    double *m, *t, *v, *mm;
    if (l == h->level_end) {
      m = h->mass;
    } else {
      wt_level_state(h, l, &m, &t, &v);
    }
    if ((rc = wt_level_mean(h, l, WT_FIELD_MEAN_MASS, &mm))) break;
    const int *mask_n = nullptr, *mask_e = nullptr;
    if (h->wav) wt_level_masks(h, l, &mask_n, &mask_e);
    wtr::RemapLevel L{D.n, D.P, D.NN, D.nsrc, D.topo, mm, nullptr, nullptr, m, nullptr, nullptr};
    const int64_t cnt = (int64_t)10 * (D.n + 1) * (D.n + 1);
    wtr::k_min_mass<<<(unsigned)((cnt + 127) / 128), 128, 0, s>>>(L, nz, bv, h->ph.ref_density, mask_n, key);
    e = cudaGetLastError();
  }
  unsigned long long k = ~0ull;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&k, key, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(bv);
  if (rc != WT_OK) return rc;
  if (e != cudaSuccess) return wt_handle_fail("min_mass", e);
  if (k == ~0ull) {
    *min_mass = 1e16;  // no node counted: the reference's starting value
  } else {
    double x;
    std::memcpy(&x, &k, 8);
    *min_mass = x;
  }
  return WT_OK;
}

}  // extern "C"
