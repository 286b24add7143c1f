// C-ABI of the host grid builder.  A Fortran host that already owns its grid
// does not need this; it exists so that a C, C++ or Python host can produce the
// same per-level geometry and ghost tables that the reference computes in
// init_grid / precompute_geometry / refine_patch2 (src/init.f90,
// src/refine_patch.f90) and hand them to wt_create.
#include <cstdio>
#include <cstring>
#include <exception>

#include "grid.hpp"
#include "../../include/wavetrisk_gpu.h"

using namespace wtg;

extern "C" {

int wt_grid_build(int min_level, int max_level, int domain_level, double radius, double omega, wt_grid** out) {
  if (!out) return WT_ERR_ARG;
  *out = nullptr;
  try {
    Grid* g = new Grid();
    build_grid(*g, min_level, max_level, domain_level, radius, omega);
    *out = reinterpret_cast<wt_grid*>(g);
    return WT_OK;
  } catch (std::exception& e) {
    std::fprintf(stderr, "wt_grid_build: %s\n", e.what());
    return WT_ERR_ARG;
  }
}

void wt_grid_free(wt_grid* g) { delete reinterpret_cast<Grid*>(g); }

int wt_grid_level_dims(const wt_grid* gh, int level, wt_level_dims* dims) {
  const Grid* g = reinterpret_cast<const Grid*>(gh);
  if (!g || !dims || level < g->min_level - 1 || level > g->max_level) return WT_ERR_ARG;
  const Level& L = g->at(level);
  dims->n = L.n;
  dims->P = L.P;
  dims->NN = L.NN;
  dims->n_halo_node = (int64_t)L.halo_node.size();
  dims->n_halo_edge = (int64_t)L.halo_edge.size();
  return WT_OK;
}

// Copies one geometry table of a level into caller memory.  Names and sizes
// (doubles unless stated): "node" 3*NN (x plane, y plane, z plane),
// "len"/"pedlen" 3*NN, "part" 6*NN, "hex_inv" NN, "triarea"/"coriolis" 2*NN,
// "overl_a" 4*NN, "overl_split" 2*NN, "ccentre" 6*NN (xyz planes of LORT then
// UPLT), "halo_node" 2*n_halo_node int64, "halo_edge" 3*n_halo_edge int64;
// above the coarsest level also "iu_wgt" 9*NN, "rf_wgt" 3*NN and "rf_conflict"
// (1 double: the largest difference between two writers of one R_F_wgt slot).
int wt_grid_copy(const wt_grid* gh, int level, const char* name, void* dst) {
  const Grid* g = reinterpret_cast<const Grid*>(gh);
  if (!g || !name || !dst || level < g->min_level - 1 || level > g->max_level) return WT_ERR_ARG;
  const Level& L = g->at(level);
  double* d = static_cast<double*>(dst);
  auto cp = [&](const std::vector<double>& v) { std::memcpy(d, v.data(), v.size() * sizeof(double)); };
  if (!std::strcmp(name, "node")) {
    for (int64_t k = 0; k < L.NN; ++k) { d[k] = L.node[k].x; d[L.NN + k] = L.node[k].y; d[2 * L.NN + k] = L.node[k].z; }
  } else if (!std::strcmp(name, "ccentre")) {
    for (int t = 0; t < 2; ++t)
      for (int64_t k = 0; k < L.NN; ++k) {
        const Coord& c = L.ccentre[t * L.NN + k];
        d[(3 * t + 0) * L.NN + k] = c.x; d[(3 * t + 1) * L.NN + k] = c.y; d[(3 * t + 2) * L.NN + k] = c.z;
      }
  } else if (!std::strcmp(name, "len")) cp(L.len);
  else if (!std::strcmp(name, "pedlen")) cp(L.pedlen);
  else if (!std::strcmp(name, "part")) cp(L.part);
  else if (!std::strcmp(name, "hex_inv")) cp(L.hex_inv);
  else if (!std::strcmp(name, "triarea")) cp(L.triarea);
  else if (!std::strcmp(name, "coriolis")) cp(L.coriolis);
  else if (!std::strcmp(name, "overl_a")) cp(L.overl_a);
  else if (!std::strcmp(name, "overl_split")) cp(L.overl_split);
  else if (!std::strcmp(name, "iu_wgt")) {
    if (L.iu_wgt.empty()) return WT_ERR_ARG;
    cp(L.iu_wgt);
  } else if (!std::strcmp(name, "rf_wgt")) {
    if (L.rf_wgt.empty()) return WT_ERR_ARG;
    cp(L.rf_wgt);
  } else if (!std::strcmp(name, "rf_conflict")) {
    if (L.rf_wgt.empty()) return WT_ERR_ARG;
    d[0] = L.rf_conflict;
  }
  else if (!std::strcmp(name, "halo_node")) {
    int64_t* o = static_cast<int64_t*>(dst);
    for (size_t k = 0; k < L.halo_node.size(); ++k) { o[2 * k] = L.halo_node[k].dst; o[2 * k + 1] = L.halo_node[k].src; }
  } else if (!std::strcmp(name, "halo_edge")) {
    int64_t* o = static_cast<int64_t*>(dst);
    for (size_t k = 0; k < L.halo_edge.size(); ++k) {
      o[3 * k] = L.halo_edge[k].dst; o[3 * k + 1] = L.halo_edge[k].src; o[3 * k + 2] = L.halo_edge[k].sign;
    }
  } else {
    return WT_ERR_ARG;
  }
  return WT_OK;
}

}  // extern "C"
