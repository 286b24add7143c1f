// Host-side icosahedral grid builder for the padded lozenge layout.
//
// The reference builds its grid on the host (Fortran) in src/init.f90 (init_grid,
// init_coordinates, assign_coord, precompute_geometry), src/refine_patch.f90
// (refine_patch2: child coordinates from parent nodes and edge midpoints) and
// src/comm.f90 (create_comm / create_comm_e / pack_idx / create_comm_pole: the
// ghost-cell copy tables).  This file restates those procedures for a layout in
// which every one of the 10 icosahedral lozenges is one domain and every level
// of a lozenge is one padded (n+4)x(n+4) array (2-cell halo, BDRY_THICKNESS=2 in
// src/shared.f90:23).  It is set-up code, run once per grid on the host, exactly
// as the reference runs it once per refinement.
#pragma once
#include <cstdint>
#include <vector>

namespace wtg {

struct Coord { double x, y, z; };

// Element-type constants, same numbering as src/shared.f90:50-63,137-143.
enum { RT = 0, DG = 1, UP = 2 };
enum { LORT = 0, UPLT = 1 };
enum { NORTH = 1, EAST = 2, SOUTH = 3, WEST = 4, NORTHEAST = 5, SOUTHEAST = 6, SOUTHWEST = 7, NORTHWEST = 8 };
constexpr int HALO = 2;          // BDRY_THICKNESS
constexpr int N_LOZ = 10;        // N_ICOSAH_LOZENGE
constexpr int POLE = -2;
constexpr int NONE = -1;

struct HaloNode { int64_t dst, src; };
struct HaloEdge { int64_t dst, src; int sign; };   // dst/src are plane*NN + node

struct Level {
  int l = 0, n = 0, P = 0;
  int64_t NN = 0;                 // 10 * P * P nodes in the padded level
  std::vector<Coord> node;        // [NN]
  std::vector<Coord> ccentre;     // [2*NN]  plane t*NN + node
  std::vector<Coord> midpt;       // [3*NN]
  std::vector<double> len, pedlen;        // [3*NN]
  std::vector<double> part;               // [6*NN]  part k at k*NN + node
  std::vector<double> hex_inv;            // [NN]
  std::vector<double> triarea, coriolis;  // [2*NN]
  std::vector<double> overl_a;            // [4*NN]  Overl_Area%a
  std::vector<double> overl_split;        // [2*NN]  Overl_Area%split
  std::vector<double> iu_wgt;             // [9*NN]  I_u_wgt%enc (k at k*NN + node); levels > min_level-1
  std::vector<double> rf_wgt;             // [3*NN]  R_F_wgt%enc (c at c*NN + node); levels > min_level-1
  std::vector<uint8_t> rf_set;            // build scratch: slot already written
  double rf_conflict = 0.0;               // largest difference between two writers of one R_F_wgt slot
  std::vector<uint8_t> valid;             // [NN] 1 where node coordinates are defined
  std::vector<HaloNode> halo_node;
  std::vector<HaloEdge> halo_edge;

  inline int64_t id(int d, int i, int j) const {
    return ((int64_t)d * P + (j + HALO)) * P + (i + HALO);
  }
  inline bool in(int i, int j) const {
    return i >= -HALO && j >= -HALO && i < n + HALO && j < n + HALO;
  }
};

struct Grid {
  int min_level = 0, max_level = 0, domain_level = 0;
  double radius = 6371.22e3, omega = 7.292e-5;
  // Lozenge connectivity (src/init.f90:init_connections with one domain per lozenge).
  int neigh[N_LOZ][9];            // 1..8 used
  int neigh_rot[N_LOZ][9];
  int neigh_over_pole[N_LOZ][2];
  bool penta[N_LOZ][9];
  std::vector<Level> lev;         // index l - (min_level-1)
  Level& at(int l) { return lev[l - (min_level - 1)]; }
  const Level& at(int l) const { return lev[l - (min_level - 1)]; }
};

// Build levels min_level-1 .. max_level (uniform, every node present).
void build_grid(Grid& g, int min_level, int max_level, int domain_level, double radius, double omega);

}  // namespace wtg
