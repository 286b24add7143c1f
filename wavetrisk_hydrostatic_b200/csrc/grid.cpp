// Host-side icosahedral grid builder (see grid.hpp for the layout).
//
// Every floating-point expression below keeps the operand order of the
// reference's Fortran so that the geometry tables come out the same; the
// file is compiled with -ffp-contract=off (no FMA contraction).
#include "grid.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <cstdio>
#include <functional>
#include <stdexcept>

namespace wtg {
namespace {

const double MATH_PI = std::acos(-1.0);
double R = 6371.22e3;  // set per build (src/shared.f90:399 default)

inline Coord C(double x, double y, double z) { return Coord{x, y, z}; }
inline Coord operator+(Coord a, Coord b) { return C(a.x + b.x, a.y + b.y, a.z + b.z); }
inline double sq(double a) { return a * a; }
inline double eps() { return R * 1e-13; }                                    // src/shared.f90:444

// src/sphere.f90 (geom_mod) restated op-for-op.
inline double dist(Coord p, Coord q) {                                         // sphere.f90:14
  return R * std::asin(std::sqrt(sq(p.y * q.z - p.z * q.y) + sq(p.z * q.x - p.x * q.z) + sq(p.x * q.y - p.y * q.x)) /
                       (R * R));
}
inline Coord project_on_sphere(Coord p) {                                      // sphere.f90:86
  double nrm = std::sqrt(sq(p.x) + sq(p.y) + sq(p.z));
  return C(p.x * (R / nrm), p.y * (R / nrm), p.z * (R / nrm));
}
inline Coord mid_pt(Coord p, Coord q) { return project_on_sphere(C(p.x + q.x, p.y + q.y, p.z + q.z)); }  // :276
inline Coord vector(Coord a, Coord b) { return C(b.x - a.x, b.y - a.y, b.z - a.z); }
inline double inner(Coord u, Coord v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
inline Coord cross(Coord u, Coord v) { return C(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x); }
inline double norm(Coord c) { return std::sqrt(sq(c.x) + sq(c.y) + sq(c.z)); }
inline double distn(Coord p, Coord q) {                                        // sphere.f90:184
  double sindist = sq(1.0 / R) * std::sqrt(sq(p.y * q.z - p.z * q.y) + sq(p.z * q.x - p.x * q.z) + sq(p.x * q.y - p.y * q.x));
  if (sindist > 1.0) return std::asin(1.0);
  return std::asin(sindist);
}
inline double triarea(Coord A, Coord B, Coord Cc) {                            // sphere.f90:163
  double ab = distn(A, B), ac = distn(A, Cc), bc = distn(B, Cc);
  double s = (ab + ac + bc) / 2;
  double t = std::tan(0.5 * s) * std::tan((s - ab) / 2.0) * std::tan((s - ac) / 2.0) * std::tan((s - bc) / 2.0);
  if (t < 1e-64) return 0.0;
  return 4.0 * (R * R) * std::atan(std::sqrt(t));
}
inline Coord circumcentre(Coord A, Coord B, Coord Cc) {                        // sphere.f90:197
  Coord centre = cross(C(A.x - B.x, A.y - B.y, A.z - B.z), C(Cc.x - B.x, Cc.y - B.y, Cc.z - B.z));
  if (norm(centre) < eps()) return centre;
  return project_on_sphere(centre);
}
inline Coord sph2cart(double lon, double lat) {                                // sphere.f90:79
  return C(R * (std::cos(lon) * std::cos(lat)), R * (std::sin(lon) * std::cos(lat)), R * std::sin(lat));
}
// sphere.f90:98 arc_inters
void arc_inters(Coord a1, Coord a2, Coord b1, Coord b2, Coord& inters, bool& does) {
  inters = b2;
  does = true;
  if (norm(vector(a2, b2)) < eps()) return;
  Coord n1 = cross(a1, a2);
  double inpr = inner(n1, b1) * inner(n1, b2);
  if (inpr > 0.0) { does = false; return; }
  Coord n2 = cross(b1, b2);
  inpr = inner(n2, a1) * inner(n2, a2);
  if (inpr > 0.0) { does = false; return; }
  inters = project_on_sphere(cross(n1, n2));
  Coord neg = C(-inters.x, -inters.y, -inters.z);
  if (norm(vector(neg, a1)) < norm(vector(inters, a1))) inters = neg;
  does = true;
}

// ---------------------------------------------------------------------------
// Lozenge connectivity: src/init.f90:init_connections (:525-615) for
// N_SUB_DOM_PER_DIM = 1, i.e. one domain per lozenge.
void init_connections(Grid& g) {
  for (int d = 0; d < N_LOZ; ++d)
    for (int s = 0; s < 9; ++s) { g.neigh[d][s] = NONE; g.neigh_rot[d][s] = 0; g.penta[d][s] = false; }
  for (int ii = 1; ii <= 2; ++ii)
    for (int jj = 1; jj <= 5; ++jj) {
      int loz = 5 * ii - 5 + (jj - 1);
      auto mod = [](int a, int b) { return ((a % b) + b) % b; };
      g.neigh_over_pole[loz][0] = 5 * ii - 5 + mod(jj + 1, 5);
      g.neigh_over_pole[loz][1] = 5 * ii - 5 + mod(jj - 3, 5);
      if (ii == 2) g.neigh[loz][NORTHWEST] = POLE;
      if (ii == 1) g.neigh[loz][SOUTHEAST] = POLE;
      g.neigh[loz][NORTH] = 5 + mod(ii + jj - 2, 5); g.neigh_rot[loz][NORTH] = ii - 1;
      g.neigh[loz][EAST] = mod(jj, 5);               g.neigh_rot[loz][EAST] = 1 - (ii - 1);
      g.neigh[loz][SOUTH] = mod(ii + jj - 3, 5);     g.neigh_rot[loz][SOUTH] = 1 - (ii - 1);
      g.neigh[loz][WEST] = 5 + mod(jj - 2, 5);       g.neigh_rot[loz][WEST] = ii - 1;
      // set_penta (src/init.f90:245-250): all four lozenge corners are icosahedron vertices
      g.penta[loz][SOUTHWEST] = g.penta[loz][SOUTHEAST] = g.penta[loz][NORTHWEST] = g.penta[loz][NORTHEAST] = true;
    }
}

// ---------------------------------------------------------------------------
// Ghost-copy tables: src/comm.f90 create_comm_e (:103-345), pack_idx (:705-750),
// create_comm specials (:370-438), create_comm_pole (:440-530), for a domain that
// is a whole lozenge at level l (PATCH_SIZE -> n).  Entries are produced in the
// reference's unpack order (source domain outermost, then the destination's
// creation order) and later writes to the same ghost win, as in cp_bdry_inside.
struct RawEntry { int src_d, si, sj; int dst_d, di, dj; int is_edge; int se, de; int sign; int order; };

// local coordinates (i,j) of boundary patch s -> domain coordinates (idx(), src/domain.f90:757)
inline void bloc(int s, int i, int j, int n, int& di, int& dj) {
  switch (s) {
    case NORTH: di = i; dj = n + j; break;
    case EAST: di = n + i; dj = j; break;
    case SOUTH: di = i; dj = j - HALO; break;
    case WEST: di = i - HALO; dj = j; break;
    case NORTHEAST: di = n + i; dj = n + j; break;
    case SOUTHEAST: di = n + i; dj = j - HALO; break;
    case SOUTHWEST: di = i - HALO; dj = j - HALO; break;
    case NORTHWEST: di = i - HALO; dj = n + j; break;
    default: throw std::runtime_error("bad side");
  }
}

void pack_idx(int i, int j, int rot, int s, int shift, int n, int& ir, int& jr, int& ip, int& jp) {
  const int LAST = n - 1;
  if (s == NORTH) { ir = i + rot * (j + shift); jr = j + n; if (rot) { ip = j; jp = LAST - i; } else { ip = i; jp = j; } }
  if (s == EAST) { ir = i + n; jr = j + rot * (i + shift); if (rot) { ip = LAST - j; jp = i; } else { ip = i; jp = j; } }
  if (s == SOUTH) { ir = i - rot * (j + shift); jr = -1 - j; if (rot) { ip = LAST - j; jp = LAST - i; } else { ip = i; jp = LAST - j; } }
  if (s == WEST) { ir = -1 - i; jr = j - rot * (i + shift); if (rot) { ip = LAST - j; jp = LAST - i; } else { ip = LAST - i; jp = j; } }
}

// shift_arr(e+1, s) of src/comm.f90:19 (column s holds e = RT, DG, UP, NODE)
const int shift_arr[5][4] = {{0, 0, 0, 0}, {0, 1, 1, 1}, {1, 1, 0, 1}, {1, 0, 0, 0}, {0, 0, 1, 0}};
constexpr int NODE_E = 3;

void build_halo(const Grid& g, Level& L) {
  const int n = L.n, LAST = n - 1, LAST_BDRY = HALO - 1;
  std::vector<RawEntry> raw;
  int order = 0;
  auto add = [&](int dst_d, int src, int ip, int jp, int is_edge, int se, int di, int dj, int de, int sign) {
    // create_pack_st2 skips partners outside the source patch (src/comm.f90:70)
    raw.push_back(RawEntry{src, ip, jp, dst_d, di, dj, is_edge, se, de, sign, order++});
  };
  for (int d = 0; d < N_LOZ; ++d) {
    for (int s = 1; s <= 8; ++s) {
      if (!g.penta[d][s]) {
        // create_comm (non-pentagon sides)
        int typ = s;
        int src = g.neigh[d][typ];
        if (src == NONE) continue;
        int rot = g.neigh_rot[d][typ];
        int orient = rot ? -1 : 1;
        for (int e = 0; e <= NODE_E; ++e) {
          int shift = shift_arr[s][e];
          int e_pack = (e + rot * ((s % 2) + 1)) % 3;
          bool ns = (s == NORTH || s == SOUTH);
          for (int a = 0; a < HALO; ++a)
            for (int b = 0; b < n; ++b) {
              int i = ns ? b : a, j = ns ? a : b;
              int ir, jr, ip, jp;
              pack_idx(i, j, rot, s, shift, n, ir, jr, ip, jp);
              if (ip < 0 || jp < 0 || ip >= n || jp >= n) continue;
              if (e == NODE_E) add(d, src, ip, jp, 0, 0, ir, jr, 0, orient);
              else add(d, src, ip, jp, 1, e_pack, ir, jr, e, orient);
            }
        }
        int di, dj;
        if (rot == 1 && typ == WEST && g.penta[d][SOUTHWEST]) {
          bloc(SOUTHWEST, LAST_BDRY, LAST_BDRY, n, di, dj);
          add(d, src, LAST, LAST, 1, RT, di, dj, RT, 1);
        }
        if (rot == 1 && typ == SOUTH && g.penta[d][SOUTHWEST]) {
          bloc(SOUTHWEST, LAST_BDRY, LAST_BDRY, n, di, dj);
          add(d, src, LAST, LAST, 1, UP, di, dj, RT, -1);
        }
        if (rot == 0 && typ == EAST && g.penta[d][SOUTHEAST]) {
          bloc(SOUTHEAST, 0, LAST_BDRY, n, di, dj);
          add(d, src, 1, 0, 0, 0, di, dj, 0, 1);
        }
        if (rot == 0 && typ == NORTH && g.penta[d][NORTHWEST]) {
          bloc(NORTHWEST, LAST_BDRY, 0, n, di, dj);
          add(d, src, 0, 1, 0, 0, di, dj, 0, 1);
        }
        if (rot == 1 && typ == EAST && g.penta[d][NORTHEAST]) {
          bloc(NORTHEAST, 0, 1, n, di, dj); add(d, src, 0, 1, 0, 0, di, dj, 0, 1);
          bloc(NORTHEAST, 1, 0, n, di, dj); add(d, src, 1, 1, 0, 0, di, dj, 0, -1);
          bloc(NORTHEAST, 0, 1, n, di, dj); add(d, src, 0, 1, 1, RT, di, dj, RT, 1);
          bloc(NORTHEAST, 0, 0, n, di, dj); add(d, src, 0, 0, 1, DG, di, dj, RT, -1);
          bloc(NORTHEAST, 0, 0, n, di, dj); add(d, src, 0, 0, 1, UP, di, dj, UP, 1);
        }
        if (rot == 1 && typ == NORTH && g.penta[d][NORTHEAST]) {
          bloc(NORTHEAST, 1, 0, n, di, dj); add(d, src, 1, 0, 0, 0, di, dj, 0, 1);
          bloc(NORTHEAST, 0, 1, n, di, dj); add(d, src, 1, 1, 0, 0, di, dj, 0, -1);
          bloc(NORTHEAST, 0, 1, n, di, dj); add(d, src, 1, 0, 1, UP, di, dj, RT, -1);
          bloc(NORTHEAST, 0, 0, n, di, dj); add(d, src, 0, 0, 1, DG, di, dj, UP, -1);
          bloc(NORTHEAST, 0, 0, n, di, dj); add(d, src, 0, 0, 1, RT, di, dj, RT, 1);
        }
      } else {
        // create_comm_pole (src/comm.f90:440)
        int typ = s;
        if (g.neigh[d][typ] != POLE) continue;
        for (int i = 0; i <= 1; ++i) {
          int src = g.neigh_over_pole[d][i];
          bool se = (s == SOUTHEAST);
          int s_side = (s == NORTHWEST) ? NORTH : EAST;
          int a, b, di, dj;
          if (i == 0) {
            int ijn[2] = {0, 1};
            if (se) std::swap(ijn[0], ijn[1]);
            bloc(s_side, ijn[0], ijn[1], n, di, dj);
            add(d, src, 0, LAST, 1, DG, di, dj, 2 * s_side - 2, 1);
            int ijn2[2] = {LAST_BDRY, 1}, ijs[2] = {1, LAST};
            if (se) { std::swap(ijn2[0], ijn2[1]); std::swap(ijs[0], ijs[1]); }
            bloc(s, ijn2[0], ijn2[1], n, di, dj);
            add(d, src, ijs[0], ijs[1], 0, 0, di, dj, 0, -1);
          }
          if (i == 1) {
            int ijn[2] = {LAST_BDRY, 0}, ijs[2] = {0, LAST};
            if (se) { std::swap(ijn[0], ijn[1]); std::swap(ijs[0], ijs[1]); }
            bloc(s, ijn[0], ijn[1], n, di, dj);
            add(d, src, ijs[0], ijs[1], 0, 0, di, dj, 0, 1);
          }
          {
            int ijn[2] = {-i + 1, 1}, ijs[2] = {0, LAST};
            if (se) { std::swap(ijn[0], ijn[1]); std::swap(ijs[0], ijs[1]); }
            bloc(s_side, ijn[0], ijn[1], n, di, dj);
            add(d, src, ijs[0], ijs[1], 0, 0, di, dj, 0, (i ? -1 : 1));
            bloc(s_side, 0, 0, n, di, dj);
            add(d, src, ijs[0], ijs[1], 1, UP - 2 * s_side + 2, di, dj, DG + i * (-2 * s_side + 3), (i ? -1 : 1));
          }
          if (i == 0) continue;
          s_side = (s == NORTHWEST) ? WEST : SOUTH;
          {
            int ijn[2] = {LAST_BDRY - 1, LAST}, ijs[2] = {1, LAST};
            if (se) { std::swap(ijn[0], ijn[1]); std::swap(ijs[0], ijs[1]); }
            bloc(s_side, ijn[0], ijn[1], n, di, dj);
            add(d, src, ijs[0], ijs[1], 0, 0, di, dj, 0, 1);
            int ijn2[2] = {LAST, LAST_BDRY};
            if (s == NORTHWEST) std::swap(ijn2[0], ijn2[1]);
            bloc(s_side, ijn2[0], ijn2[1], n, di, dj);
            a = LAST * (-s_side + 4); b = LAST * (s_side - 3);
            add(d, src, a, b, 1, DG, di, dj, 2 * s_side - 6, 1);
          }
        }
      }
    }
  }
  // Reference unpack order: source domain outermost, then creation order (stable).
  std::vector<std::vector<RawEntry>> by_src(N_LOZ);
  for (auto& r : raw) by_src[r.src_d].push_back(r);
  L.halo_node.clear();
  L.halo_edge.clear();
  std::vector<int64_t> last_node(L.NN, -1), last_edge(3 * L.NN, -1);
  std::vector<HaloNode> nodes;
  std::vector<HaloEdge> edges;
  for (int sd = 0; sd < N_LOZ; ++sd)
    for (auto& r : by_src[sd]) {
      if (!L.in(r.di, r.dj)) throw std::runtime_error("halo destination outside padded array");
      int64_t src = L.id(r.src_d, r.si, r.sj), dst = L.id(r.dst_d, r.di, r.dj);
      if (!r.is_edge) {
        last_node[dst] = (int64_t)nodes.size();
        nodes.push_back(HaloNode{dst, src});
        // keep the orientation flag of the node entry for the overlap-area swap (set_areas)
        nodes.back().dst = r.sign < 0 ? -(dst + 1) : dst;  // temporarily encode sign
      } else {
        int64_t de = (int64_t)r.de * L.NN + dst, se = (int64_t)r.se * L.NN + src;
        last_edge[de] = (int64_t)edges.size();
        edges.push_back(HaloEdge{de, se, r.sign});
      }
    }
  // Keep only the last writer of every ghost (cp_bdry_inside overwrites in order).
  for (size_t k = 0; k < nodes.size(); ++k) {
    int64_t dst = nodes[k].dst < 0 ? -nodes[k].dst - 1 : nodes[k].dst;
    if (last_node[dst] == (int64_t)k) L.halo_node.push_back(nodes[k]);
  }
  for (size_t k = 0; k < edges.size(); ++k)
    if (last_edge[edges[k].dst] == (int64_t)k) L.halo_edge.push_back(edges[k]);
}

// ---------------------------------------------------------------------------
void alloc_level(Level& L, int l) {
  L.l = l;
  L.n = 1 << l;
  L.P = L.n + 2 * HALO;
  L.NN = (int64_t)N_LOZ * L.P * L.P;
  Coord O{0, 0, 0};
  L.node.assign(L.NN, O);
  L.ccentre.assign(2 * L.NN, O);
  L.midpt.assign(3 * L.NN, O);
  L.len.assign(3 * L.NN, 0.0);
  L.pedlen.assign(3 * L.NN, 0.0);
  L.part.assign(6 * L.NN, 0.0);
  L.hex_inv.assign(L.NN, 0.0);
  L.triarea.assign(2 * L.NN, 1.0);   // extend(dom%triarea, ..., 1d0) default (src/refine_patch.f90:187)
  L.coriolis.assign(2 * L.NN, 0.0);
  L.overl_a.assign(4 * L.NN, 0.0);
  L.overl_split.assign(2 * L.NN, 0.0);
  L.valid.assign(L.NN, 0);
}

// Coordinates of level min_level-1: src/init.f90 init_coordinates (:270-318) +
// assign_coord (:617-664), for every sub-domain of DOMAIN_LEVEL inside a lozenge.
void coords_root(Grid& g, Level& L) {
  const double lat[4] = {-MATH_PI / 2.0, -std::atan(1.0 / 2.0), std::atan(1.0 / 2.0), MATH_PI / 2.0};
  double lon[10];
  for (int k = 0; k < 10; ++k) lon[k] = (MATH_PI * double(k)) / 5.0;
  auto mod = [](int a, int b) { return ((a % b) + b) % b; };
  const int DL = g.domain_level;
  const int NSD = 1 << DL;
  const int PL = (g.min_level - 1) - DL;  // PATCH_LEVEL
  if (PL < 0) throw std::runtime_error("min_level must exceed domain_level");
  const int PS = 1 << PL;
  for (int ii = 1; ii <= 2; ++ii)
    for (int jj = 1; jj <= 5; ++jj) {
      int loz = 5 * ii - 5 + (jj - 1);
      auto unit = [&](Coord c) { return C(c.x / R, c.y / R, c.z / R); };
      Coord ne = unit(sph2cart(lon[mod(ii + 2 * jj - 2, 10)], lat[ii]));
      Coord se = unit(sph2cart(lon[ii + 2 * jj - 3], lat[ii - 1]));
      Coord sw = unit(sph2cart(lon[mod(ii + 2 * jj - 4, 10)], lat[ii]));
      Coord nw = unit(sph2cart(lon[ii + 2 * jj - 3], lat[ii + 1]));
      // yrotate by YANGLE = 0 is the identity up to signed zeros; it is kept for fidelity.
      auto yrot = [](Coord c) {
        return C(c.x * std::cos(0.0) - c.z * std::sin(0.0), c.y, c.x * std::sin(0.0) + c.z * std::cos(0.0));
      };
      Coord cnr[2][2] = {{yrot(sw), yrot(nw)}, {yrot(se), yrot(ne)}};  // cnr[i][j]
      std::function<Coord(int, int, int)> J0 = [&](int i, int j, int l) -> Coord {  // get_J0_coord
        if (l > 0) return mid_pt(J0(i / 2, j / 2, l - 1), J0((i + 1) / 2, (j + 1) / 2, l - 1));
        return cnr[i][j];
      };
      for (int sj = 1; sj <= NSD; ++sj)
        for (int si = 1; si <= NSD; ++si) {
          int oi = (si - 1) * PS, oj = (sj - 1) * PS;
          auto nd = [&](int i, int j) -> Coord& { return L.node[L.id(loz, oi + i, oj + j)]; };
          auto mark = [&](int i, int j) { L.valid[L.id(loz, oi + i, oj + j)] = 1; };
          nd(PS, PS) = project_on_sphere(J0(si, sj, DL));           mark(PS, PS);
          nd(PS, 0) = project_on_sphere(J0(si, sj - 1, DL));        mark(PS, 0);
          nd(0, 0) = project_on_sphere(J0(si - 1, sj - 1, DL));     mark(0, 0);
          nd(0, PS) = project_on_sphere(J0(si - 1, sj, DL));        mark(0, PS);
          for (int l = 1; l <= PL; ++l) {
            int pc = 1 << (PL - l + 1), pf = pc / 2;
            for (int j0 = 0; j0 < PS; j0 += pc) {
              for (int i0 = 0; i0 < PS; i0 += pc) {
                nd(i0 + pf, j0) = mid_pt(nd(i0, j0), nd(i0 + pc, j0));            mark(i0 + pf, j0);
                nd(i0, j0 + pf) = mid_pt(nd(i0, j0), nd(i0, j0 + pc));            mark(i0, j0 + pf);
                nd(i0 + pf, j0 + pf) = mid_pt(nd(i0 + pc, j0 + pc), nd(i0, j0));  mark(i0 + pf, j0 + pf);
              }
              nd(PS, j0 + pf) = mid_pt(nd(PS, j0), nd(PS, j0 + pc));              mark(PS, j0 + pf);
            }
            for (int i0 = 0; i0 < PS; i0 += pc) {
              nd(i0 + pf, PS) = mid_pt(nd(i0, PS), nd(i0 + pc, PS));              mark(i0 + pf, PS);
            }
          }
        }
    }
  // comm_nodes3(get_coord, set_coord) (src/main.f90:500): ghosts take the owners' coordinates
  for (auto& h : L.halo_node) {
    int64_t dst = h.dst < 0 ? -h.dst - 1 : h.dst;
    L.node[dst] = L.node[h.src];
    L.valid[dst] = 1;
  }
}

// Child coordinates from parent nodes and edge midpoints: src/refine_patch.f90:129-155
void coords_child(const Grid& g, const Level& Pa, Level& L) {
  for (int d = 0; d < N_LOZ; ++d) {
    for (int b = -1; b <= Pa.n; ++b)
      for (int a = -1; a <= Pa.n; ++a) {
        int64_t p = Pa.id(d, a, b);
        auto set = [&](int i, int j, Coord c) {
          if (!L.in(i, j)) return;
          L.node[L.id(d, i, j)] = c;
          L.valid[L.id(d, i, j)] = 1;
        };
        set(2 * a, 2 * b, Pa.node[p]);
        set(2 * a + 1, 2 * b, Pa.midpt[RT * Pa.NN + p]);
        set(2 * a + 1, 2 * b + 1, Pa.midpt[DG * Pa.NN + p]);
        set(2 * a, 2 * b + 1, Pa.midpt[UP * Pa.NN + p]);
      }
    const int n = L.n, np = Pa.n;
    if (g.penta[d][SOUTHEAST])
      L.node[L.id(d, n, -1)] = mid_pt(Pa.node[Pa.id(d, np + 1, 0)], Pa.node[Pa.id(d, np, 0)]);
    if (g.penta[d][NORTHWEST])
      L.node[L.id(d, -1, n)] = mid_pt(Pa.node[Pa.id(d, 0, np + 1)], Pa.node[Pa.id(d, 0, np)]);
  }
}

// Reads outside the padded array return ORIGIN (the reference reads a
// neighbouring storage element there; those values are never used downstream).
struct Acc {
  Level& L; int d;
  Coord node(int i, int j) const { return L.in(i, j) ? L.node[L.id(d, i, j)] : Coord{0, 0, 0}; }
  Coord cc(int i, int j, int t) const { return L.in(i, j) ? L.ccentre[t * L.NN + L.id(d, i, j)] : Coord{0, 0, 0}; }
  Coord mp(int i, int j, int e) const { return L.in(i, j) ? L.midpt[e * L.NN + L.id(d, i, j)] : Coord{0, 0, 0}; }
  double part(int i, int j, int k) const { return L.in(i, j) ? L.part[(k - 1) * L.NN + L.id(d, i, j)] : 0.0; }
};

void geometry(Grid& g, Level& L) {
  const int n = L.n;
  for (int d = 0; d < N_LOZ; ++d) {
    Acc A{L, d};
    auto ID = [&](int i, int j) { return L.id(d, i, j); };
    // ccentre over [-BDRY, n+BDRY-1]  (src/init.f90:684 ccentre)
    for (int j = -2; j <= n + 1; ++j)
      for (int i = -2; i <= n + 1; ++i) {
        L.ccentre[LORT * L.NN + ID(i, j)] = circumcentre(A.node(i, j), A.node(i + 1, j + 1), A.node(i + 1, j));
        L.ccentre[UPLT * L.NN + ID(i, j)] = circumcentre(A.node(i, j), A.node(i, j + 1), A.node(i + 1, j + 1));
      }
    // ccentre_penta (src/init.f90:320-377)
    if (g.penta[d][SOUTHWEST]) {
      Coord c = circumcentre(A.node(0, 0), A.node(0, -1), A.node(-1, 0));
      L.ccentre[LORT * L.NN + ID(-1, -1)] = c;
      L.ccentre[UPLT * L.NN + ID(-1, -1)] = c;
      Coord pt3 = mid_pt(A.node(0, -2), A.node(-2, 0));
      L.ccentre[LORT * L.NN + ID(-1, -2)] = circumcentre(A.node(0, -1), A.node(0, -2), pt3);
      L.ccentre[UPLT * L.NN + ID(-2, -1)] = circumcentre(pt3, A.node(-2, 0), A.node(-1, 0));
    }
    if (g.penta[d][SOUTHEAST]) {
      int i = n, j = -1;
      Coord c = circumcentre(A.node(i - 1, j), A.node(i, j + 1), A.node(i + 1, j + 1));
      L.ccentre[LORT * L.NN + ID(i - 1, j)] = c;
      L.ccentre[UPLT * L.NN + ID(i, j)] = c;
    }
    if (g.penta[d][NORTHWEST]) {
      int i = -1, j = n;
      Coord c = circumcentre(A.node(i, j - 1), A.node(i + 1, j + 1), A.node(i + 1, j));
      L.ccentre[UPLT * L.NN + ID(i, j - 1)] = c;
      L.ccentre[LORT * L.NN + ID(i, j)] = c;
    }
    if (g.penta[d][NORTHEAST]) {
      int i = n, j = n;
      Coord c = circumcentre(A.node(i, j), A.node(i, j + 1), A.node(i + 1, j));
      L.ccentre[LORT * L.NN + ID(i, j)] = c;
      L.ccentre[UPLT * L.NN + ID(i, j)] = c;
    }
    // midpt over [-(BDRY-1), n+BDRY-1]  (src/init.f90:826-870)
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        int64_t id = ID(i, j);
        Coord* M = &L.midpt[0];
        if (j >= n + 1) { M[RT * L.NN + id] = mid_pt(A.node(i, j), A.node(i + 1, j)); continue; }
        if (i >= n + 1) { M[UP * L.NN + id] = mid_pt(A.node(i, j), A.node(i, j + 1)); continue; }
        if (j == -1) {
          if (i == -1 && g.penta[d][SOUTHWEST]) { M[DG * L.NN + id] = A.cc(i, j, LORT); continue; }
          if (i == n && g.penta[d][SOUTHEAST]) { M[UP * L.NN + id] = A.cc(i, j, UPLT); continue; }
        } else if (j == n && g.penta[d][NORTHWEST] && i == -1) {
          M[RT * L.NN + id] = A.cc(i, j, LORT);
          continue;
        }
        M[RT * L.NN + id] = mid_pt(A.node(i, j), A.node(i + 1, j));
        M[DG * L.NN + id] = mid_pt(A.node(i + 1, j + 1), A.node(i, j));
        M[UP * L.NN + id] = mid_pt(A.node(i, j), A.node(i, j + 1));
        if (j == n && i == n && g.penta[d][NORTHEAST]) M[DG * L.NN + id] = A.cc(i, j, LORT);
      }
    // lengths (src/init.f90:379-414)
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        int64_t id = ID(i, j);
        if (j >= n + 1) { L.len[RT * L.NN + id] = dist(A.node(i, j), A.node(i + 1, j)); continue; }
        if (i >= n + 1) { L.len[UP * L.NN + id] = dist(A.node(i, j), A.node(i, j + 1)); continue; }
        L.len[RT * L.NN + id] = dist(A.node(i, j), A.node(i + 1, j));
        L.len[DG * L.NN + id] = dist(A.node(i + 1, j + 1), A.node(i, j));
        L.len[UP * L.NN + id] = dist(A.node(i, j), A.node(i, j + 1));
        L.pedlen[RT * L.NN + id] = dist(A.cc(i, j - 1, UPLT), A.cc(i, j, LORT));
        L.pedlen[DG * L.NN + id] = dist(A.cc(i, j, UPLT), A.cc(i, j, LORT));
        L.pedlen[UP * L.NN + id] = dist(A.cc(i, j, UPLT), A.cc(i - 1, j, LORT));
        if (i == -1 && j == -1 && g.penta[d][SOUTHWEST]) {
          L.pedlen[DG * L.NN + id] = 0;
          L.len[RT * L.NN + id] = dist(A.node(i + 1, j), A.node(i, j + 1));
        }
        if (i == n && j == n && g.penta[d][NORTHEAST]) L.len[DG * L.NN + id] = dist(A.node(i + 1, j), A.node(i, j + 1));
      }
    // cpt_areas (src/init.f90:666-700; init_Areas in src/sphere.f90:296)
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        Coord c = A.node(i, j);
        Coord corners[6] = {A.cc(i, j, LORT), A.cc(i, j, UPLT), A.cc(i - 1, j, LORT),
                            A.cc(i - 1, j - 1, UPLT), A.cc(i - 1, j - 1, LORT), A.cc(i, j - 1, UPLT)};
        Coord mids[6] = {A.mp(i, j, RT), A.mp(i, j, DG), A.mp(i, j, UP),
                         A.mp(i - 1, j, RT), A.mp(i - 1, j - 1, DG), A.mp(i, j - 1, UP)};
        double part[6];
        for (int k = 0; k < 6; ++k) part[k] = triarea(c, corners[k], mids[k]) + triarea(c, corners[k], mids[(k + 1) % 6]);
        double sum = 0.0;
        for (int k = 0; k < 6; ++k) sum += part[k];
        double hex_inv = 1.0;
        if (sum != 0.0) hex_inv = 1.0 / sum;
        int64_t id = ID(i, j);
        int k0 = 0, k1 = 6;
        bool full = true;
        if (j >= n + 1) { k0 = 3; k1 = 6; full = false; }
        else if (i >= n + 1) { k0 = 2; k1 = 5; full = false; }
        for (int k = k0; k < k1; ++k) L.part[k * L.NN + id] = part[k];
        if (full) L.hex_inv[id] = hex_inv;
      }
    // cpt_triarea and coriolis (src/init.f90:760-824)
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        int64_t id = ID(i, j);
        double lort = A.part(i, j, 1) + A.part(i + 1, j, 3) + A.part(i + 1, j + 1, 5);
        double uplt = A.part(i, j, 2) + A.part(i + 1, j + 1, 4) + A.part(i, j + 1, 6);
        L.triarea[LORT * L.NN + id] = lort;
        L.triarea[UPLT * L.NN + id] = uplt;
        L.coriolis[LORT * L.NN + id] = L.ccentre[LORT * L.NN + id].z / R * 2.0 * g.omega * lort;
        L.coriolis[UPLT * L.NN + id] = L.ccentre[UPLT * L.NN + id].z / R * 2.0 * g.omega * uplt;
      }
  }
}

// Overlap areas of child nodes: set_RF_wgts + get_overl_areas (src/wavelet.f90:1512-1566,1408-1475)
const int no_adj_tri[10][3] = {{0, 0, LORT}, {0, -1, UPLT}, {-1, -1, LORT}, {-1, -1, UPLT}, {-1, 0, LORT},
                               {0, 0, UPLT}, {0, 0, LORT}, {0, -1, UPLT}, {-1, -1, LORT}, {-1, -1, UPLT}};
const int hex_s_offs[3] = {2, 0, 4};
const int bfly_tri[3][4][3] = {  // [e][k][:]
    {{-1, -1, LORT}, {0, -1, LORT}, {1, 0, UPLT}, {0, 0, UPLT}},
    {{0, 1, LORT}, {-1, 0, LORT}, {0, -1, UPLT}, {1, 0, UPLT}},
    {{0, 0, LORT}, {0, 1, LORT}, {-1, 0, UPLT}, {-1, -1, UPLT}}};
const int adj_tri[3][2][3] = {{{0, -1, UPLT}, {0, 0, LORT}}, {{0, 0, UPLT}, {0, 0, LORT}}, {{0, 0, UPLT}, {-1, 0, LORT}}};

enum { INSIDE = 0, OUTER1 = 1, OUTER2 = 2 };  // src/shared.f90:65-67

// typ[0..1] is the reference's typ(1:2): how the two coarse dual edges cross the child hexagon.
void get_overl_areas(Level& Pa, Level& L, int d, int ip, int jp, int ic, int jc, int e, double area[8], int typ[2]) {
  Acc P{Pa, d}, Cc{L, d};
  for (int k = 0; k < 8; ++k) area[k] = 0.0;
  typ[0] = typ[1] = 0;
  Coord hex[6];
  for (int i = 0; i < 6; ++i) {
    const int* t = no_adj_tri[i + hex_s_offs[-e + 2]];
    hex[i] = Cc.cc(ic + t[0], jc + t[1], t[2]);
  }
  auto ptri = [&](const int* t) { return P.cc(ip + t[0], jp + t[1], t[2]); };
  Coord tri[3][2];
  tri[0][0] = ptri(bfly_tri[e][3]); tri[1][0] = ptri(adj_tri[e][1]); tri[2][0] = ptri(bfly_tri[e][2]);
  tri[0][1] = ptri(bfly_tri[e][1]); tri[1][1] = ptri(adj_tri[e][0]); tri[2][1] = ptri(bfly_tri[e][0]);
  Coord pt = Cc.node(ic, jc);
  // Fortran 1-based area(1..8) -> area[0..7]; hex(1..6) -> hex[0..5]
  area[0] = triarea(hex[5], hex[0], pt);
  area[1] = triarea(hex[2], hex[3], pt);
  for (int i = 1; i <= 2; ++i) {
    Coord ip0, ip1;
    bool d0, d1;
    arc_inters(tri[0][i - 1], tri[1][i - 1], hex[3 * i - 3], hex[3 * i - 2], ip0, d0);
    arc_inters(tri[2][i - 1], tri[1][i - 1], hex[3 * i - 1], hex[3 * i - 2], ip1, d1);
    if (d0 && d1) {
      area[i + 3] = triarea(ip0, tri[1][i - 1], hex[3 * i - 2]);
      area[i + 5] = triarea(tri[1][i - 1], hex[3 * i - 2], ip1);
      area[i + 1] = area[i + 3] + area[i + 5];
      area[i - 1] = area[i - 1] + triarea(hex[3 * i - 3], ip0, pt) + triarea(ip0, pt, tri[1][i - 1]);
      area[-i + 2] = area[-i + 2] + triarea(ip1, hex[3 * i - 1], pt) + triarea(tri[1][i - 1], pt, ip1);
      typ[-i + 2] = INSIDE;
    } else if (!d0 && !d1) {
      area[i + 1] = 0.0;
      arc_inters(tri[1][0], tri[1][1], hex[3 * i - 3], hex[3 * i - 2], ip0, d0);
      arc_inters(tri[1][1], tri[1][0], hex[3 * i - 2], hex[3 * i - 1], ip1, d1);
      if (!d0 && d1) {
        area[i - 1] = area[i - 1] + triarea(hex[3 * i - 3], hex[3 * i - 2], pt) + triarea(hex[3 * i - 2], ip1, pt);
        area[-i + 2] = area[-i + 2] + triarea(ip1, hex[3 * i - 1], pt);
        typ[-i + 2] = OUTER2;
      } else if (d0 && !d1) {
        area[i - 1] = area[i - 1] + triarea(hex[3 * i - 3], ip0, pt);
        area[-i + 2] = area[-i + 2] + triarea(hex[3 * i - 2], hex[3 * i - 1], pt) + triarea(ip0, hex[3 * i - 2], pt);
        typ[-i + 2] = OUTER1;
      } else {
        std::fprintf(stderr, "wtg: overlap area case A at d=%d (%d,%d)\n", d, ic, jc);
      }
    } else {
      std::fprintf(stderr, "wtg: overlap area case B at d=%d (%d,%d)\n", d, ic, jc);
    }
  }
}

void overlap_areas(Level& Pa, Level& L) {
  for (int d = 0; d < N_LOZ; ++d)
    for (int jp = 0; jp < Pa.n; ++jp)
      for (int ip = 0; ip < Pa.n; ++ip) {
        int ic = 2 * ip, jc = 2 * jp;
        const int ce[3][2] = {{ic + 1, jc}, {ic + 1, jc + 1}, {ic, jc + 1}};
        for (int e = 0; e < 3; ++e) {
          double area[8];
          int typ[2];
          get_overl_areas(Pa, L, d, ip, jp, ce[e][0], ce[e][1], e, area, typ);
          int64_t id = L.id(d, ce[e][0], ce[e][1]);
          for (int k = 0; k < 4; ++k) L.overl_a[k * L.NN + id] = area[k];
          L.overl_split[id] = area[4];
          L.overl_split[L.NN + id] = area[5];
        }
      }
}

// ---- outer velocity interpolation weights I_u_wgt -------------------------
// set_WT_wgts / outer_velo_weights (src/wavelet.f90:1567-1705) with the
// helpers local_coord (:1500), coords_to_rowd (:1769), coord2local (:1749),
// normalize2 (:1477), normalize_Coord and direction (src/sphere.f90:7,256).

inline Coord normalize_coord(Coord c) {
  const double nrm = std::sqrt(sq(c.x) + sq(c.y) + sq(c.z));
  if (nrm >= eps()) return C(c.x / nrm, c.y / nrm, c.z / nrm);
  return C(0.0, 0.0, 0.0);
}
inline Coord direction(Coord a, Coord b) { return normalize_coord(vector(a, b)); }

struct Row6 { double v[6]; };
inline Row6 operator-(const Row6& a, const Row6& b) {
  Row6 r;
  for (int k = 0; k < 6; ++k) r.v[k] = a.v[k] - b.v[k];
  return r;
}

inline Row6 coords_to_rowd(Coord midpt, Coord dirvec, Coord x, Coord y) {
  const double q0 = inner(dirvec, x), q1 = inner(dirvec, y);
  const double nrm = std::sqrt(sq(q0) + sq(q1));
  const double u = q0 / nrm, v = q1 / nrm;
  const double x0 = inner(midpt, x), x1 = inner(midpt, y);
  return Row6{{u, u * x0, u * x1, v, v * x0, v * x1}};
}

// Vendored DGESV path for a 6x6 system (src/dgesv.f90: DGETRF -> DGETF2 since
// ILAENV's block size exceeds 6, then DGETRS), with the reference BLAS loops of
// IDAMAX, DSWAP, DSCAL, DGER and DTRSM.  a is column-major: a[c*6 + r].  On a
// singular factor b is left as DGESV leaves it (unsolved).
bool dgesv6(double a[36], double b[6]) {
  auto A = [&](int r, int c) -> double& { return a[c * 6 + r]; };
  const double sfmin = std::numeric_limits<double>::min();  // DLAMCH('S')
  int ipiv[6];
  int info = 0;
  for (int j = 0; j < 6; ++j) {
    int jp = j;
    double dmax = std::fabs(A(j, j));
    for (int i = j + 1; i < 6; ++i)
      if (std::fabs(A(i, j)) > dmax) { dmax = std::fabs(A(i, j)); jp = i; }
    ipiv[j] = jp;
    if (A(jp, j) != 0.0) {
      if (jp != j)
        for (int c = 0; c < 6; ++c) std::swap(A(j, c), A(jp, c));
      if (j < 5) {
        if (std::fabs(A(j, j)) >= sfmin) {
          const double r = 1.0 / A(j, j);
          for (int i = j + 1; i < 6; ++i) A(i, j) = r * A(i, j);
        } else {
          for (int i = j + 1; i < 6; ++i) A(i, j) = A(i, j) / A(j, j);
        }
      }
    } else if (info == 0) {
      info = j + 1;
    }
    if (j < 5)
      for (int c = j + 1; c < 6; ++c)
        if (A(j, c) != 0.0) {
          const double temp = -1.0 * A(j, c);
          for (int i = j + 1; i < 6; ++i) A(i, c) = A(i, c) + A(i, j) * temp;
        }
  }
  if (info != 0) return false;
  for (int i = 0; i < 6; ++i)
    if (ipiv[i] != i) std::swap(b[i], b[ipiv[i]]);
  for (int k = 0; k < 6; ++k)
    if (b[k] != 0.0)
      for (int i = k + 1; i < 6; ++i) b[i] = b[i] - b[k] * A(i, k);
  for (int k = 5; k >= 0; --k)
    if (b[k] != 0.0) {
      b[k] = b[k] / A(k, k);
      for (int i = 0; i < k; ++i) b[i] = b[i] - b[k] * A(i, k);
    }
  return true;
}

// Stencil tables of src/shared.f90:287-324 (0-based edge index, k = 0, 1).
const int END_PT[3][2][2] = {{{0, 0}, {1, 0}}, {{1, 1}, {0, 0}}, {{0, 0}, {0, 1}}};
const int OPP_NO[3][2][2] = {{{0, -1}, {1, 1}}, {{0, 1}, {1, 0}}, {{1, 1}, {-1, 0}}};
const int HEX_SIDES[10][3] = {{0, 0, RT},  {0, 0, DG},   {0, 0, UP}, {-1, 0, RT}, {-1, -1, DG},
                              {0, -1, UP}, {0, 0, RT},   {0, 0, DG}, {0, 0, UP},  {-1, 0, RT}};
const int HEX_S_OFFS[3] = {2, 0, 4};
const double IU_BASE[9] = {16.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0, -1.0 / 16.0,
                           -1.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0};

struct OuterWeights {
  const Grid& g;
  const Level& Pa;
  int d;
  Coord x, y;
  int bad = 0;  // reads of undefined node coordinates

  Coord node(int i, int j) {
    if (!Pa.in(i, j) || !Pa.valid[Pa.id(d, i, j)]) { ++bad; return C(0.0, 0.0, 0.0); }
    return Pa.node[Pa.id(d, i, j)];
  }
  // get_coord: the pentagon corners take the node the reference's boundary
  // patches hold there (nidx of IMINUS/JMINUS/JPLUS/IPLUS/IJPLUS).
  Coord get_coord(int i, int j, int e) {
    const int n = Pa.n;
    if (i == -1) {
      if (j == -1 && g.penta[d][SOUTHWEST]) {
        if (e == RT) return node(-1, 0);
        if (e == UP) return node(0, -1);
        ++bad;  // the reference returns an undefined value here; never reached
        return C(0.0, 0.0, 0.0);
      }
      if (j == n && g.penta[d][NORTHWEST]) return node(0, n + 1);
      return node(i, j);
    }
    if (i == n && j == -1 && g.penta[d][SOUTHEAST]) return node(n + 1, 0);
    if (i == n + 1 && j == n + 1 && g.penta[d][NORTHEAST]) return node(n + 1, n);
    return node(i, j);
  }
  Row6 row(int i0, int j0, const int* off1, const int* off2, int e00) {
    const int i = i0 + off1[0] + off2[0], j = j0 + off1[1] + off2[1], e = off2[2];
    const Coord p1 = get_coord(i + END_PT[e][0][0], j + END_PT[e][0][1], e00);
    const Coord p2 = get_coord(i + END_PT[e][1][0], j + END_PT[e][1][1], e00);
    return coords_to_rowd(mid_pt(p1, p2), vector(p1, p2), x, y);
  }
  // outer_velo_weights(dom, p, i0, j0, e0): 9 entries of I_u_wgt%enc.
  void compute(int i0, int j0, int e0, double out[9]) {
    const int n = Pa.n;
    (void)n;
    const Coord mid = Pa.midpt[(int64_t)e0 * Pa.NN + Pa.id(d, i0, j0)];
    const Coord e1 = Pa.node[Pa.id(d, i0 + END_PT[e0][0][0], j0 + END_PT[e0][0][1])];
    const Coord e2 = Pa.node[Pa.id(d, i0 + END_PT[e0][1][0], j0 + END_PT[e0][1][1])];
    x = direction(e1, e2);
    y = normalize_coord(cross(x, mid));
    double w[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int hs = HEX_S_OFFS[e0];
    const int zero2[2] = {0, 0};
    const int self3[3] = {0, 0, e0};
    for (int k = 1; k <= 2; ++k) {
      const int* ep_k = END_PT[e0][k - 1];
      const int* ep_o = END_PT[e0][2 - k];  // end_pt(:, -k+3)
      const int* op_k = OPP_NO[e0][k - 1];
      const int s = 3 * k - 3;
      Row6 G[6];
      G[0] = row(i0, j0, zero2, self3, e0);
      G[1] = row(i0, j0, ep_o, HEX_SIDES[hs + 2 + s], e0);
      G[2] = row(i0, j0, ep_k, HEX_SIDES[(hs + 3) - s], e0);
      G[3] = row(i0, j0, op_k, HEX_SIDES[hs + 1 + s], e0) - row(i0, j0, ep_k, HEX_SIDES[hs + 2 + s], e0);
      G[4] = row(i0, j0, ep_o, HEX_SIDES[(hs + 3) - s], e0) - row(i0, j0, op_k, HEX_SIDES[(hs + 4) - s], e0);
      G[5] = row(i0, j0, ep_k, HEX_SIDES[(hs + 5) - s], e0) - row(i0, j0, ep_o, HEX_SIDES[hs + 0 + s], e0);
      double a[36];
      for (int c = 0; c < 6; ++c)
        for (int r = 0; r < 6; ++r) a[c * 6 + r] = G[c].v[r];
      const Coord n1 = Pa.node[Pa.id(d, i0 + END_PT[e0][0][0], j0 + END_PT[e0][0][1])];
      const Coord n2 = Pa.node[Pa.id(d, i0 + END_PT[e0][1][0], j0 + END_PT[e0][1][1])];
      Row6 bb = coords_to_rowd(mid_pt(mid, n2), vector(n1, n2), x, y);
      double b[6];
      for (int r = 0; r < 6; ++r) b[r] = bb.v[r];
      dgesv6(a, b);
      w[0] = w[0] + b[0];
      w[2 * k - 1] = w[2 * k - 1] + b[1];
      w[2 * k] = w[2 * k] + b[2];
      w[2 * k + 3] = b[3];
      w[2 * k + 4] = b[4];
      w[-2 * k + 5] = w[-2 * k + 5] + b[5];
      w[-2 * k + 6] = w[-2 * k + 6] - b[5];
    }
    for (int q = 0; q < 9; ++q) out[q] = 0.5 * w[q] - IU_BASE[q];
  }
};

// set_WT_wgts over the parents [0, n_par)^2 of every lozenge
// (apply_interscale_to_patch3(..., 0, 0) in refine_patch2): RT weights at the
// child (2i+1, 2j), DG at (2i, 2j), UP at (2i, 2j+1).  Other nodes, ghosts
// included, keep zero weights, as in the reference's extend(I_u_wgt, 0).
void velo_weights(const Grid& g, const Level& Pa, Level& L) {
  L.iu_wgt.assign((size_t)9 * L.NN, 0.0);
  int bad = 0;
  for (int d = 0; d < N_LOZ; ++d) {
    OuterWeights W{g, Pa, d, C(0, 0, 0), C(0, 0, 0)};
    for (int jp = 0; jp < Pa.n; ++jp)
      for (int ip = 0; ip < Pa.n; ++ip) {
        const int tgt[3][2] = {{2 * ip + 1, 2 * jp}, {2 * ip, 2 * jp}, {2 * ip, 2 * jp + 1}};
        for (int e = 0; e < 3; ++e) {
          double w[9];
          W.compute(ip, jp, e, w);
          const int64_t id = L.id(d, tgt[e][0], tgt[e][1]);
          for (int q = 0; q < 9; ++q) L.iu_wgt[(int64_t)q * L.NN + id] = w[q];
        }
      }
    bad += W.bad;
  }
  if (bad) std::fprintf(stderr, "wtg: %d undefined node reads in velocity weights (level %d)\n", bad, L.l);
}

// ---- flux-restriction weights R_F_wgt ----------------------------------------
// set_RF_wgts / basic_F_restr_wgt (src/wavelet.f90:1512-1540, 1176-1360) with
// get_indices' stencil naming (src/shared.f90:84-112) and nghb_pt (:285).
// R_F_wgt lives on the child level (3 components, component c at c*NN + node)
// and is not ghost-copied.  Two parents write some slots (RT k=1 of (i,j) and
// UP k=1 of (i+1,j) describe the same coarse LORT triangle; UP k=0 of (i,j)
// and RT k=0 of (i,j+1) the same UPLT triangle); the last write wins, in the
// order lozenge, j, i, then RT before UP, i.e. the reference's loop order for a
// patch covering the whole lozenge.
enum { S_UZM = 0, S_UPZ, S_UMZ, S_UZP, S_VMM, S_VPM, S_VMP, S_VPP, S_WMM, S_WPM, S_WMP, S_WPP, S_WMMM, S_WPPP,
       S_VMPP, S_VPMM };
const int NGHB_PT[10][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 0}, {-1, -1}, {0, -1}, {1, 0}, {1, 1}, {0, 1}, {-1, 0}};

struct RFWeights {
  const Level& Pa;
  Level& L;
  int d;
  Coord x, y;
  int bad = 0;  // reads outside the padded child level
  double conflict = 0.0;  // largest change of a slot by a second writer

  Coord node(int i, int j) {
    if (!L.in(i, j)) { ++bad; return C(0.0, 0.0, 0.0); }
    return L.node[L.id(d, i, j)];
  }
  Coord cc(int i, int j, const int* t) {
    const int ii = i + t[0], jj = j + t[1];
    if (!L.in(ii, jj)) { ++bad; return C(0.0, 0.0, 0.0); }
    return L.ccentre[(int64_t)t[2] * L.NN + L.id(d, ii, jj)];
  }
  // coords_to_row (:1336-1359): row of the flux at edge ije, scaled by its dual length.
  Row6 row(const int* ije) {
    const int i = ije[0], j = ije[1], e = ije[2];
    const Coord p1 = node(i + END_PT[e][0][0], j + END_PT[e][0][1]);
    const Coord p2 = node(i + END_PT[e][1][0], j + END_PT[e][1][1]);
    const double ped = dist(cc(i, j, adj_tri[e][0]), cc(i, j, adj_tri[e][1]));
    Row6 r = coords_to_rowd(mid_pt(p1, p2), vector(p1, p2), x, y);
    for (int q = 0; q < 6; ++q) r.v[q] = r.v[q] * ped;
    return r;
  }
  // interp_F_wgts (:1288-1321)
  void interp(int k1, const int* lcsd, Coord endpt_o, int ije[16][3], const int st[9], double w[6]) {
    const Coord c = cc(lcsd[0], lcsd[1], adj_tri[lcsd[2]][1 - k1]);
    const Coord m = L.in(lcsd[0], lcsd[1]) ? L.midpt[(int64_t)lcsd[2] * L.NN + L.id(d, lcsd[0], lcsd[1])]
                                           : C(0.0, 0.0, 0.0);
    x = direction(c, m);
    y = normalize_coord(cross(x, c));
    Row6 G[6];
    G[0] = row(ije[st[0]]);
    G[1] = row(ije[st[1]]);
    G[2] = row(ije[st[2]]);
    G[3] = row(ije[st[3]]) - row(ije[st[4]]);
    G[4] = row(ije[st[5]]) - row(ije[st[6]]);
    G[5] = row(ije[st[7]]) - row(ije[st[8]]);
    double a[36];
    for (int col = 0; col < 6; ++col)
      for (int r = 0; r < 6; ++r) a[col * 6 + r] = G[col].v[r];
    // coords_to_row_perp (:1323-1334)
    const Coord mid = mid_pt(c, endpt_o);
    const Coord dir = cross(vector(c, endpt_o), mid);
    Row6 b = coords_to_rowd(mid, dir, x, y);
    const double dd = dist(c, endpt_o);
    for (int q = 0; q < 6; ++q) w[q] = b.v[q] * dd;
    dgesv6(a, w);
  }
  void store(int i, int j, const double* v) {
    if (!L.in(i, j)) { ++bad; return; }
    const int64_t id = L.id(d, i, j);
    for (int c = 0; c < 3; ++c) {
      double& s = L.rf_wgt[(int64_t)c * L.NN + id];
      if (L.rf_set[id]) conflict = std::max(conflict, std::fabs(s - v[c]));
      s = v[c];
    }
    L.rf_set[id] = 1;
  }
  // basic_F_restr_wgt for parent (ip, jp), edge e in {RT, UP}, overlap types typ[0..1].
  void compute(int ip, int jp, int e, const int typ[2]) {
    const int i0 = 2 * ip, j0 = 2 * jp;
    int enc[4][2];
    int i, j;
    if (e == UP) {
      const int t[4][2] = {{i0 - 2, j0}, {i0 - 2, j0 + 1}, {i0 + 1, j0}, {i0 + 1, j0 + 1}};
      std::memcpy(enc, t, sizeof t);
      i = i0;
      j = j0 + 1;
    } else {
      const int t[4][2] = {{i0, j0}, {i0, j0 + 1}, {i0 + 1, j0 - 2}, {i0 + 1, j0 - 1}};
      std::memcpy(enc, t, sizeof t);
      i = i0 + 1;
      j = j0;
    }
    const int hs = HEX_S_OFFS[e];
    int ije[16][3];
    auto set = [&](int s, int bi, int bj, const int* h) { ije[s][0] = bi + h[0]; ije[s][1] = bj + h[1]; ije[s][2] = h[2]; };
    set(S_UMZ, i, j, HEX_SIDES[hs + 1]);
    set(S_UPZ, i, j, HEX_SIDES[hs + 4]);
    set(S_WMP, i, j, HEX_SIDES[hs + 0]);
    set(S_VPP, i, j, HEX_SIDES[hs + 5]);
    set(S_WPM, i, j, HEX_SIDES[hs + 3]);
    set(S_VMM, i, j, HEX_SIDES[hs + 2]);
    const int mp[2] = {i + NGHB_PT[hs + 0][0], j + NGHB_PT[hs + 0][1]};
    const int pp[2] = {i + NGHB_PT[hs + 5][0], j + NGHB_PT[hs + 5][1]};
    const int pm[2] = {i + NGHB_PT[hs + 3][0], j + NGHB_PT[hs + 3][1]};
    const int mm[2] = {i + NGHB_PT[hs + 2][0], j + NGHB_PT[hs + 2][1]};
    set(S_VMP, mp[0], mp[1], HEX_SIDES[hs + 2]);
    set(S_VMPP, mp[0], mp[1], HEX_SIDES[hs + 5]);
    set(S_UZP, mp[0], mp[1], HEX_SIDES[hs + 4]);
    set(S_WPPP, pp[0], pp[1], HEX_SIDES[hs + 0]);
    set(S_WPP, pp[0], pp[1], HEX_SIDES[hs + 3]);
    set(S_VPM, pm[0], pm[1], HEX_SIDES[hs + 5]);
    set(S_VPMM, pm[0], pm[1], HEX_SIDES[hs + 2]);
    set(S_UZM, pm[0], pm[1], HEX_SIDES[hs + 1]);
    set(S_WMMM, mm[0], mm[1], HEX_SIDES[hs + 3]);
    set(S_WMM, mm[0], mm[1], HEX_SIDES[hs + 0]);
    static const int ST1[9] = {S_VPP, S_WMP, S_UZP, S_UPZ, S_WPP, S_VMP, S_UMZ, S_WPPP, S_VMPP};
    static const int ST0[9] = {S_VMM, S_WPM, S_UZM, S_UMZ, S_WMM, S_VPM, S_UPZ, S_WMMM, S_VPMM};
    for (int k = 1; k >= 0; --k) {
      const int* ta = adj_tri[e][k];
      const Coord po = Pa.ccentre[(int64_t)ta[2] * Pa.NN + Pa.id(d, ip + ta[0], jp + ta[1])];
      const int* u = ije[k == 1 ? S_UZP : S_UZM];
      const int slot = k == 1 ? 0 : 2;
      if (dist(po, cc(u[0], u[1], adj_tri[u[2]][1 - k])) < eps()) {  // coinciding circumcentres
        const double z[3] = {0.0, 0.0, 0.0};
        store(enc[slot][0], enc[slot][1], z);
        store(enc[slot + 1][0], enc[slot + 1][1], z);
        continue;
      }
      const int* lcsd;
      if (typ[k] == OUTER1) lcsd = ije[k == 1 ? S_VPP : S_VMM];
      else if (typ[k] == OUTER2) lcsd = ije[k == 1 ? S_WMP : S_WPM];
      else lcsd = ije[k == 1 ? S_UZP : S_UZM];
      double w[6];
      interp(k, lcsd, po, ije, k == 1 ? ST1 : ST0, w);
      double o[6];
      if (e == RT) {
        const double t[6] = {w[1], w[2], w[0], w[4], w[5], w[3]};
        std::memcpy(o, t, sizeof t);
      } else {
        const double t[6] = {w[2], w[0], w[1], w[5], w[3], w[4]};
        std::memcpy(o, t, sizeof t);
      }
      store(enc[slot][0], enc[slot][1], o);
      store(enc[slot + 1][0], enc[slot + 1][1], o + 3);
    }
  }
};

// set_RF_wgts over the parents [0, n_par)^2 of every lozenge: the overlap
// type of the RT child (2i+1, 2j) feeds the RT weights, that of the UP child
// (2i, 2j+1) the UP weights.
void rf_weights(Level& Pa, Level& L) {
  L.rf_wgt.assign((size_t)3 * L.NN, 0.0);
  L.rf_set.assign((size_t)L.NN, 0);
  int bad = 0;
  double conflict = 0.0;
  for (int d = 0; d < N_LOZ; ++d) {
    RFWeights W{Pa, L, d, C(0, 0, 0), C(0, 0, 0)};
    for (int jp = 0; jp < Pa.n; ++jp)
      for (int ip = 0; ip < Pa.n; ++ip) {
        double area[8];
        int typ[2];
        get_overl_areas(Pa, L, d, ip, jp, 2 * ip + 1, 2 * jp, RT, area, typ);
        W.compute(ip, jp, RT, typ);
        get_overl_areas(Pa, L, d, ip, jp, 2 * ip, 2 * jp + 1, UP, area, typ);
        W.compute(ip, jp, UP, typ);
      }
    bad += W.bad;
    conflict = std::max(conflict, W.conflict);
  }
  L.rf_conflict = conflict;
  L.rf_set.clear();
  if (bad) std::fprintf(stderr, "wtg: %d reads outside the padded level in flux-restriction weights (level %d)\n",
                        bad, L.l);
}

// comm_nodes9(get_areas, set_areas) + area_post_comm (src/refine_patch.f90:436-486)
void comm_areas(const Grid& g, Level& L) {
  for (auto& h : L.halo_node) {
    bool neg = h.dst < 0;
    int64_t dst = neg ? -h.dst - 1 : h.dst;
    double a[4];
    for (int k = 0; k < 4; ++k) a[k] = L.overl_a[k * L.NN + h.src];
    if (neg) { std::swap(a[0], a[1]); std::swap(a[2], a[3]); }
    for (int k = 0; k < 4; ++k) L.overl_a[k * L.NN + dst] = a[k];
    L.overl_split[dst] = L.overl_split[h.src];
    L.overl_split[L.NN + dst] = L.overl_split[L.NN + h.src];
    L.hex_inv[dst] = L.hex_inv[h.src];
  }
  for (int d = 0; d < N_LOZ; ++d) {
    if (g.penta[d][SOUTHEAST])
      for (int k = 0; k < 4; ++k) L.overl_a[k * L.NN + L.id(d, L.n, -1)] = 0.0;
    if (g.penta[d][NORTHWEST])
      for (int k = 0; k < 4; ++k) L.overl_a[k * L.NN + L.id(d, -1, L.n)] = 0.0;
  }
}

}  // namespace

void build_grid(Grid& g, int min_level, int max_level, int domain_level, double radius, double omega) {
  if (min_level < 2 || max_level < min_level || max_level > 11) throw std::runtime_error("bad levels");
  R = radius;
  g.min_level = min_level;
  g.max_level = max_level;
  g.domain_level = domain_level;
  g.radius = radius;
  g.omega = omega;
  init_connections(g);
  g.lev.clear();
  g.lev.resize(max_level - min_level + 2);
  for (int l = min_level - 1; l <= max_level; ++l) {
    Level& L = g.at(l);
    alloc_level(L, l);
    build_halo(g, L);
    if (l == min_level - 1) {
      coords_root(g, L);
    } else {
      coords_child(g, g.at(l - 1), L);
    }
    geometry(g, L);
    if (l > min_level - 1) {
      overlap_areas(g.at(l - 1), L);
      velo_weights(g, g.at(l - 1), L);
      rf_weights(g.at(l - 1), L);
    }
    comm_areas(g, L);
  }
  // Strip the temporary sign encoding of node entries (kept only for the area swap).
  for (auto& L : g.lev)
    for (auto& h : L.halo_node)
      if (h.dst < 0) h.dst = -h.dst - 1;
}

}  // namespace wtg
