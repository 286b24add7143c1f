// ORACLE -- test infrastructure only.
//
// The oracle's own icosahedral grid: a CPU FP64 restatement, written from the
// reference's Fortran and nothing else, of the host set-up that produces the
// geometry and ghost tables the hot path consumes.  It exists so that the
// oracle (and the timed CPU baseline) never take geometry from the product's
// builder; tests/test_oracle_grid.py compares every table of the two builders.
//
// Followed, routine by routine (reference file:line):
//   sphere.f90            dist :14, distn :184, triarea :163, circumcentre :197,
//                         project_on_sphere :86, mid_pt :276, arc_inters :92,
//                         normalize_Coord :282, init_Areas (sphere.f90:305)
//   init.f90              init_coordinates :270-318 (icosahedron corners,
//                         get_J0_coord), assign_coord :617-664, ccentre :745,
//                         ccentre_penta :320-384, midpt :829-876, lengths
//                         :386-420, cpt_areas :666-711, cpt_triarea :763-780,
//                         coriolis :782-800, init_connections :525-615
//   refine_patch.f90      refine_patch2 :106-262 (child coordinates, geometry
//                         on [-2|-1, n+1], the two pentagon corner nodes),
//                         set_areas / get_areas / area_post_comm :436-486
//   comm.f90              create_comm_e :103-345, pack_idx :594-645,
//                         create_comm :370-438, create_comm_pole :440-530,
//                         create_pack_st(2) :64-81,764-774, cp_bdry_inside
//                         :785-806 (unpack order: source domain outermost)
//   wavelet.f90           get_overl_areas :1408-1475, set_RF_wgts :1512-1540,
//                         basic_F_restr_wgt :1176-1345, set_WT_wgts :1567-1584,
//                         outer_velo_weights :1586-1705, local_coord :1500,
//                         coords_to_rowd :1769, Iu_Base_Wgt :1765
//   dgesv.f90             DGESV -> DGETF2 (reciprocal scaling when |pivot| >=
//                         sfmin) + DGETRS with the reference BLAS loops (the
//                         vendored LAPACK path; the reference's build links a
//                         system LAPACK instead, whose operation order may differ)
//   shared.f90:285-330    nghb_pt, end_pt, opp_no, adj_tri, no_adj_tri,
//                         hex_sides, hex_s_offs, bfly_tri
//
// Layout: one domain per lozenge (N_SUB_DOM_PER_DIM = 1 for the ghost tables;
// DOMAIN_LEVEL sub-domains only set the root coordinates through
// get_J0_coord), every level of a lozenge one padded (n+4)^2 array with the
// reference's 2-cell halo: slot (d, i, j), i, j in [-2, n+1], at
// (d*P + j+2)*P + i+2.  Reads beyond the padded array give ORIGIN / 0 (the
// reference reads a neighbouring storage element there; none of those values
// reaches an owned result).  Arithmetic in the reference's operand order,
// compiled without FMA contraction.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <vector>

namespace og {

struct C3 { double x, y, z; };
static inline C3 mk(double x, double y, double z) { return C3{x, y, z}; }

enum { RT = 0, DG = 1, UP = 2, NODE = 3 };
enum { LORT = 0, UPLT = 1 };
enum { NORTH = 1, EAST = 2, SOUTH = 3, WEST = 4, NORTHEAST = 5, SOUTHEAST = 6, SOUTHWEST = 7, NORTHWEST = 8 };
enum { INSIDE = 0, OUTER1 = 1, OUTER2 = 2 };
constexpr int BDRY = 2, LAST_BDRY = BDRY - 1;
constexpr int NLOZ = 10;
constexpr int POLE_ = -2, NONE_ = -1;

// -------------------------------------------------------------- sphere.f90 --
struct Sphere {
  double R = 6371.22e3, omega = 7.292e-5;
  double eps() const { return R * 1e-13; }
  static double sq(double a) { return a * a; }
  double dist(C3 p, C3 q) const {
    return R * std::asin(std::sqrt(sq(p.y * q.z - p.z * q.y) + sq(p.z * q.x - p.x * q.z) + sq(p.x * q.y - p.y * q.x)) /
                         (R * R));
  }
  double distn(C3 p, C3 q) const {
    double s = ((1.0 / R) * (1.0 / R)) *
               std::sqrt(sq(p.y * q.z - p.z * q.y) + sq(p.z * q.x - p.x * q.z) + sq(p.x * q.y - p.y * q.x));
    if (s > 1.0) return std::asin(1.0);
    return std::asin(s);
  }
  double triarea(C3 A, C3 B, C3 C) const {
    double ab = distn(A, B), ac = distn(A, C), bc = distn(B, C);
    double s = (ab + ac + bc) / 2;
    double t = std::tan(0.5 * s) * std::tan((s - ab) / 2.0) * std::tan((s - ac) / 2.0) * std::tan((s - bc) / 2.0);
    if (t < 1e-64) return 0.0;
    return 4.0 * (R * R) * std::atan(std::sqrt(t));
  }
  static double norm(C3 c) { return std::sqrt(sq(c.x) + sq(c.y) + sq(c.z)); }
  static C3 cross(C3 u, C3 v) { return mk(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x); }
  static double inner(C3 u, C3 v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
  static C3 vec(C3 a, C3 b) { return mk(b.x - a.x, b.y - a.y, b.z - a.z); }
  C3 project(C3 p) const {
    double nrm = std::sqrt(sq(p.x) + sq(p.y) + sq(p.z));
    return mk(p.x * (R / nrm), p.y * (R / nrm), p.z * (R / nrm));
  }
  C3 mid_pt(C3 p, C3 q) const { return project(mk(p.x + q.x, p.y + q.y, p.z + q.z)); }
  C3 circumcentre(C3 A, C3 B, C3 C) const {
    C3 c = cross(mk(A.x - B.x, A.y - B.y, A.z - B.z), mk(C.x - B.x, C.y - B.y, C.z - B.z));
    if (norm(c) < eps()) return c;
    return project(c);
  }
  C3 normalize(C3 s) const {
    double nrm = std::sqrt(sq(s.x) + sq(s.y) + sq(s.z));
    if (nrm >= eps()) return mk(s.x / nrm, s.y / nrm, s.z / nrm);
    return mk(0, 0, 0);
  }
  C3 direction(C3 a, C3 b) const { return normalize(vec(a, b)); }
  C3 sph2cart(double lon, double lat) const {
    return mk(R * (std::cos(lon) * std::cos(lat)), R * (std::sin(lon) * std::cos(lat)), R * std::sin(lat));
  }
  void arc_inters(C3 a1, C3 a2, C3 b1, C3 b2, C3& pt, bool& does) const {
    pt = b2;
    does = true;
    if (norm(vec(a2, b2)) < eps()) return;
    C3 n1 = cross(a1, a2);
    double inpr = inner(n1, b1) * inner(n1, b2);
    if (inpr > 0.0) { does = false; return; }
    C3 n2 = cross(b1, b2);
    inpr = inner(n2, a1) * inner(n2, a2);
    if (inpr > 0.0) { does = false; return; }
    pt = project(cross(n1, n2));
    C3 neg = mk(-pt.x, -pt.y, -pt.z);
    if (norm(vec(neg, a1)) < norm(vec(pt, a1))) pt = neg;
    does = true;
  }
};

// ------------------------------------------------------------- one level --
struct HNode { int64_t dst, src; int sign; };
struct HEdge { int64_t dst, src; int sign; };   // plane*NN + node

struct Lev {
  int l = 0, n = 0, P = 0;
  int64_t NN = 0;
  std::vector<C3> node, cc, mp;
  std::vector<double> len, pedlen, part, hexinv, tri, cor, oa, os, iu, rf;
  std::vector<HNode> hn;
  std::vector<HEdge> he;
  int64_t id(int d, int i, int j) const { return ((int64_t)d * P + (j + BDRY)) * P + (i + BDRY); }
  bool in(int i, int j) const { return i >= -BDRY && j >= -BDRY && i < n + BDRY && j < n + BDRY; }
  C3 nd(int d, int i, int j) const { return in(i, j) ? node[id(d, i, j)] : mk(0, 0, 0); }
  C3 c(int d, int i, int j, int t) const { return in(i, j) ? cc[t * NN + id(d, i, j)] : mk(0, 0, 0); }
  C3 m(int d, int i, int j, int e) const { return in(i, j) ? mp[e * NN + id(d, i, j)] : mk(0, 0, 0); }
  double pt(int d, int i, int j, int k) const { return in(i, j) ? part[(k - 1) * NN + id(d, i, j)] : 0.0; }
};

struct Grid {
  Sphere S;
  int min_level = 0, max_level = 0, domain_level = 0;
  int neigh[NLOZ][9], rot[NLOZ][9], over_pole[NLOZ][2];
  std::vector<Lev> L;  // index l - (min_level - 1)
  Lev& at(int l) { return L[l - (min_level - 1)]; }
};

// ---------------------------------------------- init.f90:init_connections --
// One sub-domain per lozenge: N_SUB_DOM_PER_DIM = 1, so i = j = 1 in the loops.
static void connections(Grid& g) {
  auto mod = [](int a, int b) { return ((a % b) + b) % b; };
  for (int ii = 1; ii <= 2; ++ii)
    for (int jj = 1; jj <= 5; ++jj) {
      const int loz = 5 * ii - 5 + (jj - 1);
      for (int s = 0; s < 9; ++s) g.neigh[loz][s] = NONE_, g.rot[loz][s] = 0;
      g.over_pole[loz][0] = 5 * ii - 5 + mod(jj + 1, 5);
      g.over_pole[loz][1] = 5 * ii - 5 + mod(jj - 3, 5);
      if (ii - 1 == 1) g.neigh[loz][NORTHWEST] = POLE_;
      else g.neigh[loz][SOUTHEAST] = POLE_;
      g.neigh[loz][NORTH] = 5 + mod(ii + jj - 2, 5), g.rot[loz][NORTH] = ii - 1;
      g.neigh[loz][EAST] = mod(jj, 5), g.rot[loz][EAST] = 1 - (ii - 1);
      g.neigh[loz][SOUTH] = mod(ii + jj - 3, 5), g.rot[loz][SOUTH] = 1 - (ii - 1);
      g.neigh[loz][WEST] = 5 + mod(jj - 2, 5), g.rot[loz][WEST] = ii - 1;
    }
}

// ------------------------------------------------------ comm.f90 tables --
// Boundary-patch local (i, j) of side s -> lozenge slot (nidx of the
// boundary patches: north/south dims (n, BDRY), east/west (BDRY, n)).
static void bdry_slot(int s, int i, int j, int n, int& a, int& b) {
  switch (s) {
    case NORTH: a = i; b = n + j; return;
    case EAST: a = n + i; b = j; return;
    case SOUTH: a = i; b = j - BDRY; return;
    case WEST: a = i - BDRY; b = j; return;
    case NORTHEAST: a = n + i; b = n + j; return;
    case SOUTHEAST: a = n + i; b = j - BDRY; return;
    case SOUTHWEST: a = i - BDRY; b = j - BDRY; return;
    case NORTHWEST: a = i - BDRY; b = n + j; return;
  }
  throw std::runtime_error("bdry_slot");
}

struct Entry { int src_d, si, sj, se; int dst_d, di, dj, de; int sign; bool edge; };

static void pack_idx(int i, int j, int rot, int s, int shift, int n, int& ir, int& jr, int& ip, int& jp) {
  const int LAST = n - 1;
  if (s == NORTH) { ir = i + rot * (j + shift); jr = j + n; ip = rot ? j : i; jp = rot ? LAST - i : j; }
  if (s == EAST) { ir = i + n; jr = j + rot * (i + shift); ip = rot ? LAST - j : i; jp = rot ? i : j; }
  if (s == SOUTH) { ir = i - rot * (j + shift); jr = -1 - j; ip = rot ? LAST - j : i; jp = rot ? LAST - i : LAST - j; }
  if (s == WEST) { ir = -1 - i; jr = j - rot * (i + shift); ip = rot ? LAST - j : LAST - i; jp = rot ? LAST - i : j; }
}

static void ghost_tables(Grid& g, Lev& V) {
  const int n = V.n, LAST = n - 1;
  // shift_arr (comm.f90:19), column s = 1..4 holds e = RT, DG, UP, NODE
  static const int shift_arr[4][4] = {{0, 1, 1, 1}, {1, 1, 0, 1}, {1, 0, 0, 0}, {0, 0, 1, 0}};
  std::vector<std::vector<Entry>> list(NLOZ);  // per destination, creation order
  for (int d = 0; d < NLOZ; ++d) {
    auto& out = list[d];
    auto pack_st = [&](bool edge, int src, int si, int sj, int se, int s, int bi, int bj, int de, int sign) {
      int a, b;
      bdry_slot(s, bi, bj, n, a, b);
      out.push_back(Entry{src, si, sj, se, d, a, b, de, sign, edge});
    };
    for (int s = 1; s <= 8; ++s) {
      if (s <= 4) {  // create_comm: the four sides of a lozenge are never pentagons
        const int src = g.neigh[d][s];
        if (src == NONE_) continue;
        const int rot = g.rot[d][s], orient = rot ? -1 : 1;
        for (int e = 0; e <= NODE; ++e) {
          const int shift = shift_arr[s - 1][e];
          const int e_pack = (e + rot * ((s % 2) + 1)) % 3;
          const bool ns = (s == NORTH || s == SOUTH);
          for (int o = 1; o <= BDRY; ++o)
            for (int q = 1; q <= n; ++q) {
              const int i = ns ? q : o, j = ns ? o : q;
              int ir, jr, ip, jp;
              pack_idx(i - 1, j - 1, rot, s, shift, n, ir, jr, ip, jp);
              if (ip < 0 || jp < 0 || ip >= n || jp >= n) continue;  // create_pack_st2
              out.push_back(Entry{src, ip, jp, e == NODE ? 0 : e_pack, d, ir, jr, e == NODE ? 0 : e, orient,
                                  e != NODE});
            }
        }
        if (rot == 1 && s == WEST)   // SW corner is always a pentagon here
          pack_st(true, src, LAST, LAST, RT, SOUTHWEST, LAST_BDRY, LAST_BDRY, RT, 1);
        if (rot == 1 && s == SOUTH)
          pack_st(true, src, LAST, LAST, UP, SOUTHWEST, LAST_BDRY, LAST_BDRY, RT, -1);
        if (rot == 0 && s == EAST) pack_st(false, src, 1, 0, 0, SOUTHEAST, 0, LAST_BDRY, 0, 1);
        if (rot == 0 && s == NORTH) pack_st(false, src, 0, 1, 0, NORTHWEST, LAST_BDRY, 0, 0, 1);
        if (rot == 1 && s == EAST) {
          pack_st(false, src, 0, 1, 0, NORTHEAST, 0, 1, 0, 1);
          pack_st(false, src, 1, 1, 0, NORTHEAST, 1, 0, 0, -1);
          pack_st(true, src, 0, 1, RT, NORTHEAST, 0, 1, RT, 1);
          pack_st(true, src, 0, 0, DG, NORTHEAST, 0, 0, RT, -1);
          pack_st(true, src, 0, 0, UP, NORTHEAST, 0, 0, UP, 1);
        }
        if (rot == 1 && s == NORTH) {
          pack_st(false, src, 1, 0, 0, NORTHEAST, 1, 0, 0, 1);
          pack_st(false, src, 1, 1, 0, NORTHEAST, 0, 1, 0, -1);
          pack_st(true, src, 1, 0, UP, NORTHEAST, 0, 1, RT, -1);
          pack_st(true, src, 0, 0, DG, NORTHEAST, 0, 0, UP, -1);
          pack_st(true, src, 0, 0, RT, NORTHEAST, 0, 0, RT, 1);
        }
      } else {  // corners are pentagons: create_comm_pole for k = 0, 1
        if (g.neigh[d][s] != POLE_) continue;
        for (int i = 0; i <= 1; ++i) {
          const int src = g.over_pole[d][i];
          const bool se = (s == SOUTHEAST);
          int s_side = (s == NORTHWEST) ? NORTH : EAST;
          auto sw = [&](int v[2]) { if (se) { int t = v[0]; v[0] = v[1]; v[1] = t; } };
          if (i == 0) {
            int ijn[2] = {0, 1};
            sw(ijn);
            pack_st(true, src, 0, LAST, DG, s_side, ijn[0], ijn[1], 2 * s_side - 2, 1);
            int ijn2[2] = {LAST_BDRY, 1}, ijs[2] = {1, LAST};
            sw(ijn2);
            sw(ijs);
            pack_st(false, src, ijs[0], ijs[1], 0, s, ijn2[0], ijn2[1], 0, -1);
          }
          if (i == 1) {
            int ijn[2] = {LAST_BDRY, 0}, ijs[2] = {0, LAST};
            sw(ijn);
            sw(ijs);
            pack_st(false, src, ijs[0], ijs[1], 0, s, ijn[0], ijn[1], 0, 1);
          }
          {
            int ijn[2] = {-i + 1, 1}, ijs[2] = {0, LAST};
            sw(ijn);
            sw(ijs);
            const int sg = i ? -1 : 1;
            pack_st(false, src, ijs[0], ijs[1], 0, s_side, ijn[0], ijn[1], 0, sg);
            pack_st(true, src, ijs[0], ijs[1], UP - 2 * s_side + 2, s_side, 0, 0, DG + i * (-2 * s_side + 3), sg);
          }
          if (i == 0) continue;
          s_side = (s == NORTHWEST) ? WEST : SOUTH;
          {
            int ijn[2] = {LAST_BDRY - 1, LAST}, ijs[2] = {1, LAST};
            sw(ijn);
            sw(ijs);
            pack_st(false, src, ijs[0], ijs[1], 0, s_side, ijn[0], ijn[1], 0, 1);
            int ijn2[2] = {LAST, LAST_BDRY};
            if (s == NORTHWEST) { int t = ijn2[0]; ijn2[0] = ijn2[1]; ijn2[1] = t; }
            pack_st(true, src, LAST * (-s_side + 4), LAST * (s_side - 3), DG, s_side, ijn2[0], ijn2[1],
                    2 * s_side - 6, 1);
          }
        }
      }
    }
  }
  // cp_bdry_inside: source domain outermost, then every destination, each
  // list in creation order; later writes to one slot overwrite earlier ones.
  std::vector<int64_t> lastn(V.NN, -1), laste(3 * V.NN, -1);
  std::vector<HNode> nodes;
  std::vector<HEdge> edges;
  for (int src = 0; src < NLOZ; ++src)
    for (int d = 0; d < NLOZ; ++d)
      for (const Entry& E : list[d]) {
        if (E.src_d != src) continue;
        if (!V.in(E.di, E.dj)) throw std::runtime_error("ghost destination outside the padded level");
        const int64_t dn = V.id(E.dst_d, E.di, E.dj), sn = V.id(E.src_d, E.si, E.sj);
        if (E.edge) {
          const int64_t de = (int64_t)E.de * V.NN + dn;
          laste[de] = (int64_t)edges.size();
          edges.push_back(HEdge{de, (int64_t)E.se * V.NN + sn, E.sign});
        } else {
          lastn[dn] = (int64_t)nodes.size();
          nodes.push_back(HNode{dn, sn, E.sign});
        }
      }
  V.hn.clear();
  V.he.clear();
  for (size_t k = 0; k < nodes.size(); ++k)
    if (lastn[nodes[k].dst] == (int64_t)k) V.hn.push_back(nodes[k]);
  for (size_t k = 0; k < edges.size(); ++k)
    if (laste[edges[k].dst] == (int64_t)k) V.he.push_back(edges[k]);
}

// ----------------------------------------------------------- coordinates --
static void alloc(Lev& V, int l) {
  V.l = l;
  V.n = 1 << l;
  V.P = V.n + 2 * BDRY;
  V.NN = (int64_t)NLOZ * V.P * V.P;
  const C3 O = mk(0, 0, 0);
  V.node.assign(V.NN, O);
  V.cc.assign(2 * V.NN, O);
  V.mp.assign(3 * V.NN, O);
  V.len.assign(3 * V.NN, 0.0);
  V.pedlen.assign(3 * V.NN, 0.0);
  V.part.assign(6 * V.NN, 0.0);
  V.hexinv.assign(V.NN, 0.0);
  V.tri.assign(2 * V.NN, 1.0);   // extend (dom%triarea, ..., 1d0), refine_patch.f90:187
  V.cor.assign(2 * V.NN, 0.0);
  V.oa.assign(4 * V.NN, 0.0);
  V.os.assign(2 * V.NN, 0.0);
  V.iu.assign(9 * V.NN, 0.0);
  V.rf.assign(3 * V.NN, 0.0);
}

// init_coordinates + assign_coord for level min_level-1 (every sub-domain of
// DOMAIN_LEVEL), then comm_nodes3 (get_coord, set_coord).
static void root_coordinates(Grid& g, Lev& V) {
  const Sphere& S = g.S;
  const double PI = std::acos(-1.0);
  const double lat[4] = {-PI / 2.0, -std::atan(1.0 / 2.0), std::atan(1.0 / 2.0), PI / 2.0};
  double lon[10];
  for (int k = 0; k < 10; ++k) lon[k] = (PI * double(k)) / 5.0;
  auto mod = [](int a, int b) { return ((a % b) + b) % b; };
  const int DL = g.domain_level, NSD = 1 << DL;
  const int PL = (g.min_level - 1) - DL;
  if (PL < 0) throw std::runtime_error("min_level - 1 < DOMAIN_LEVEL");
  const int PS = 1 << PL;
  const double YANGLE = 0.0;
  for (int ii = 1; ii <= 2; ++ii)
    for (int jj = 1; jj <= 5; ++jj) {
      const int loz = 5 * ii - 5 + (jj - 1);
      auto unit = [&](C3 c) { return mk(c.x / S.R, c.y / S.R, c.z / S.R); };
      C3 ne = unit(S.sph2cart(lon[mod(ii + 2 * jj - 2, 10)], lat[ii]));
      C3 se = unit(S.sph2cart(lon[ii + 2 * jj - 3], lat[ii - 1]));
      C3 sw = unit(S.sph2cart(lon[mod(ii + 2 * jj - 4, 10)], lat[ii]));
      C3 nw = unit(S.sph2cart(lon[ii + 2 * jj - 3], lat[ii + 1]));
      auto yrot = [&](C3 c) {
        return mk(c.x * std::cos(YANGLE) - c.z * std::sin(YANGLE), c.y, c.x * std::sin(YANGLE) + c.z * std::cos(YANGLE));
      };
      C3 cnr[2][2];  // cnr(i+1, j+1) of get_J0_coord
      cnr[0][1] = yrot(nw), cnr[1][1] = yrot(ne), cnr[0][0] = yrot(sw), cnr[1][0] = yrot(se);
      std::function<C3(int, int, int)> J0 = [&](int i, int j, int l) -> C3 {
        if (l > 0) return S.mid_pt(J0(i / 2, j / 2, l - 1), J0((i + 1) / 2, (j + 1) / 2, l - 1));
        return cnr[i][j];
      };
      for (int sj = 1; sj <= NSD; ++sj)
        for (int si = 1; si <= NSD; ++si) {
          const int oi = (si - 1) * PS, oj = (sj - 1) * PS;
          auto at = [&](int i, int j) -> C3& { return V.node[V.id(loz, oi + i, oj + j)]; };
          at(PS, PS) = S.project(J0(si, sj, DL));
          at(PS, 0) = S.project(J0(si, sj - 1, DL));
          at(0, 0) = S.project(J0(si - 1, sj - 1, DL));
          at(0, PS) = S.project(J0(si - 1, sj, DL));
          for (int l = 1; l <= PL; ++l) {
            const int pc = 1 << (PL - l + 1), pf = pc / 2;
            for (int j = 1; j <= PS; j += pc) {
              for (int i = 1; i <= PS; i += pc) {
                at(i + pf - 1, j - 1) = S.mid_pt(at(i - 1, j - 1), at(i + pc - 1, j - 1));
                at(i - 1, j + pf - 1) = S.mid_pt(at(i - 1, j - 1), at(i - 1, j + pc - 1));
                at(i + pf - 1, j + pf - 1) = S.mid_pt(at(i + pc - 1, j + pc - 1), at(i - 1, j - 1));
              }
              at(PS, j + pf - 1) = S.mid_pt(at(PS, j - 1), at(PS, j + pc - 1));
            }
            for (int i = 1; i <= PS; i += pc) at(i + pf - 1, PS) = S.mid_pt(at(i - 1, PS), at(i + pc - 1, PS));
          }
        }
    }
  for (const HNode& h : V.hn) V.node[h.dst] = V.node[h.src];
}

// refine_patch2 (refine_patch.f90:129-155) over a whole lozenge.
static void child_coordinates(Grid& g, const Lev& Pa, Lev& V) {
  const Sphere& S = g.S;
  for (int d = 0; d < NLOZ; ++d) {
    for (int b = -1; b <= Pa.n; ++b)
      for (int a = -1; a <= Pa.n; ++a) {
        const int64_t p = Pa.id(d, a, b);
        V.node[V.id(d, 2 * a, 2 * b)] = Pa.node[p];
        V.node[V.id(d, 2 * a + 1, 2 * b)] = Pa.mp[RT * Pa.NN + p];
        V.node[V.id(d, 2 * a + 1, 2 * b + 1)] = Pa.mp[DG * Pa.NN + p];
        V.node[V.id(d, 2 * a, 2 * b + 1)] = Pa.mp[UP * Pa.NN + p];
      }
    // the two pentagon corner nodes of the south-east and north-west corners
    V.node[V.id(d, V.n, -1)] = S.mid_pt(Pa.nd(d, Pa.n + 1, 0), Pa.nd(d, Pa.n, 0));
    V.node[V.id(d, -1, V.n)] = S.mid_pt(Pa.nd(d, 0, Pa.n + 1), Pa.nd(d, 0, Pa.n));
  }
}

// ------------------------------------------------------------- geometry --
static void geometry(Grid& g, Lev& V) {
  const Sphere& S = g.S;
  const int n = V.n;
  for (int d = 0; d < NLOZ; ++d) {
    // ccentre on [-2, n+1]^2 (apply_onescale2 with -BDRY, BDRY)
    for (int j = -2; j <= n + 1; ++j)
      for (int i = -2; i <= n + 1; ++i) {
        const int64_t id = V.id(d, i, j);
        V.cc[LORT * V.NN + id] = S.circumcentre(V.nd(d, i, j), V.nd(d, i + 1, j + 1), V.nd(d, i + 1, j));
        V.cc[UPLT * V.NN + id] = S.circumcentre(V.nd(d, i, j), V.nd(d, i, j + 1), V.nd(d, i + 1, j + 1));
      }
    // ccentre_penta at the four lozenge corners (every corner is a pentagon)
    auto CC = [&](int i, int j, int t) -> C3& { return V.cc[t * V.NN + V.id(d, i, j)]; };
    {
      CC(-1, -1, LORT) = S.circumcentre(V.nd(d, 0, 0), V.nd(d, 0, -1), V.nd(d, -1, 0));
      CC(-1, -1, UPLT) = CC(-1, -1, LORT);
      C3 pt3 = S.mid_pt(V.nd(d, 0, -2), V.nd(d, -2, 0));
      CC(-1, -2, LORT) = S.circumcentre(V.nd(d, 0, -1), V.nd(d, 0, -2), pt3);
      CC(-2, -1, UPLT) = S.circumcentre(pt3, V.nd(d, -2, 0), V.nd(d, -1, 0));
    }
    {
      const int i = n, j = -1;
      CC(i - 1, j, LORT) = S.circumcentre(V.nd(d, i - 1, j), V.nd(d, i, j + 1), V.nd(d, i + 1, j + 1));
      CC(i, j, UPLT) = CC(i - 1, j, LORT);
    }
    {
      const int i = -1, j = n;
      CC(i, j - 1, UPLT) = S.circumcentre(V.nd(d, i, j - 1), V.nd(d, i + 1, j + 1), V.nd(d, i + 1, j));
      CC(i, j, LORT) = CC(i, j - 1, UPLT);
    }
    {
      const int i = n, j = n;
      CC(i, j, LORT) = S.circumcentre(V.nd(d, i, j), V.nd(d, i, j + 1), V.nd(d, i + 1, j));
      CC(i, j, UPLT) = CC(i, j, LORT);
    }
    // midpt on [-1, n+1]^2
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        const int64_t id = V.id(d, i, j);
        C3* M = &V.mp[0];
        auto set = [&](int e, C3 v) { M[e * V.NN + id] = v; };
        if (j >= n + 1) { set(RT, S.mid_pt(V.nd(d, i, j), V.nd(d, i + 1, j))); continue; }
        if (i >= n + 1) { set(UP, S.mid_pt(V.nd(d, i, j), V.nd(d, i, j + 1))); continue; }
        if (j == -1) {
          if (i == -1) { set(DG, CC(i, j, LORT)); continue; }
          if (i == n) { set(UP, CC(i, j, UPLT)); continue; }
        } else if (j == n && i == -1) {
          set(RT, CC(i, j, LORT));
          continue;
        }
        set(RT, S.mid_pt(V.nd(d, i, j), V.nd(d, i + 1, j)));
        set(DG, S.mid_pt(V.nd(d, i + 1, j + 1), V.nd(d, i, j)));
        set(UP, S.mid_pt(V.nd(d, i, j), V.nd(d, i, j + 1)));
        if (j == n && i == n) set(DG, CC(i, j, LORT));
      }
    // cpt_areas on [-1, n+1]^2
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        const int64_t id = V.id(d, i, j);
        const C3 ctr = V.nd(d, i, j);
        const C3 cor[6] = {V.c(d, i, j, LORT), V.c(d, i, j, UPLT), V.c(d, i - 1, j, LORT),
                           V.c(d, i - 1, j - 1, UPLT), V.c(d, i - 1, j - 1, LORT), V.c(d, i, j - 1, UPLT)};
        const C3 mid[6] = {V.m(d, i, j, RT), V.m(d, i, j, DG), V.m(d, i, j, UP),
                           V.m(d, i - 1, j, RT), V.m(d, i - 1, j - 1, DG), V.m(d, i, j - 1, UP)};
        double part[6];
        for (int k = 0; k < 6; ++k)
          part[k] = S.triarea(ctr, cor[k], mid[k]) + S.triarea(ctr, cor[k], mid[(k + 1) % 6]);
        double sum = 0.0;
        for (int k = 0; k < 6; ++k) sum += part[k];
        const double hinv = (sum != 0.0) ? 1.0 / sum : 1.0;
        int k0 = 0, k1 = 6;
        bool whole = true;
        if (j >= n + 1) k0 = 3, k1 = 6, whole = false;          // part(4:6)
        else if (i >= n + 1) k0 = 2, k1 = 5, whole = false;     // part(3:5)
        for (int k = k0; k < k1; ++k) V.part[k * V.NN + id] = part[k];
        if (whole) V.hexinv[id] = hinv;
      }
    // lengths on [-1, n+1]^2 (after cpt_areas in refine_patch2; the values do not depend on the order)
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        const int64_t id = V.id(d, i, j);
        if (j >= n + 1) { V.len[RT * V.NN + id] = S.dist(V.nd(d, i, j), V.nd(d, i + 1, j)); continue; }
        if (i >= n + 1) { V.len[UP * V.NN + id] = S.dist(V.nd(d, i, j), V.nd(d, i, j + 1)); continue; }
        V.len[RT * V.NN + id] = S.dist(V.nd(d, i, j), V.nd(d, i + 1, j));
        V.len[DG * V.NN + id] = S.dist(V.nd(d, i + 1, j + 1), V.nd(d, i, j));
        V.len[UP * V.NN + id] = S.dist(V.nd(d, i, j), V.nd(d, i, j + 1));
        V.pedlen[RT * V.NN + id] = S.dist(V.c(d, i, j - 1, UPLT), V.c(d, i, j, LORT));
        V.pedlen[DG * V.NN + id] = S.dist(V.c(d, i, j, UPLT), V.c(d, i, j, LORT));
        V.pedlen[UP * V.NN + id] = S.dist(V.c(d, i, j, UPLT), V.c(d, i - 1, j, LORT));
        if (i == -1 && j == -1) {
          V.pedlen[DG * V.NN + id] = 0;
          V.len[RT * V.NN + id] = S.dist(V.nd(d, i + 1, j), V.nd(d, i, j + 1));
        }
        if (i == n && j == n) V.len[DG * V.NN + id] = S.dist(V.nd(d, i + 1, j), V.nd(d, i, j + 1));
      }
    // cpt_triarea and coriolis on [-1, n+1]^2
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) {
        const int64_t id = V.id(d, i, j);
        const double tl = V.pt(d, i, j, 1) + V.pt(d, i + 1, j, 3) + V.pt(d, i + 1, j + 1, 5);
        const double tu = V.pt(d, i, j, 2) + V.pt(d, i + 1, j + 1, 4) + V.pt(d, i, j + 1, 6);
        V.tri[LORT * V.NN + id] = tl;
        V.tri[UPLT * V.NN + id] = tu;
        V.cor[LORT * V.NN + id] = V.cc[LORT * V.NN + id].z / S.R * 2.0 * S.omega * tl;
        V.cor[UPLT * V.NN + id] = V.cc[UPLT * V.NN + id].z / S.R * 2.0 * S.omega * tu;
      }
  }
}

// ---------------------------------------------------- shared.f90 stencils --
// Fortran arrays stored column by column; accessors take the reference's
// 1-based indices.
static const int nghb_pt_[20] = {1, 0, 1, 1, 0, 1, -1, 0, -1, -1, 0, -1, 1, 0, 1, 1, 0, 1, -1, 0};
static const int end_pt_[12] = {0, 0, 1, 0, 1, 1, 0, 0, 0, 0, 0, 1};
static const int opp_no_[12] = {0, -1, 1, 1, 0, 1, 1, 0, 1, 1, -1, 0};
static const int adj_tri_[18] = {0, -1, UPLT, 0, 0, LORT, 0, 0, UPLT, 0, 0, LORT, 0, 0, UPLT, -1, 0, LORT};
static const int no_adj_tri_[30] = {0, 0, LORT, 0, -1, UPLT, -1, -1, LORT, -1, -1, UPLT, -1, 0, LORT,
                                    0, 0, UPLT, 0, 0, LORT, 0, -1, UPLT, -1, -1, LORT, -1, -1, UPLT};
static const int hex_sides_[30] = {0, 0, RT, 0, 0, DG, 0, 0, UP, -1, 0, RT, -1, -1, DG,
                                   0, -1, UP, 0, 0, RT, 0, 0, DG, 0, 0, UP, -1, 0, RT};
static const int hex_s_offs_[3] = {2, 0, 4};
static const int bfly_tri_[36] = {-1, -1, LORT, 0, -1, LORT, 1, 0, UPLT, 0, 0, UPLT, 0, 1, LORT, -1, 0, LORT,
                                  0, -1, UPLT, 1, 0, UPLT, 0, 0, LORT, 0, 1, LORT, -1, 0, UPLT, -1, -1, UPLT};
struct I3 { int a, b, c; };
static inline I3 nghb_pt(int k) { return I3{nghb_pt_[2 * (k - 1)], nghb_pt_[2 * (k - 1) + 1], 0}; }
static inline I3 end_pt(int k, int e1) { const int* p = end_pt_ + 2 * ((k - 1) + 2 * (e1 - 1)); return I3{p[0], p[1], 0}; }
static inline I3 opp_no(int k, int e1) { const int* p = opp_no_ + 2 * ((k - 1) + 2 * (e1 - 1)); return I3{p[0], p[1], 0}; }
static inline I3 adj_tri(int k, int e1) { const int* p = adj_tri_ + 3 * ((k - 1) + 2 * (e1 - 1)); return I3{p[0], p[1], p[2]}; }
static inline I3 no_adj_tri(int k) { const int* p = no_adj_tri_ + 3 * (k - 1); return I3{p[0], p[1], p[2]}; }
static inline I3 hex_sides(int k) { const int* p = hex_sides_ + 3 * (k - 1); return I3{p[0], p[1], p[2]}; }
static inline int hex_s_offs(int e1) { return hex_s_offs_[e1 - 1]; }
static inline I3 bfly_tri(int k, int e1) { const int* p = bfly_tri_ + 3 * ((k - 1) + 4 * (e1 - 1)); return I3{p[0], p[1], p[2]}; }

// -------------------------------------------------------------- dgesv ----
// DGESV = DGETF2 + DGETRS of the vendored LAPACK (column-major a(6,6), b(6)).
static void dgesv6(double a[36], double b[6]) {
  const int N = 6;
  auto A = [&](int i, int j) -> double& { return a[(i - 1) + N * (j - 1)]; };
  int ipiv[7];
  const double sfmin = 2.2250738585072014e-308;  // DLAMCH('S')
  for (int j = 1; j <= N; ++j) {
    int jp = j;  // IDAMAX over A(j:N, j)
    double dmax = std::fabs(A(j, j));
    for (int i = j + 1; i <= N; ++i)
      if (std::fabs(A(i, j)) > dmax) { jp = i; dmax = std::fabs(A(i, j)); }
    ipiv[j] = jp;
    if (A(jp, j) != 0.0) {
      if (jp != j)
        for (int k = 1; k <= N; ++k) { double t = A(j, k); A(j, k) = A(jp, k); A(jp, k) = t; }
      if (j < N) {
        if (std::fabs(A(j, j)) >= sfmin) {
          const double r = 1.0 / A(j, j);
          for (int i = j + 1; i <= N; ++i) A(i, j) = r * A(i, j);
        } else {
          for (int i = j + 1; i <= N; ++i) A(i, j) = A(i, j) / A(j, j);
        }
      }
    }
    if (j < N)  // DGER: A(j+1:, j+1:) -= A(j+1:, j) * A(j, j+1:)
      for (int k = j + 1; k <= N; ++k)
        if (A(j, k) != 0.0) {
          const double t = -1.0 * A(j, k);
          for (int i = j + 1; i <= N; ++i) A(i, k) = A(i, k) + A(i, j) * t;
        }
  }
  for (int i = 1; i <= N; ++i)  // DLASWP
    if (ipiv[i] != i) { double t = b[i - 1]; b[i - 1] = b[ipiv[i] - 1]; b[ipiv[i] - 1] = t; }
  for (int k = 1; k <= N; ++k)  // DTRSM lower, unit diagonal
    if (b[k - 1] != 0.0)
      for (int i = k + 1; i <= N; ++i) b[i - 1] = b[i - 1] - b[k - 1] * A(i, k);
  for (int k = N; k >= 1; --k)  // DTRSM upper
    if (b[k - 1] != 0.0) {
      b[k - 1] = b[k - 1] / A(k, k);
      for (int i = 1; i <= k - 1; ++i) b[i - 1] = b[i - 1] - b[k - 1] * A(i, k);
    }
}

// -------------------------------------------------- wavelet.f90 helpers --
static void normalize2(double q0, double q1, double& u, double& v) {
  const double nrm = std::sqrt(q0 * q0 + q1 * q1);
  u = q0 / nrm;
  v = q1 / nrm;
}
static void coords_to_rowd(C3 midpt, C3 dirvec, C3 x, C3 y, double row[6]) {
  double u, v;
  normalize2(Sphere::inner(dirvec, x), Sphere::inner(dirvec, y), u, v);
  const double xy0 = Sphere::inner(midpt, x), xy1 = Sphere::inner(midpt, y);
  row[0] = u, row[1] = u * xy0, row[2] = u * xy1, row[3] = v, row[4] = v * xy0, row[5] = v * xy1;
}
static void local_coord(const Sphere& S, C3 midpt, C3 e1, C3 e2, C3& x, C3& y) {
  x = S.direction(e1, e2);
  y = S.normalize(Sphere::cross(x, midpt));
}

// get_overl_areas (wavelet.f90:1408-1475) for the child slot (ic, jc) of
// parent (ip, jp) and parent edge e.
static void overl_areas(const Sphere& S, const Lev& Pa, const Lev& V, int d, int ip, int jp, int ic, int jc, int e,
                        double area[8], int typ[2]) {
  for (int k = 0; k < 8; ++k) area[k] = 0.0;
  typ[0] = typ[1] = 0;
  auto ccd = [&](const Lev& Z, int i, int j, I3 t) { return Z.c(d, i + t.a, j + t.b, t.c); };
  C3 hex[7];
  for (int i = 0; i < 6; ++i) hex[i + 1] = ccd(V, ic, jc, no_adj_tri(i + hex_s_offs(-e + 3) + 1));
  C3 tri[4][3];  // tri(1..3, 1..2)
  tri[1][1] = ccd(Pa, ip, jp, bfly_tri(4, e + 1));
  tri[2][1] = ccd(Pa, ip, jp, adj_tri(2, e + 1));
  tri[3][1] = ccd(Pa, ip, jp, bfly_tri(3, e + 1));
  tri[1][2] = ccd(Pa, ip, jp, bfly_tri(2, e + 1));
  tri[2][2] = ccd(Pa, ip, jp, adj_tri(1, e + 1));
  tri[3][2] = ccd(Pa, ip, jp, bfly_tri(1, e + 1));
  const C3 pt = V.nd(d, ic, jc);
  double* A = area - 1;  // 1-based
  int* T = typ - 1;
  A[1] = S.triarea(hex[6], hex[1], pt);
  A[2] = S.triarea(hex[3], hex[4], pt);
  for (int i = 1; i <= 2; ++i) {
    C3 p0, p1;
    bool d0, d1;
    S.arc_inters(tri[1][i], tri[2][i], hex[3 * i - 2], hex[3 * i - 1], p0, d0);
    S.arc_inters(tri[3][i], tri[2][i], hex[3 * i], hex[3 * i - 1], p1, d1);
    if (d0 && d1) {
      A[i + 4] = S.triarea(p0, tri[2][i], hex[3 * i - 1]);
      A[i + 6] = S.triarea(tri[2][i], hex[3 * i - 1], p1);
      A[i + 2] = A[i + 4] + A[i + 6];
      A[i] = A[i] + S.triarea(hex[3 * i - 2], p0, pt) + S.triarea(p0, pt, tri[2][i]);
      A[-i + 3] = A[-i + 3] + S.triarea(p1, hex[3 * i], pt) + S.triarea(tri[2][i], pt, p1);
      T[-i + 3] = INSIDE;
    } else if (!d0 && !d1) {
      A[i + 2] = 0.0;
      S.arc_inters(tri[2][1], tri[2][2], hex[3 * i - 2], hex[3 * i - 1], p0, d0);
      S.arc_inters(tri[2][2], tri[2][1], hex[3 * i - 1], hex[3 * i], p1, d1);
      if (!d0 && d1) {
        A[i] = A[i] + S.triarea(hex[3 * i - 2], hex[3 * i - 1], pt) + S.triarea(hex[3 * i - 1], p1, pt);
        A[-i + 3] = A[-i + 3] + S.triarea(p1, hex[3 * i], pt);
        T[-i + 3] = OUTER2;
      } else if (d0 && !d1) {
        A[i] = A[i] + S.triarea(hex[3 * i - 2], p0, pt);
        A[-i + 3] = A[-i + 3] + S.triarea(hex[3 * i - 1], hex[3 * i], pt) + S.triarea(p0, hex[3 * i - 1], pt);
        T[-i + 3] = OUTER1;
      } else {
        throw std::runtime_error("overlap area: unexpected intersection case A");
      }
    } else {
      throw std::runtime_error("overlap area: unexpected intersection case B");
    }
  }
}

// Child-level (i0, j0) + offset -> (i, j, e) triples of basic_F_restr_wgt.
struct IJE { int i, j, e; };
static inline IJE operator+(IJE a, I3 b) { return IJE{a.i + b.a, a.j + b.b, a.e + b.c}; }

// Positions of the ije array of basic_F_restr_wgt (shared.f90 names).
enum { UMZ = 0, UPZ, WMP, VPP, WPM, VMM, VMP, VMPP, UZP, WPPP, WPP, VPM, VPMM, UZM, WMMM, WMM };

// basic_F_restr_wgt (wavelet.f90:1176-1345)
static void rf_weights_edge(const Sphere& S, const Lev& Pa, Lev& V, int d, int ip, int jp, int e, int i0, int j0,
                            const int typ[2]) {
  int enc[4][2];
  int i, j;
  if (e == UP) {
    int t[4][2] = {{i0 - 2, j0}, {i0 - 2, j0 + 1}, {i0 + 1, j0}, {i0 + 1, j0 + 1}};
    std::memcpy(enc, t, sizeof t);
    i = i0, j = j0 + 1;
  } else {
    int t[4][2] = {{i0, j0}, {i0, j0 + 1}, {i0 + 1, j0 - 2}, {i0 + 1, j0 - 1}};
    std::memcpy(enc, t, sizeof t);
    i = i0 + 1, j = j0;
  }
  const int hso = hex_s_offs(e + 1);
  IJE ije[16];
  const IJE b0{i, j, 0};
  ije[UMZ] = b0 + hex_sides(hso + 1 + 1);
  ije[UPZ] = b0 + hex_sides(hso + 4 + 1);
  ije[WMP] = b0 + hex_sides(hso + 0 + 1);
  ije[VPP] = b0 + hex_sides(hso + 5 + 1);
  ije[WPM] = b0 + hex_sides(hso + 3 + 1);
  ije[VMM] = b0 + hex_sides(hso + 2 + 1);
  const I3 nmp = nghb_pt(hso + 0 + 1), npp = nghb_pt(hso + 5 + 1), npm = nghb_pt(hso + 3 + 1),
           nmm = nghb_pt(hso + 2 + 1);
  const IJE mp{i + nmp.a, j + nmp.b, 0}, pp{i + npp.a, j + npp.b, 0}, pm{i + npm.a, j + npm.b, 0},
      mm{i + nmm.a, j + nmm.b, 0};
  ije[VMP] = mp + hex_sides(hso + 4 - 2 + 1);
  ije[VMPP] = mp + hex_sides(hso + 1 + 4 + 1);
  ije[UZP] = mp + hex_sides(hso + 0 + 4 + 1);
  ije[WPPP] = pp + hex_sides(hso + 4 - 4 + 1);
  ije[WPP] = pp + hex_sides(hso + 1 + 2 + 1);
  ije[VPM] = pm + hex_sides(hso + 1 + 4 + 1);
  ije[VPMM] = pm + hex_sides(hso + 4 - 2 + 1);
  ije[UZM] = pm + hex_sides(hso + 3 - 2 + 1);
  ije[WMMM] = mm + hex_sides(hso + 1 + 2 + 1);
  ije[WMM] = mm + hex_sides(hso + 4 - 4 + 1);

  auto ccP = [&](I3 t) { return Pa.c(d, ip + t.a, jp + t.b, t.c); };
  auto ccC = [&](int a, int b, I3 t) { return V.c(d, a + t.a, b + t.b, t.c); };
  auto rowC = [&](IJE q, const C3& x, const C3& y, double row[6]) {
    const I3 p1 = end_pt(1, q.e + 1), p2 = end_pt(2, q.e + 1);
    const C3 e1 = V.nd(d, q.i + p1.a, q.j + p1.b), e2 = V.nd(d, q.i + p2.a, q.j + p2.b);
    const double ped = S.dist(ccC(q.i, q.j, adj_tri(1, q.e + 1)), ccC(q.i, q.j, adj_tri(2, q.e + 1)));
    coords_to_rowd(S.mid_pt(e1, e2), Sphere::vec(e1, e2), x, y, row);
    for (int r = 0; r < 6; ++r) row[r] = row[r] * ped;
  };
  auto interp = [&](int k1, IJE lcsd, C3 endpt_o, const int st[9], double w[6]) {
    const I3 at = adj_tri(-k1 + 2, lcsd.e + 1);
    const C3 ctri = V.c(d, lcsd.i + at.a, lcsd.j + at.b, at.c);
    C3 x, y;
    local_coord(S, ctri, ctri, V.m(d, lcsd.i, lcsd.j, lcsd.e), x, y);
    double G[36], r0[6], r1[6];
    for (int c = 0; c < 3; ++c) {
      rowC(ije[st[c]], x, y, r0);
      for (int r = 0; r < 6; ++r) G[r + 6 * c] = r0[r];
    }
    for (int c = 0; c < 3; ++c) {
      rowC(ije[st[3 + 2 * c]], x, y, r0);
      rowC(ije[st[4 + 2 * c]], x, y, r1);
      for (int r = 0; r < 6; ++r) G[r + 6 * (3 + c)] = r0[r] - r1[r];
    }
    // coords_to_row_perp of (ctri, endpt)
    const C3 mid = S.mid_pt(ctri, endpt_o);
    const C3 dir = Sphere::cross(Sphere::vec(ctri, endpt_o), mid);
    double b[6];
    coords_to_rowd(mid, dir, x, y, b);
    const double dd = S.dist(ctri, endpt_o);
    for (int r = 0; r < 6; ++r) b[r] = b[r] * dd;
    dgesv6(G, b);
    for (int r = 0; r < 6; ++r) w[r] = b[r];
  };
  auto store = [&](int a, int bj, const double* w) {
    if (!V.in(a, bj)) throw std::runtime_error("R_F_wgt slot outside the padded level");
    for (int c = 0; c < 3; ++c) V.rf[c * V.NN + V.id(d, a, bj)] = w[c];
  };
  for (int k : {1, 0}) {
    const I3 pt = adj_tri(k + 1, e + 1);
    const C3 cpar = ccP(pt);
    const IJE q = (k == 1) ? ije[UZP] : ije[UZM];
    const I3 at = adj_tri(-k + 2, q.e + 1);
    const double dst = S.dist(cpar, V.c(d, q.i + at.a, q.j + at.b, at.c));
    double w[6] = {0, 0, 0, 0, 0, 0};
    const int* e2 = (k == 1) ? enc[0] : enc[2];
    const int* e3 = (k == 1) ? enc[1] : enc[3];
    if (dst < S.eps()) {
      store(e2[0], e2[1], w);
      store(e3[0], e3[1], w);
      continue;
    }
    IJE lcsd;
    if (k == 1) lcsd = typ[1] == OUTER1 ? ije[VPP] : typ[1] == OUTER2 ? ije[WMP] : ije[UZP];
    else lcsd = typ[0] == OUTER1 ? ije[VMM] : typ[0] == OUTER2 ? ije[WPM] : ije[UZM];
    static const int st1[9] = {VPP, WMP, UZP, UPZ, WPP, VMP, UMZ, WPPP, VMPP};
    static const int st0[9] = {VMM, WPM, UZM, UMZ, WMM, VPM, UPZ, WMMM, VPMM};
    interp(k, lcsd, cpar, k == 1 ? st1 : st0, w);
    double r[6];
    if (e == RT) { double t[6] = {w[1], w[2], w[0], w[4], w[5], w[3]}; std::memcpy(r, t, sizeof t); }
    else { double t[6] = {w[2], w[0], w[1], w[5], w[3], w[4]}; std::memcpy(r, t, sizeof t); }
    store(e2[0], e2[1], r);
    store(e3[0], e3[1], r + 3);
  }
}

// outer_velo_weights (wavelet.f90:1586-1705) of parent edge (i0, j0, e0).
static void iu_weights(const Sphere& S, const Lev& Pa, int d, int i0, int j0, int e0, double out[9]) {
  const int n = Pa.n;
  auto get_coord = [&](int i, int j, int e) -> C3 {
    // the four lozenge corners are pentagons (is_penta of the corner patch)
    if (i == -1) {
      if (j == -1) {
        if (e == RT) return Pa.nd(d, -1, 0);   // nidx(LAST_BDRY, 0, IMINUS)
        if (e == UP) return Pa.nd(d, 0, -1);   // nidx(0, LAST_BDRY, JMINUS)
        // other edges fall through to the plain slot, as the reference
      } else if (j == n) {
        return Pa.nd(d, 0, n + 1);             // nidx(0, 1, JPLUS)
      }
      return Pa.nd(d, i, j);
    }
    if (i == n && j == -1) return Pa.nd(d, n + 1, 0);                 // nidx(1, 0, IPLUS)
    if (i == n + 1 && j == n + 1) return Pa.nd(d, n + 1, n);          // nidx(1, 0, IJPLUS)
    return Pa.nd(d, i, j);
  };
  const I3 ep1 = end_pt(1, e0 + 1), ep2 = end_pt(2, e0 + 1);
  C3 x, y;
  local_coord(S, Pa.m(d, i0, j0, e0), Pa.nd(d, i0 + ep1.a, j0 + ep1.b), Pa.nd(d, i0 + ep2.a, j0 + ep2.b), x, y);
  auto row = [&](I3 o1, I3 o2, double r[6]) {
    const int i = i0 + o1.a + o2.a, j = j0 + o1.b + o2.b, e = o2.c;
    const I3 a1 = end_pt(1, e + 1), a2 = end_pt(2, e + 1);
    const C3 p1 = get_coord(i + a1.a, j + a1.b, e0), p2 = get_coord(i + a2.a, j + a2.b, e0);
    coords_to_rowd(S.mid_pt(p1, p2), Sphere::vec(p1, p2), x, y, r);
  };
  double w[10] = {0};  // 1-based
  const int hso = hex_s_offs(e0 + 1);
  for (int k = 1; k <= 2; ++k) {
    double G[36], r0[6], r1[6];
    auto col = [&](int c, const double* v) { for (int r = 0; r < 6; ++r) G[r + 6 * (c - 1)] = v[r]; };
    row(I3{0, 0, 0}, I3{0, 0, e0}, r0); col(1, r0);
    row(end_pt(-k + 3, e0 + 1), hex_sides(hso + 2 + 3 * k - 3 + 1), r0); col(2, r0);
    row(end_pt(k, e0 + 1), hex_sides((hso + 3) - (3 * k - 3) + 1), r0); col(3, r0);
    row(opp_no(k, e0 + 1), hex_sides(hso + 1 + 3 * k - 3 + 1), r0);
    row(end_pt(k, e0 + 1), hex_sides(hso + 2 + 3 * k - 3 + 1), r1);
    for (int r = 0; r < 6; ++r) r0[r] = r0[r] - r1[r];
    col(4, r0);
    row(end_pt(-k + 3, e0 + 1), hex_sides((hso + 3) - (3 * k - 3) + 1), r0);
    row(opp_no(k, e0 + 1), hex_sides((hso + 4) - (3 * k - 3) + 1), r1);
    for (int r = 0; r < 6; ++r) r0[r] = r0[r] - r1[r];
    col(5, r0);
    row(end_pt(k, e0 + 1), hex_sides((hso + 5) - (3 * k - 3) + 1), r0);
    row(end_pt(-k + 3, e0 + 1), hex_sides(hso + 0 + 3 * k - 3 + 1), r1);
    for (int r = 0; r < 6; ++r) r0[r] = r0[r] - r1[r];
    col(6, r0);
    const C3 n1 = Pa.nd(d, i0 + ep1.a, j0 + ep1.b), n2 = Pa.nd(d, i0 + ep2.a, j0 + ep2.b);
    double b[6];
    coords_to_rowd(S.mid_pt(Pa.m(d, i0, j0, e0), n2), Sphere::vec(n1, n2), x, y, b);
    dgesv6(G, b);
    w[1] = w[1] + b[0];
    w[2 * k] = w[2 * k] + b[1];
    w[2 * k + 1] = w[2 * k + 1] + b[2];
    w[2 * k + 4] = b[3];
    w[2 * k + 5] = b[4];
    w[-2 * k + 6] = w[-2 * k + 6] + b[5];
    w[-2 * k + 7] = w[-2 * k + 7] - b[5];
  }
  static const double base[9] = {16.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0, -1.0 / 16.0,
                                 -1.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0};
  for (int k = 0; k < 9; ++k) out[k] = 0.5 * w[k + 1] - base[k];
}

// set_WT_wgts and set_RF_wgts of every parent (a, b) in [0, n_par)^2
// (apply_interscale_to_patch3 with st = en = 0).
static void interscale(Grid& g, Lev& Pa, Lev& V) {
  const Sphere& S = g.S;
  for (int d = 0; d < NLOZ; ++d)
    for (int b = 0; b < Pa.n; ++b)
      for (int a = 0; a < Pa.n; ++a) {
        const int ic = 2 * a, jc = 2 * b;
        double w[9];
        iu_weights(S, Pa, d, a, b, RT, w);
        for (int k = 0; k < 9; ++k) V.iu[k * V.NN + V.id(d, ic + 1, jc)] = w[k];
        iu_weights(S, Pa, d, a, b, DG, w);
        for (int k = 0; k < 9; ++k) V.iu[k * V.NN + V.id(d, ic, jc)] = w[k];
        iu_weights(S, Pa, d, a, b, UP, w);
        for (int k = 0; k < 9; ++k) V.iu[k * V.NN + V.id(d, ic, jc + 1)] = w[k];
      }
  for (int d = 0; d < NLOZ; ++d)
    for (int b = 0; b < Pa.n; ++b)
      for (int a = 0; a < Pa.n; ++a) {
        const int ic = 2 * a, jc = 2 * b;
        double area[8];
        int typ[2];
        auto put = [&](int i, int j) {
          const int64_t id = V.id(d, i, j);
          for (int k = 0; k < 4; ++k) V.oa[k * V.NN + id] = area[k];
          V.os[id] = area[4];
          V.os[V.NN + id] = area[5];
        };
        overl_areas(S, Pa, V, d, a, b, ic + 1, jc, RT, area, typ);
        put(ic + 1, jc);
        rf_weights_edge(S, Pa, V, d, a, b, RT, ic, jc, typ);
        overl_areas(S, Pa, V, d, a, b, ic + 1, jc + 1, DG, area, typ);
        put(ic + 1, jc + 1);
        overl_areas(S, Pa, V, d, a, b, ic, jc + 1, UP, area, typ);
        put(ic, jc + 1);
        rf_weights_edge(S, Pa, V, d, a, b, UP, ic, jc, typ);
      }
}

// comm_nodes9 (get_areas, set_areas) and area_post_comm on one level.
static void areas_to_ghosts(Lev& V) {
  for (const HNode& h : V.hn) {
    double a[4] = {V.oa[h.src], V.oa[V.NN + h.src], V.oa[2 * V.NN + h.src], V.oa[3 * V.NN + h.src]};
    if (h.sign < 0) { double t[4] = {a[1], a[0], a[3], a[2]}; std::memcpy(a, t, sizeof t); }
    for (int k = 0; k < 4; ++k) V.oa[k * V.NN + h.dst] = a[k];
    V.os[h.dst] = V.os[h.src];
    V.os[V.NN + h.dst] = V.os[V.NN + h.src];
    V.hexinv[h.dst] = V.hexinv[h.src];
  }
  for (int d = 0; d < NLOZ; ++d)
    for (int k = 0; k < 4; ++k) {
      V.oa[k * V.NN + V.id(d, V.n, -1)] = 0.0;   // south-east corner (IPLUSJMINUS)
      V.oa[k * V.NN + V.id(d, -1, V.n)] = 0.0;   // north-west corner (IMINUSJPLUS)
    }
}

static void build(Grid& g, int min_level, int max_level, int domain_level, double radius, double omega) {
  g.S.R = radius;
  g.S.omega = omega;
  g.min_level = min_level;
  g.max_level = max_level;
  g.domain_level = domain_level;
  connections(g);
  g.L.resize(max_level - min_level + 2);
  for (int l = min_level - 1; l <= max_level; ++l) {
    Lev& V = g.at(l);
    alloc(V, l);
    ghost_tables(g, V);
    if (l == min_level - 1) root_coordinates(g, V);
    else child_coordinates(g, g.at(l - 1), V);
    geometry(g, V);
    if (l > min_level - 1) interscale(g, g.at(l - 1), V);
  }
  for (int l = min_level - 1; l <= max_level; ++l) areas_to_ghosts(g.at(l));
}

}  // namespace og

// ----------------------------------------------------------------- C ABI --
extern "C" {

void* orc_grid_build(int min_level, int max_level, int domain_level, double radius, double omega) {
  try {
    og::Grid* g = new og::Grid();
    og::build(*g, min_level, max_level, domain_level, radius, omega);
    return g;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_grid_build: %s\n", e.what());
    return nullptr;
  }
}

void orc_grid_free(void* g) { delete static_cast<og::Grid*>(g); }

// n, P, NN, node ghost entries, edge ghost entries
int orc_grid_dims(void* gp, int l, int64_t* out) {
  og::Grid& g = *static_cast<og::Grid*>(gp);
  if (l < g.min_level - 1 || l > g.max_level) return -1;
  const og::Lev& V = g.at(l);
  out[0] = V.n, out[1] = V.P, out[2] = V.NN, out[3] = (int64_t)V.hn.size(), out[4] = (int64_t)V.he.size();
  return 0;
}

// Copies table `name` of level l into dst (layouts as the product's level descriptors).
int orc_grid_copy(void* gp, int l, const char* name, void* dst) {
  og::Grid& g = *static_cast<og::Grid*>(gp);
  if (l < g.min_level - 1 || l > g.max_level || !name || !dst) return -1;
  const og::Lev& V = g.at(l);
  double* D = static_cast<double*>(dst);
  auto vec = [&](const std::vector<double>& v) { std::memcpy(D, v.data(), v.size() * sizeof(double)); };
  if (!std::strcmp(name, "node")) {
    for (int64_t k = 0; k < V.NN; ++k) D[k] = V.node[k].x, D[V.NN + k] = V.node[k].y, D[2 * V.NN + k] = V.node[k].z;
  } else if (!std::strcmp(name, "ccentre")) {
    for (int t = 0; t < 2; ++t)
      for (int64_t k = 0; k < V.NN; ++k) {
        const og::C3& c = V.cc[t * V.NN + k];
        D[(3 * t + 0) * V.NN + k] = c.x, D[(3 * t + 1) * V.NN + k] = c.y, D[(3 * t + 2) * V.NN + k] = c.z;
      }
  } else if (!std::strcmp(name, "len")) vec(V.len);
  else if (!std::strcmp(name, "pedlen")) vec(V.pedlen);
  else if (!std::strcmp(name, "part")) vec(V.part);
  else if (!std::strcmp(name, "hex_inv")) vec(V.hexinv);
  else if (!std::strcmp(name, "triarea")) vec(V.tri);
  else if (!std::strcmp(name, "coriolis")) vec(V.cor);
  else if (!std::strcmp(name, "overl_a")) vec(V.oa);
  else if (!std::strcmp(name, "overl_split")) vec(V.os);
  else if (!std::strcmp(name, "iu_wgt")) vec(V.iu);
  else if (!std::strcmp(name, "rf_wgt")) vec(V.rf);
  else if (!std::strcmp(name, "halo_node")) {
    int64_t* I = static_cast<int64_t*>(dst);
    for (size_t k = 0; k < V.hn.size(); ++k) I[2 * k] = V.hn[k].dst, I[2 * k + 1] = V.hn[k].src;
  } else if (!std::strcmp(name, "halo_edge")) {
    int64_t* I = static_cast<int64_t*>(dst);
    for (size_t k = 0; k < V.he.size(); ++k) I[3 * k] = V.he[k].dst, I[3 * k + 1] = V.he[k].src, I[3 * k + 2] = V.he[k].sign;
  } else {
    return -1;
  }
  return 0;
}

}  // extern "C"
