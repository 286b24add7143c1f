// ORACLE (test infrastructure only): CPU FP64 restatement of the reference's
// wavelet transforms of the prognostic variables (layer mass, potential
// temperature and velocity, every layer) on a uniform hierarchy of padded
// lozenge levels, the threshold mask and compression.  Imported only by tests/.
//
// Routines, op for op and in evaluation order:
//   forward_wavelet_transform (jmin_in = level_start+1)   src/wavelet.f90:20-98
//   inverse_wavelet_transform                             src/wavelet.f90:208-296
//   Restrict_scalar, Prolong_scalar, Reconstruct_scalar   src/wavelet.f90:520-640
//   Compute_scalar_wavelets, Interp_node                  src/wavelet.f90:642-670,1487-1498
//   Compute_velo_wavelets, Compute_velo_wavelets_penta    src/wavelet.f90:672-781
//   velo_interp_penta_corr                                src/wavelet.f90:927-952
//   Reconstruct_outer_velo, Reconstruct_inner_velo        src/wavelet.f90:954-1003
//   Interp_inner_velo, Interp_outer_velo                  src/wavelet.f90:1005-1094
//   Reconstruct_velo_penta, Restrict_velo                 src/wavelet.f90:1096-1174
//   mask_tol_vars                                         src/mask.f90:102-156
//   compress_wavelets, compress_scalar, compress_vector   src/adapt.f90:79-232
//   WT_after_step                                         src/adapt.f90:192-237
//   adapt's mask sequence without tree surgery            src/adapt.f90:14-65
//     init_masks_zero, mask_active, mask_adj_same_scale, mask_restrict_same_scale,
//     mask_adj_finer_scale, complete_masks, mask_trsk      src/mask.f90:7-100,734-768
//     mask_parent_nodes/edges, mask_adj_same_scale_nodes_edges, mask_restrict_flux,
//     mask_adj_child, mask_edges_consist(2), mask_edges_if_both_nodes,
//     mask_nodes_if_all_edges, prolong_node_adjzone, div_grad_stencil  src/mask.f90:158-867
//     comm_masks (serial comm_masks_mpi)                  src/comm.f90:531-553
//   check_child_required                                  src/refine_patch.f90:289-327
// Iteration sets are those of apply_interscale_d (parents [0, n_par)),
// apply_interscale_d with +1 (parents [0, n_par], "+1 to include poles"),
// apply_interscale_d2 (parents [0, n_par]: every child patch is extended) and
// apply_onescale (nodes [st, n-1+en]) on one domain per lozenge.  Every
// lozenge corner is a pentagon (set_penta).  update_bdry is the level's ghost
// copy (cp_bdry_inside) of every level, applied where the reference's drivers
// call it.
// Reads outside the padded array take 0.  The layers of a transform run on the
// oracle's worker threads (orc_set_threads); layers share no data.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

extern "C" int orc_get_threads(void);  // oracle_trisk.cpp

namespace {

enum { RT = 0, DG = 1, UP = 2 };
enum { LORT = 0, UPLT = 1 };
constexpr int H = 2;
constexpr int FROZEN = 32, TOLRNZ = 16, ADJSPACE = 14, RESTRCT = 12, ADJZONE = 8, TRSK = 2, ZERO = 0;

// Stencil tables of src/shared.f90:287-324 (0-based edge index, k = 0, 1).
const int END_PT[3][2][2] = {{{0, 0}, {1, 0}}, {{1, 1}, {0, 0}}, {{0, 0}, {0, 1}}};
const int OPP_NO[3][2][2] = {{{0, -1}, {1, 1}}, {{0, 1}, {1, 0}}, {{1, 1}, {-1, 0}}};
const int HEX_SIDES[10][3] = {{0, 0, RT},  {0, 0, DG},   {0, 0, UP}, {-1, 0, RT}, {-1, -1, DG},
                              {0, -1, UP}, {0, 0, RT},   {0, 0, DG}, {0, 0, UP},  {-1, 0, RT}};
const int HEX_S_OFFS[3] = {2, 0, 4};
// Iu_Base_Wgt (src/wavelet.f90:1764)
const double IU_BASE[9] = {16.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0, -1.0 / 16.0,
                           -1.0 / 16.0, -1.0 / 16.0, 1.0 / 16.0, 1.0 / 16.0};

}  // namespace

extern "C" {
struct orc_wlevel {
  int level, n, P;
  int64_t NN;
  const double *len, *triarea, *hex_inv, *overl_a, *iu_wgt;  // iu_wgt may be null on the coarsest level
  const int64_t* hn;
  int64_t nhn;
  const int64_t* he;
  int64_t nhe;
  int32_t *mask_n, *mask_e;                                  // [NN], [3*NN]
  double *s_m, *s_t, *s_v;                                   // scaling [nz][NN], [nz][NN], [nz][3*NN]
  double *w_m, *w_t, *w_v;                                   // wavelets, same shapes
};
}

namespace {

// Runs f(k) for the layers k = 0..nz-1 on the oracle's worker count: the
// transforms of different layers share no data, so the order does not matter.
template <class F>
void par_k(int nz, F f) {
  const int nt = std::min(std::max(1, orc_get_threads()), nz);
  if (nt <= 1) {
    for (int k = 0; k < nz; ++k) f(k);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (int k = t; k < nz; k += nt) f(k);
    });
  for (auto& x : th) x.join();
}

struct W {
  orc_wlevel* lv;
  int ls, le, nz;

  orc_wlevel& L(int l) const { return lv[l - ls]; }
  static int64_t id(const orc_wlevel& g, int d, int i, int j) {
    return ((int64_t)d * g.P + (j + H)) * g.P + (i + H);
  }
  static bool in(const orc_wlevel& g, int i, int j) {
    return i >= -H && j >= -H && i < g.n + H && j < g.n + H;
  }
  // node field of one layer
  static double rn(const orc_wlevel& g, const double* f, int d, int i, int j) {
    return in(g, i, j) ? f[id(g, d, i, j)] : 0.0;
  }
  // edge field of one layer (planes of NN)
  static double re(const orc_wlevel& g, const double* f, int e, int d, int i, int j) {
    return in(g, i, j) ? f[(int64_t)e * g.NN + id(g, d, i, j)] : 0.0;
  }
  static double oa(const orc_wlevel& g, int d, int i, int j, int k) {
    return in(g, i, j) ? g.overl_a[(int64_t)(k - 1) * g.NN + id(g, d, i, j)] : 0.0;
  }
  static double hinv(const orc_wlevel& g, int d, int i, int j) { return in(g, i, j) ? g.hex_inv[id(g, d, i, j)] : 0.0; }
  static double len(const orc_wlevel& g, int e, int d, int i, int j) {
    return in(g, i, j) ? g.len[(int64_t)e * g.NN + id(g, d, i, j)] : 0.0;
  }
  static double tri(const orc_wlevel& g, int t, int d, int i, int j) {
    return in(g, i, j) ? g.triarea[(int64_t)t * g.NN + id(g, d, i, j)] : 0.0;
  }
  static int mn(const orc_wlevel& g, int d, int i, int j) { return in(g, i, j) ? g.mask_n[id(g, d, i, j)] : ZERO; }
  static int me(const orc_wlevel& g, int e, int d, int i, int j) {
    return in(g, i, j) ? g.mask_e[(int64_t)e * g.NN + id(g, d, i, j)] : ZERO;
  }
  static double iu(const orc_wlevel& g, int q, int d, int i, int j) {
    return (g.iu_wgt && in(g, i, j)) ? g.iu_wgt[(int64_t)q * g.NN + id(g, d, i, j)] : 0.0;
  }

  // ---- ghost copies (update_bdry of one level, all layers)
  void halo_n(int l, double* f) {
    const orc_wlevel& g = L(l);
    for (int k = 0; k < nz; ++k) {
      double* b = f + (int64_t)k * g.NN;
      for (int64_t q = 0; q < g.nhn; ++q) b[g.hn[2 * q]] = b[g.hn[2 * q + 1]];
    }
  }
  void halo_e(int l, double* f) {
    const orc_wlevel& g = L(l);
    for (int k = 0; k < nz; ++k) {
      double* b = f + (int64_t)k * 3 * g.NN;
      for (int64_t q = 0; q < g.nhe; ++q) {
        const double v = b[g.he[3 * q + 1]];
        b[g.he[3 * q]] = g.he[3 * q + 2] < 0 ? -v : v;
      }
    }
  }
  // update_bdry in the serial build (src/comm_ser.f90) is cp_bdry_inside of
  // the whole field: every level's ghosts, whatever level is named.
  void halo_scalars(int, bool wav) {
    for (int m = ls; m <= le; ++m) {
      orc_wlevel& g = L(m);
      halo_n(m, wav ? g.w_m : g.s_m);
      halo_n(m, wav ? g.w_t : g.s_t);
    }
  }
  void halo_velo(int, bool wav) {
    for (int m = ls; m <= le; ++m) halo_e(m, wav ? L(m).w_v : L(m).s_v);
  }
  void zero_wavelets() {
    for (int l = ls; l <= le; ++l) {
      orc_wlevel& g = L(l);
      for (int64_t q = 0; q < (int64_t)nz * g.NN; ++q) g.w_m[q] = g.w_t[q] = 0.0;
      for (int64_t q = 0; q < (int64_t)nz * 3 * g.NN; ++q) g.w_v[q] = 0.0;
    }
  }

  // ---- scalars (one layer of one variable)
  static double interp_node(const orc_wlevel& C, const double* s, int d, int i, int j, int i1, int j1, int i2, int j2,
                            int i3, int j3, int i4, int j4) {
    return (oa(C, d, i, j, 1) * rn(C, s, d, i1, j1) + oa(C, d, i, j, 2) * rn(C, s, d, i2, j2) +
            oa(C, d, i, j, 3) * rn(C, s, d, i3, j3) + oa(C, d, i, j, 4) * rn(C, s, d, i4, j4)) *
           hinv(C, d, i, j);
  }
  void compute_scalar_wavelets(int l, const double* s, double* wc) {
    const orc_wlevel& C = L(l + 1);
    const int np = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < np; ++jp)
        for (int ip = 0; ip < np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          if (mn(C, d, i + 1, j) >= ADJZONE)
            wc[id(C, d, i + 1, j)] = rn(C, s, d, i + 1, j) - interp_node(C, s, d, i + 1, j, i, j, i + 2, j, i + 2, j + 2, i, j - 2);
          if (mn(C, d, i + 1, j + 1) >= ADJZONE)
            wc[id(C, d, i + 1, j + 1)] =
                rn(C, s, d, i + 1, j + 1) - interp_node(C, s, d, i + 1, j + 1, i + 2, j + 2, i, j, i + 2, j, i, j + 2);
          if (mn(C, d, i, j + 1) >= ADJZONE)
            wc[id(C, d, i, j + 1)] = rn(C, s, d, i, j + 1) - interp_node(C, s, d, i, j + 1, i, j, i, j + 2, i - 2, j, i + 2, j + 2);
        }
  }
  void restrict_scalar(int l, const double* s, const double* wc, double* sp) {
    const orc_wlevel& C = L(l + 1);
    const orc_wlevel& Pa = L(l);
    const int np = Pa.n;
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= np; ++jp)
        for (int ip = 0; ip <= np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          if (mn(C, d, i, j) == 0) continue;
          const double sum =
              rn(C, wc, d, i + 1, j) * oa(C, d, i + 1, j, 1) + rn(C, wc, d, i + 1, j + 1) * oa(C, d, i + 1, j + 1, 2) +
              rn(C, wc, d, i + 2, j + 1) * oa(C, d, i + 2, j + 1, 3) + rn(C, wc, d, i + 1, j + 2) * oa(C, d, i + 1, j + 2, 4) +
              rn(C, wc, d, i, j + 1) * oa(C, d, i, j + 1, 1) + rn(C, wc, d, i - 1, j) * oa(C, d, i - 1, j, 2) +
              rn(C, wc, d, i - 1, j + 1) * oa(C, d, i - 1, j + 1, 3) + rn(C, wc, d, i - 2, j - 1) * oa(C, d, i - 2, j - 1, 4) +
              rn(C, wc, d, i - 1, j - 1) * oa(C, d, i - 1, j - 1, 1) + rn(C, wc, d, i, j - 1) * oa(C, d, i, j - 1, 2) +
              rn(C, wc, d, i - 1, j - 2) * oa(C, d, i - 1, j - 2, 3) + rn(C, wc, d, i + 1, j - 1) * oa(C, d, i + 1, j - 1, 4);
          sp[id(Pa, d, ip, jp)] = rn(C, s, d, i, j) + sum * hinv(Pa, d, ip, jp);
        }
  }
  void prolong_scalar(int l, const double* sp, const double* wc, double* s) {
    const orc_wlevel& C = L(l + 1);
    const orc_wlevel& Pa = L(l);
    const int np = Pa.n;
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= np; ++jp)
        for (int ip = 0; ip <= np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          if (mn(C, d, i, j) == FROZEN) continue;
          const double sum =
              rn(C, wc, d, i + 1, j) * oa(C, d, i + 1, j, 1) + rn(C, wc, d, i + 1, j + 1) * oa(C, d, i + 1, j + 1, 2) +
              rn(C, wc, d, i + 2, j + 1) * oa(C, d, i + 2, j + 1, 3) + rn(C, wc, d, i, j + 1) * oa(C, d, i, j + 1, 1) +
              rn(C, wc, d, i - 1, j) * oa(C, d, i - 1, j, 2) + rn(C, wc, d, i - 1, j + 1) * oa(C, d, i - 1, j + 1, 3) +
              rn(C, wc, d, i - 2, j - 1) * oa(C, d, i - 2, j - 1, 4) + rn(C, wc, d, i - 1, j - 1) * oa(C, d, i - 1, j - 1, 1) +
              rn(C, wc, d, i, j - 1) * oa(C, d, i, j - 1, 2) + rn(C, wc, d, i - 1, j - 2) * oa(C, d, i - 1, j - 2, 3) +
              rn(C, wc, d, i + 1, j - 1) * oa(C, d, i + 1, j - 1, 4);
          s[id(C, d, i, j)] = rn(Pa, sp, d, ip, jp) - sum * hinv(Pa, d, ip, jp);
        }
  }
  void reconstruct_scalar(int l, const double* wc, double* s) {
    const orc_wlevel& C = L(l + 1);
    const int np = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < np; ++jp)
        for (int ip = 0; ip < np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          s[id(C, d, i + 1, j)] = interp_node(C, s, d, i + 1, j, i, j, i + 2, j, i + 2, j + 2, i, j - 2) + rn(C, wc, d, i + 1, j);
          s[id(C, d, i + 1, j + 1)] =
              interp_node(C, s, d, i + 1, j + 1, i + 2, j + 2, i, j, i + 2, j, i, j + 2) + rn(C, wc, d, i + 1, j + 1);
          s[id(C, d, i, j + 1)] = interp_node(C, s, d, i, j + 1, i, j, i, j + 2, i - 2, j, i + 2, j + 2) + rn(C, wc, d, i, j + 1);
        }
  }

  // ---- velocity (one layer)
  // velocity at the parent-level edge ed_idx(ip + off, jp + off, hex side)
  static double ved(const orc_wlevel& Pa, const double* vp, int d, int ip, int jp, const int* off, const int* hs) {
    return re(Pa, vp, hs[2], d, ip + off[0] + hs[0], jp + off[1] + hs[1]);
  }
  // Interp_outer_velo(dom, i_par, j_par, ide, e): child weights at node (ic, jc)
  static double interp_outer(const orc_wlevel& Pa, const orc_wlevel& C, const double* vp, int d, int ip, int jp, int ic,
                             int jc, int e) {
    const int hs = HEX_S_OFFS[e];
    const int* e1 = END_PT[e][0];
    const int* e2 = END_PT[e][1];
    const int* o1 = OPP_NO[e][0];
    const int* o2 = OPP_NO[e][1];
    double t[9];
    t[0] = re(Pa, vp, e, d, ip, jp);
    t[1] = ved(Pa, vp, d, ip, jp, e2, HEX_SIDES[hs + 2]);
    t[2] = ved(Pa, vp, d, ip, jp, e1, HEX_SIDES[hs + 3]);
    t[3] = ved(Pa, vp, d, ip, jp, e1, HEX_SIDES[hs + 5]);
    t[4] = ved(Pa, vp, d, ip, jp, e2, HEX_SIDES[hs + 0]);
    t[5] = ved(Pa, vp, d, ip, jp, o1, HEX_SIDES[hs + 1]) - ved(Pa, vp, d, ip, jp, e1, HEX_SIDES[hs + 2]);
    t[6] = ved(Pa, vp, d, ip, jp, e2, HEX_SIDES[hs + 3]) - ved(Pa, vp, d, ip, jp, o1, HEX_SIDES[hs + 4]);
    t[7] = ved(Pa, vp, d, ip, jp, o2, HEX_SIDES[hs + 4]) - ved(Pa, vp, d, ip, jp, e2, HEX_SIDES[hs + 5]);
    t[8] = ved(Pa, vp, d, ip, jp, e1, HEX_SIDES[hs + 0]) - ved(Pa, vp, d, ip, jp, o2, HEX_SIDES[hs + 1]);
    double sum = 0.0;
    for (int q = 0; q < 9; ++q) sum = sum + (IU_BASE[q] + iu(C, q, d, ic, jc)) * t[q];
    return sum;
  }
  // Interp_inner_velo: the six inner child edges of parent (ip, jp)
  static void interp_inner(const orc_wlevel& Pa, const orc_wlevel& C, const double* vp, const double* v, int d, int ip,
                           int jp, double u[6]) {
    double curl[2];
    for (int t = LORT; t <= UPLT; ++t) {
      const int i1 = ip - t + 1, j1 = jp, i2 = ip, j2 = jp + t;
      curl[t] = (re(Pa, vp, DG, d, ip, jp) * len(Pa, DG, d, ip, jp) + re(Pa, vp, UP, d, i1, j1) * len(Pa, UP, d, i1, j1) +
                 re(Pa, vp, RT, d, i2, j2) * len(Pa, RT, d, i2, j2)) /
                tri(Pa, t, d, ip, jp);
    }
    const int i = 2 * ip, j = 2 * jp;
    auto pr = [&](int e, int a, int b) { return re(C, v, e, d, a, b) * len(C, e, d, a, b); };
    u[0] = (tri(C, LORT, d, i, j) * curl[LORT] - pr(RT, i, j) - pr(DG, i, j)) / len(C, UP, d, i + 1, j);
    u[1] = (tri(C, LORT, d, i + 1, j) * curl[LORT] - pr(RT, i + 1, j) - pr(UP, i + 2, j)) / len(C, DG, d, i + 1, j);
    u[2] = (tri(C, LORT, d, i + 1, j + 1) * curl[LORT] - pr(DG, i + 1, j + 1) - pr(UP, i + 2, j + 1)) /
           len(C, RT, d, i + 1, j + 1);
    u[3] = (tri(C, UPLT, d, i, j) * curl[UPLT] - pr(UP, i, j) - pr(DG, i, j)) / len(C, RT, d, i, j + 1);
    u[4] = (tri(C, UPLT, d, i, j + 1) * curl[UPLT] - pr(UP, i, j + 1) - pr(RT, i, j + 2)) / len(C, DG, d, i, j + 1);
    u[5] = (tri(C, UPLT, d, i + 1, j + 1) * curl[UPLT] - pr(DG, i + 1, j + 1) - pr(RT, i + 1, j + 2)) /
           len(C, UP, d, i + 1, j + 1);
  }
  static double& ee(const orc_wlevel& g, double* f, int e, int d, int i, int j) {
    return f[(int64_t)e * g.NN + id(g, d, i, j)];
  }
  void restrict_velo(int l, const double* v, double* vp) {
    const orc_wlevel& C = L(l + 1);
    const orc_wlevel& Pa = L(l);
    const int np = Pa.n;
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < np; ++jp)
        for (int ip = 0; ip < np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          if (me(C, RT, d, i, j) > 0) ee(Pa, vp, RT, d, ip, jp) = 0.5 * (re(C, v, RT, d, i, j) + re(C, v, RT, d, i + 1, j));
          if (me(C, DG, d, i, j) > 0)
            ee(Pa, vp, DG, d, ip, jp) = 0.5 * (re(C, v, DG, d, i + 1, j + 1) + re(C, v, DG, d, i, j));
          if (me(C, UP, d, i, j) > 0) ee(Pa, vp, UP, d, ip, jp) = 0.5 * (re(C, v, UP, d, i, j) + re(C, v, UP, d, i, j + 1));
        }
  }
  // velo_interp_penta_corr at the south-west corner
  void penta_corr(int l, const double* vp, int d, double u[2]) {
    const orc_wlevel& C = L(l + 1);
    const orc_wlevel& Pa = L(l);
    u[0] = (IU_BASE[8] + iu(C, 8, d, 0, 1)) *
           ((-re(Pa, vp, UP, d, 0, -1) - (-re(Pa, vp, RT, d, -1, -1))) -
            (re(Pa, vp, DG, d, -1, -1) - re(Pa, vp, UP, d, -1, -1)));
    u[1] = (IU_BASE[5] + iu(C, 5, d, 1, 0)) *
           (re(Pa, vp, RT, d, -1, -1) + re(Pa, vp, RT, d, -1, 0) - (re(Pa, vp, RT, d, -1, -1) - re(Pa, vp, DG, d, -1, -1)));
  }
  void compute_velo_wavelets(int l, const double* vp, const double* v, double* wc) {
    const orc_wlevel& C = L(l + 1);
    const orc_wlevel& Pa = L(l);
    const int np = Pa.n, nc = C.n;
    for (int d = 0; d < 10; ++d) {
      for (int jp = 0; jp < np; ++jp)
        for (int ip = 0; ip < np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          for (int e = 0; e < 3; ++e) {
            const int a1 = i + END_PT[e][0][0], b1 = j + END_PT[e][0][1];
            const int a2 = i + END_PT[e][1][0], b2 = j + END_PT[e][1][1];
            if (me(C, e, d, a2, b2) < ADJZONE) continue;
            const double u = interp_outer(Pa, C, vp, d, ip, jp, a2, b2, e);
            ee(C, wc, e, d, a2, b2) = re(C, v, e, d, a2, b2) - u;
            ee(C, wc, e, d, a1, b1) = -ee(C, wc, e, d, a2, b2);
          }
          double u[6];
          interp_inner(Pa, C, vp, v, d, ip, jp, u);
          if (me(C, UP, d, i + 1, j) >= ADJZONE) ee(C, wc, UP, d, i + 1, j) = re(C, v, UP, d, i + 1, j) - u[0];
          if (me(C, DG, d, i + 1, j) >= ADJZONE) ee(C, wc, DG, d, i + 1, j) = re(C, v, DG, d, i + 1, j) - u[1];
          if (me(C, RT, d, i + 1, j + 1) >= ADJZONE) ee(C, wc, RT, d, i + 1, j + 1) = re(C, v, RT, d, i + 1, j + 1) - u[2];
          if (me(C, RT, d, i, j + 1) >= ADJZONE) ee(C, wc, RT, d, i, j + 1) = re(C, v, RT, d, i, j + 1) - u[3];
          if (me(C, DG, d, i, j + 1) >= ADJZONE) ee(C, wc, DG, d, i, j + 1) = re(C, v, DG, d, i, j + 1) - u[4];
          if (me(C, UP, d, i + 1, j + 1) >= ADJZONE) ee(C, wc, UP, d, i + 1, j + 1) = re(C, v, UP, d, i + 1, j + 1) - u[5];
        }
      // Compute_velo_wavelets_penta, corners in the order NE, SE, SW, NW
      {  // SE (IPLUSJMINUS)
        const double vv = (IU_BASE[6] + iu(C, 6, d, nc - 1, 0)) * (re(Pa, vp, RT, d, np, 0) + re(Pa, vp, UP, d, np, -1));
        if (me(C, RT, d, nc - 2, 0) >= ADJZONE) {
          ee(C, wc, RT, d, nc - 2, 0) = ee(C, wc, RT, d, nc - 2, 0) - vv;
          ee(C, wc, RT, d, nc - 1, 0) = ee(C, wc, RT, d, nc - 1, 0) + vv;
        }
      }
      {  // SW (IJMINUS)
        double u[2];
        penta_corr(l, vp, d, u);
        if (me(C, UP, d, 0, 0) >= ADJZONE) {
          ee(C, wc, UP, d, 0, 0) = ee(C, wc, UP, d, 0, 0) + u[0];
          ee(C, wc, UP, d, 0, 1) = ee(C, wc, UP, d, 0, 1) - u[0];
        }
        if (me(C, RT, d, 0, 0) >= ADJZONE) {
          ee(C, wc, RT, d, 0, 0) = ee(C, wc, RT, d, 0, 0) + u[1];
          ee(C, wc, RT, d, 1, 0) = ee(C, wc, RT, d, 1, 0) - u[1];
        }
      }
      {  // NW (IMINUSJPLUS)
        const double vv = -(IU_BASE[7] + iu(C, 7, d, 0, nc - 1)) * (re(Pa, vp, UP, d, 0, np) + re(Pa, vp, RT, d, -1, np));
        if (me(C, UP, d, 0, nc - 2) >= ADJZONE) {
          ee(C, wc, UP, d, 0, nc - 2) = ee(C, wc, UP, d, 0, nc - 2) - vv;
          ee(C, wc, UP, d, 0, nc - 1) = ee(C, wc, UP, d, 0, nc - 1) + vv;
        }
      }
    }
  }
  void reconstruct_outer_velo(int l, const double* vp, const double* wc, double* v) {
    const orc_wlevel& C = L(l + 1);
    const orc_wlevel& Pa = L(l);
    const int np = Pa.n, nc = C.n;
    for (int d = 0; d < 10; ++d) {
      for (int jp = 0; jp <= np; ++jp)
        for (int ip = 0; ip <= np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          for (int e = 0; e < 3; ++e) {
            const int a1 = i + END_PT[e][0][0], b1 = j + END_PT[e][0][1];
            const int a2 = i + END_PT[e][1][0], b2 = j + END_PT[e][1][1];
            const double u = interp_outer(Pa, C, vp, d, ip, jp, a2, b2, e);
            ee(C, v, e, d, a2, b2) = u + re(C, wc, e, d, a2, b2);
            ee(C, v, e, d, a1, b1) = 2.0 * re(Pa, vp, e, d, ip, jp) - ee(C, v, e, d, a2, b2);
          }
        }
      // Reconstruct_velo_penta, corners in the order NE, SE, SW, NW
      {  // SE
        const double vv =
            -(IU_BASE[6] + iu(C, 6, d, nc - 1, 0)) * (re(Pa, vp, RT, d, np, 0) + re(Pa, vp, UP, d, np, -1));
        ee(C, v, RT, d, nc - 2, 0) = ee(C, v, RT, d, nc - 2, 0) - vv;
        ee(C, v, RT, d, nc - 1, 0) = ee(C, v, RT, d, nc - 1, 0) + vv;
      }
      {  // SW
        double u[2];
        penta_corr(l, vp, d, u);
        ee(C, v, UP, d, 0, 0) = ee(C, v, UP, d, 0, 0) - u[0];
        ee(C, v, UP, d, 0, 1) = ee(C, v, UP, d, 0, 1) + u[0];
        ee(C, v, RT, d, 0, 0) = ee(C, v, RT, d, 0, 0) - u[1];
        ee(C, v, RT, d, 1, 0) = ee(C, v, RT, d, 1, 0) + u[1];
      }
      {  // NW
        const double vv = (IU_BASE[7] + iu(C, 7, d, 0, nc - 1)) * (re(Pa, vp, UP, d, 0, np) + re(Pa, vp, RT, d, -1, np));
        ee(C, v, UP, d, 0, nc - 2) = ee(C, v, UP, d, 0, nc - 2) - vv;
        ee(C, v, UP, d, 0, nc - 1) = ee(C, v, UP, d, 0, nc - 1) + vv;
      }
    }
  }
  void reconstruct_inner_velo(int l, const double* vp, const double* wc, double* v) {
    const orc_wlevel& C = L(l + 1);
    const orc_wlevel& Pa = L(l);
    const int np = Pa.n;
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < np; ++jp)
        for (int ip = 0; ip < np; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          double u[6];
          interp_inner(Pa, C, vp, v, d, ip, jp, u);
          ee(C, v, UP, d, i + 1, j) = u[0] + re(C, wc, UP, d, i + 1, j);
          ee(C, v, DG, d, i + 1, j) = u[1] + re(C, wc, DG, d, i + 1, j);
          ee(C, v, RT, d, i + 1, j + 1) = u[2] + re(C, wc, RT, d, i + 1, j + 1);
          ee(C, v, RT, d, i, j + 1) = u[3] + re(C, wc, RT, d, i, j + 1);
          ee(C, v, DG, d, i, j + 1) = u[4] + re(C, wc, DG, d, i, j + 1);
          ee(C, v, UP, d, i + 1, j + 1) = u[5] + re(C, wc, UP, d, i + 1, j + 1);
        }
  }

  // layer pointers
  double* SM(int l, int k) { return L(l).s_m + (int64_t)k * L(l).NN; }
  double* ST(int l, int k) { return L(l).s_t + (int64_t)k * L(l).NN; }
  double* SV(int l, int k) { return L(l).s_v + (int64_t)k * 3 * L(l).NN; }
  double* WM(int l, int k) { return L(l).w_m + (int64_t)k * L(l).NN; }
  double* WT(int l, int k) { return L(l).w_t + (int64_t)k * L(l).NN; }
  double* WV(int l, int k) { return L(l).w_v + (int64_t)k * 3 * L(l).NN; }

  void forward() {
    zero_wavelets();
    for (int l = le - 1; l >= ls; --l) {
      halo_scalars(l + 1, false);
      par_k(nz, [&](int k) {
        compute_scalar_wavelets(l, SM(l + 1, k), WM(l + 1, k));
        compute_scalar_wavelets(l, ST(l + 1, k), WT(l + 1, k));
      });
      halo_scalars(l + 1, true);
      par_k(nz, [&](int k) {
        restrict_scalar(l, SM(l + 1, k), WM(l + 1, k), SM(l, k));
        restrict_scalar(l, ST(l + 1, k), WT(l + 1, k), ST(l, k));
        restrict_velo(l, SV(l + 1, k), SV(l, k));
      });
    }
    for (int l = ls; l <= le; ++l) halo_velo(l, false);
    for (int l = le - 1; l >= ls; --l)
      par_k(nz, [&](int k) { compute_velo_wavelets(l, SV(l, k), SV(l + 1, k), WV(l + 1, k)); });
  }

  void inverse() {
    for (int l = ls; l <= le; ++l) {
      halo_scalars(l, true);
      halo_velo(l, true);
    }
    for (int l = ls; l <= le; ++l) {
      halo_scalars(l, false);
      halo_velo(l, false);
    }
    for (int l = ls; l <= le - 1; ++l) {
      par_k(nz, [&](int k) {
        prolong_scalar(l, SM(l, k), WM(l + 1, k), SM(l + 1, k));
        prolong_scalar(l, ST(l, k), WT(l + 1, k), ST(l + 1, k));
      });
      if (l > ls) halo_velo(l, false);
      halo_scalars(l + 1, false);
      par_k(nz, [&](int k) { reconstruct_outer_velo(l, SV(l, k), WV(l + 1, k), SV(l + 1, k)); });
      halo_velo(l + 1, false);
      par_k(nz, [&](int k) {
        reconstruct_scalar(l, WM(l + 1, k), SM(l + 1, k));
        reconstruct_scalar(l, WT(l + 1, k), ST(l + 1, k));
      });
      par_k(nz, [&](int k) { reconstruct_inner_velo(l, SV(l, k), WV(l + 1, k), SV(l + 1, k)); });
    }
  }

  // mask_tol_vars on nodes [st, n-1+en]^2 of level l
  void mask_tol(int l, int st, int en, const double* thr, int level_fill) {
    orc_wlevel& g = L(l);
    for (int d = 0; d < 10; ++d)
      for (int j = st; j <= g.n - 1 + en; ++j)
        for (int i = st; i <= g.n - 1 + en; ++i) {
          if (!in(g, i, j)) continue;
          const int64_t x = id(g, d, i, j);
          if (g.mask_n[x] == FROZEN) continue;
          bool active = false;
          for (int k = 0; k < nz; ++k) {
            const double wm = g.w_m[(int64_t)k * g.NN + x], wt = g.w_t[(int64_t)k * g.NN + x];
            if (std::fabs(wm) >= thr[0 * nz + k] || l < level_fill) active = true;
            if (std::fabs(wt) >= thr[1 * nz + k] || l < level_fill) active = true;
          }
          if (active)
            g.mask_n[x] = TOLRNZ;
          else if (g.mask_n[x] > ADJZONE)
            g.mask_n[x] = ADJZONE;
          for (int e = 0; e < 3; ++e) {
            const int64_t xe = (int64_t)e * g.NN + x;
            active = false;
            for (int k = 0; k < nz; ++k)
              if (std::fabs(g.w_v[(int64_t)k * 3 * g.NN + xe]) >= thr[2 * nz + k] || l < level_fill) active = true;
            if (active)
              g.mask_e[xe] = TOLRNZ;
            else if (g.mask_e[xe] > ADJZONE)
              g.mask_e[xe] = ADJZONE;
          }
        }
  }

  void compress() {
    for (int l = ls; l <= le; ++l) {
      halo_scalars(l, true);
      halo_velo(l, true);
    }
    par_k(nz, [&](int k) {
      for (int l = ls + 1; l <= le; ++l) {
        orc_wlevel& g = L(l);
        for (int d = 0; d < 10; ++d) {
          for (int j = 0; j <= g.n; ++j)
            for (int i = 0; i <= g.n; ++i) {
              const int64_t x = id(g, d, i, j);
              if (g.mask_n[x] < ADJZONE) {
                WM(l, k)[x] = 0.0;
                WT(l, k)[x] = 0.0;
              }
            }
          for (int j = 0; j < g.n; ++j)
            for (int i = 0; i < g.n; ++i) {
              const int64_t x = id(g, d, i, j);
              for (int e = 0; e < 3; ++e)
                if (g.mask_e[(int64_t)e * g.NN + x] < ADJZONE) WV(l, k)[(int64_t)e * g.NN + x] = 0.0;
            }
        }
      }
    });
  }

  // ---- masks (one level; out-of-array reads are ZERO, writes are skipped)
  static void at_least(int32_t* m, int64_t x, int typ) {
    if (m[x] < typ) m[x] = typ;
  }
  static void sn(orc_wlevel& g, int d, int i, int j, int typ) {
    if (in(g, i, j)) at_least(g.mask_n, id(g, d, i, j), typ);
  }
  static void se(orc_wlevel& g, int e, int d, int i, int j, int typ) {
    if (in(g, i, j)) at_least(g.mask_e, (int64_t)e * g.NN + id(g, d, i, j), typ);
  }
  // serial comm_masks_mpi: every level's node and edge masks to their ghost copies
  void comm_masks() {
    for (int l = ls; l <= le; ++l) {
      orc_wlevel& g = L(l);
      for (int64_t q = 0; q < g.nhn; ++q) g.mask_n[g.hn[2 * q]] = g.mask_n[g.hn[2 * q + 1]];
      for (int64_t q = 0; q < g.nhe; ++q) g.mask_e[g.he[3 * q]] = g.mask_e[g.he[3 * q + 1]];
    }
  }
  void init_masks_zero() {
    for (int l = ls + 1; l <= le; ++l) {
      orc_wlevel& g = L(l);
      for (int64_t x = 0; x < g.NN; ++x) g.mask_n[x] = ZERO;
      for (int64_t x = 0; x < 3 * g.NN; ++x) g.mask_e[x] = ZERO;
    }
  }
  void mask_parent_nodes(int l) {  // parents [0, np]
    orc_wlevel& Pa = L(l);
    orc_wlevel& C = L(l + 1);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= Pa.n; ++jp)
        for (int ip = 0; ip <= Pa.n; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          if (mn(C, d, i + 1, j) == TOLRNZ || mn(C, d, i + 1, j + 1) == TOLRNZ || mn(C, d, i, j + 1) == TOLRNZ ||
              mn(C, d, i - 1, j) == TOLRNZ || mn(C, d, i - 1, j - 1) == TOLRNZ || mn(C, d, i, j - 1) == TOLRNZ) {
            sn(Pa, d, ip, jp, TOLRNZ);
            sn(C, d, i, j, TOLRNZ);
          }
        }
  }
  void mask_parent_edges(int l) {  // parents [0, np)
    orc_wlevel& Pa = L(l);
    orc_wlevel& C = L(l + 1);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < Pa.n; ++jp)
        for (int ip = 0; ip < Pa.n; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          auto T = [&](int e, int a, int b) { return me(C, e, d, a, b) == TOLRNZ; };
          if (T(RT, i, j) || T(RT, i + 1, j) || T(DG, i, j - 1) || T(DG, i + 1, j) || T(UP, i + 1, j) || T(UP, i + 1, j - 1))
            se(Pa, RT, d, ip, jp, TOLRNZ);
          if (T(RT, i, j + 1) || T(RT, i + 1, j + 1) || T(DG, i, j) || T(DG, i + 1, j + 1) || T(UP, i + 1, j + 1) ||
              T(UP, i + 1, j))
            se(Pa, DG, d, ip, jp, TOLRNZ);
          if (T(RT, i, j + 1) || T(RT, i - 1, j + 1) || T(DG, i, j + 1) || T(DG, i - 1, j) || T(UP, i, j) || T(UP, i, j + 1))
            se(Pa, UP, d, ip, jp, TOLRNZ);
        }
  }
  void mask_adj_same_scale(int l) {  // nodes [0, n]
    orc_wlevel& g = L(l);
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= g.n; ++j)
        for (int i = 0; i <= g.n; ++i) {
          if (mn(g, d, i + 1, j) == TOLRNZ || mn(g, d, i + 1, j + 1) == TOLRNZ || mn(g, d, i, j + 1) == TOLRNZ ||
              mn(g, d, i - 1, j) == TOLRNZ || mn(g, d, i - 1, j - 1) == TOLRNZ || mn(g, d, i, j - 1) == TOLRNZ)
            sn(g, d, i, j, ADJSPACE);
          auto T = [&](int e, int a, int b) { return me(g, e, d, a, b) == TOLRNZ; };
          if (T(DG, i, j) || T(UP, i, j - 1) || T(DG, i, j - 1) || T(UP, i + 1, j)) se(g, RT, d, i, j, ADJSPACE);
          if (T(UP, i, j) || T(RT, i, j) || T(UP, i + 1, j) || T(RT, i, j + 1)) se(g, DG, d, i, j, ADJSPACE);
          if (T(DG, i, j) || T(RT, i - 1, j) || T(DG, i - 1, j) || T(RT, i, j + 1)) se(g, UP, d, i, j, ADJSPACE);
        }
  }
  void mask_restrict_flux(int l) {  // nodes [0, n)
    orc_wlevel& g = L(l);
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j < g.n; ++j)
        for (int i = 0; i < g.n; ++i) {
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
  }
  void mask_adj_child(int l) {  // parents [0, np]
    orc_wlevel& Pa = L(l);
    orc_wlevel& C = L(l + 1);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= Pa.n; ++jp)
        for (int ip = 0; ip <= Pa.n; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          auto PE = [&](int e, int a, int b, int typ) { return me(Pa, e, d, a, b) >= typ; };
          if (mn(Pa, d, ip, jp) >= TOLRNZ) {
            const int nb[13][2] = {{0, 0},  {1, 0},  {1, 1},  {0, 1},  {-1, 0}, {-1, -1}, {0, -1},
                                   {-1, 1}, {1, -1}, {2, 1},  {1, 2},  {-1, -2}, {-2, -1}};
            for (auto& q : nb) sn(C, d, i + q[0], j + q[1], ADJZONE);
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
          if (PE(RT, ip, jp, ADJSPACE) || PE(DG, ip, jp, ADJSPACE) || PE(UP, ip, jp, ADJSPACE) ||
              PE(RT, ip - 1, jp, ADJSPACE) || PE(DG, ip - 1, jp - 1, ADJSPACE) || PE(UP, ip, jp - 1, ADJSPACE))
            sn(Pa, d, ip, jp, RESTRCT);
        }
  }
  void mask_edges_if_both_nodes(int l) {  // nodes [0, n)
    orc_wlevel& g = L(l);
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j < g.n; ++j)
        for (int i = 0; i < g.n; ++i)
          if (mn(g, d, i, j) >= ADJZONE) {
            if (mn(g, d, i + 1, j) >= ADJZONE) se(g, RT, d, i, j, ADJZONE);
            if (mn(g, d, i + 1, j + 1) >= ADJZONE) se(g, DG, d, i, j, ADJZONE);
            if (mn(g, d, i, j + 1) >= ADJZONE) se(g, UP, d, i, j, ADJZONE);
          }
  }
  void mask_edges_consist(int l) {  // parents [0, np]
    orc_wlevel& Pa = L(l);
    orc_wlevel& C = L(l + 1);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= Pa.n; ++jp)
        for (int ip = 0; ip <= Pa.n; ++ip) {
          const int i = 2 * ip, j = 2 * jp;
          auto A = [&](int e, int a, int b) { return me(C, e, d, a, b) >= ADJZONE; };
          if (A(RT, i, j) || A(RT, i + 1, j) || A(DG, i, j - 1) || A(DG, i + 1, j) || A(UP, i + 1, j - 1) || A(UP, i + 1, j)) {
            se(C, RT, d, i, j, ADJZONE);
            se(C, RT, d, i + 1, j, ADJZONE);
            se(Pa, RT, d, ip, jp, ADJZONE);
          }
          if (A(RT, i, j + 1) || A(RT, i + 1, j + 1) || A(DG, i, j) || A(DG, i + 1, j + 1) || A(UP, i + 1, j) ||
              A(UP, i + 1, j + 1)) {
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
  }
  void mask_edges_consist2(int l) {  // parents [0, np)
    orc_wlevel& Pa = L(l);
    orc_wlevel& C = L(l + 1);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < Pa.n; ++jp)
        for (int ip = 0; ip < Pa.n; ++ip) {
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
  }
  void mask_nodes_if_all_edges(int l) {  // nodes [0, n]
    orc_wlevel& g = L(l);
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= g.n; ++j)
        for (int i = 0; i <= g.n; ++i)
          if (me(g, RT, d, i, j) >= ADJZONE && me(g, DG, d, i, j) >= ADJZONE && me(g, UP, d, i, j) >= ADJZONE &&
              me(g, RT, d, i - 1, j) >= ADJZONE && me(g, DG, d, i - 1, j - 1) >= ADJZONE && me(g, UP, d, i, j - 1) >= ADJZONE)
            sn(g, d, i, j, ADJZONE);
  }
  void prolong_node_adjzone(int l) {  // parents [0, np]
    orc_wlevel& Pa = L(l);
    orc_wlevel& C = L(l + 1);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= Pa.n; ++jp)
        for (int ip = 0; ip <= Pa.n; ++ip)
          if (mn(C, d, 2 * ip, 2 * jp) >= ADJZONE) sn(Pa, d, ip, jp, ADJZONE);
  }
  void mask_node_trsk(int l) {  // nodes [-2, n+1]: div_grad_stencil (no Laplacian diffusion)
    orc_wlevel& g = L(l);
    for (int d = 0; d < 10; ++d)
      for (int j = -2; j <= g.n + 1; ++j)
        for (int i = -2; i <= g.n + 1; ++i)
          if (mn(g, d, i, j) >= ADJZONE) {
            const int nb[7][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}, {-1, 0}, {-1, -1}, {0, -1}};
            for (auto& q : nb) sn(g, d, i + q[0], j + q[1], TRSK);
            se(g, RT, d, i, j, TRSK);
            se(g, DG, d, i, j, TRSK);
            se(g, UP, d, i, j, TRSK);
            se(g, RT, d, i - 1, j, TRSK);
            se(g, DG, d, i - 1, j - 1, TRSK);
            se(g, UP, d, i, j - 1, TRSK);
          }
  }
  // check_child_required for every parent patch of level l (patch side ps) and
  // child quadrant c = 0 NE, 1 SE, 2 SW, 3 NW (chd_offs).
  void child_required(int l, int ps, uint8_t* out) {
    const orc_wlevel& g = L(l);
    const int np = g.n / ps;
    const int offs[4][2] = {{ps / 2, ps / 2}, {ps / 2, 0}, {0, 0}, {0, ps / 2}};
    int64_t o = 0;
    for (int d = 0; d < 10; ++d)
      for (int pj = 0; pj < np; ++pj)
        for (int pi = 0; pi < np; ++pi)
          for (int c = 0; c < 4; ++c) {
            bool req = false;
            for (int jj = -2; jj <= ps / 2 + 1 && !req; ++jj)
              for (int ii = -2; ii <= ps / 2 + 1 && !req; ++ii) {
                const int i = pi * ps + offs[c][0] + ii, j = pj * ps + offs[c][1] + jj;
                req = mn(g, d, i, j) >= ADJZONE || me(g, RT, d, i, j) >= RESTRCT || me(g, DG, d, i, j) >= RESTRCT ||
                      me(g, UP, d, i, j) >= RESTRCT;
              }
            out[o++] = req ? 1 : 0;
          }
  }
  // adapt (src/adapt.f90:14-65) without tree surgery: every patch exists.
  void mask_build(const double* thr, int level_fill, int max_level, int ps, uint8_t* required) {
    mask_phase1(thr, level_fill, max_level, ps, required, le - 1);
    mask_phase2();
  }
  // adapt up to refine(): init_masks_zero, mask_active, mask_adj_same_scale,
  // mask_restrict_same_scale, then check_child_required of the parent levels
  // ls .. req_hi (refine visits every existing patch, level_end's included).
  void mask_phase1(const double* thr, int level_fill, int max_level, int ps, uint8_t* required, int req_hi) {
    init_masks_zero();
    // mask_active
    for (int l = ls; l <= le; ++l) {
      halo_scalars(l, true);
      halo_velo(l, true);
    }
    mask_tol(le, 0, 1, thr, level_fill);
    comm_masks();
    for (int l = le - 1; l >= ls; --l) {
      mask_tol(l, -1, 2, thr, level_fill);
      mask_parent_nodes(l);
      mask_parent_edges(l);
      comm_masks();
    }
    comm_masks();
    for (int l = ls; l <= le; ++l) mask_adj_same_scale(l);
    comm_masks();
    for (int l = ls; l <= (le < max_level - 1 ? le : max_level - 1); ++l) mask_restrict_flux(l);
    comm_masks();
    if (required) {
      uint8_t* o = required;
      for (int l = ls; l <= req_hi; ++l) {
        child_required(l, ps, o);
        o += (int64_t)10 * (L(l).n / ps) * (L(l).n / ps) * 4;
      }
    }
  }
  // adapt after refine() (post_refine's comm_masks, mask_adj_finer_scale,
  // complete_masks, mask_trsk) on levels ls .. le, le being the level_end that
  // refine left.
  void mask_phase2() {
    comm_masks();  // post_refine
    for (int l = le - 1; l >= ls; --l) {
      mask_adj_child(l);
      mask_edges_if_both_nodes(l + 1);
    }
    comm_masks();
    // complete_masks
    for (int l = le - 1; l >= ls + 1; --l) {
      mask_edges_consist(l);
      comm_masks();
      mask_edges_consist2(l);
      comm_masks();
    }
    if (ls < le) {
      mask_edges_consist(ls);
      comm_masks();
      comm_masks();
    }
    for (int l = le - 1; l >= ls + 1; --l) {
      mask_nodes_if_all_edges(l + 1);
      prolong_node_adjzone(l);
    }
    if (ls + 1 <= le) mask_nodes_if_all_edges(ls + 1);
    comm_masks();
    // mask_trsk
    for (int l = ls; l <= le; ++l) mask_node_trsk(l);
  }

  void wt_after_step() {
    zero_wavelets();
    for (int l = ls; l <= le; ++l) {
      halo_scalars(l, false);
      halo_velo(l, false);
    }
    par_k(nz, [&](int k) {
      for (int l = ls; l <= le - 1; ++l) {
        compute_scalar_wavelets(l, SM(l + 1, k), WM(l + 1, k));
        compute_scalar_wavelets(l, ST(l + 1, k), WT(l + 1, k));
        compute_velo_wavelets(l, SV(l, k), SV(l + 1, k), WV(l + 1, k));
      }
    });
    compress();
    inverse();
  }
};

}  // namespace

extern "C" {

int orc_wt_forward(orc_wlevel* lv, int ls, int le, int nz) {
  W w{lv, ls, le, nz};
  w.forward();
  return 0;
}

int orc_wt_inverse(orc_wlevel* lv, int ls, int le, int nz) {
  W w{lv, ls, le, nz};
  w.inverse();
  return 0;
}

// mask_active's threshold pass: level_end on (0, 1), coarser levels on (-1, 2)
// after the ghost copy of the wavelets (update_bdry1(wav_coeff, ...)).
int orc_mask_tol(orc_wlevel* lv, int ls, int le, int nz, const double* threshold, int level_fill) {
  W w{lv, ls, le, nz};
  for (int l = ls; l <= le; ++l) {
    w.halo_scalars(l, true);
    w.halo_velo(l, true);
  }
  w.mask_tol(le, 0, 1, threshold, level_fill);
  for (int l = le - 1; l >= ls; --l) w.mask_tol(l, -1, 2, threshold, level_fill);
  return 0;
}

int orc_mask_build(orc_wlevel* lv, int ls, int le, int nz, const double* threshold, int level_fill, int max_level,
                   int patch_size, uint8_t* child_required) {
  W w{lv, ls, le, nz};
  w.mask_build(threshold, level_fill, max_level, patch_size, child_required);
  return 0;
}

// The two halves of adapt's mask sequence around refine(): the first on levels
// ls..le with the check_child_required flags of parent levels ls..req_hi, the
// second on ls..le as refine left level_end.
int orc_mask_phase1(orc_wlevel* lv, int ls, int le, int nz, const double* threshold, int level_fill, int max_level,
                    int patch_size, uint8_t* child_required, int req_hi) {
  W w{lv, ls, le, nz};
  w.mask_phase1(threshold, level_fill, max_level, patch_size, child_required, req_hi);
  return 0;
}

int orc_mask_phase2(orc_wlevel* lv, int ls, int le, int nz) {
  W w{lv, ls, le, nz};
  w.mask_phase2();
  return 0;
}

// mask_adj_child of the parents of level l (l in [ls, le-1]) alone, as
// init_structures applies it to the root level (src/main.f90:514).
int orc_mask_adj_child(orc_wlevel* lv, int ls, int le, int nz, int l) {
  if (l < ls || l >= le) return 1;
  W w{lv, ls, le, nz};
  w.mask_adj_child(l);
  return 0;
}

int orc_compress(orc_wlevel* lv, int ls, int le, int nz) {
  W w{lv, ls, le, nz};
  w.compress();
  return 0;
}

int orc_wt_after_step(orc_wlevel* lv, int ls, int le, int nz) {
  W w{lv, ls, le, nz};
  w.wt_after_step();
  return 0;
}

}  // extern "C"
