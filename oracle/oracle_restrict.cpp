// ORACLE (test infrastructure only): CPU FP64 restatement of the reference's
// coarse-level compute-or-restrict operators of the multi-level trend, on one
// parent/child pair of uniform padded lozenge levels.  Imported only by tests/.
//
// Routines, op for op and in evaluation order:
//   cpt_or_restr_scalar, scalar_cpt_restr        src/multi_level.f90:311-345
//   cpt_or_restr_u_source, u_source_cpt_restr    src/multi_level.f90:347-392
//     (restriction part; the parent's own u_source is the single-level trend)
//   cpt_or_restr_flux, flux_cpt_restr            src/multi_level.f90:394-451
//   interp_flux                                  src/multi_level.f90:453-482
//   complete_coarse_flux                         src/multi_level.f90:484-508
//   part_coarse_flux                             src/multi_level.f90:510-538
//   coarse_flux                                  src/multi_level.f90:540-573
//   get_indices                                  src/multi_level.f90:617-659
// Iteration sets: apply_interscale_to_patch3(.., 0, 1) visits parents
// [0, n_par]^2 of each lozenge; flux_cpt_restr returns for children at
// PATCH_SIZE, leaving parents [0, n_par)^2; apply_interscale_to_patch(.., 0, 0)
// visits parents [0, n_par)^2.  The child flux and child dscalar are
// ghost-copied first (update_bdry of level l+1 in trend_ml).  A read of dscalar
// outside the padded child level returns 0 and is counted when the area weight
// it multiplies is non-zero (the reference reads past its 2-cell boundary patch
// there).
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle_restrict.h"

namespace {

enum { RT = 0, DG = 1, UP = 2 };
constexpr int RESTRCT = 12, ADJZONE = 8;
enum { UZM = 0, UPZ, UMZ, UZP, VMM, VPM, VMP, VPP, WMM, WPM, WMP, WPP, WMMM, WPPP, VMPP, VPMM };

// src/shared.f90:285-330
const int NGHB_PT[10][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 0}, {-1, -1}, {0, -1}, {1, 0}, {1, 1}, {0, 1}, {-1, 0}};
const int HEX_SIDES[10][3] = {{0, 0, RT},  {0, 0, DG}, {0, 0, UP}, {-1, 0, RT}, {-1, -1, DG},
                              {0, -1, UP}, {0, 0, RT}, {0, 0, DG}, {0, 0, UP},  {-1, 0, RT}};
const int HEX_S_OFFS[3] = {2, 0, 4};
const int BFLY_NO2[3][4][2] = {{{-3, -2}, {1, -2}, {3, 2}, {-1, 2}},
                               {{1, 3}, {-3, -1}, {-1, -3}, {3, 1}},
                               {{2, -1}, {2, 3}, {-2, 1}, {-2, -3}}};

struct Lv {
  const orc_rlevel& g;
  int d;
  bool in(int i, int j) const { return i >= -2 && j >= -2 && i < g.n + 2 && j < g.n + 2; }
  int64_t id(int i, int j) const { return ((int64_t)d * g.P + j + 2) * g.P + i + 2; }
  int64_t ed(int i, int j, const int* hs) const { return (int64_t)hs[2] * g.NN + id(i + hs[0], j + hs[1]); }
  double a(int i, int j, int k) const { return g.overl_a[(int64_t)k * g.NN + id(i, j)]; }
  double split(int i, int j, int k) const { return g.overl_split[(int64_t)k * g.NN + id(i, j)]; }
  double hinv(int i, int j) const { return g.hex_inv[id(i, j)]; }
  const double* rf(int i, int j, double out[3]) const {
    for (int c = 0; c < 3; ++c) out[c] = g.rf_wgt[(int64_t)c * g.NN + id(i, j)];
    return out;
  }
};

// get_indices: edge slots (plane*NN + node) of the 16 stencil fluxes and the four
// diagonal neighbours MP, PP, PM, MM as (i, j).
struct Ind {
  int64_t e[16];
  int nb[4][2];  // MP, PP, PM, MM
};

Ind get_indices(const Lv& C, int i, int j, int e) {
  Ind r;
  const int hs = HEX_S_OFFS[e];
  r.e[UMZ] = C.ed(i, j, HEX_SIDES[hs + 1]);
  r.e[UPZ] = C.ed(i, j, HEX_SIDES[hs + 4]);
  r.e[WMP] = C.ed(i, j, HEX_SIDES[hs + 0]);
  r.e[VPP] = C.ed(i, j, HEX_SIDES[hs + 5]);
  r.e[WPM] = C.ed(i, j, HEX_SIDES[hs + 3]);
  r.e[VMM] = C.ed(i, j, HEX_SIDES[hs + 2]);
  const int off[4] = {0, 5, 3, 2};
  for (int q = 0; q < 4; ++q) {
    r.nb[q][0] = i + NGHB_PT[hs + off[q]][0];
    r.nb[q][1] = j + NGHB_PT[hs + off[q]][1];
  }
  const int *mp = r.nb[0], *pp = r.nb[1], *pm = r.nb[2], *mm = r.nb[3];
  r.e[VMP] = C.ed(mp[0], mp[1], HEX_SIDES[hs + 2]);
  r.e[VMPP] = C.ed(mp[0], mp[1], HEX_SIDES[hs + 5]);
  r.e[UZP] = C.ed(mp[0], mp[1], HEX_SIDES[hs + 4]);
  r.e[WPPP] = C.ed(pp[0], pp[1], HEX_SIDES[hs + 0]);
  r.e[WPP] = C.ed(pp[0], pp[1], HEX_SIDES[hs + 3]);
  r.e[VPM] = C.ed(pm[0], pm[1], HEX_SIDES[hs + 5]);
  r.e[VPMM] = C.ed(pm[0], pm[1], HEX_SIDES[hs + 2]);
  r.e[UZM] = C.ed(pm[0], pm[1], HEX_SIDES[hs + 1]);
  r.e[WMMM] = C.ed(mm[0], mm[1], HEX_SIDES[hs + 3]);
  r.e[WMM] = C.ed(mm[0], mm[1], HEX_SIDES[hs + 0]);
  return r;
}

// Fortran SUM of three products, first to last.
inline double sum3(const double* h, const int64_t* e, const int s[3], const double w[3]) {
  double t = h[e[s[0]]] * w[0];
  t = t + h[e[s[1]]] * w[1];
  return t + h[e[s[2]]] * w[2];
}
inline double sum3d(const double* h, const int64_t* e, const int p[3], const int m[3], const double w[3]) {
  double t = (h[e[p[0]]] - h[e[m[0]]]) * w[0];
  t = t + (h[e[p[1]]] - h[e[m[1]]]) * w[1];
  return t + (h[e[p[2]]] - h[e[m[2]]]) * w[2];
}

struct Restrict {
  const Lv C;
  const double* h;   // child flux, one layer, ghost-copied
  const double* ds;  // child dscalar, one layer, ghost-copied
  int64_t oob = 0;

  double dsr(int i, int j, double wgt) {
    if (!C.in(i, j)) {
      if (wgt != 0.0) ++oob;
      return 0.0;
    }
    return ds[C.id(i, j)];
  }

  void interp_flux(int i, int j, double sm[4]) {
    double w0[3], w1[3];
    Ind id = get_indices(C, i + 1, j, RT);
    {
      const int a[3] = {WPM, UZM, VMM}, p[3] = {VPM, WMMM, UMZ}, m[3] = {UPZ, VPMM, WMM};
      sm[0] = -sum3(h, id.e, a, C.rf(i + 1, j - 2, w0)) - sum3d(h, id.e, p, m, C.rf(i + 1, j - 1, w1));
    }
    {
      const int a[3] = {WMP, UZP, VPP}, p[3] = {VMP, WPPP, UPZ}, m[3] = {UMZ, VMPP, WPP};
      sm[1] = sum3(h, id.e, a, C.rf(i, j, w0)) + sum3d(h, id.e, p, m, C.rf(i, j + 1, w1));
    }
    id = get_indices(C, i, j + 1, UP);
    {
      const int a[3] = {UZM, VMM, WPM}, p[3] = {WMMM, UMZ, VPM}, m[3] = {VPMM, WMM, UPZ};
      sm[2] = -sum3(h, id.e, a, C.rf(i + 1, j, w0)) - sum3d(h, id.e, p, m, C.rf(i + 1, j + 1, w1));
    }
    {
      const int a[3] = {UZP, VPP, WMP}, p[3] = {WPPP, UPZ, VMP}, m[3] = {VMPP, WPP, UMZ};
      sm[3] = sum3(h, id.e, a, C.rf(i - 2, j, w0)) + sum3d(h, id.e, p, m, C.rf(i - 2, j + 1, w1));
    }
  }

  double part_coarse_flux(int i, int j, int e) {
    const Ind id = get_indices(C, i, j, e);
    double area[2] = {C.a(i, j, 0), C.a(i, j, 1)};
    double ol[4];
    ol[0] = C.split(i, j, 0);
    ol[1] = C.split(i, j, 1);
    ol[2] = C.a(i, j, 2) - ol[0];
    ol[3] = C.a(i, j, 3) - ol[1];
    area[0] = area[0] + ol[0] + ol[3];
    area[1] = area[1] + ol[1] + ol[2];
    const double s = area[0] + area[1];
    area[0] = area[0] / s;
    area[1] = area[1] / s;
    const int *mp = id.nb[0], *pp = id.nb[1], *pm = id.nb[2], *mm = id.nb[3];
    ol[0] = C.split(pp[0], pp[1], 0);
    ol[1] = C.split(mm[0], mm[1], 1);
    ol[2] = C.a(mp[0], mp[1], 2) - C.split(mp[0], mp[1], 0);
    ol[3] = C.a(pm[0], pm[1], 3) - C.split(pm[0], pm[1], 1);
    double t = h[id.e[UPZ]] * area[0];
    t = t + h[id.e[UMZ]] * area[1];
    t = t - (h[id.e[VMM]] + h[id.e[WMP]]) * area[1];
    t = t - (h[id.e[WPM]] + h[id.e[VPP]]) * area[0];
    t = t + ol[2] * ds[C.id(mp[0], mp[1])];
    t = t - ol[3] * ds[C.id(pm[0], pm[1])];
    t = t - ol[0] * ds[C.id(pp[0], pp[1])];
    return t + ol[1] * ds[C.id(mm[0], mm[1])];
  }

  double coarse_flux(int i, int j, int e) {
    const int hs = HEX_S_OFFS[e];
    auto nb = [&](int k, int& x, int& y) { x = i + NGHB_PT[hs + k][0]; y = j + NGHB_PT[hs + k][1]; };
    int mz[2], pz[2], mp[2], pp[2], pm[2], mm[2];
    nb(1, mz[0], mz[1]);
    nb(4, pz[0], pz[1]);
    nb(0, mp[0], mp[1]);
    nb(5, pp[0], pp[1]);
    nb(3, pm[0], pm[1]);
    nb(2, mm[0], mm[1]);
    const int(*b2)[2] = BFLY_NO2[e];
    const double wpp = C.a(pp[0], pp[1], 2) * C.a(pp[0], pp[1], 3) * C.hinv(pp[0], pp[1]);
    const double wpm = C.a(pm[0], pm[1], 2) * C.a(pm[0], pm[1], 3) * C.hinv(pm[0], pm[1]);
    const double wmp = C.a(mp[0], mp[1], 2) * C.a(mp[0], mp[1], 3) * C.hinv(mp[0], mp[1]);
    const double wmm = C.a(mm[0], mm[1], 2) * C.a(mm[0], mm[1], 3) * C.hinv(mm[0], mm[1]);
    const double d_mm2 = dsr(i + b2[0][0], j + b2[0][1], wmm);
    const double d_pm2 = dsr(i + b2[1][0], j + b2[1][1], wpm);
    const double d_pp2 = dsr(i + b2[2][0], j + b2[2][1], wpp);
    const double d_mp2 = dsr(i + b2[3][0], j + b2[3][1], wmp);
    const double dmz = ds[C.id(mz[0], mz[1])], dpz = ds[C.id(pz[0], pz[1])];
    double c = C.a(i, j, 0) * C.a(i, j, 1) * C.hinv(i, j);
    c = c + C.a(mp[0], mp[1], 1) * C.a(mp[0], mp[1], 2) * C.hinv(mp[0], mp[1]);
    c = c + C.a(pp[0], pp[1], 0) * C.a(pp[0], pp[1], 2) * C.hinv(pp[0], pp[1]);
    c = c + C.a(pm[0], pm[1], 0) * C.a(pm[0], pm[1], 3) * C.hinv(pm[0], pm[1]);
    c = c + C.a(mm[0], mm[1], 1) * C.a(mm[0], mm[1], 3) * C.hinv(mm[0], mm[1]);
    double t = c * (dpz - dmz);
    t = t + wpp * 0.5 * (d_pp2 - dmz);
    t = t + wpm * 0.5 * (d_pm2 - dmz);
    t = t + wmp * 0.5 * (dpz - d_mp2);
    return t + wmm * 0.5 * (dpz - d_mm2);
  }

  double complete(const double sm[4], int ic, int jc, int e) {
    if (e == RT) {
      const double p = part_coarse_flux(ic + 1, jc, RT), c = coarse_flux(ic + 1, jc, RT);
      return p + c + sm[0] + sm[1];
    }
    if (e == DG) {
      const double p = part_coarse_flux(ic + 1, jc + 1, DG), c = coarse_flux(ic + 1, jc + 1, DG);
      return p + c + sm[1] + sm[2];
    }
    const double p = part_coarse_flux(ic, jc + 1, UP), c = coarse_flux(ic, jc + 1, UP);
    return p + c + sm[2] + sm[3];
  }
};

void halo_nodes(const orc_rlevel& g, double* f) {
  for (int64_t q = 0; q < g.nhn; ++q) f[g.hn[2 * q]] = f[g.hn[2 * q + 1]];
}
void halo_edges(const orc_rlevel& g, double* f) {
  for (int64_t q = 0; q < g.nhe; ++q) {
    const double v = f[g.he[3 * q + 1]];
    f[g.he[3 * q]] = g.he[3 * q + 2] < 0 ? -v : v;
  }
}

}  // namespace

extern "C" {

// scalar_cpt_restr of the node scalar `scal` from child to parent, every layer.
int orc_restrict_scalar(const orc_rlevel* par, const orc_rlevel* chd, int nz) {
  for (int k = 0; k < nz; ++k)
    for (int d = 0; d < 10; ++d) {
      Lv Pa{*par, d}, C{*chd, d};
      double* sp = par->scal + (int64_t)k * par->NN;
      const double* sc = chd->scal + (int64_t)k * chd->NN;
      for (int jp = 0; jp <= par->n; ++jp)
        for (int ip = 0; ip <= par->n; ++ip)
          if (par->mask_n[Pa.id(ip, jp)] >= RESTRCT) sp[Pa.id(ip, jp)] = sc[C.id(2 * ip, 2 * jp)];
    }
  return 0;
}

// flux_cpt_restr from the child's flux and dscalar, every layer.  Returns the
// number of non-zero-weighted dscalar reads outside the padded child level.
int64_t orc_restrict_flux(const orc_rlevel* par, const orc_rlevel* chd, int nz) {
  int64_t oob = 0;
  std::vector<double> hc(3 * chd->NN), dc(chd->NN);
  for (int k = 0; k < nz; ++k) {
    std::memcpy(hc.data(), chd->flux + 3 * k * chd->NN, 3 * chd->NN * sizeof(double));
    std::memcpy(dc.data(), chd->dscal + k * chd->NN, chd->NN * sizeof(double));
    halo_edges(*chd, hc.data());
    halo_nodes(*chd, dc.data());
    double* fp = par->flux + 3 * k * par->NN;
    for (int d = 0; d < 10; ++d) {
      Lv Pa{*par, d};
      Restrict R{Lv{*chd, d}, hc.data(), dc.data()};
      for (int jp = 0; jp < par->n; ++jp)
        for (int ip = 0; ip < par->n; ++ip) {
          const int64_t idp = Pa.id(ip, jp);
          const int32_t* me = par->mask_e;
          const int m0 = me[idp], m1 = me[par->NN + idp], m2 = me[2 * par->NN + idp];
          int mx = m0 > m1 ? m0 : m1;
          mx = mx > m2 ? mx : m2;
          double sm[4] = {0.0, 0.0, 0.0, 0.0};
          if (mx >= RESTRCT) R.interp_flux(2 * ip, 2 * jp, sm);
          if (m0 >= RESTRCT) fp[idp] = R.complete(sm, 2 * ip, 2 * jp, RT);
          if (m1 >= RESTRCT) fp[par->NN + idp] = R.complete(sm, 2 * ip, 2 * jp, DG);
          if (m2 >= RESTRCT) fp[2 * par->NN + idp] = R.complete(sm, 2 * ip, 2 * jp, UP);
        }
      oob += R.oob;
    }
  }
  return oob;
}

// Restriction part of u_source_cpt_restr, every layer.
int orc_restrict_u_source(const orc_rlevel* par, const orc_rlevel* chd, int nz) {
  for (int k = 0; k < nz; ++k) {
    double* vp = par->dvelo + 3 * k * par->NN;
    const double* vc = chd->dvelo + 3 * k * chd->NN;
    const int64_t NC = chd->NN, NP = par->NN;
    for (int d = 0; d < 10; ++d) {
      Lv Pa{*par, d}, C{*chd, d};
      for (int jp = 0; jp < par->n; ++jp)
        for (int ip = 0; ip < par->n; ++ip) {
          const int64_t idp = Pa.id(ip, jp), idc = C.id(2 * ip, 2 * jp);
          const int64_t idE = C.id(2 * ip + 1, 2 * jp), idNE = C.id(2 * ip + 1, 2 * jp + 1),
                        idN = C.id(2 * ip, 2 * jp + 1);
          if (chd->mask_e[idc] >= ADJZONE) vp[idp] = vc[idc] + vc[idE];
          if (chd->mask_e[NC + idc] >= ADJZONE) vp[NP + idp] = vc[NC + idc] + vc[NC + idNE];
          if (chd->mask_e[2 * NC + idc] >= ADJZONE) vp[2 * NP + idp] = vc[2 * NC + idc] + vc[2 * NC + idN];
        }
    }
  }
  return 0;
}

}  // extern "C"
