// ORACLE (test infrastructure only): CPU FP64 restatement of the barotropic
// pieces of the reference's mode-split step on one uniform level of padded
// lozenge arrays.  Imported only by tests/.
//
// Routines, op for op:
//   flux_divergence (one level)               src/barotropic_2d.f90:326-366
//   step1 itype 4 (comput :229-244, comp_SW :420-437)    src/ops.f90
//   cal_div, div                              src/ops.f90:1325-1355
//   rhs_elliptic, cal_rhs_elliptic            src/barotropic_2d.f90:151-185
//   grad_eta (one level)                      src/barotropic_2d.f90:455-474
//   step1 itype 3 (comput :225-228, comp_SW :416-419), porosity 1   src/ops.f90
//   u_update                                  src/barotropic_2d.f90:131-149
//   step1 itypes 1, 5, 6, 7 (comput :198-262, comp_SW :396-455)     src/ops.f90
//   step1 itype 8 (comput :256-271, comp_SW :460-471) + post_vort :1159-1228
//     in the reference's visiting order for a patch covering the lozenge:
//     nodes [0, n)^2 row by row, the north row and (n, n), the east column.
//   flux_divergence over a hierarchy, with cpt_or_restr_flux    src/barotropic_2d.f90:326-366
//   rhs_elliptic over a hierarchy                               src/barotropic_2d.f90:151-185
//   grad_eta over a hierarchy, with cpt_or_restr_eta            src/barotropic_2d.f90:414-474
//   u_update over a hierarchy                                   src/barotropic_2d.f90:131-149
// In grad_eta the restricted copy of eta is not ghost-copied again: the west
// and south ghosts keep the values of the first update_bdry, the east and
// north ghost rows (parents [0, n]) are restricted directly.
// step1 visits nodes [0, n]^2 of each lozenge and runs comp_SW on the south
// and west borders; update_bdry is the level's ghost copy.  u_update is
// applied to the edges grad_eta writes (the reference's element range also
// covers ghost edges, which the next ghost copy overwrites).
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle_restrict.h"

extern "C" {
struct orc_blevel {
  int n, P;
  int64_t NN;
  const double *len, *pedlen, *hex_inv;
  const int64_t* hn;
  int64_t nhn;
  const int64_t* he;
  int64_t nhe;
};
}

namespace {

enum { RT = 0, DG = 1, UP = 2 };

inline double interp(double a, double b) { return 0.5 * (a + b); }

struct B {
  const orc_blevel& L;
  int64_t id(int d, int i, int j) const { return ((int64_t)d * L.P + j + 2) * L.P + i + 2; }
  void halo_n(double* f) const {
    for (int64_t q = 0; q < L.nhn; ++q) f[L.hn[2 * q]] = f[L.hn[2 * q + 1]];
  }
  void halo_e(double* f) const {
    for (int64_t q = 0; q < L.nhe; ++q) {
      const double v = f[L.he[3 * q + 1]];
      f[L.he[3 * q]] = L.he[3 * q + 2] < 0 ? -v : v;
    }
  }
};

}  // namespace

extern "C" {

int orc_rhs_elliptic(const orc_blevel* Lp, int nz, const double* mass, const double* mean_m, const double* velo,
                     const double* eta, const double* div_old, double dt, double theta2, double rho0, double* hflux,
                     double* div, double* rhs) {
  const orc_blevel& L = *Lp;
  B b{L};
  const int64_t NN = L.NN;
  const int P = L.P;
  std::vector<double> m(mass, mass + nz * NN), v(velo, velo + 3 * nz * NN), e(eta, eta + NN), dold(div_old, div_old + NN);
  for (int k = 0; k < nz; ++k) {
    b.halo_n(m.data() + k * NN);
    b.halo_e(v.data() + 3 * k * NN);
  }
  b.halo_n(e.data());
  b.halo_n(dold.data());
  std::memset(hflux, 0, 3 * NN * sizeof(double));
  // step1 itype 4
  for (int d = 0; d < 10; ++d)
    for (int j = 0; j <= L.n; ++j)
      for (int i = 0; i <= L.n; ++i) {
        const int64_t id = b.id(d, i, j);
        const int64_t idE = id + 1, idN = id + P, idNE = id + P + 1, idW = id - 1, idS = id - P, idSW = id - P - 1;
        double f[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < nz; ++k) {
          const double* M = m.data() + k * NN;
          const double* A = mean_m + k * NN;
          const double* V = v.data() + 3 * k * NN;
          const double dz0 = M[id] + A[id];
          double dz = interp(dz0, M[idE] + A[idE]);
          f[RT] = f[RT] + V[RT * NN + id] * dz;
          dz = interp(dz0, M[idNE] + A[idNE]);
          f[DG] = f[DG] + V[DG * NN + id] * dz;
          dz = interp(dz0, M[idN] + A[idN]);
          f[UP] = f[UP] + V[UP * NN + id] * dz;
        }
        for (int q = 0; q < 3; ++q) hflux[q * NN + id] = f[q] * L.pedlen[q * NN + id];
        if (i == 0 || j == 0) {  // comp_SW
          double g[3] = {0.0, 0.0, 0.0};
          for (int k = 0; k < nz; ++k) {
            const double* M = m.data() + k * NN;
            const double* A = mean_m + k * NN;
            const double* V = v.data() + 3 * k * NN;
            const double dz0 = M[id] + A[id];
            double dz = interp(dz0, M[idW] + A[idW]);
            g[0] = g[0] + V[RT * NN + idW] * dz;
            dz = interp(dz0, M[idSW] + A[idSW]);
            g[1] = g[1] + V[DG * NN + idSW] * dz;
            dz = interp(dz0, M[idS] + A[idS]);
            g[2] = g[2] + V[UP * NN + idS] * dz;
          }
          hflux[RT * NN + idW] = g[0] * L.pedlen[RT * NN + idW];
          hflux[DG * NN + idSW] = g[1] * L.pedlen[DG * NN + idSW];
          hflux[UP * NN + idS] = g[2] * L.pedlen[UP * NN + idS];
        }
      }
  b.halo_e(hflux);
  std::memset(div, 0, NN * sizeof(double));
  for (int d = 0; d < 10; ++d)
    for (int j = 0; j <= L.n; ++j)
      for (int i = 0; i <= L.n; ++i) {
        const int64_t id = b.id(d, i, j);
        div[id] = (hflux[RT * NN + id] - hflux[RT * NN + id - 1] + hflux[DG * NN + id - P - 1] - hflux[DG * NN + id] +
                   hflux[UP * NN + id] - hflux[UP * NN + id - P]) *
                  L.hex_inv[id];
      }
  b.halo_n(div);
  std::memset(rhs, 0, NN * sizeof(double));
  for (int d = 0; d < 10; ++d)
    for (int j = 0; j <= L.n; ++j)
      for (int i = 0; i <= L.n; ++i) {
        const int64_t id = b.id(d, i, j);
        rhs[id] = -e[id] + dt * (theta2 * div[id] + (1.0 - theta2) * dold[id]) / rho0;
      }
  return 0;
}

int orc_u_update(const orc_blevel* Lp, int nz, double grav, const double* eta, double dt, double theta1, double* velo,
                 double* grad) {
  const orc_blevel& L = *Lp;
  B b{L};
  const int64_t NN = L.NN;
  const int P = L.P;
  std::vector<double> e(eta, eta + NN);
  b.halo_n(e.data());
  std::memset(grad, 0, 3 * NN * sizeof(double));
  std::vector<char> written(3 * NN, 0);
  for (int d = 0; d < 10; ++d)
    for (int j = 0; j <= L.n; ++j)
      for (int i = 0; i <= L.n; ++i) {
        const int64_t id = b.id(d, i, j);
        grad[RT * NN + id] = grav * (e[id + 1] / 1.0 - e[id] / 1.0) / L.len[RT * NN + id];
        grad[DG * NN + id] = grav * (e[id] / 1.0 - e[id + P + 1] / 1.0) / L.len[DG * NN + id];
        grad[UP * NN + id] = grav * (e[id + P] / 1.0 - e[id] / 1.0) / L.len[UP * NN + id];
        written[RT * NN + id] = written[DG * NN + id] = written[UP * NN + id] = 1;
        if (i == 0 || j == 0) {  // comp_SW
          grad[RT * NN + id - 1] = -(grav * (e[id - 1] / 1.0 - e[id] / 1.0) / L.len[RT * NN + id - 1]);
          grad[DG * NN + id - P - 1] = -(grav * (e[id] / 1.0 - e[id - P - 1] / 1.0) / L.len[DG * NN + id - P - 1]);
          grad[UP * NN + id - P] = -(grav * (e[id - P] / 1.0 - e[id] / 1.0) / L.len[UP * NN + id - P]);
          written[RT * NN + id - 1] = written[DG * NN + id - P - 1] = written[UP * NN + id - P] = 1;
        }
      }
  const double s = theta1 * dt;
  for (int k = 0; k < nz; ++k)
    for (int64_t x = 0; x < 3 * NN; ++x)
      if (written[x]) velo[3 * k * NN + x] = velo[3 * k * NN + x] - s * grad[x];
  return 0;
}

// One layer: s (NN, itypes 1 and 6), v (3*NN), mass, mean_m (NN); flux (3*NN out).
int orc_step1_flux(const orc_blevel* Lp, int itype, const double* s_in, const double* v_in, const double* m_in,
                   const double* mean_m, double* flux) {
  const orc_blevel& L = *Lp;
  B b{L};
  const int64_t NN = L.NN;
  const int P = L.P;
  std::vector<double> s(NN, 0.0), v(v_in, v_in + 3 * NN), m(m_in, m_in + NN);
  if (s_in) s.assign(s_in, s_in + NN);
  b.halo_n(s.data());
  b.halo_n(m.data());
  b.halo_e(v.data());
  std::memset(flux, 0, 3 * NN * sizeof(double));
  const double* ped = L.pedlen;
  const double* len = L.len;
  for (int d = 0; d < 10; ++d)
    for (int j = 0; j <= L.n; ++j)
      for (int i = 0; i <= L.n; ++i) {
        const int64_t id = b.id(d, i, j);
        const int64_t idE = id + 1, idN = id + P, idNE = id + P + 1, idW = id - 1, idS = id - P, idSW = id - P - 1;
        const int64_t rt = RT * NN + id, dg = DG * NN + id, up = UP * NN + id;
        const int64_t wrt = RT * NN + idW, swdg = DG * NN + idSW, sup = UP * NN + idS;
        const bool sw = (i == 0 || j == 0);
        if (itype == 1) {
          flux[rt] = (s[idE] - s[id]) / len[rt] * ped[rt];
          flux[dg] = (s[id] - s[idNE]) / len[dg] * ped[dg];
          flux[up] = (s[idN] - s[id]) / len[up] * ped[up];
          if (sw) {
            flux[wrt] = -((s[idW] - s[id]) / len[wrt] * ped[wrt]);
            flux[swdg] = -((s[id] - s[idSW]) / len[swdg] * ped[swdg]);
            flux[sup] = -((s[idS] - s[id]) / len[sup] * ped[sup]);
          }
        } else if (itype == 5) {
          flux[rt] = v[rt] * ped[rt];
          flux[dg] = v[dg] * ped[dg];
          flux[up] = v[up] * ped[up];
          if (sw) {
            flux[wrt] = v[wrt] * ped[wrt];
            flux[swdg] = v[swdg] * ped[swdg];
            flux[sup] = v[sup] * ped[sup];
          }
        } else if (itype == 6) {
          flux[rt] = (s[idE] - s[id]) * v[rt] * ped[rt] / 4.0;
          flux[dg] = (s[id] - s[idNE]) * v[dg] * ped[dg] / 4.0;
          flux[up] = (s[idN] - s[id]) * v[up] * ped[up] / 4.0;
          if (sw) {
            flux[wrt] = -((s[idW] - s[id]) * v[wrt] * ped[wrt] / 4.0);
            flux[swdg] = -((s[id] - s[idSW]) * v[swdg] * ped[swdg] / 4.0);
            flux[sup] = -((s[idS] - s[id]) * v[sup] * ped[sup] / 4.0);
          }
        } else if (itype == 7) {
          const double dz0 = m[id] + mean_m[id];
          flux[rt] = v[rt] * ped[rt] * interp(dz0, m[idE] + mean_m[idE]);
          flux[dg] = v[dg] * ped[dg] * interp(dz0, m[idNE] + mean_m[idNE]);
          flux[up] = v[up] * ped[up] * interp(dz0, m[idN] + mean_m[idN]);
          if (sw) {
            flux[wrt] = v[wrt] * ped[wrt] * interp(dz0, m[idW] + mean_m[idW]);
            flux[swdg] = v[swdg] * ped[swdg] * interp(dz0, m[idSW] + mean_m[idSW]);
            flux[sup] = v[sup] * ped[sup] * interp(dz0, m[idS] + mean_m[idS]);
          }
        } else {
          return -1;
        }
      }
  return 0;
}

// One layer's velocity v (3*NN) -> vort (2*NN, LORT plane then UPLT plane).
int orc_step1_vort(const orc_blevel* Lp, const double* triarea, const double* v_in, double* vort) {
  const orc_blevel& L = *Lp;
  B b{L};
  const int64_t NN = L.NN;
  const int P = L.P, n = L.n;
  std::vector<double> v(v_in, v_in + 3 * NN);
  b.halo_e(v.data());
  std::memset(vort, 0, 2 * NN * sizeof(double));
  auto up = [&](int e, int64_t x) { return v[e * NN + x] * L.len[e * NN + x]; };
  auto put = [&](int t, int64_t x, double c) { vort[t * NN + x] = c / triarea[t * NN + x]; };
  enum { LORT = 0, UPLT = 1 };
  for (int d = 0; d < 10; ++d) {
    auto node = [&](int i, int j) {
      const int64_t id = b.id(d, i, j);
      const int64_t idN = id + P, idE = id + 1, idS = id - P, idW = id - 1, idSW = id - P - 1;
      // comput
      const double u_RT = up(RT, id), u_RT_N = up(RT, idN), u_RT_W = up(RT, idW);
      const double u_DG = up(DG, id), u_DG_S = up(DG, idS), u_DG_W = up(DG, idW);
      const double u_UP = up(UP, id), u_UP_E = up(UP, idE), u_UP_S = up(UP, idS);
      const double c_LORT = u_RT + u_UP_E + u_DG;
      const double c_UPLT = -(u_DG + u_UP + u_RT_N);
      const double c_W_LORT = u_RT_W + u_UP + u_DG_W;
      const double c_S_UPLT = -(u_RT + u_DG_S + u_UP_S);
      put(LORT, id, c_LORT);
      put(UPLT, id, c_UPLT);
      put(LORT, idW, c_W_LORT);
      put(UPLT, idS, c_S_UPLT);
      if (i == 0 || j == 0) {  // comp_SW
        const double w_RT_W = up(RT, idW), w_RT_SW = up(RT, idSW), w_DG_SW = up(DG, idSW);
        const double w_UP_S = up(UP, idS), w_UP_SW = up(UP, idSW);
        put(LORT, idSW, w_RT_SW + w_UP_S + w_DG_SW);
        put(UPLT, idSW, -(w_RT_W + w_DG_SW + w_UP_SW));
      }
    };
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) node(i, j);
    for (int i = 0; i < n; ++i) node(i, n);
    node(n, n);
    for (int j = 0; j < n; ++j) node(n, j);
    // post_vort at the four pentagon corners
    {
      const int64_t idS = b.id(d, 0, -1), idSW = b.id(d, -1, -1), idW = b.id(d, -1, 0);
      put(LORT, idSW, up(UP, idS) - up(RT, idW) + up(RT, idSW));
      vort[UPLT * NN + idSW] = vort[LORT * NN + idSW];
    }
    {
      const int64_t id = b.id(d, n, 0), idS = b.id(d, n, -1), idSW = b.id(d, n - 1, -1);
      put(LORT, idSW, -up(RT, id) + up(RT, idSW) + up(DG, idSW));
      vort[UPLT * NN + idS] = vort[LORT * NN + idSW];
    }
    {
      const int64_t id = b.id(d, 0, n), idSW = b.id(d, -1, n - 1), idW = b.id(d, -1, n);
      put(UPLT, idSW, up(UP, id) - up(DG, idSW) - up(UP, idSW));
      vort[LORT * NN + idW] = vort[UPLT * NN + idSW];
    }
    {
      const int64_t id = b.id(d, n, n), idN = b.id(d, n, n + 1);
      put(LORT, id, up(RT, id) - up(RT, idN) - up(UP, id));
      vort[UPLT * NN + id] = vort[LORT * NN + id];
    }
  }
  return 0;
}

// One level of a hierarchy for the barotropic pieces: the level record, the
// compute-or-restrict record (masks, overlap areas, R_F_wgt) and the level's
// fields.
struct orc_bml {
  orc_blevel b;
  orc_rlevel r;                     // flux / dscal / scal / dvelo pointers unused
  const double *mass, *mean_m;      // [nz][NN]
  double* velo;                     // [nz][3*NN], updated by orc_u_update_multi
  const double *eta, *div_old;      // [NN]
  double *div, *rhs, *grad;         // out: [NN], [NN], [3*NN]
};

// flux_divergence + rhs_elliptic over levels lv[0..nlev-1] (level_start first).
int orc_rhs_elliptic_multi(orc_bml* lv, int nlev, int nz, double dt, double theta2, double rho0) {
  std::vector<std::vector<double>> flux(nlev);
  for (int q = nlev - 1; q >= 0; --q) {
    orc_bml& M = lv[q];
    const orc_blevel& L = M.b;
    B b{L};
    const int64_t NN = L.NN;
    const int P = L.P;
    std::vector<double> m(M.mass, M.mass + nz * NN), v(M.velo, M.velo + 3 * nz * NN);
    for (int k = 0; k < nz; ++k) {
      b.halo_n(m.data() + k * NN);
      b.halo_e(v.data() + 3 * k * NN);
    }
    flux[q].assign(3 * NN, 0.0);
    double* hf = flux[q].data();
    // step1 itype 4
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= L.n; ++j)
        for (int i = 0; i <= L.n; ++i) {
          const int64_t id = b.id(d, i, j);
          const int64_t idE = id + 1, idN = id + P, idNE = id + P + 1, idW = id - 1, idS = id - P, idSW = id - P - 1;
          double f[3] = {0.0, 0.0, 0.0};
          for (int k = 0; k < nz; ++k) {
            const double* Mm = m.data() + k * NN;
            const double* A = M.mean_m + k * NN;
            const double* V = v.data() + 3 * k * NN;
            const double dz0 = Mm[id] + A[id];
            double dz = interp(dz0, Mm[idE] + A[idE]);
            f[RT] = f[RT] + V[RT * NN + id] * dz;
            dz = interp(dz0, Mm[idNE] + A[idNE]);
            f[DG] = f[DG] + V[DG * NN + id] * dz;
            dz = interp(dz0, Mm[idN] + A[idN]);
            f[UP] = f[UP] + V[UP * NN + id] * dz;
          }
          for (int e = 0; e < 3; ++e) hf[e * NN + id] = f[e] * L.pedlen[e * NN + id];
          if (i == 0 || j == 0) {
            double g[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < nz; ++k) {
              const double* Mm = m.data() + k * NN;
              const double* A = M.mean_m + k * NN;
              const double* V = v.data() + 3 * k * NN;
              const double dz0 = Mm[id] + A[id];
              double dz = interp(dz0, Mm[idW] + A[idW]);
              g[0] = g[0] + V[RT * NN + idW] * dz;
              dz = interp(dz0, Mm[idSW] + A[idSW]);
              g[1] = g[1] + V[DG * NN + idSW] * dz;
              dz = interp(dz0, Mm[idS] + A[idS]);
              g[2] = g[2] + V[UP * NN + idS] * dz;
            }
            hf[RT * NN + idW] = g[0] * L.pedlen[RT * NN + idW];
            hf[DG * NN + idSW] = g[1] * L.pedlen[DG * NN + idSW];
            hf[UP * NN + idS] = g[2] * L.pedlen[UP * NN + idS];
          }
        }
    if (q < nlev - 1) {  // cpt_or_restr_flux with dscalar => div_flux of the child
      orc_rlevel Pr = M.r, Cr = lv[q + 1].r;
      Pr.flux = hf;
      Cr.flux = flux[q + 1].data();
      Cr.dscal = lv[q + 1].div;
      orc_restrict_flux(&Pr, &Cr, 1);
    }
    b.halo_e(hf);
    std::memset(M.div, 0, NN * sizeof(double));
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= L.n; ++j)
        for (int i = 0; i <= L.n; ++i) {
          const int64_t id = b.id(d, i, j);
          M.div[id] = (hf[RT * NN + id] - hf[RT * NN + id - 1] + hf[DG * NN + id - P - 1] - hf[DG * NN + id] +
                       hf[UP * NN + id] - hf[UP * NN + id - P]) *
                      L.hex_inv[id];
        }
    b.halo_n(M.div);
  }
  for (int q = nlev - 1; q >= 0; --q) {  // cal_rhs_elliptic on every level
    orc_bml& M = lv[q];
    const orc_blevel& L = M.b;
    B b{L};
    const int64_t NN = L.NN;
    std::vector<double> e(M.eta, M.eta + NN), dold(M.div_old, M.div_old + NN);
    b.halo_n(e.data());
    b.halo_n(dold.data());
    std::memset(M.rhs, 0, NN * sizeof(double));
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= L.n; ++j)
        for (int i = 0; i <= L.n; ++i) {
          const int64_t id = b.id(d, i, j);
          M.rhs[id] = -e[id] + dt * (theta2 * M.div[id] + (1.0 - theta2) * dold[id]) / rho0;
        }
  }
  return 0;
}

// grad_eta + u_update over the hierarchy.
int orc_u_update_multi(orc_bml* lv, int nlev, int nz, double grav, double dt, double theta1) {
  constexpr int RESTRCT = 12;
  std::vector<std::vector<double>> ew(nlev);
  for (int q = 0; q < nlev; ++q) {  // update_bdry(sol(S_MASS, zlevels+1)); copy to the work field
    B b{lv[q].b};
    ew[q].assign(lv[q].eta, lv[q].eta + lv[q].b.NN);
    b.halo_n(ew[q].data());
  }
  for (int q = nlev - 1; q >= 0; --q) {
    orc_bml& M = lv[q];
    const orc_blevel& L = M.b;
    B b{L};
    const int64_t NN = L.NN;
    const int P = L.P;
    double* e = ew[q].data();
    if (q < nlev - 1) {  // cpt_or_restr_eta: parents [0, n]^2 with mask_n >= RESTRCT
      const orc_blevel& Lc = lv[q + 1].b;
      B bc{Lc};
      for (int d = 0; d < 10; ++d)
        for (int jp = 0; jp <= L.n; ++jp)
          for (int ip = 0; ip <= L.n; ++ip)
            if (M.r.mask_n[b.id(d, ip, jp)] >= RESTRCT) e[b.id(d, ip, jp)] = ew[q + 1][bc.id(d, 2 * ip, 2 * jp)];
    }
    std::memset(M.grad, 0, 3 * NN * sizeof(double));
    std::vector<char> written(3 * NN, 0);
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= L.n; ++j)
        for (int i = 0; i <= L.n; ++i) {
          const int64_t id = b.id(d, i, j);
          double* g = M.grad;
          g[RT * NN + id] = grav * (e[id + 1] / 1.0 - e[id] / 1.0) / L.len[RT * NN + id];
          g[DG * NN + id] = grav * (e[id] / 1.0 - e[id + P + 1] / 1.0) / L.len[DG * NN + id];
          g[UP * NN + id] = grav * (e[id + P] / 1.0 - e[id] / 1.0) / L.len[UP * NN + id];
          written[RT * NN + id] = written[DG * NN + id] = written[UP * NN + id] = 1;
          if (i == 0 || j == 0) {
            g[RT * NN + id - 1] = -(grav * (e[id - 1] / 1.0 - e[id] / 1.0) / L.len[RT * NN + id - 1]);
            g[DG * NN + id - P - 1] = -(grav * (e[id] / 1.0 - e[id - P - 1] / 1.0) / L.len[DG * NN + id - P - 1]);
            g[UP * NN + id - P] = -(grav * (e[id - P] / 1.0 - e[id] / 1.0) / L.len[UP * NN + id - P]);
            written[RT * NN + id - 1] = written[DG * NN + id - P - 1] = written[UP * NN + id - P] = 1;
          }
        }
    const double s = theta1 * dt;
    for (int k = 0; k < nz; ++k)
      for (int64_t x = 0; x < 3 * NN; ++x)
        if (written[x]) M.velo[3 * k * NN + x] = M.velo[3 * k * NN + x] - s * M.grad[x];
  }
  return 0;
}

}  // extern "C"
