// ORACLE (test infrastructure only): CPU FP64 restatement of the reference's
// barotropic elliptic operator, scalar wavelet restriction/prolongation and
// multigrid solvers on a uniform hierarchy of padded lozenge levels.  Imported
// only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
//
// Routines follow, op for op and in evaluation order:
//   elliptic_lo, complete_elliptic_lo      src/barotropic_2d.f90:187-250
//   step1 itype 2 (flux)                   src/ops.f90:202-216, comp_SW :420-434
//   cal_div, div                           src/ops.f90:1325-1355
//   elliptic_lo_diag (exact = .false.)     src/barotropic_2d.f90:252-324
//   FMG, v_cycle                           src/lin_solve.f90:33-140
//   SRJ, SRJ_iter                          src/lin_solve.f90:142-231
//   restrict, prolong, prol_fun            src/lin_solve.f90:233-269
//   Jacobi, Jacobi_iteration, cal_jacobi   src/lin_solve.f90:271-359
//   bicgstab                               src/lin_solve.f90:361-431
//   l2, dp, lc, residual, res_err          src/lin_solve.f90:433-618
//   forward_scalar_transform_0             src/wavelet.f90:105-155
//   inverse_scalar_transform_0             src/wavelet.f90:298-346
//   Compute_scalar_wavelets, Interp_node   src/wavelet.f90:642-670,1487-1498
//   Restrict_scalar, Prolong_scalar        src/wavelet.f90:520-612
//   Reconstruct_scalar                     src/wavelet.f90:614-640
// Iteration sets follow the reference's apply_onescale ranges: (0,1) on a
// domain is [0, n_d]^2, so nodes on the north/east rows of every
// DOMAIN_LEVEL sub-domain (and the pole copies) enter l2/dp more than once,
// exactly as in the reference's sums.  Reads outside the padded array (which
// the reference takes from a neighbouring storage element, only for ghost
// rows whose results are later overwritten or weighted by zero) read 0.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

enum { RT = 0, DG = 1, UP = 2 };
constexpr int H = 2;

struct ELevel {
  int n, P;
  int64_t NN;
  const double *len, *pedlen, *hex_inv, *overl_a, *topo;
  const int64_t* hn;
  int64_t nhn;
  const int64_t* he;
  int64_t nhe;
  const double* eta_old;  // old free surface (Laplacian_scalar(S_TEMP) of eta_update), ghosts copied; null = 0
};

struct EParams {
  double grav, dt, theta1, theta2;
  int domain_level;
  int coarse_iter, max_vcycle, pre_iter, down_iter, up_iter, post_iter, max_srj_iter;
  double fine_tol, coarse_tol;
};

inline double interp(double a, double b) { return 0.5 * (a + b); }

struct Solver {
  std::vector<ELevel> lev;
  int ls, le;
  EParams p;
  std::vector<int64_t> off;  // node offset of each level in a multi-level field
  int64_t total = 0;
  // persistent module fields of the reference
  std::vector<double> hflux, dsc, wc_mass, wc_temp, Au, diag, res, corr, s_, As_, Ap_, res0_, p_, corr_b, pf;

  const ELevel& L(int l) const { return lev[l - ls]; }
  int64_t id(int l, int d, int i, int j) const {
    const ELevel& g = L(l);
    return off[l - ls] + ((int64_t)d * g.P + (j + H)) * g.P + (i + H);
  }
  bool in(int l, int i, int j) const { int n = L(l).n; return i >= -H && j >= -H && i < n + H && j < n + H; }
  int64_t loc(int l, int64_t gid) const { return gid - off[l - ls]; }
  double rd(const std::vector<double>& f, int l, int d, int i, int j) const { return in(l, i, j) ? f[id(l, d, i, j)] : 0.0; }
  double oa(int l, int d, int i, int j, int k) const {  // overl_areas%a(k), k = 1..4
    if (!in(l, i, j)) return 0.0;
    const ELevel& g = L(l);
    return g.overl_a[(int64_t)(k - 1) * g.NN + (id(l, d, i, j) - off[l - ls])];
  }
  double hinv(int l, int64_t gid) const { return L(l).hex_inv[gid - off[l - ls]]; }

  void init() {
    off.clear();
    total = 0;
    for (auto& g : lev) { off.push_back(total); total += g.NN; }
    for (auto* v : {&dsc, &wc_mass, &wc_temp, &Au, &diag, &res, &corr, &s_, &As_, &Ap_, &res0_, &p_, &corr_b, &pf})
      v->assign(total, 0.0);
    hflux.assign(3 * total, 0.0);
  }

  // cp_bdry_inside of a node field at level l
  void halo(std::vector<double>& f, int l) {
    const ELevel& g = L(l);
    double* b = f.data() + off[l - ls];
    for (int64_t k = 0; k < g.nhn; ++k) b[g.hn[2 * k]] = b[g.hn[2 * k + 1]];
  }
  void halo_e(std::vector<double>& f, int l) {
    const ELevel& g = L(l);
    double* b = f.data() + 3 * off[l - ls];
    for (int64_t k = 0; k < g.nhe; ++k) {
      double v = b[g.he[3 * k + 1]];
      b[g.he[3 * k]] = g.he[3 * k + 2] < 0 ? -v : v;
    }
  }
  // zero_float_field over [-(BDRY-1), BDRY] of levels lmin..lmax
  void zero(std::vector<double>& f, int lmin, int lmax) {
    for (int l = lmin; l <= lmax; ++l) {
      int n = L(l).n;
      for (int d = 0; d < 10; ++d)
        for (int j = -1; j <= n + 1; ++j)
          for (int i = -1; i <= n + 1; ++i) f[id(l, d, i, j)] = 0.0;
    }
  }
  // multiplicity of node (i, j) of a lozenge in the union of the (0,1) ranges
  // of the DOMAIN_LEVEL sub-domains (1, 2 or 4)
  int mult(int l, int i, int j) const {
    int n = L(l).n, nd = n >> p.domain_level;
    if (nd < 1) nd = 1;
    int a = (i > 0 && i < n && i % nd == 0) ? 2 : 1;
    int b = (j > 0 && j < n && j % nd == 0) ? 2 : 1;
    return a * b;
  }

  // ---- elliptic operator (phi = 1; eta_old the old free surface, 0 when absent)
  double eta_old(int l, int64_t gid) const {
    const ELevel& g = L(l);
    return g.eta_old ? g.eta_old[gid - off[l - ls]] : 0.0;
  }
  double csq(int l, int64_t gid) const {
    const ELevel& g = L(l);
    double c = std::fabs(g.topo[gid - off[l - ls]]) * 1.0 + eta_old(l, gid);
    return p.grav * c;
  }
  void flux_node(const std::vector<double>& q, int l, int d, int i, int j, bool sw) {
    const ELevel& g = L(l);
    int64_t NN = g.NN, base = 3 * off[l - ls];
    auto F = [&](int e, int64_t gid) -> double& { return hflux[base + (int64_t)e * NN + (gid - off[l - ls])]; };
    int64_t id0 = id(l, d, i, j);
    const double* len = g.len;
    const double* ped = g.pedlen;
    auto LEN = [&](int e, int64_t gid) { return len[(int64_t)e * NN + (gid - off[l - ls])]; };
    auto PED = [&](int e, int64_t gid) { return ped[(int64_t)e * NN + (gid - off[l - ls])]; };
    double c0 = csq(l, id0);
    if (!sw) {
      int64_t idE = id(l, d, i + 1, j), idNE = id(l, d, i + 1, j + 1), idN = id(l, d, i, j + 1);
      double c1 = csq(l, idE), c2 = csq(l, idNE), c3 = csq(l, idN);
      F(RT, id0) = interp(c0, c1) * (q[idE] / 1.0 - q[id0] / 1.0) / LEN(RT, id0) * PED(RT, id0);
      F(DG, id0) = interp(c0, c2) * (q[id0] / 1.0 - q[idNE] / 1.0) / LEN(DG, id0) * PED(DG, id0);
      F(UP, id0) = interp(c0, c3) * (q[idN] / 1.0 - q[id0] / 1.0) / LEN(UP, id0) * PED(UP, id0);
    } else {
      int64_t idW = id(l, d, i - 1, j), idSW = id(l, d, i - 1, j - 1), idS = id(l, d, i, j - 1);
      double c1 = csq(l, idW), c2 = csq(l, idSW), c3 = csq(l, idS);
      F(RT, idW) = -(interp(c0, c1) * (q[idW] / 1.0 - q[id0] / 1.0) / LEN(RT, idW) * PED(RT, idW));
      F(DG, idSW) = -(interp(c0, c2) * (q[id0] / 1.0 - q[idSW] / 1.0) / LEN(DG, idSW) * PED(DG, idSW));
      F(UP, idS) = -(interp(c0, c3) * (q[idS] / 1.0 - q[id0] / 1.0) / LEN(UP, idS) * PED(UP, idS));
    }
  }
  // elliptic_lo: out = theta1*theta2*dt^2 * div(flux(q)) - q on [0, n]^2 of level l
  void elliptic_lo(std::vector<double>& q, int l, std::vector<double>& out) {
    halo(q, l);
    zero(out, ls, le);
    int n = L(l).n;
    for (int d = 0; d < 10; ++d) {
      // step1 itype 2 traversal: owned nodes, then north row and NE point, then east column
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          flux_node(q, l, d, i, j, false);
          if (i == 0 || j == 0) flux_node(q, l, d, i, j, true);
        }
      for (int i = 0; i < n; ++i) {
        flux_node(q, l, d, i, n, false);
        if (i == 0) flux_node(q, l, d, i, n, true);
      }
      flux_node(q, l, d, n, n, false);
      for (int j = 0; j < n; ++j) {
        flux_node(q, l, d, n, j, false);
        if (j == 0) flux_node(q, l, d, n, j, true);
      }
    }
    halo_e(hflux, l);
    const ELevel& g = L(l);
    int64_t NN = g.NN, base = 3 * off[l - ls];
    auto Fr = [&](int e, int64_t gid) { return hflux[base + (int64_t)e * NN + (gid - off[l - ls])]; };
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t id0 = id(l, d, i, j), idS = id(l, d, i, j - 1), idW = id(l, d, i - 1, j), idSW = id(l, d, i - 1, j - 1);
          dsc[id0] = (Fr(RT, id0) - Fr(RT, idW) + Fr(DG, idSW) - Fr(DG, id0) + Fr(UP, id0) - Fr(UP, idS)) * hinv(l, id0);
        }
    halo(dsc, l);
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t id0 = id(l, d, i, j);
          out[id0] = p.theta1 * p.theta2 * (p.dt * p.dt) * dsc[id0] - q[id0];
        }
  }
  void elliptic_lo_diag(int l, std::vector<double>& out) {
    zero(out, ls, le);
    int n = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t id0 = id(l, d, i, j);
          double depth = std::fabs(L(l).topo[id0 - off[l - ls]]) + eta_old(l, id0) / 1.0;
          double wgt = 2.0 * std::sqrt(3.0) * depth;
          double lap = -(p.grav * wgt * (p.dt * p.dt) * hinv(l, id0));
          out[id0] = p.theta1 * p.theta2 * lap - 1.0;
        }
  }
  // ---- linear algebra on level l
  void residual(std::vector<double>& f, std::vector<double>& u, int l, std::vector<double>& r) {
    halo(f, l);
    elliptic_lo(u, l, Au);
    halo(Au, l);
    int n = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t k = id(l, d, i, j);
          r[k] = f[k] - Au[k];
        }
  }
  double l2(const std::vector<double>& s, int l) {
    double acc = 0.0;
    int n = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          double v = s[id(l, d, i, j)];
          int m = mult(l, i, j);
          for (int q = 0; q < m; ++q) acc = acc + v * v;
        }
    return std::sqrt(acc);
  }
  double dp(std::vector<double>& a, std::vector<double>& b, int l) {
    halo(a, l);
    halo(b, l);
    double acc = 0.0;
    int n = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t k = id(l, d, i, j);
          int m = mult(l, i, j);
          for (int q = 0; q < m; ++q) acc = acc + a[k] * b[k];
        }
    return acc;
  }
  void lc(std::vector<double>& s, double a1, const std::vector<double>& s1, double a2, const std::vector<double>& s2, int l) {
    int n = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t k = id(l, d, i, j);
          s[k] = a1 * s1[k] + a2 * s2[k];
        }
    halo(s, l);
  }
  void jacobi_iteration(std::vector<double>& u, std::vector<double>& f, double w, int l) {
    elliptic_lo(u, l, Au);
    halo(Au, l);
    elliptic_lo_diag(l, diag);
    halo(diag, l);
    int n = L(l).n;
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t k = id(l, d, i, j);
          u[k] = u[k] + w * (f[k] - Au[k]) / diag[k];
        }
  }
  void jacobi(std::vector<double>& u, std::vector<double>& f, int l, int iters) {
    halo(f, l);
    for (int it = 0; it < iters; ++it) jacobi_iteration(u, f, 1.0, l);
  }
  double res_err(std::vector<double>& f, std::vector<double>& u, double nrm_f, int l) {
    std::vector<double>& r = corr_b;  // "res = u; zero_float_field(res, AT_NODE, l)"
    r = u;
    zero(r, l, l);
    residual(f, u, l, r);
    return l2(r, l) / nrm_f;
  }
  void bicgstab(std::vector<double>& u, std::vector<double>& f, double nrm_f, int l, double tol, int iter_max,
                double* err_out, int* iter_out) {
    halo(f, l);
    halo(u, l);
    std::vector<double> rr = u, cc = u;
    zero(rr, ls, ls);
    zero(cc, ls, ls);
    residual(f, u, l, rr);
    std::vector<double> r0 = rr, pp = r0, ss = r0, Ap, As;
    Ap.assign(total, 0.0);
    elliptic_lo(pp, l, Ap);
    halo(Ap, l);
    As = Ap;
    double rho = dp(r0, rr, l), err = 0.0;
    int iter;
    for (iter = 1; iter <= iter_max; ++iter) {
      double alph = rho / dp(Ap, r0, l);
      lc(ss, 1.0, rr, -alph, Ap, l);
      elliptic_lo(ss, l, As);
      halo(As, l);
      double omga = dp(As, ss, l) / dp(As, As, l);
      lc(cc, alph, pp, omga, ss, l);
      lc(u, 1.0, u, 1.0, cc, l);
      lc(rr, 1.0, ss, -omga, As, l);
      err = l2(rr, l) / nrm_f;
      if (err <= tol) break;
      double rho_old = rho;
      rho = dp(r0, rr, l);
      double b = (alph / omga) * (rho / rho_old);
      lc(cc, 1.0, pp, -omga, Ap, l);
      lc(pp, 1.0, rr, b, cc, l);
      elliptic_lo(pp, l, Ap);
      halo(Ap, l);
    }
    if (err_out) *err_out = err;
    if (iter_out) *iter_out = iter;
  }
  // ---- wavelet transforms between levels c and c+1
  double interp_node(const std::vector<double>& s, int l, int d, int i, int j, int i1, int j1, int i2, int j2, int i3,
                     int j3, int i4, int j4) {
    int64_t k = id(l, d, i, j);
    return (oa(l, d, i, j, 1) * rd(s, l, d, i1, j1) + oa(l, d, i, j, 2) * rd(s, l, d, i2, j2) +
            oa(l, d, i, j, 3) * rd(s, l, d, i3, j3) + oa(l, d, i, j, 4) * rd(s, l, d, i4, j4)) *
           hinv(l, k);
  }
  void forward_scalar(std::vector<double>& s, std::vector<double>& wc, int c) {
    std::fill(wc.begin(), wc.end(), 0.0);   // zero_float(wavelet)
    int f = c + 1, np = L(c).n;
    halo(s, f);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < np; ++jp)
        for (int ip = 0; ip < np; ++ip) {
          int i = 2 * ip, j = 2 * jp;
          wc[id(f, d, i + 1, j)] = rd(s, f, d, i + 1, j) - interp_node(s, f, d, i + 1, j, i, j, i + 2, j, i + 2, j + 2, i, j - 2);
          wc[id(f, d, i + 1, j + 1)] =
              rd(s, f, d, i + 1, j + 1) - interp_node(s, f, d, i + 1, j + 1, i + 2, j + 2, i, j, i + 2, j, i, j + 2);
          wc[id(f, d, i, j + 1)] = rd(s, f, d, i, j + 1) - interp_node(s, f, d, i, j + 1, i, j, i, j + 2, i - 2, j, i + 2, j + 2);
        }
    halo(wc, f);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= np; ++jp)
        for (int ip = 0; ip <= np; ++ip) {
          int i = 2 * ip, j = 2 * jp;
          double sum = rd(wc, f, d, i + 1, j) * oa(f, d, i + 1, j, 1) + rd(wc, f, d, i + 1, j + 1) * oa(f, d, i + 1, j + 1, 2) +
                       rd(wc, f, d, i + 2, j + 1) * oa(f, d, i + 2, j + 1, 3) +
                       rd(wc, f, d, i + 1, j + 2) * oa(f, d, i + 1, j + 2, 4) + rd(wc, f, d, i, j + 1) * oa(f, d, i, j + 1, 1) +
                       rd(wc, f, d, i - 1, j) * oa(f, d, i - 1, j, 2) + rd(wc, f, d, i - 1, j + 1) * oa(f, d, i - 1, j + 1, 3) +
                       rd(wc, f, d, i - 2, j - 1) * oa(f, d, i - 2, j - 1, 4) +
                       rd(wc, f, d, i - 1, j - 1) * oa(f, d, i - 1, j - 1, 1) + rd(wc, f, d, i, j - 1) * oa(f, d, i, j - 1, 2) +
                       rd(wc, f, d, i - 1, j - 2) * oa(f, d, i - 1, j - 2, 3) +
                       rd(wc, f, d, i + 1, j - 1) * oa(f, d, i + 1, j - 1, 4);
          int64_t kp = id(c, d, ip, jp);
          s[kp] = rd(s, f, d, i, j) + sum * hinv(c, kp);
        }
  }
  void inverse_scalar(std::vector<double>& wc, std::vector<double>& s, int f) {
    int c = f - 1, np = L(c).n;
    halo(wc, c);
    halo(wc, f);
    halo(s, c);
    halo(s, f);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp <= np; ++jp)
        for (int ip = 0; ip <= np; ++ip) {
          int i = 2 * ip, j = 2 * jp;
          double sum = rd(wc, f, d, i + 1, j) * oa(f, d, i + 1, j, 1) + rd(wc, f, d, i + 1, j + 1) * oa(f, d, i + 1, j + 1, 2) +
                       rd(wc, f, d, i + 2, j + 1) * oa(f, d, i + 2, j + 1, 3) + rd(wc, f, d, i, j + 1) * oa(f, d, i, j + 1, 1) +
                       rd(wc, f, d, i - 1, j) * oa(f, d, i - 1, j, 2) + rd(wc, f, d, i - 1, j + 1) * oa(f, d, i - 1, j + 1, 3) +
                       rd(wc, f, d, i - 2, j - 1) * oa(f, d, i - 2, j - 1, 4) +
                       rd(wc, f, d, i - 1, j - 1) * oa(f, d, i - 1, j - 1, 1) + rd(wc, f, d, i, j - 1) * oa(f, d, i, j - 1, 2) +
                       rd(wc, f, d, i - 1, j - 2) * oa(f, d, i - 1, j - 2, 3) +
                       rd(wc, f, d, i + 1, j - 1) * oa(f, d, i + 1, j - 1, 4);
          int64_t kp = id(c, d, ip, jp);
          s[id(f, d, i, j)] = s[kp] - sum * hinv(c, kp);
        }
    halo(s, f);
    for (int d = 0; d < 10; ++d)
      for (int jp = 0; jp < np; ++jp)
        for (int ip = 0; ip < np; ++ip) {
          int i = 2 * ip, j = 2 * jp;
          s[id(f, d, i + 1, j)] = interp_node(s, f, d, i + 1, j, i, j, i + 2, j, i + 2, j + 2, i, j - 2) + rd(wc, f, d, i + 1, j);
          s[id(f, d, i + 1, j + 1)] =
              interp_node(s, f, d, i + 1, j + 1, i + 2, j + 2, i, j, i + 2, j, i, j + 2) + rd(wc, f, d, i + 1, j + 1);
          s[id(f, d, i, j + 1)] = interp_node(s, f, d, i, j + 1, i, j, i, j + 2, i - 2, j, i + 2, j + 2) + rd(wc, f, d, i, j + 1);
        }
  }
  // ---- solvers
  struct Report {
    double nrm_res[2][16];
    int iterations[16];
  };
  void fmg(std::vector<double>& u, std::vector<double>& f, Report& rep) {
    for (int l = ls; l <= le; ++l) halo(f, l);
    res = u;
    zero(res, ls, le);
    zero(wc_mass, ls, le);
    std::vector<double> nrm_f(le - ls + 1);
    for (int l = ls; l <= le; ++l) {
      nrm_f[l - ls] = l2(f, l);
      if (nrm_f[l - ls] == 0.0) nrm_f[l - ls] = 1.0;
      rep.nrm_res[0][l - ls] = res_err(f, u, nrm_f[l - ls], l);
      rep.nrm_res[1][l - ls] = 0.0;
      rep.iterations[l - ls] = 0;
    }
    int l = ls;
    bicgstab(u, f, nrm_f[0], l, p.coarse_tol, p.coarse_iter, &rep.nrm_res[1][0], &rep.iterations[0]);
    for (l = ls + 1; l <= le; ++l) {
      if (rep.nrm_res[0][l - ls] < p.fine_tol) continue;
      inverse_scalar(wc_mass, u, l);   // prolong
      jacobi(u, f, l, p.pre_iter);
      for (int iter = 1; iter <= p.max_vcycle; ++iter) {
        v_cycle(u, f, l, nrm_f[l - ls], rep);
        rep.iterations[l - ls] = iter;
        if (rep.nrm_res[1][l - ls] <= p.fine_tol) break;
      }
    }
  }
  void v_cycle(std::vector<double>& u, std::vector<double>& f, int l, double nrmf, Report& rep) {
    corr = u;
    for (int j = ls; j <= l; ++j) zero(corr, ls, l);
    residual(f, u, l, res);
    for (int j = l; j >= ls + 1; --j) {
      jacobi(corr, res, j, p.down_iter);
      residual(res, corr, j, res);
      forward_scalar(res, wc_temp, j - 1);   // restrict
    }
    int j = ls;
    double nrm_rhs = l2(res, j);
    if (nrm_rhs == 0.0) nrm_rhs = 1.0;
    bicgstab(corr, res, nrm_rhs, j, p.coarse_tol, p.coarse_iter, nullptr, nullptr);
    for (j = ls + 1; j <= l; ++j) {
      // prol_fun: zero wav_coeff(S_TEMP,1) at level j, interpolate a copy of corr
      zero(wc_temp, j, j);
      pf = corr;
      inverse_scalar(wc_temp, pf, j);
      lc(corr, 1.0, corr, 1.0, pf, j);
      jacobi(corr, res, j, p.up_iter);
    }
    lc(u, 1.0, u, 1.0, corr, l);
    jacobi(u, f, l, p.post_iter);
    rep.nrm_res[1][l - ls] = res_err(f, u, nrmf, l);
  }
  void srj(std::vector<double>& u, std::vector<double>& f, Report& rep) {
    for (int l = ls; l <= le; ++l) halo(f, l);
    zero(wc_mass, ls, le);
    std::vector<double> nrm_f(le - ls + 1);
    for (int l = ls; l <= le; ++l) {
      nrm_f[l - ls] = l2(f, l);
      if (nrm_f[l - ls] == 0.0) nrm_f[l - ls] = 1.0;
      rep.nrm_res[0][l - ls] = rep.nrm_res[1][l - ls] = 0.0;
      rep.iterations[l - ls] = 0;
    }
    const int m = 8;
    const double k1 = 3e-2, k2 = 1.8;
    double w[m];
    int max_iter = p.max_srj_iter;
    if (max_iter < m) {
      for (int n = 0; n < m; ++n) w[n] = 1.0;
    } else {
      max_iter = m * (max_iter / m);
      const double PI = std::acos(-1.0);
      for (int n = 1; n <= m; ++n)
        w[n - 1] = 2.0 / (k1 + k2 - (k2 - k1) * std::cos(PI * (2.0 * double(n) - 1.0) / (2.0 * double(m))));
    }
    int l = ls;
    bicgstab(u, f, nrm_f[0], l, p.coarse_tol, p.coarse_iter, &rep.nrm_res[1][0], &rep.iterations[0]);
    for (l = ls + 1; l <= le; ++l) {
      inverse_scalar(wc_mass, u, l);
      int ii = 0;
      for (int iter = 1; iter <= max_iter; ++iter) {
        ii = ii + 1;
        if (ii > m) {
          if (rep.nrm_res[1][l - ls] < p.fine_tol) break;
          ii = 1;
        }
        halo(f, l);
        jacobi_iteration(u, f, w[ii - 1], l);
        rep.nrm_res[1][l - ls] = res_err(f, u, nrm_f[l - ls], l);
        rep.iterations[l - ls] = iter;
        if (rep.nrm_res[1][l - ls] <= p.fine_tol) break;
      }
    }
  }
};

}  // namespace

extern "C" {

struct orc_elevel {
  int level, n, P;
  int64_t NN;
  const double *len, *pedlen, *hex_inv, *overl_a, *topo;
  const int64_t* halo_node;
  int64_t n_halo_node;
  const int64_t* halo_edge;
  int64_t n_halo_edge;
  const double* eta_old;
};

struct orc_eparams {
  double grav, dt, theta1, theta2;
  int domain_level;
  int coarse_iter, max_vcycle, pre_iter, down_iter, up_iter, post_iter, max_srj_iter;
  double fine_tol, coarse_tol;
};

static void setup(Solver& S, const orc_elevel* lv, int nlev, const orc_eparams* p) {
  S.ls = lv[0].level;
  S.le = lv[nlev - 1].level;
  for (int q = 0; q < nlev; ++q)
    S.lev.push_back(ELevel{lv[q].n, lv[q].P, lv[q].NN, lv[q].len, lv[q].pedlen, lv[q].hex_inv, lv[q].overl_a, lv[q].topo,
                           lv[q].halo_node, lv[q].n_halo_node, lv[q].halo_edge, lv[q].n_halo_edge, lv[q].eta_old});
  S.p = EParams{p->grav, p->dt, p->theta1, p->theta2, p->domain_level, p->coarse_iter, p->max_vcycle, p->pre_iter,
                p->down_iter, p->up_iter, p->post_iter, p->max_srj_iter, p->fine_tol, p->coarse_tol};
  S.init();
}

// out = elliptic_lo(q) at level l; q and out are multi-level fields (all levels
// concatenated in level order); q's ghosts are refreshed in place.
int orc_elliptic_apply(const orc_elevel* lv, int nlev, const orc_eparams* p, int level, double* q, double* out) {
  Solver S;
  setup(S, lv, nlev, p);
  std::vector<double> qq(q, q + S.total), oo(S.total, 0.0);
  S.elliptic_lo(qq, level, oo);
  std::memcpy(q, qq.data(), S.total * 8);
  std::memcpy(out, oo.data(), S.total * 8);
  return 0;
}

// Fills levels coarser than level_end of s by repeated restriction (forward
// scalar transform), as restrict(s, l) does one level at a time.
int orc_restrict_all(const orc_elevel* lv, int nlev, const orc_eparams* p, double* s) {
  Solver S;
  setup(S, lv, nlev, p);
  std::vector<double> ss(s, s + S.total);
  for (int c = S.le - 1; c >= S.ls; --c) S.forward_scalar(ss, S.wc_temp, c);
  std::memcpy(s, ss.data(), S.total * 8);
  return 0;
}

// prolong(s, fine): inverse scalar transform with zero wavelets, level fine-1 -> fine
int orc_prolong(const orc_elevel* lv, int nlev, const orc_eparams* p, int fine, double* s) {
  Solver S;
  setup(S, lv, nlev, p);
  std::vector<double> ss(s, s + S.total);
  S.inverse_scalar(S.wc_mass, ss, fine);
  std::memcpy(s, ss.data(), S.total * 8);
  return 0;
}

double orc_l2(const orc_elevel* lv, int nlev, const orc_eparams* p, int level, const double* s) {
  Solver S;
  setup(S, lv, nlev, p);
  std::vector<double> ss(s, s + S.total);
  return S.l2(ss, level);
}

// method 0 = FMG, 1 = SRJ.  u (in/out) and f are multi-level fields.
// nrm_res_out[2*nlev] = initial/final normalised residual per level, iters_out[nlev].
int orc_elliptic_solve(const orc_elevel* lv, int nlev, const orc_eparams* p, int method, double* u, double* f,
                       double* nrm_res_out, int* iters_out) {
  Solver S;
  setup(S, lv, nlev, p);
  std::vector<double> uu(u, u + S.total), ff(f, f + S.total);
  Solver::Report rep{};
  if (method == 0) S.fmg(uu, ff, rep);
  else S.srj(uu, ff, rep);
  std::memcpy(u, uu.data(), S.total * 8);
  for (int q = 0; q < nlev; ++q) {
    nrm_res_out[2 * q] = rep.nrm_res[0][q];
    nrm_res_out[2 * q + 1] = rep.nrm_res[1][q];
    iters_out[q] = rep.iterations[q];
  }
  return 0;
}

}  // extern "C"
