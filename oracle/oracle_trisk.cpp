// ORACLE (test infrastructure only): CPU FP64 restatement of the reference's
// TRiSK trend and RK4 stepper on one uniform level of the padded lozenge layout.
// It is imported only by tests/, by __graft_entry__.smoke() and by bench.py's
// CPU-baseline leg, as the checker; the product path never calls it.
//
// Parity pin: the reference is Fortran and no Fortran compiler exists in this
// build container, so the restatement is checked against the properties the
// reference itself relies on (mass conservation, TRiSK energy neutrality,
// rest-state balance) rather than against reference output.  Parity against the
// reference binary is therefore "unpinned"; the CUDA path is checked against
// this file.
//
// Routines follow, op for op and in evaluation order:
//   trend_ml                       src/multi_level.f90:5-47
//   basic_operators                src/multi_level.f90:49-100
//   cal_surf_press/column_mass     src/ops.f90:1023-1072
//   set_surf_geopot                src/ops.f90:1074-1092
//   integrate_pressure_up          src/ops.f90:1094-1131
//   step1 (itype 0) comput/comp_SW src/ops.f90:14-524
//   post_step1                     src/ops.f90:526-737
//   scalar_trend, div              src/ops.f90:739-755,1325-1343
//   du_source, Qperp, get_weights  src/ops.f90:757-785,834-901,1006-1021
//   du_grad, gradi_e               src/ops.f90:787-832,1280-1301
//   RK4, RK_sub_step               src/time_integr.f90:78-103,206-225
//   cp_bdry_inside                 src/comm.f90:785-808
//   trend_ml over a hierarchy (orc_trend_multi): basic_operators with the
//   compute-or-restrict of Bernoulli, Exner and fluxes, cal_scalar_trend,
//   velocity_trend_source with cpt_or_restr_u_source, velocity_trend_grad
//   (src/multi_level.f90:5-188, 311-392) and the masks of scalar_trend,
//   du_source and du_grad (src/ops.f90:750,773,803); the restrictions are
//   those of oracle_restrict.cpp.
// Compiled with -O2 -ffp-contract=off (no FMA), like gfortran -O2 on x86-64.
#include <cstdint>
#include <cstring>
#include <vector>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>

#include "oracle_restrict.h"

namespace {

enum { RT = 0, DG = 1, UP = 2 };
enum { LORT = 0, UPLT = 1 };
constexpr int H = 2;

struct Lev {
  int n, P;
  int64_t NN;
  const double *len, *pedlen, *part, *hex_inv, *triarea, *coriolis;
  const int64_t* hnode;  // pairs (dst, src)
  int64_t n_hnode;
  const int64_t* hedge;  // triples (dst, src, sign)
  int64_t n_hedge;
};

struct Phys { double grav, ref_density, p_top; };

inline double interp(double a, double b) { return 0.5 * (a + b); }   // src/utils.f90:528

// Minimal persistent worker pool: run(fn) calls fn(d) for d = 0..9 (the ten
// lozenge domains) spread over the workers and returns when all are done.
// Results do not depend on the thread count (no cross-domain reductions).
class Pool {
 public:
  void set_threads(int n) {
    stop();
    n = n < 1 ? 1 : (n > 10 ? 10 : n);
    nthreads_ = n;
    // a new worker waits for the next run: it starts from the current
    // generation, not from 0 (a stale generation would replay the last run's
    // function, which no longer exists)
    uint64_t g0;
    {
      std::unique_lock<std::mutex> lk(m_);
      g0 = gen_;
    }
    for (int t = 1; t < n; ++t) workers_.emplace_back([this, t, g0] { loop(t, g0); });
  }
  int threads() const { return nthreads_; }
  void run(const std::function<void(int)>& fn) {
    if (nthreads_ <= 1) { for (int d = 0; d < 10; ++d) fn(d); return; }
    {
      std::unique_lock<std::mutex> lk(m_);
      fn_ = &fn; pending_ = nthreads_ - 1; ++gen_;
    }
    cv_.notify_all();
    for (int d = 0; d < 10; d += nthreads_) fn(d);
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
  }
  ~Pool() { stop(); }
 private:
  void loop(int t, uint64_t seen) {
    for (;;) {
      const std::function<void(int)>* fn;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
        if (quit_) return;
        seen = gen_; fn = fn_;
      }
      for (int d = t; d < 10; d += nthreads_) (*fn)(d);
      std::unique_lock<std::mutex> lk(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  void stop() {
    { std::unique_lock<std::mutex> lk(m_); quit_ = true; }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
    workers_.clear();
    quit_ = false;
    nthreads_ = 1;
  }
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* fn_ = nullptr;
  uint64_t gen_ = 0;
  int pending_ = 0, nthreads_ = 1;
  bool quit_ = false;
};
Pool& pool() { static Pool p; return p; }

struct Ctx {
  const Lev& L;
  const Phys& ph;
  int d = 0;
  // per-layer field pointers (the reference's module pointers mass, temp, velo, ...)
  double *mass, *temp, *velo;
  const double *mean_m, *mean_t;
  double *qe, *vort, *ke, *bernoulli, *exner;
  double *hflux_m, *hflux_t;
  double *geopot, *geopot_lower, *press, *press_lower, *surf_press;
  const double* topo;
  Ctx(const Lev& l, const Phys& p) : L(l), ph(p) {}
  inline int64_t id(int i, int j) const { return ((int64_t)d * L.P + (j + H)) * L.P + (i + H); }
  inline int64_t E(int e, int64_t node) const { return (int64_t)e * L.NN + node; }
  inline double part(int64_t node, int k) const { return L.part[(int64_t)(k - 1) * L.NN + node]; }
};

void halo_nodes(const Lev& L, double* f) {
  for (int64_t k = 0; k < L.n_hnode; ++k) f[L.hnode[2 * k]] = f[L.hnode[2 * k + 1]];
}
void halo_edges(const Lev& L, double* f) {
  for (int64_t k = 0; k < L.n_hedge; ++k) {
    double v = f[L.hedge[3 * k + 1]];
    f[L.hedge[3 * k]] = L.hedge[3 * k + 2] < 0 ? -v : v;
  }
}

// --- step1 itype 0 --------------------------------------------------------
struct Step1State {  // host-associated locals of step1 shared by comput and comp_SW
  double u_dual_RT_W, u_dual_DG_SW, u_dual_UP_S;
  double pv_W_LORT, pv_S_UPLT;
};

void comput(Ctx& c, Step1State& st, int i, int j) {
  const Lev& L = c.L;
  int64_t id = c.id(i, j), idN = c.id(i, j + 1), idE = c.id(i + 1, j), idS = c.id(i, j - 1), idW = c.id(i - 1, j),
          idNE = c.id(i + 1, j + 1), idSW = c.id(i - 1, j - 1);
  // rho_dz(0:NORTHEAST) at (id, idN, idE, idS, idW, idNE) for mass and temp
  int64_t ids[6] = {id, idN, idE, idS, idW, idNE};
  double rm[6], rt[6];
  for (int k = 0; k < 6; ++k) { rm[k] = c.mass[ids[k]] + c.mean_m[ids[k]]; rt[k] = c.temp[ids[k]] + c.mean_t[ids[k]]; }
  enum { O = 0, N_ = 1, E_ = 2, S_ = 3, W_ = 4, NE_ = 5 };
  const double* v = c.velo;
  double u_dual_RT = v[c.E(RT, id)] * L.pedlen[c.E(RT, id)];
  double u_dual_DG = v[c.E(DG, id)] * L.pedlen[c.E(DG, id)];
  double u_dual_UP = v[c.E(UP, id)] * L.pedlen[c.E(UP, id)];
  st.u_dual_RT_W = v[c.E(RT, idW)] * L.pedlen[c.E(RT, idW)];
  st.u_dual_DG_SW = v[c.E(DG, idSW)] * L.pedlen[c.E(DG, idSW)];
  st.u_dual_UP_S = v[c.E(UP, idS)] * L.pedlen[c.E(UP, idS)];

  double u_prim_RT = v[c.E(RT, id)] * L.len[c.E(RT, id)];
  double u_prim_RT_N = v[c.E(RT, idN)] * L.len[c.E(RT, idN)];
  double u_prim_RT_W = v[c.E(RT, idW)] * L.len[c.E(RT, idW)];
  double u_prim_DG = v[c.E(DG, id)] * L.len[c.E(DG, id)];
  double u_prim_DG_S = v[c.E(DG, idS)] * L.len[c.E(DG, idS)];
  double u_prim_DG_SW = v[c.E(DG, idSW)] * L.len[c.E(DG, idSW)];
  double u_prim_DG_W = v[c.E(DG, idW)] * L.len[c.E(DG, idW)];
  double u_prim_UP = v[c.E(UP, id)] * L.len[c.E(UP, id)];
  double u_prim_UP_E = v[c.E(UP, idE)] * L.len[c.E(UP, idE)];
  double u_prim_UP_S = v[c.E(UP, idS)] * L.len[c.E(UP, idS)];

  double circ_LORT = u_prim_RT + u_prim_UP_E + u_prim_DG;
  double circ_UPLT = -(u_prim_DG + u_prim_UP + u_prim_RT_N);
  double circ_W_LORT = u_prim_RT_W + u_prim_UP + u_prim_DG_W;
  double circ_S_UPLT = -(u_prim_RT + u_prim_DG_S + u_prim_UP_S);

  double pv_mass1 = rm[O] * c.part(id, 1) + rm[E_] * c.part(idE, 3) + rm[NE_] * c.part(idNE, 5);
  double pv_mass2 = rm[O] * c.part(id, 2) + rm[NE_] * c.part(idNE, 4) + rm[N_] * c.part(idN, 6);
  double pv_mass3 = rm[W_] * c.part(idW, 1) + rm[O] * c.part(id, 3) + rm[N_] * c.part(idN, 5);
  double pv_mass4 = rm[S_] * c.part(idS, 2) + rm[E_] * c.part(idE, 4) + rm[O] * c.part(id, 6);

  double pv_LORT = (L.coriolis[c.E(LORT, id)] + circ_LORT) / pv_mass1;
  double pv_UPLT = (L.coriolis[c.E(UPLT, id)] + circ_UPLT) / pv_mass2;
  st.pv_W_LORT = (L.coriolis[c.E(LORT, idW)] + circ_W_LORT) / pv_mass3;
  st.pv_S_UPLT = (L.coriolis[c.E(UPLT, idS)] + circ_S_UPLT) / pv_mass4;

  c.qe[c.E(RT, id)] = interp(st.pv_S_UPLT, pv_LORT);
  c.qe[c.E(DG, id)] = interp(pv_UPLT, pv_LORT);
  c.qe[c.E(UP, id)] = interp(pv_UPLT, st.pv_W_LORT);

  c.vort[c.E(LORT, id)] = circ_LORT / L.triarea[c.E(LORT, id)];
  c.vort[c.E(UPLT, id)] = circ_UPLT / L.triarea[c.E(UPLT, id)];
  c.vort[c.E(LORT, idW)] = circ_W_LORT / L.triarea[c.E(LORT, idW)];
  c.vort[c.E(UPLT, idS)] = circ_S_UPLT / L.triarea[c.E(UPLT, idS)];

  c.ke[id] = (u_prim_UP * u_dual_UP + u_prim_DG * u_dual_DG + u_prim_RT * u_dual_RT + u_prim_UP_S * st.u_dual_UP_S +
              u_prim_DG_SW * st.u_dual_DG_SW + u_prim_RT_W * st.u_dual_RT_W) *
             L.hex_inv[id] / 4.0;

  double Phi_k = interp(c.geopot[id], c.geopot_lower[id]);
  // incompressible: phi_node = 1 (no penalization)
  c.bernoulli[id] = c.ke[id] + Phi_k + c.press[id] / (c.ph.ref_density * 1.0);
  c.exner[id] = -Phi_k;

  // physics_scalar_flux = 0 for the configs of this path
  c.hflux_m[c.E(RT, id)] = u_dual_RT * interp(rm[O], rm[E_]) + 0.0;
  c.hflux_m[c.E(DG, id)] = u_dual_DG * interp(rm[O], rm[NE_]) + 0.0;
  c.hflux_m[c.E(UP, id)] = u_dual_UP * interp(rm[O], rm[N_]) + 0.0;
  c.hflux_t[c.E(RT, id)] = u_dual_RT * interp(rt[O], rt[E_]) + 0.0;
  c.hflux_t[c.E(DG, id)] = u_dual_DG * interp(rt[O], rt[NE_]) + 0.0;
  c.hflux_t[c.E(UP, id)] = u_dual_UP * interp(rt[O], rt[N_]) + 0.0;
}

void comp_SW(Ctx& c, Step1State& st, int i, int j) {
  const Lev& L = c.L;
  int64_t id = c.id(i, j), idW = c.id(i - 1, j), idSW = c.id(i - 1, j - 1), idS = c.id(i, j - 1);
  // rho_dz(0:SOUTHWEST) at (id, id, id, idS, idW, id, id, idSW)
  double rm0 = c.mass[id] + c.mean_m[id], rmS = c.mass[idS] + c.mean_m[idS], rmW = c.mass[idW] + c.mean_m[idW],
         rmSW = c.mass[idSW] + c.mean_m[idSW];
  double rt0 = c.temp[id] + c.mean_t[id], rtS = c.temp[idS] + c.mean_t[idS], rtW = c.temp[idW] + c.mean_t[idW],
         rtSW = c.temp[idSW] + c.mean_t[idSW];
  const double* v = c.velo;
  double u_prim_RT_W = v[c.E(RT, idW)] * L.len[c.E(RT, idW)];
  double u_prim_DG_SW = v[c.E(DG, idSW)] * L.len[c.E(DG, idSW)];
  double u_prim_UP_S = v[c.E(UP, idS)] * L.len[c.E(UP, idS)];
  double u_prim_RT_SW = v[c.E(RT, idSW)] * L.len[c.E(RT, idSW)];
  double u_prim_UP_SW = v[c.E(UP, idSW)] * L.len[c.E(UP, idSW)];

  double circ_SW_LORT = u_prim_RT_SW + u_prim_UP_S + u_prim_DG_SW;
  double circ_SW_UPLT = -(u_prim_RT_W + u_prim_DG_SW + u_prim_UP_SW);

  double pv_mass1 = rmSW * c.part(idSW, 1) + rmS * c.part(idS, 3) + rm0 * c.part(id, 5);
  double pv_mass2 = rmSW * c.part(idSW, 2) + rm0 * c.part(id, 4) + rmW * c.part(idW, 6);

  double pv_SW_LORT = (L.coriolis[c.E(LORT, idSW)] + circ_SW_LORT) / pv_mass1;
  double pv_SW_UPLT = (L.coriolis[c.E(UPLT, idSW)] + circ_SW_UPLT) / pv_mass2;

  c.qe[c.E(RT, idW)] = interp(st.pv_W_LORT, pv_SW_UPLT);
  c.qe[c.E(DG, idSW)] = interp(pv_SW_LORT, pv_SW_UPLT);
  c.qe[c.E(UP, idS)] = interp(pv_SW_LORT, st.pv_S_UPLT);

  c.vort[c.E(LORT, idSW)] = circ_SW_LORT / L.triarea[c.E(LORT, idSW)];
  c.vort[c.E(UPLT, idSW)] = circ_SW_UPLT / L.triarea[c.E(UPLT, idSW)];

  c.hflux_m[c.E(RT, idW)] = st.u_dual_RT_W * interp(rm0, rmW) + 0.0;
  c.hflux_m[c.E(DG, idSW)] = st.u_dual_DG_SW * interp(rm0, rmSW) + 0.0;
  c.hflux_m[c.E(UP, idS)] = st.u_dual_UP_S * interp(rm0, rmS) + 0.0;
  c.hflux_t[c.E(RT, idW)] = st.u_dual_RT_W * interp(rt0, rtW) + 0.0;
  c.hflux_t[c.E(DG, idSW)] = st.u_dual_DG_SW * interp(rt0, rtSW) + 0.0;
  c.hflux_t[c.E(UP, idS)] = st.u_dual_UP_S * interp(rt0, rtS) + 0.0;
}

// Domain-level traversal of step1 for a lozenge that is one patch with all
// four sides on the domain boundary (S_bdry = W_bdry = true).
void step1(Ctx& c) {
  const int n = c.L.n;
  Step1State st{};
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      comput(c, st, i, j);
      if (i == 0 || j == 0) comp_SW(c, st, i, j);
    }
  // north ghost row and the north-east point
  for (int i = 0; i < n; ++i) {
    comput(c, st, i, n);
    if (i == 0) comp_SW(c, st, i, n);
  }
  comput(c, st, n, n);
  // east ghost column
  for (int j = 0; j < n; ++j) {
    comput(c, st, n, j);
    if (j == 0) comp_SW(c, st, n, j);
  }
}

void post_step1(Ctx& c, int corner) {
  const Lev& L = c.L;
  const int n = c.L.n;
  auto rho = [&](int64_t k) { return c.mass[k] + c.mean_m[k]; };
  auto pr = [&](int e, int64_t k) { return c.velo[c.E(e, k)] * L.len[c.E(e, k)]; };
  if (corner == 7) {  // IJMINUS
    int64_t id = c.id(0, 0), idN = c.id(0, 1), idE = c.id(1, 0), idS = c.id(0, -1), idW = c.id(-1, 0), idSW = c.id(-1, -1);
    double r0 = rho(id), rN = rho(idN), rE = rho(idE), rS = rho(idS), rW = rho(idW);
    double u_prim_RT_W = pr(RT, idW), u_prim_RT_SW = pr(RT, idSW), u_prim_UP_S = pr(UP, idS);
    double circ_SW_LORT = u_prim_UP_S - u_prim_RT_W + u_prim_RT_SW;
    double circ_W_LORT = c.vort[c.E(LORT, idW)] * L.triarea[c.E(LORT, idW)];
    double circ_S_UPLT = c.vort[c.E(UPLT, idS)] * L.triarea[c.E(UPLT, idS)];
    c.vort[c.E(LORT, idSW)] = circ_SW_LORT / L.triarea[c.E(LORT, idSW)];
    c.vort[c.E(UPLT, idSW)] = c.vort[c.E(LORT, idSW)];
    double pm1 = rW * c.part(idW, 6) + r0 * (c.part(id, 4) + c.part(id, 5)) + rS * c.part(idS, 3);
    double pm2 = rW * c.part(idW, 1) + r0 * c.part(id, 3) + rN * c.part(idN, 5);
    double pm3 = rS * c.part(idS, 2) + rE * c.part(idE, 4) + r0 * c.part(id, 6);
    double pv_W_LORT = (L.coriolis[c.E(LORT, idW)] + circ_W_LORT) / pm1;
    double pv_SW_LORT = (L.coriolis[c.E(LORT, idSW)] + circ_SW_LORT) / pm2;
    double pv_S_UPLT = (L.coriolis[c.E(UPLT, idS)] + circ_S_UPLT) / pm3;
    double pv_SW_UPLT = pv_SW_LORT;
    c.qe[c.E(RT, idW)] = interp(pv_W_LORT, pv_SW_UPLT);
    c.qe[c.E(UP, idS)] = interp(pv_S_UPLT, pv_SW_LORT);
  }
  if (corner == 6) {  // IPLUSJMINUS
    int64_t id = c.id(n, 0), idE = c.id(n + 1, 0), idS = c.id(n, -1), idW = c.id(n - 1, 0), idNE = c.id(n + 1, 1),
            idSW = c.id(n - 1, -1);
    double r0 = rho(id), rE = rho(idE), rS = rho(idS), rW = rho(idW), rNE = rho(idNE), rSW = rho(idSW);
    double u_prim_RT_SW = pr(RT, idSW), u_prim_DG_SW = pr(DG, idSW), u_prim_RT = pr(RT, id);
    double circ_SW_LORT = -u_prim_RT + u_prim_RT_SW + u_prim_DG_SW;
    double circ_LORT = c.vort[c.E(LORT, id)] * L.triarea[c.E(LORT, id)];
    double circ_SW_UPLT = c.vort[c.E(UPLT, idSW)] * L.triarea[c.E(UPLT, idSW)];
    c.vort[c.E(LORT, idSW)] = circ_SW_LORT / L.triarea[c.E(LORT, idSW)];
    c.vort[c.E(UPLT, idS)] = c.vort[c.E(LORT, idSW)];
    double pm1 = rSW * c.part(idSW, 1) + rS * c.part(idS, 3) + r0 * (c.part(id, 5) + c.part(id, 6));
    double pm2 = r0 * c.part(id, 1) + rE * c.part(idE, 3) + rNE * c.part(idNE, 5);
    double pm3 = rSW * c.part(idSW, 2) + r0 * c.part(id, 4) + rW * c.part(idW, 6);
    double pv_SW_LORT = (L.coriolis[c.E(LORT, idSW)] + circ_SW_LORT) / pm1;
    double pv_LORT = (L.coriolis[c.E(LORT, id)] + circ_LORT) / pm2;
    double pv_SW_UPLT = (L.coriolis[c.E(UPLT, idSW)] + circ_SW_UPLT) / pm3;
    double pv_S_UPLT = pv_SW_LORT;
    c.qe[c.E(RT, id)] = interp(pv_S_UPLT, pv_LORT);
    c.qe[c.E(DG, idSW)] = interp(pv_SW_LORT, pv_SW_UPLT);
  }
  if (corner == 8) {  // IMINUSJPLUS
    int64_t id = c.id(0, n), idN = c.id(0, n + 1), idS = c.id(0, n - 1), idW = c.id(-1, n), idNE = c.id(1, n + 1),
            idSW = c.id(-1, n - 1);
    double r0 = rho(id), rN = rho(idN), rS = rho(idS), rW = rho(idW), rNE = rho(idNE), rSW = rho(idSW);
    double u_prim_UP = pr(UP, id), u_prim_DG_SW = pr(DG, idSW), u_prim_UP_SW = pr(UP, idSW);
    double circ_SW_UPLT = u_prim_UP - u_prim_DG_SW - u_prim_UP_SW;
    double circ_UPLT = c.vort[c.E(UPLT, id)] * L.triarea[c.E(UPLT, id)];
    double circ_SW_LORT = c.vort[c.E(LORT, idSW)] * L.triarea[c.E(LORT, idSW)];
    c.vort[c.E(UPLT, idSW)] = circ_SW_UPLT / L.triarea[c.E(UPLT, idSW)];
    c.vort[c.E(LORT, idW)] = c.vort[c.E(UPLT, idSW)];
    double pm1 = rSW * c.part(idSW, 2) + r0 * (c.part(id, 3) + c.part(id, 4)) + rW * c.part(idW, 6);
    double pm2 = r0 * c.part(id, 2) + rNE * c.part(idNE, 4) + rN * c.part(idN, 6);
    double pm3 = rSW * c.part(idSW, 1) + rS * c.part(idS, 3) + r0 * c.part(id, 5);
    double pv_SW_UPLT = (L.coriolis[c.E(UPLT, idSW)] + circ_SW_UPLT) / pm1;
    double pv_UPLT = (L.coriolis[c.E(UPLT, id)] + circ_UPLT) / pm2;
    double pv_SW_LORT = (L.coriolis[c.E(LORT, idSW)] + circ_SW_LORT) / pm3;
    double pv_W_LORT = pv_SW_UPLT;
    c.qe[c.E(UP, id)] = interp(pv_W_LORT, pv_UPLT);
    c.qe[c.E(DG, idSW)] = interp(pv_SW_LORT, pv_SW_UPLT);
  }
  if (corner == 5) {  // IJPLUS
    int64_t id = c.id(n, n), idN = c.id(n, n + 1), idE = c.id(n + 1, n), idS = c.id(n, n - 1), idW = c.id(n - 1, n);
    double r0 = rho(id), rN = rho(idN), rE = rho(idE), rS = rho(idS), rW = rho(idW);
    double u_prim_RT = pr(RT, id), u_prim_RT_N = pr(RT, idN), u_prim_UP = pr(UP, id);
    double circ_LORT = u_prim_RT - u_prim_RT_N - u_prim_UP;
    double circ_W_LORT = c.vort[c.E(LORT, idW)] * L.triarea[c.E(LORT, idW)];
    double circ_S_UPLT = c.vort[c.E(UPLT, idS)] * L.triarea[c.E(UPLT, idS)];
    c.vort[c.E(LORT, id)] = circ_LORT / L.triarea[c.E(LORT, id)];
    c.vort[c.E(UPLT, id)] = c.vort[c.E(LORT, id)];
    double pm1 = rE * c.part(idE, 3) + r0 * (c.part(id, 1) + c.part(id, 2)) + rN * c.part(idN, 6);
    double pm2 = rW * c.part(idW, 1) + r0 * c.part(id, 3) + rN * c.part(idN, 5);
    double pm3 = rS * c.part(idS, 2) + rE * c.part(idE, 4) + r0 * c.part(id, 6);
    double pv_LORT = (L.coriolis[c.E(LORT, id)] + circ_LORT) / pm1;
    double pv_W_LORT = (L.coriolis[c.E(LORT, idW)] + circ_W_LORT) / pm2;
    double pv_S_UPLT = (L.coriolis[c.E(UPLT, idS)] + circ_S_UPLT) / pm3;
    double pv_UPLT = pv_LORT;
    c.qe[c.E(RT, id)] = interp(pv_LORT, pv_S_UPLT);
    c.qe[c.E(UP, id)] = interp(pv_UPLT, pv_W_LORT);
  }
}

double divg(const Ctx& c, const double* hf, int i, int j) {   // div, src/ops.f90:1325
  int64_t id = c.id(i, j), idS = c.id(i, j - 1), idW = c.id(i - 1, j), idSW = c.id(i - 1, j - 1);
  return (hf[c.E(RT, id)] - hf[c.E(RT, idW)] + hf[c.E(DG, idSW)] - hf[c.E(DG, id)] + hf[c.E(UP, id)] - hf[c.E(UP, idS)]) *
         c.L.hex_inv[id];
}

void get_weights(const Ctx& c, int64_t id, int offs, double w[5]) {   // src/ops.f90:1006
  double wgt[5];
  wgt[0] = c.part(id, 1 + offs);
  for (int i = 2; i <= 5; ++i) wgt[i - 1] = wgt[i - 2] + c.part(id, ((i + offs - 1) % 6) + 1);
  for (int i = 0; i < 5; ++i) wgt[i] = 0.5 - wgt[i] * c.L.hex_inv[id];
  w[0] = wgt[0]; w[1] = -wgt[1]; w[2] = wgt[2]; w[3] = -wgt[3]; w[4] = wgt[4];
}

void Qperp(const Ctx& c, int i, int j, double Q[3]) {   // src/ops.f90:834
  const double* hm = c.hflux_m;
  const double* qe = c.qe;
  int64_t id = c.id(i, j), idNW = c.id(i - 1, j + 1), idN = c.id(i, j + 1), idNE = c.id(i + 1, j + 1), idW = c.id(i - 1, j),
          idE = c.id(i + 1, j), idSW = c.id(i - 1, j - 1), idS = c.id(i, j - 1), idSE = c.id(i + 1, j - 1);
  auto T = [&](int e1, int64_t n1, int e0, int64_t n0, double w) {
    return hm[c.E(e1, n1)] * interp(qe[c.E(e1, n1)], qe[c.E(e0, n0)]) * w;
  };
  double w1[5], w2[5];
  get_weights(c, id, 0, w1);
  get_weights(c, idE, 3, w2);
  Q[RT] = T(DG, id, RT, id, w1[0]) + T(UP, id, RT, id, w1[1]) + T(RT, idW, RT, id, w1[2]) + T(DG, idSW, RT, id, w1[3]) +
          T(UP, idS, RT, id, w1[4]) + T(DG, idS, RT, id, w2[0]) + T(UP, idSE, RT, id, w2[1]) + T(RT, idE, RT, id, w2[2]) +
          T(DG, idE, RT, id, w2[3]) + T(UP, idE, RT, id, w2[4]);
  get_weights(c, id, 1, w1);
  get_weights(c, idNE, 4, w2);
  Q[DG] = T(UP, id, DG, id, w1[0]) + T(RT, idW, DG, id, w1[1]) + T(DG, idSW, DG, id, w1[2]) + T(UP, idS, DG, id, w1[3]) +
          T(RT, id, DG, id, w1[4]) + T(UP, idE, DG, id, w2[0]) + T(RT, idNE, DG, id, w2[1]) + T(DG, idNE, DG, id, w2[2]) +
          T(UP, idNE, DG, id, w2[3]) + T(RT, idN, DG, id, w2[4]);
  get_weights(c, id, 2, w1);
  get_weights(c, idN, 5, w2);
  Q[UP] = T(RT, idW, UP, id, w1[0]) + T(DG, idSW, UP, id, w1[1]) + T(UP, idS, UP, id, w1[2]) + T(RT, id, UP, id, w1[3]) +
          T(DG, id, UP, id, w1[4]) + T(RT, idN, UP, id, w2[0]) + T(DG, idN, UP, id, w2[1]) + T(UP, idN, UP, id, w2[2]) +
          T(RT, idNW, UP, id, w2[3]) + T(DG, idW, UP, id, w2[4]);
}

struct Work {
  std::vector<double> qe, vort, ke, bernoulli, exner, hflux_m, hflux_t, geopot, geopot_lower, press, press_lower, surf_press;
  explicit Work(int64_t NN)
      : qe(3 * NN), vort(2 * NN), ke(NN), bernoulli(NN), exner(NN), hflux_m(3 * NN), hflux_t(3 * NN), geopot(NN),
        geopot_lower(NN), press(NN), press_lower(NN), surf_press(NN) {}
};

// trend_ml on one uniform level (level_start == level_end).  q is updated in
// place by the initial halo copy (update_bdry), as in the reference.
void trend_ml(const Lev& L, const Phys& ph, int nz, double* mass, double* temp, double* velo, const double* mean_m,
              const double* mean_t, const double* topo, double* dmass, double* dtemp, double* dvelo, Work& w) {
  const int64_t NN = L.NN;
  const int n = L.n;
  for (int k = 0; k < nz; ++k) {
    halo_nodes(L, mass + k * NN);
    halo_nodes(L, temp + k * NN);
    halo_edges(L, velo + k * 3 * NN);
  }
  // Every lozenge is an independent domain between ghost copies (the
  // reference's MPI decomposition); the per-lozenge loops run in parallel.
  auto ctx = [&](int d) {
    Ctx c(L, ph);
    c.d = d;
    c.qe = w.qe.data(); c.vort = w.vort.data(); c.ke = w.ke.data(); c.bernoulli = w.bernoulli.data();
    c.exner = w.exner.data(); c.hflux_m = w.hflux_m.data(); c.hflux_t = w.hflux_t.data(); c.geopot = w.geopot.data();
    c.geopot_lower = w.geopot_lower.data(); c.press = w.press.data(); c.press_lower = w.press_lower.data();
    c.surf_press = w.surf_press.data(); c.topo = topo;
    return c;
  };
  // zero_float_field over [-(BDRY-1), BDRY] (src/utils.f90:1217)
  pool().run([&](int d) {
    Ctx c = ctx(d);
    for (int k = 0; k < nz; ++k)
      for (int j = -1; j <= n + 1; ++j)
        for (int i = -1; i <= n + 1; ++i) {
          int64_t id = c.id(i, j);
          dmass[k * NN + id] = 0.0;
          dtemp[k * NN + id] = 0.0;
          for (int e = 0; e < 3; ++e) dvelo[k * 3 * NN + e * NN + id] = 0.0;
        }
  });
  // cal_surf_press: set_surf_geopot over [-1, n+1]; column_mass over [0, n]
  for (int64_t id = 0; id < NN; ++id) w.surf_press[id] = 0.0;
  pool().run([&](int d) {
    Ctx c = ctx(d);
    for (int j = -1; j <= n + 1; ++j)
      for (int i = -1; i <= n + 1; ++i) w.geopot[c.id(i, j)] = ph.grav * topo[c.id(i, j)];
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t id = c.id(i, j);
          double rho_dz = mean_m[k * NN + id] + mass[k * NN + id];
          double rho_dz_theta = mean_t[k * NN + id] + temp[k * NN + id];
          w.surf_press[id] = w.surf_press[id] + (rho_dz - rho_dz_theta);
        }
  });
  for (int64_t id = 0; id < NN; ++id) {
    w.surf_press[id] = ph.grav * w.surf_press[id] + ph.p_top;
    w.press_lower[id] = w.surf_press[id];
  }
  for (int k = 0; k < nz; ++k) {
    // basic_operators: integrate_pressure_up then step1, per lozenge; post_step1 at the corners
    pool().run([&](int d) {
      Ctx c = ctx(d);
      c.mass = mass + k * NN; c.temp = temp + k * NN; c.velo = velo + k * 3 * NN;
      c.mean_m = mean_m + k * NN; c.mean_t = mean_t + k * NN;
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t id = c.id(i, j);
          double rho_dz = c.mean_m[id] + c.mass[id];
          double rho_dz_theta = c.mean_t[id] + c.temp[id];
          w.geopot_lower[id] = w.geopot[id];
          double p_upper = w.press_lower[id] - ph.grav * (rho_dz - rho_dz_theta);
          w.press[id] = interp(w.press_lower[id], p_upper);
          w.geopot[id] = w.geopot_lower[id] + ph.grav * rho_dz / (ph.ref_density * 1.0);
          w.press_lower[id] = p_upper;
        }
      step1(c);
      for (int corner = 5; corner <= 8; ++corner) post_step1(c, corner);   // apply_to_penta_d order NE..NW
    });
    // cal_scalar_trend: update_bdry(horiz_flux) then scalar_trend over [0, n]
    halo_edges(L, w.hflux_m.data());
    halo_edges(L, w.hflux_t.data());
    double* dv = dvelo + k * 3 * NN;
    pool().run([&](int d) {
      Ctx c = ctx(d);
      c.mass = mass + k * NN; c.temp = temp + k * NN; c.velo = velo + k * 3 * NN;
      c.mean_m = mean_m + k * NN; c.mean_t = mean_t + k * NN;
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          int64_t id = c.id(i, j);
          dmass[k * NN + id] = -divg(c, w.hflux_m.data(), i, j);
          dtemp[k * NN + id] = -divg(c, w.hflux_t.data(), i, j);
        }
      // velocity_trend_source (du_source) then velocity_trend_grad (du_grad) on owned nodes
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          int64_t id = c.id(i, j);
          double Q[3];
          Qperp(c, i, j, Q);
          for (int e = 0; e < 3; ++e) dv[e * NN + id] = -Q[e] + 0.0 * L.len[e * NN + id];
        }
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          int64_t id = c.id(i, j), idE = c.id(i + 1, j), idN = c.id(i, j + 1), idNE = c.id(i + 1, j + 1);
          int64_t ids[4] = {id, idE, idNE, idN};
          double theta[4];
          for (int q = 0; q < 4; ++q) {
            double rdz = c.mean_m[ids[q]] + c.mass[ids[q]];
            double rdzt = c.mean_t[ids[q]] + c.temp[ids[q]];
            theta[q] = rdzt / rdz;
          }
          double theta_e[3] = {interp(theta[0], theta[1]), interp(theta[0], theta[2]), interp(theta[0], theta[3])};
          const double* B = w.bernoulli.data();
          const double* X = w.exner.data();
          double gradB[3] = {(B[idE] - B[id]) / L.len[RT * NN + id], (B[id] - B[idNE]) / L.len[DG * NN + id],
                             (B[idN] - B[id]) / L.len[UP * NN + id]};
          double gradE[3] = {(X[idE] - X[id]) / L.len[RT * NN + id], (X[id] - X[idNE]) / L.len[DG * NN + id],
                             (X[idN] - X[id]) / L.len[UP * NN + id]};
          for (int e = 0; e < 3; ++e)
            dv[e * NN + id] = dv[e * NN + id] / L.len[e * NN + id] - gradB[e] - theta_e[e] * gradE[e];
        }
    });
  }
}

void rk_sub_step(int64_t count, const double* sol, const double* trend, double h, double* dest) {
  for (int64_t i = 0; i < count; ++i) dest[i] = sol[i] + h * trend[i];
}

}  // namespace

extern "C" {

void orc_set_threads(int n) { pool().set_threads(n); }

int orc_get_threads(void) { return pool().threads(); }

struct orc_level {
  int n, P;
  int64_t NN;
  const double *len, *pedlen, *part, *hex_inv, *triarea, *coriolis;
  const int64_t* halo_node;
  int64_t n_halo_node;
  const int64_t* halo_edge;
  int64_t n_halo_edge;
};

static Lev to_lev(const orc_level* o) {
  return Lev{o->n, o->P, o->NN, o->len, o->pedlen, o->part, o->hex_inv, o->triarea, o->coriolis,
             o->halo_node, o->n_halo_node, o->halo_edge, o->n_halo_edge};
}

// One evaluation of trend_ml.  mass/temp/velo are updated in place by the
// halo copy; dmass/dtemp/dvelo receive the trends; diag (optional, may be NULL)
// receives qe (3*NN), bernoulli (NN), exner (NN) of the last layer.
int orc_trend(const orc_level* lev, int nz, double grav, double ref_density, double p_top, double* mass, double* temp,
              double* velo, const double* mean_m, const double* mean_t, const double* topo, double* dmass, double* dtemp,
              double* dvelo) {
  Lev L = to_lev(lev);
  Phys ph{grav, ref_density, p_top};
  Work w(L.NN);
  trend_ml(L, ph, nz, mass, temp, velo, mean_m, mean_t, topo, dmass, dtemp, dvelo, w);
  return 0;
}

// nsteps of the low-storage RK4 of src/time_integr.f90:78-103 with
// WT_after_step reduced to its halo copy (uniform grid: level_start == level_end).
int orc_rk4(const orc_level* lev, int nz, double grav, double ref_density, double p_top, double dt, int nsteps,
            double* mass, double* temp, double* velo, const double* mean_m, const double* mean_t, const double* topo) {
  Lev L = to_lev(lev);
  Phys ph{grav, ref_density, p_top};
  Work w(L.NN);
  const int64_t NN = L.NN, nn = nz * NN, ne = nz * 3 * NN;
  std::vector<double> m1(mass, mass + nn), t1(temp, temp + nn), v1(velo, velo + ne);
  std::vector<double> dm(nn, 0.0), dtt(nn, 0.0), dv(ne, 0.0);
  const double hs[4] = {dt / 4.0, dt / 3.0, dt / 2.0, dt};
  for (int s = 0; s < nsteps; ++s) {
    for (int stage = 0; stage < 4; ++stage) {
      double* qm = stage == 0 ? mass : m1.data();
      double* qt = stage == 0 ? temp : t1.data();
      double* qv = stage == 0 ? velo : v1.data();
      trend_ml(L, ph, nz, qm, qt, qv, mean_m, mean_t, topo, dm.data(), dtt.data(), dv.data(), w);
      double* om = stage == 3 ? mass : m1.data();
      double* ot = stage == 3 ? temp : t1.data();
      double* ov = stage == 3 ? velo : v1.data();
      rk_sub_step(nn, mass, dm.data(), hs[stage], om);
      rk_sub_step(nn, temp, dtt.data(), hs[stage], ot);
      rk_sub_step(ne, velo, dv.data(), hs[stage], ov);
      // WT_after_step: update_bdry of the new state
      for (int k = 0; k < nz; ++k) {
        halo_nodes(L, om + k * NN);
        halo_nodes(L, ot + k * NN);
        halo_edges(L, ov + k * 3 * NN);
      }
    }
  }
  return 0;
}

// One level of a uniform hierarchy for trend_ml over levels level_start ..
// level_end: geometry, weights, masks, state (updated in place by the halo
// copy) and trends (out).
struct orc_mlevel {
  orc_level geo;
  const double *overl_a, *overl_split, *rf_wgt;  // rf_wgt may be NULL on level_start
  const int32_t *mask_n, *mask_e;
  double *mass, *temp, *velo;                    // [nz][NN], [nz][NN], [nz][3*NN]
  const double *mean_m, *mean_t, *topo;
  double *dmass, *dtemp, *dvelo;                 // out, same shapes
};

int orc_trend_multi(const orc_mlevel* lv, int nlev, int nz, double grav, double ref_density, double p_top) {
  constexpr int TRSK = 2, ADJZONE = 8;
  Phys ph{grav, ref_density, p_top};
  std::vector<Lev> L;
  std::vector<Work> W;
  for (int q = 0; q < nlev; ++q) {
    L.push_back(to_lev(&lv[q].geo));
    W.emplace_back(L[q].NN);
  }
  auto ctx = [&](int q, int d, int k) {
    Ctx c(L[q], ph);
    Work& w = W[q];
    const orc_mlevel& m = lv[q];
    const int64_t NN = L[q].NN;
    c.d = d;
    c.qe = w.qe.data(); c.vort = w.vort.data(); c.ke = w.ke.data(); c.bernoulli = w.bernoulli.data();
    c.exner = w.exner.data(); c.hflux_m = w.hflux_m.data(); c.hflux_t = w.hflux_t.data(); c.geopot = w.geopot.data();
    c.geopot_lower = w.geopot_lower.data(); c.press = w.press.data(); c.press_lower = w.press_lower.data();
    c.surf_press = w.surf_press.data(); c.topo = m.topo;
    c.mass = m.mass + k * NN; c.temp = m.temp + k * NN; c.velo = m.velo + k * 3 * NN;
    c.mean_m = m.mean_m + k * NN; c.mean_t = m.mean_t + k * NN;
    return c;
  };
  // restriction records of level q with the given layer fields
  auto rlev = [&](int q, double* scal, double* dscal, double* flux, double* dvelo) {
    const orc_mlevel& m = lv[q];
    return orc_rlevel{L[q].n, L[q].P, L[q].NN, L[q].hex_inv, m.overl_a, m.overl_split, m.rf_wgt,
                      L[q].hnode, L[q].n_hnode, L[q].hedge, L[q].n_hedge, m.mask_n, m.mask_e,
                      scal, dscal, flux, dvelo};
  };
  // update_bdry(q, NONE) and zero_float_field of the trends
  for (int q = 0; q < nlev; ++q) {
    const int64_t NN = L[q].NN;
    for (int k = 0; k < nz; ++k) {
      halo_nodes(L[q], lv[q].mass + k * NN);
      halo_nodes(L[q], lv[q].temp + k * NN);
      halo_edges(L[q], lv[q].velo + k * 3 * NN);
    }
    std::memset(lv[q].dmass, 0, nz * NN * sizeof(double));
    std::memset(lv[q].dtemp, 0, nz * NN * sizeof(double));
    std::memset(lv[q].dvelo, 0, 3 * nz * NN * sizeof(double));
  }
  // cal_surf_press on every level
  for (int q = 0; q < nlev; ++q) {
    const int64_t NN = L[q].NN;
    const int n = L[q].n;
    Work& w = W[q];
    const orc_mlevel& m = lv[q];
    for (int64_t id = 0; id < NN; ++id) w.surf_press[id] = 0.0;
    for (int d = 0; d < 10; ++d) {
      Ctx c = ctx(q, d, 0);
      for (int j = -1; j <= n + 1; ++j)
        for (int i = -1; i <= n + 1; ++i) w.geopot[c.id(i, j)] = ph.grav * m.topo[c.id(i, j)];
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j <= n; ++j)
          for (int i = 0; i <= n; ++i) {
            const int64_t id = c.id(i, j);
            const double rho_dz = m.mean_m[k * NN + id] + m.mass[k * NN + id];
            const double rho_dz_theta = m.mean_t[k * NN + id] + m.temp[k * NN + id];
            w.surf_press[id] = w.surf_press[id] + (rho_dz - rho_dz_theta);
          }
    }
    for (int64_t id = 0; id < NN; ++id) {
      w.surf_press[id] = ph.grav * w.surf_press[id] + ph.p_top;
      w.press_lower[id] = w.surf_press[id];
    }
  }
  for (int k = 0; k < nz; ++k) {
    for (int q = nlev - 1; q >= 0; --q) {
      const Lev& Lq = L[q];
      const int64_t NN = Lq.NN;
      const int n = Lq.n;
      Work& w = W[q];
      const orc_mlevel& m = lv[q];
      // basic_operators
      pool().run([&](int d) {
        Ctx c = ctx(q, d, k);
        for (int j = 0; j <= n; ++j)
          for (int i = 0; i <= n; ++i) {
            const int64_t id = c.id(i, j);
            const double rho_dz = c.mean_m[id] + c.mass[id];
            const double rho_dz_theta = c.mean_t[id] + c.temp[id];
            w.geopot_lower[id] = w.geopot[id];
            const double p_upper = w.press_lower[id] - ph.grav * (rho_dz - rho_dz_theta);
            w.press[id] = interp(w.press_lower[id], p_upper);
            w.geopot[id] = w.geopot_lower[id] + ph.grav * rho_dz / (ph.ref_density * 1.0);
            w.press_lower[id] = p_upper;
          }
        step1(c);
        for (int corner = 5; corner <= 8; ++corner) post_step1(c, corner);
      });
      if (q < nlev - 1) {
        Work& wc = W[q + 1];
        const int64_t NC = L[q + 1].NN;
        orc_rlevel P = rlev(q, w.bernoulli.data(), nullptr, nullptr, nullptr);
        orc_rlevel C = rlev(q + 1, wc.bernoulli.data(), nullptr, nullptr, nullptr);
        orc_restrict_scalar(&P, &C, 1);
        P.scal = w.exner.data();
        C.scal = wc.exner.data();
        orc_restrict_scalar(&P, &C, 1);
        P.flux = w.hflux_m.data();
        C.flux = wc.hflux_m.data();
        C.dscal = lv[q + 1].dmass + k * NC;
        orc_restrict_flux(&P, &C, 1);
        P.flux = w.hflux_t.data();
        C.flux = wc.hflux_t.data();
        C.dscal = lv[q + 1].dtemp + k * NC;
        orc_restrict_flux(&P, &C, 1);
      }
      // cal_scalar_trend: update_bdry(horiz_flux, l), scalar_trend over [0, n]
      halo_edges(Lq, w.hflux_m.data());
      halo_edges(Lq, w.hflux_t.data());
      pool().run([&](int d) {
        Ctx c = ctx(q, d, k);
        for (int j = 0; j <= n; ++j)
          for (int i = 0; i <= n; ++i) {
            const int64_t id = c.id(i, j);
            const bool on = m.mask_n[id] >= TRSK;
            m.dmass[k * NN + id] = on ? -divg(c, w.hflux_m.data(), i, j) : 0.0;
            m.dtemp[k * NN + id] = on ? -divg(c, w.hflux_t.data(), i, j) : 0.0;
          }
      });
      // velocity_trend_source
      double* dv = m.dvelo + k * 3 * NN;
      auto u_source = [&](Ctx& c, int i, int j) {
        const int64_t id = c.id(i, j);
        if (m.mask_n[id] >= TRSK) {
          double Q[3];
          Qperp(c, i, j, Q);
          for (int e = 0; e < 3; ++e) dv[e * NN + id] = -Q[e] + 0.0 * Lq.len[e * NN + id];
        } else {
          for (int e = 0; e < 3; ++e) dv[e * NN + id] = 0.0;
        }
      };
      if (q == nlev - 1) {
        pool().run([&](int d) {
          Ctx c = ctx(q, d, k);
          for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) u_source(c, i, j);
        });
      } else {
        const Lev& Lc = L[q + 1];
        const int32_t* mc = lv[q + 1].mask_e;
        pool().run([&](int d) {
          Ctx c = ctx(q, d, k);
          for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
              const int64_t idc = ((int64_t)d * Lc.P + 2 * j + 2) * Lc.P + 2 * i + 2;
              int mn = mc[idc];
              for (int e = 1; e < 3; ++e) mn = mc[e * Lc.NN + idc] < mn ? mc[e * Lc.NN + idc] : mn;
              if (mn < ADJZONE) u_source(c, i, j);
            }
        });
        orc_rlevel P = rlev(q, nullptr, nullptr, nullptr, dv);
        orc_rlevel C = rlev(q + 1, nullptr, nullptr, nullptr, lv[q + 1].dvelo + k * 3 * Lc.NN);
        orc_restrict_u_source(&P, &C, 1);
      }
    }
    // velocity_trend_grad on every level
    for (int q = 0; q < nlev; ++q) {
      const Lev& Lq = L[q];
      const int64_t NN = Lq.NN;
      const int n = Lq.n;
      Work& w = W[q];
      const orc_mlevel& m = lv[q];
      double* dv = m.dvelo + k * 3 * NN;
      pool().run([&](int d) {
        Ctx c = ctx(q, d, k);
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const int64_t id = c.id(i, j), idE = c.id(i + 1, j), idN = c.id(i, j + 1), idNE = c.id(i + 1, j + 1);
            if (m.mask_n[id] < TRSK) {
              for (int e = 0; e < 3; ++e) dv[e * NN + id] = 0.0;
              continue;
            }
            const int64_t ids[4] = {id, idE, idNE, idN};
            double theta[4];
            for (int t = 0; t < 4; ++t) {
              const double rdz = c.mean_m[ids[t]] + c.mass[ids[t]];
              const double rdzt = c.mean_t[ids[t]] + c.temp[ids[t]];
              theta[t] = rdzt / rdz;
            }
            const double theta_e[3] = {interp(theta[0], theta[1]), interp(theta[0], theta[2]),
                                       interp(theta[0], theta[3])};
            const double* B = w.bernoulli.data();
            const double* X = w.exner.data();
            const double gradB[3] = {(B[idE] - B[id]) / Lq.len[RT * NN + id], (B[id] - B[idNE]) / Lq.len[DG * NN + id],
                                     (B[idN] - B[id]) / Lq.len[UP * NN + id]};
            const double gradE[3] = {(X[idE] - X[id]) / Lq.len[RT * NN + id], (X[id] - X[idNE]) / Lq.len[DG * NN + id],
                                     (X[idN] - X[id]) / Lq.len[UP * NN + id]};
            for (int e = 0; e < 3; ++e)
              dv[e * NN + id] = dv[e * NN + id] / Lq.len[e * NN + id] - gradB[e] - theta_e[e] * gradE[e];
          }
      });
    }
  }
  return 0;
}

}  // extern "C"
