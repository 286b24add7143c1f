// Elliptic free-surface solver: device data, the reference's FMG / SRJ /
// BiCGSTAB control flow (src/lin_solve.f90) driving the kernels of
// elliptic_kernels.cuh, and an FP64 iterative refinement around FP32 V-cycles.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/wavetrisk_gpu.h"
#include "elliptic_kernels.cuh"
#include "wt_handle.cuh"

using namespace wte;

#define CKE(x)                                                 \
  do {                                                         \
    cudaError_t e_ = (x);                                      \
    if (e_ != cudaSuccess) return wt_handle_fail(#x, e_);     \
  } while (0)

namespace {

constexpr int TPB = 256;
inline unsigned nb(int64_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

// One multi-level field: a device buffer per level.
struct MField {
  std::vector<double*> lv;
  std::vector<float*> lvf;
};

struct ELevelDev {
  int level = 0, n = 0, P = 0, nd = 1;
  int64_t NN = 0;
  double *Ie = nullptr, *diag = nullptr;
  int *nsrc = nullptr, *esrc = nullptr;
  float *Kf = nullptr, *hinvf = nullptr, *diagf = nullptr;
};

struct Ell {
  wt_handle* h = nullptr;
  int ls = 0, le = 0;
  double dt = 0, th1 = 1, th2 = 1, cf = 0;
  int domain_level = 2;
  std::vector<ELevelDev> L;
  MField u, f, res, corr, pf, wc_mass, wc_temp, tmp, au, rr, r0, pp, ss, ap, as_, cc, rr2;
  MField eta_wc;                   // the free surface's wavelets of its last WT_after_step
  bool eta_wc_valid = false;
  MField u32, f32, r32, c32, t32;  // FP32 V-cycle work
  double* partial = nullptr;
  double* scal = nullptr;  // device scalars
  cudaGraphExec_t cycle_exec[2] = {nullptr, nullptr};  // captured correction cycles (FP32, FP64)
  int cycle_key[2] = {-1, -1};
  std::vector<const void*> cycle_ptrs[2];  // rotating() at each cycle graph's capture
  int nbmax = 0;
  std::vector<void*> allocs;
  void* lp = nullptr;  // learned preconditioner (wt_learned.cuh)

  EllLev view(int l) const {
    const DevLevel& D = const_cast<wt_handle*>(h)->at(l);
    const ELevelDev& E = L[l - ls];
    return EllLev{D.n, D.P, E.nd, D.NN, D.len, D.pedlen, D.hex_inv, D.overl_a, E.Ie, E.diag, E.nsrc, E.esrc,
                  E.Kf, E.hinvf, E.diagf};
  }
  int m(int l) const { return L[l - ls].n + 1; }
  cudaStream_t s() const { return h->stream; }

  // The buffers whose roles the solvers rotate by swapping pointers: jacobi's
  // u/tmp and corr/tmp ping-pong, v_cycle's res/au swap and the FP32 cycle's
  // c32/t32 ping-pong.  A captured graph holds the addresses it was captured
  // with, so it may be replayed only while these are as they were then.
  std::vector<const void*> rotating() const {
    std::vector<const void*> v;
    for (const MField* F : {&u, &tmp, &corr, &res, &au})
      for (double* p : F->lv) v.push_back(p);
    for (const MField* F : {&c32, &t32})
      for (float* p : F->lvf) v.push_back(p);
    return v;
  }
  void set_rotating(const std::vector<const void*>& v) {
    size_t k = 0;
    for (MField* F : {&u, &tmp, &corr, &res, &au})
      for (double*& p : F->lv) p = const_cast<double*>(static_cast<const double*>(v[k++]));
    for (MField* F : {&c32, &t32})
      for (float*& p : F->lvf) p = const_cast<float*>(static_cast<const float*>(v[k++]));
  }
};

// Captures body() on the solver's stream into ex.  The sweeps inside body()
// swap pointers while they are captured; afterwards the host-side pointers are
// put back to what they were at the start, which is the state every replay
// of the graph starts from, and that state is stored in *ptrs as the graph's
// key (a replay is valid while E.rotating() == *ptrs).
template <class Body>
int capture_graph(Ell& E, cudaGraphExec_t& ex, std::vector<const void*>& ptrs, const char* what, Body body) {
  if (ex) {
    cudaGraphExecDestroy(ex);
    ex = nullptr;
  }
  std::vector<const void*> start = E.rotating();
  cudaGraph_t g;
  cudaError_t ce = cudaStreamBeginCapture(E.s(), cudaStreamCaptureModeThreadLocal);
  if (ce != cudaSuccess) return wt_handle_fail(what, ce);
  body();
  ce = cudaStreamEndCapture(E.s(), &g);
  E.set_rotating(start);
  if (ce != cudaSuccess) return wt_handle_fail(what, ce);
  ce = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    ex = nullptr;
    return wt_handle_fail(what, ce);
  }
  ptrs = std::move(start);
  return WT_OK;
}

template <class T>
int dalloc(Ell& E, T** p, int64_t n) {
  cudaError_t e = cudaMalloc(p, sizeof(T) * std::max<int64_t>(1, n));
  if (e != cudaSuccess) return wt_handle_fail("elliptic alloc", e);
  cudaMemset(*p, 0, sizeof(T) * std::max<int64_t>(1, n));
  E.allocs.push_back(*p);
  return WT_OK;
}

int alloc_field(Ell& E, MField& F, bool fp32 = false) {
  for (int l = E.ls; l <= E.le; ++l) {
    int64_t NN = E.h->at(l).NN;
    if (fp32) {
      float* p;
      if (int rc = dalloc(E, &p, NN)) return rc;
      F.lvf.push_back(p);
    } else {
      double* p;
      if (int rc = dalloc(E, &p, NN)) return rc;
      F.lv.push_back(p);
    }
  }
  return WT_OK;
}

}  // namespace

// ---------------------------------------------------------------- setup ----
void lp_release(void* p);

static void ell_free(Ell* E) {
  if (!E) return;
  lp_release(E->lp);
  for (auto& ex : E->cycle_exec)
    if (ex) cudaGraphExecDestroy(ex);
  for (void* p : E->allocs) cudaFree(p);
  delete E;
}

void wt_handle::release_extra() {
  if (ell) ell_free(static_cast<Ell*>(ell));
  ell = nullptr;
  wt_trend_ml_release(this);
  wt_wavelet_release(this);
  wt_barotropic_release(this);
}

extern "C" int wt_elliptic_setup(wt_handle* h, double dt, double theta1, double theta2, int domain_level) {
  if (!h || h->lev.empty() || dt <= 0) return WT_ERR_ARG;
  if (h->ell) { ell_free(static_cast<Ell*>(h->ell)); h->ell = nullptr; }
  Ell* E = new Ell();
  E->h = h;
  E->ls = h->level_start;
  E->le = h->level_end;
  E->dt = dt;
  E->th1 = theta1;
  E->th2 = theta2;
  E->cf = theta1 * theta2 * (dt * dt);
  E->domain_level = domain_level;
  const double g = h->ph.grav;
  int rc = WT_OK;
  for (int l = E->ls; l <= E->le && rc == WT_OK; ++l) {
    DevLevel& D = h->at(l);
    ELevelDev X;
    X.level = l;
    X.n = D.n;
    X.P = D.P;
    X.NN = D.NN;
    X.nd = std::max(1, D.n >> domain_level);
    const int64_t NN = D.NN;
    // host copies of the level tables needed to build the operator coefficients
    std::vector<double> topo(NN), len(3 * NN), ped(3 * NN), hinv(NN);
    cudaMemcpy(topo.data(), D.topo, 8 * NN, cudaMemcpyDeviceToHost);
    cudaMemcpy(len.data(), D.len, 8 * 3 * NN, cudaMemcpyDeviceToHost);
    cudaMemcpy(ped.data(), D.pedlen, 8 * 3 * NN, cudaMemcpyDeviceToHost);
    cudaMemcpy(hinv.data(), D.hex_inv, 8 * NN, cudaMemcpyDeviceToHost);
    // csq = g (|H| phi + eta_old) with phi = 1, eta_old = 0 (src/ops.f90:203-208)
    auto csq = [&](int64_t k) { return g * (std::fabs(topo[k]) * 1.0 + 0.0); };
    std::vector<double> Ie(3 * NN, 0.0), diag(NN, 0.0);
    std::vector<float> Kf(3 * NN, 0.f), hinvf(NN, 0.f), diagf(NN, 0.f);
    const int P = D.P;
    for (int64_t k = 0; k < NN; ++k) {
      int64_t r = k % ((int64_t)P * P);
      int i = (int)(r % P) - 2, j = (int)(r / P) - 2;
      double c0 = csq(k);
      if (i + 1 <= D.n + 1) Ie[RT * NN + k] = 0.5 * (c0 + csq(k + 1));
      if (i + 1 <= D.n + 1 && j + 1 <= D.n + 1) Ie[DG * NN + k] = 0.5 * (c0 + csq(k + P + 1));
      if (j + 1 <= D.n + 1) Ie[UP * NN + k] = 0.5 * (c0 + csq(k + P));
      // elliptic_lo_diag, exact = .false. (src/barotropic_2d.f90:283-296)
      double depth = std::fabs(topo[k]) + 0.0 / 1.0;
      double wgt = 2.0 * std::sqrt(3.0) * depth;
      double lap = -(g * wgt * (dt * dt) * hinv[k]);
      diag[k] = theta1 * theta2 * lap - 1.0;
      hinvf[k] = (float)hinv[k];
      diagf[k] = (float)diag[k];
      for (int e = 0; e < 3; ++e) {
        int64_t q = e * NN + k;
        if (len[q] > 0) Kf[q] = (float)(E->cf * Ie[q] * ped[q] / len[q]);
      }
    }
    if ((rc = dalloc(*E, &X.Ie, 3 * NN))) break;
    if ((rc = dalloc(*E, &X.diag, NN))) break;
    X.nsrc = D.nsrc;
    X.esrc = D.esrc;
    if ((rc = dalloc(*E, &X.Kf, 3 * NN))) break;
    if ((rc = dalloc(*E, &X.hinvf, NN))) break;
    if ((rc = dalloc(*E, &X.diagf, NN))) break;
    cudaMemcpy(X.Ie, Ie.data(), 8 * 3 * NN, cudaMemcpyHostToDevice);
    cudaMemcpy(X.diag, diag.data(), 8 * NN, cudaMemcpyHostToDevice);
    cudaMemcpy(X.Kf, Kf.data(), 4 * 3 * NN, cudaMemcpyHostToDevice);
    cudaMemcpy(X.hinvf, hinvf.data(), 4 * NN, cudaMemcpyHostToDevice);
    cudaMemcpy(X.diagf, diagf.data(), 4 * NN, cudaMemcpyHostToDevice);
    E->L.push_back(X);
    E->nbmax = std::max<int>(E->nbmax, (int)nb(10 * (int64_t)(D.n + 1) * (D.n + 1)));
  }
  MField* fields[] = {&E->u, &E->f, &E->res, &E->corr, &E->pf, &E->wc_mass, &E->wc_temp, &E->tmp, &E->au,
                      &E->rr, &E->r0, &E->pp, &E->ss, &E->ap, &E->as_, &E->cc, &E->rr2, &E->eta_wc};
  for (MField* F : fields)
    if (rc == WT_OK) rc = alloc_field(*E, *F);
  MField* f32[] = {&E->u32, &E->f32, &E->r32, &E->c32, &E->t32};
  for (MField* F : f32)
    if (rc == WT_OK) rc = alloc_field(*E, *F, true);
  if (rc == WT_OK) rc = dalloc(*E, &E->partial, E->nbmax);
  if (rc == WT_OK) rc = dalloc(*E, &E->scal, 64);
  if (rc != WT_OK) {
    ell_free(E);
    return rc;
  }
  h->ell = E;
  return WT_OK;
}

// ------------------------------------------------------------ operators ----
namespace {

void op(Ell& E, int OPK, int l, const double* q, const double* f, double* out, double w = 1.0) {
  EllLev V = E.view(l);
  unsigned g = nb(10 * E.m(l) * E.m(l));
  if (OPK == OP_APPLY) k_ell_op<OP_APPLY><<<g, TPB, 0, E.s()>>>(V, E.cf, q, f, out, w);
  if (OPK == OP_RESID) k_ell_op<OP_RESID><<<g, TPB, 0, E.s()>>>(V, E.cf, q, f, out, w);
  if (OPK == OP_JACOBI) k_ell_op<OP_JACOBI><<<g, TPB, 0, E.s()>>>(V, E.cf, q, f, out, w);
}

// weighted dot / l2 into device scalar slot; returns nothing (async)
void dot_dev(Ell& E, int l, const double* a, const double* b, int slot, int mode, const double* den = nullptr) {
  EllLev V = E.view(l);
  unsigned g = nb(10 * E.m(l) * E.m(l));
  k_ell_dot<TPB><<<g, TPB, 0, E.s()>>>(V, a, b, E.partial);
  k_final_sum<<<1, 256, 0, E.s()>>>(E.partial, (int)g, E.scal + slot, mode, den);
}

double fetch(Ell& E, int slot) {
  double v = 0;
  cudaMemcpyAsync(&v, E.scal + slot, 8, cudaMemcpyDeviceToHost, E.s());
  cudaStreamSynchronize(E.s());
  return v;
}

double l2(Ell& E, int l, const double* a) {
  dot_dev(E, l, a, a, 0, 1);
  return fetch(E, 0);
}
double dp(Ell& E, int l, const double* a, const double* b) {
  dot_dev(E, l, a, b, 0, 0);
  return fetch(E, 0);
}

void lc(Ell& E, int l, double* s, double a1, const double* s1, double a2, const double* s2) {
  EllLev V = E.view(l);
  k_ell_lc<<<nb(10 * E.m(l) * E.m(l)), TPB, 0, E.s()>>>(V, s, a1, nullptr, s1, a2, nullptr, 1.0, s2);
}

void copy_level(Ell& E, int l, double* dst, const double* src) {
  cudaMemcpyAsync(dst, src, 8 * E.L[l - E.ls].NN, cudaMemcpyDeviceToDevice, E.s());
}
void zero_level(Ell& E, int l, double* p) { cudaMemsetAsync(p, 0, 8 * E.L[l - E.ls].NN, E.s()); }

// Jacobi sweeps (src/lin_solve.f90:271-359), ping-pong through the tmp field.
void jacobi(Ell& E, MField& u, MField& f, int l, int iters, double w = 1.0) {
  for (int it = 0; it < iters; ++it) {
    op(E, OP_JACOBI, l, u.lv[l - E.ls], f.lv[l - E.ls], E.tmp.lv[l - E.ls], w);
    std::swap(u.lv[l - E.ls], E.tmp.lv[l - E.ls]);
  }
}

void residual(Ell& E, MField& f, MField& u, int l, MField& r) {
  op(E, OP_RESID, l, u.lv[l - E.ls], f.lv[l - E.ls], r.lv[l - E.ls]);
}

// forward_scalar_transform(s, wc, c, c+1): wavelets at c+1, lifted restriction to c
void restrict_level(Ell& E, MField& s, MField& wc, int c) {
  for (int l = E.ls; l <= E.le; ++l) zero_level(E, l, wc.lv[l - E.ls]);   // zero_float(wavelet)
  EllLev C = E.view(c), F = E.view(c + 1);
  int n = E.L[c - E.ls].n;
  k_wc_compute<<<nb(10 * n * n), TPB, 0, E.s()>>>(C, F, s.lv[c + 1 - E.ls], wc.lv[c + 1 - E.ls]);
  k_restrict<<<nb(10 * (n + 1) * (n + 1)), TPB, 0, E.s()>>>(C, F, s.lv[c + 1 - E.ls], wc.lv[c + 1 - E.ls],
                                                              s.lv[c - E.ls]);
}

// inverse_scalar_transform(wc, s, f-1, f)
void prolong_level(Ell& E, MField& wc, MField& s, int fl) {
  int c = fl - 1;
  EllLev C = E.view(c), F = E.view(fl);
  int n = E.L[c - E.ls].n;
  k_prolong_even<<<nb(10 * (n + 1) * (n + 1)), TPB, 0, E.s()>>>(C, F, s.lv[c - E.ls], wc.lv[fl - E.ls], s.lv[fl - E.ls]);
  k_prolong_odd<<<nb(10 * n * n), TPB, 0, E.s()>>>(C, F, s.lv[fl - E.ls], wc.lv[fl - E.ls]);
}

double res_err(Ell& E, MField& f, MField& u, double nrm_f, int l) {
  residual(E, f, u, l, E.rr2);
  return l2(E, l, E.rr2.lv[l - E.ls]) / nrm_f;
}

// bicgstab (src/lin_solve.f90:361-431) at level l
void bicgstab(Ell& E, MField& u, MField& f, double nrm_f, int l, double tol, int iter_max, double* err_out,
              int* iter_out) {
  const int q = l - E.ls;
  double* U = u.lv[q];
  double* F = f.lv[q];
  double *R = E.rr.lv[q], *R0 = E.r0.lv[q], *Pp = E.pp.lv[q], *S = E.ss.lv[q], *AP = E.ap.lv[q], *AS = E.as_.lv[q],
         *CC = E.cc.lv[q];
  zero_level(E, l, CC);
  op(E, OP_RESID, l, U, F, R);
  copy_level(E, l, R0, R);
  copy_level(E, l, Pp, R);
  copy_level(E, l, S, R);
  op(E, OP_APPLY, l, Pp, nullptr, AP);
  double rho = dp(E, l, R0, R), err = 0.0;
  int iter;
  for (iter = 1; iter <= iter_max; ++iter) {
    double alph = rho / dp(E, l, AP, R0);
    lc(E, l, S, 1.0, R, -alph, AP);
    op(E, OP_APPLY, l, S, nullptr, AS);
    dot_dev(E, l, AS, S, 1, 0);
    dot_dev(E, l, AS, AS, 2, 0);
    double two[2];
    cudaMemcpyAsync(two, E.scal + 1, 16, cudaMemcpyDeviceToHost, E.s());
    cudaStreamSynchronize(E.s());
    double omga = two[0] / two[1];
    lc(E, l, CC, alph, Pp, omga, S);
    lc(E, l, U, 1.0, U, 1.0, CC);
    lc(E, l, R, 1.0, S, -omga, AS);
    err = l2(E, l, R) / nrm_f;
    if (err <= tol) break;
    double rho_old = rho;
    rho = dp(E, l, R0, R);
    double b = (alph / omga) * (rho / rho_old);
    lc(E, l, CC, 1.0, Pp, -omga, AP);
    lc(E, l, Pp, 1.0, R, b, CC);
    op(E, OP_APPLY, l, Pp, nullptr, AP);
  }
  if (err_out) *err_out = err;
  if (iter_out) *iter_out = iter;
}

void v_cycle(Ell& E, const wt_solver_opts& o, MField& u, MField& f, int l, double nrmf, wt_solver_report& rep) {
  for (int j = E.ls; j <= l; ++j) zero_level(E, j, E.corr.lv[j - E.ls]);
  residual(E, f, u, l, E.res);
  for (int j = l; j >= E.ls + 1; --j) {
    jacobi(E, E.corr, E.res, j, o.down_iter);
    op(E, OP_RESID, j, E.corr.lv[j - E.ls], E.res.lv[j - E.ls], E.au.lv[j - E.ls]);
    std::swap(E.res.lv[j - E.ls], E.au.lv[j - E.ls]);
    restrict_level(E, E.res, E.wc_temp, j - 1);
  }
  int j = E.ls;
  double nrm_rhs = l2(E, j, E.res.lv[0]);
  if (nrm_rhs == 0.0) nrm_rhs = 1.0;
  bicgstab(E, E.corr, E.res, nrm_rhs, j, o.coarse_tol, o.coarse_iter, nullptr, nullptr);
  for (j = E.ls + 1; j <= l; ++j) {
    zero_level(E, j, E.wc_temp.lv[j - E.ls]);
    copy_level(E, j - 1, E.pf.lv[j - 1 - E.ls], E.corr.lv[j - 1 - E.ls]);
    prolong_level(E, E.wc_temp, E.pf, j);
    lc(E, j, E.corr.lv[j - E.ls], 1.0, E.corr.lv[j - E.ls], 1.0, E.pf.lv[j - E.ls]);
    jacobi(E, E.corr, E.res, j, o.up_iter);
  }
  lc(E, l, u.lv[l - E.ls], 1.0, u.lv[l - E.ls], 1.0, E.corr.lv[l - E.ls]);
  jacobi(E, u, f, l, o.post_iter);
  rep.nrm_res_final[l - E.ls] = res_err(E, f, u, nrmf, l);
}

void fmg(Ell& E, const wt_solver_opts& o, wt_solver_report& rep) {
  MField& u = E.u;
  MField& f = E.f;
  for (int l = E.ls; l <= E.le; ++l) zero_level(E, l, E.wc_mass.lv[l - E.ls]);
  std::vector<double> nrm_f(E.le - E.ls + 1);
  for (int l = E.ls; l <= E.le; ++l) {
    nrm_f[l - E.ls] = l2(E, l, f.lv[l - E.ls]);
    if (nrm_f[l - E.ls] == 0.0) nrm_f[l - E.ls] = 1.0;
    rep.nrm_res_init[l - E.ls] = res_err(E, f, u, nrm_f[l - E.ls], l);
  }
  int l = E.ls;
  bicgstab(E, u, f, nrm_f[0], l, o.coarse_tol, o.coarse_iter, &rep.nrm_res_final[0], &rep.iterations[0]);
  for (l = E.ls + 1; l <= E.le; ++l) {
    if (rep.nrm_res_init[l - E.ls] < o.fine_tol) continue;
    prolong_level(E, E.wc_mass, u, l);
    jacobi(E, u, f, l, o.pre_iter);
    for (int iter = 1; iter <= o.max_vcycle; ++iter) {
      v_cycle(E, o, u, f, l, nrm_f[l - E.ls], rep);
      rep.iterations[l - E.ls] = iter;
      if (rep.nrm_res_final[l - E.ls] <= o.fine_tol) break;
    }
  }
}

void srj(Ell& E, const wt_solver_opts& o, wt_solver_report& rep) {
  MField& u = E.u;
  MField& f = E.f;
  for (int l = E.ls; l <= E.le; ++l) zero_level(E, l, E.wc_mass.lv[l - E.ls]);
  std::vector<double> nrm_f(E.le - E.ls + 1);
  for (int l = E.ls; l <= E.le; ++l) {
    nrm_f[l - E.ls] = l2(E, l, f.lv[l - E.ls]);
    if (nrm_f[l - E.ls] == 0.0) nrm_f[l - E.ls] = 1.0;
  }
  const int m = 8;
  const double k1 = 3e-2, k2 = 1.8;
  double w[m];
  int max_iter = o.max_srj_iter;
  if (max_iter < m) {
    for (int n = 0; n < m; ++n) w[n] = 1.0;
  } else {
    max_iter = m * (max_iter / m);
    const double PI = std::acos(-1.0);
    for (int n = 1; n <= m; ++n)
      w[n - 1] = 2.0 / (k1 + k2 - (k2 - k1) * std::cos(PI * (2.0 * double(n) - 1.0) / (2.0 * double(m))));
  }
  int l = E.ls;
  bicgstab(E, u, f, nrm_f[0], l, o.coarse_tol, o.coarse_iter, &rep.nrm_res_final[0], &rep.iterations[0]);
  for (l = E.ls + 1; l <= E.le; ++l) {
    prolong_level(E, E.wc_mass, u, l);
    int ii = 0;
    for (int iter = 1; iter <= max_iter; ++iter) {
      ii = ii + 1;
      if (ii > m) {
        if (rep.nrm_res_final[l - E.ls] < o.fine_tol) break;
        ii = 1;
      }
      jacobi(E, u, f, l, 1, w[ii - 1]);
      rep.nrm_res_final[l - E.ls] = res_err(E, f, u, nrm_f[l - E.ls], l);
      rep.iterations[l - E.ls] = iter;
      if (rep.nrm_res_final[l - E.ls] <= o.fine_tol) break;
    }
  }
}

}  // namespace

#include "wt_elliptic_mixed.cuh"
#include "wt_learned.cuh"

// ---------------------------------------------------------------- C-ABI ----
extern "C" {

int wt_elliptic_upload(wt_handle* h, const double* u, const double* f) {
  if (!h || !h->ell) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  int64_t o = 0;
  for (int l = E.ls; l <= E.le; ++l) {
    int64_t NN = E.L[l - E.ls].NN;
    if (u) CKE(cudaMemcpyAsync(E.u.lv[l - E.ls], u + o, 8 * NN, cudaMemcpyHostToDevice, E.s()));
    if (f) CKE(cudaMemcpyAsync(E.f.lv[l - E.ls], f + o, 8 * NN, cudaMemcpyHostToDevice, E.s()));
    o += NN;
  }
  CKE(cudaStreamSynchronize(E.s()));
  return WT_OK;
}

int wt_elliptic_download(wt_handle* h, double* u, double* f) {
  if (!h || !h->ell) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  int64_t o = 0;
  for (int l = E.ls; l <= E.le; ++l) {
    int64_t NN = E.L[l - E.ls].NN;
    if (u) CKE(cudaMemcpyAsync(u + o, E.u.lv[l - E.ls], 8 * NN, cudaMemcpyDeviceToHost, E.s()));
    if (f) CKE(cudaMemcpyAsync(f + o, E.f.lv[l - E.ls], 8 * NN, cudaMemcpyDeviceToHost, E.s()));
    o += NN;
  }
  CKE(cudaStreamSynchronize(E.s()));
  return WT_OK;
}

int wt_elliptic_apply(wt_handle* h, int level) {
  if (!h || !h->ell) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  if (level < E.ls || level > E.le) return WT_ERR_ARG;
  op(E, OP_APPLY, level, E.u.lv[level - E.ls], nullptr, E.f.lv[level - E.ls]);
  CKE(cudaStreamSynchronize(E.s()));
  CKE(cudaGetLastError());
  return WT_OK;
}

int wt_elliptic_restrict(wt_handle* h) {
  if (!h || !h->ell) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  for (int c = E.le - 1; c >= E.ls; --c) restrict_level(E, E.f, E.wc_temp, c);
  CKE(cudaStreamSynchronize(E.s()));
  CKE(cudaGetLastError());
  return WT_OK;
}

int wt_elliptic_prolong(wt_handle* h, int fine) {
  if (!h || !h->ell) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  if (fine <= E.ls || fine > E.le) return WT_ERR_ARG;
  for (int l = E.ls; l <= E.le; ++l) zero_level(E, l, E.wc_mass.lv[l - E.ls]);
  prolong_level(E, E.wc_mass, E.u, fine);
  CKE(cudaStreamSynchronize(E.s()));
  CKE(cudaGetLastError());
  return WT_OK;
}

int wt_elliptic_l2(wt_handle* h, int level, int which, double* out) {
  if (!h || !h->ell || !out) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  if (level < E.ls || level > E.le) return WT_ERR_ARG;
  *out = l2(E, level, (which == 0 ? E.u : E.f).lv[level - E.ls]);
  CKE(cudaGetLastError());
  return WT_OK;
}

int wt_elliptic_solve(wt_handle* h, const wt_solver_opts* opts, wt_solver_report* rep) {
  if (!h || !h->ell || !opts || !rep) return WT_ERR_ARG;
  Ell& E = *static_cast<Ell*>(h->ell);
  std::memset(rep, 0, sizeof(*rep));
  CKE(cudaStreamSynchronize(E.s()));
  auto t0 = std::chrono::steady_clock::now();
  int rc = WT_OK;
  if (opts->method == WT_SOLVER_FMG) fmg(E, *opts, *rep);
  else if (opts->method == WT_SOLVER_SRJ) srj(E, *opts, *rep);
  else if (opts->method == WT_SOLVER_MIXED_IR) rc = mixed_ir(E, *opts, *rep);
  else if (opts->method == WT_SOLVER_MG64) rc = mixed_ir(E, *opts, *rep, true);
  else if (opts->method == WT_SOLVER_FCG_LEARNED) rc = fcg_solve(E, *opts, *rep, PRE_NET);
  else if (opts->method == WT_SOLVER_FCG) rc = fcg_solve(E, *opts, *rep, PRE_NONE);
  else if (opts->method == WT_SOLVER_FCG_MG) rc = fcg_solve(E, *opts, *rep, PRE_MG);
  else return WT_ERR_ARG;
  CKE(cudaStreamSynchronize(E.s()));
  auto t1 = std::chrono::steady_clock::now();
  rep->ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  // true FP64 relative residual on the finest level
  const int l = E.le;
  double nf = l2(E, l, E.f.lv[l - E.ls]);
  if (nf == 0.0) nf = 1.0;
  rep->true_rel_residual = res_err(E, E.f, E.u, nf, l);
  CKE(cudaGetLastError());
  if (rc) return rc;
  if (!std::isfinite(rep->true_rel_residual)) return WT_ERR_NONFINITE;
  return WT_OK;
}

int wt_elliptic_autotune(wt_handle* h, const wt_solver_opts* base, const int* cand, int ncand, int repeats,
                         wt_solver_opts* best, double* best_ms) {
  if (!h || !h->ell || !base || !best || !best_ms || repeats < 1) return WT_ERR_ARG;
  const int m = base->method;
  if (m != WT_SOLVER_MIXED_IR && m != WT_SOLVER_MG64 && m != WT_SOLVER_FCG_LEARNED && m != WT_SOLVER_FCG_MG)
    return WT_ERR_ARG;
  Ell& E = *static_cast<Ell*>(h->ell);
  std::vector<int> set;
  if (cand) {
    if (ncand < 1) return WT_ERR_ARG;
    set.assign(cand, cand + 3 * ncand);
  } else {
    for (int d = 1; d <= 3; ++d)
      for (int c : {2, 4, 6, 10, 20}) set.insert(set.end(), {d, d, c});
  }
  const int q = E.le - E.ls;
  const int64_t NN = E.L[q].NN;
  double* u0 = nullptr;
  CKE(cudaMalloc(&u0, 8 * NN));
  cudaMemcpyAsync(u0, E.u.lv[q], 8 * NN, cudaMemcpyDeviceToDevice, E.s());
  double tbest = -1.0;
  int rc = WT_OK;
  for (size_t k = 0; k + 2 < set.size() && rc == WT_OK; k += 3) {
    wt_solver_opts o = *base;
    o.down_iter = set[k];
    o.up_iter = set[k + 1];
    o.coarse_iter = set[k + 2];
    if (o.down_iter < 0 || o.up_iter < 0 || o.coarse_iter < 0) continue;
    double t = -1.0;
    for (int r = 0; r < repeats; ++r) {
      cudaMemcpyAsync(E.u.lv[q], u0, 8 * NN, cudaMemcpyDeviceToDevice, E.s());
      wt_solver_report rep;
      const int src = wt_elliptic_solve(h, &o, &rep);
      if (src == WT_ERR_CUDA) rc = src;
      if (src != WT_OK) {
        t = -1.0;
        break;
      }
      t = t < 0 ? rep.ms : std::min(t, rep.ms);
    }
    if (t >= 0 && (tbest < 0 || t < tbest)) {
      tbest = t;
      *best = o;
    }
  }
  cudaMemcpyAsync(E.u.lv[q], u0, 8 * NN, cudaMemcpyDeviceToDevice, E.s());
  cudaStreamSynchronize(E.s());
  cudaFree(u0);
  if (rc != WT_OK) return rc;
  *best_ms = tbest;
  return tbest < 0 ? WT_ERR_NOT_CONVERGED : WT_OK;
}

}  // extern "C"

// ------------------------------------------------------- free surface ----
int wt_level_baro_fields(wt_handle* h, int l, double** eta, double** rhs, double** div, double** div_old);
int wt_level_barotropic_correction(wt_handle* h, double* const* m, double* const* t);

namespace {

// The free surface's inverse transform from its wavelets in E.eta_wc,
// compressed first under the current masks (compress_scalar), from
// level_start up (Prolong_scalar + Reconstruct_scalar).
int eta_inverse(wt_handle* h, Ell& E, const std::vector<double*>& eta) {
  for (int l = E.ls + 1; l <= E.le; ++l) {
    const int q = l - E.ls;
    const int *mn, *me;
    wt_level_masks(h, l, &mn, &me);
    k_compress_wc<<<nb(E.L[q].NN), TPB, 0, E.s()>>>(E.L[q].NN, mn, E.eta_wc.lv[q]);
  }
  for (int l = E.ls + 1; l <= E.le; ++l) {   // from level_start up
    const int q = l - E.ls, n = E.L[q - 1].n;
    const EllLev C = E.view(l - 1), F = E.view(l);
    k_prolong_even<<<nb(10 * (n + 1) * (n + 1)), TPB, 0, E.s()>>>(C, F, eta[q - 1], E.eta_wc.lv[q], eta[q]);
    k_prolong_odd<<<nb(10 * n * n), TPB, 0, E.s()>>>(C, F, eta[q], E.eta_wc.lv[q]);
  }
  CKE(cudaGetLastError());
  CKE(cudaStreamSynchronize(E.s()));
  return WT_OK;
}

int eta_fields(wt_handle* h, Ell& E, std::vector<double*>& eta) {
  eta.resize(E.le - E.ls + 1);
  for (int l = E.ls; l <= E.le; ++l)
    if (int rc = wt_level_baro_fields(h, l, &eta[l - E.ls], nullptr, nullptr, nullptr)) return rc;
  return WT_OK;
}

// WT_after_step of the free surface (it is layer zlevels+1 of sol): every
// wavelet from the surface as it is, compress_scalar, inverse transform.
// The wavelets stay in E.eta_wc for the inverse transform after adapt.
int eta_after_step(wt_handle* h, Ell& E) {
  E.eta_wc_valid = true;
  std::vector<double*> eta;
  if (int rc = eta_fields(h, E, eta)) return rc;
  for (int l = E.ls + 1; l <= E.le; ++l) {
    const int q = l - E.ls;
    double* wc = E.eta_wc.lv[q];
    zero_level(E, l, wc);
    const int n = E.L[q - 1].n;
    k_wc_compute<<<nb(10 * n * n), TPB, 0, E.s()>>>(E.view(l - 1), E.view(l), eta[q], wc);
  }
  return eta_inverse(h, E, eta);
}

}  // namespace

extern "C" {

// free_surface_update (src/time_integr.f90:465-478) on the hierarchy: eta_update
// (rhs_elliptic over the hierarchy, the operator's coefficients from the old
// free surface, the elliptic solve with opts, src/barotropic_2d.f90:118-129),
// barotropic_correction, u_update and WT_after_step.
int wt_free_surface_update(wt_handle* h, double dt, double theta1, double theta2, const wt_solver_opts* opts,
                           wt_solver_report* rep) {
  if (!h || !opts || !rep || dt <= 0) return WT_ERR_ARG;
  if (!h->ell || !h->wav || h->flux_bits != 64) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  if (E.ls != h->level_start || E.le != h->level_end || E.dt != dt || E.th1 != theta1 || E.th2 != theta2)
    return WT_ERR_STATE;  // wt_elliptic_setup with this dt and theta on this hierarchy
  if (int rc = wt_rhs_elliptic_multi(h, dt, theta2)) return rc;
  const double g = h->ph.grav;
  for (int l = E.ls; l <= E.le; ++l) {
    const int q = l - E.ls;
    double *eta, *rhs;
    if (int rc = wt_level_baro_fields(h, l, &eta, &rhs, nullptr, nullptr)) return rc;
    const DevLevel& D = h->at(l);
    ELevelDev& X = E.L[q];
    k_ell_coeffs<<<nb(D.NN), TPB, 0, E.s()>>>(D.n, D.P, D.NN, D.topo, eta, D.nsrc, D.len, D.pedlen, D.hex_inv, g, dt,
                                                theta1, theta2, E.cf, X.Ie, X.diag, X.Kf, X.diagf);
    // the solve starts from the current free surface (elliptic_solver(sol(S_MASS, zlevels+1), ...))
    CKE(cudaMemcpyAsync(E.u.lv[q], eta, 8 * D.NN, cudaMemcpyDeviceToDevice, E.s()));
    CKE(cudaMemcpyAsync(E.f.lv[q], rhs, 8 * D.NN, cudaMemcpyDeviceToDevice, E.s()));
  }
  CKE(cudaGetLastError());
  int rc = wt_elliptic_solve(h, opts, rep);
  if (rc != WT_OK && rc != WT_ERR_NOT_CONVERGED) return rc;
  for (int l = E.ls; l <= E.le; ++l) {
    double* eta;
    if (int r2 = wt_level_baro_fields(h, l, &eta, nullptr, nullptr, nullptr)) return r2;
    CKE(cudaMemcpyAsync(eta, E.u.lv[l - E.ls], 8 * h->at(l).NN, cudaMemcpyDeviceToDevice, E.s()));
  }
  if (int r2 = wt_level_barotropic_correction(h, nullptr, nullptr)) return r2;
  if (int r2 = wt_u_update_multi(h, dt, theta1)) return r2;
  if (int r2 = wt_wt_after_step(h)) return r2;
  // WT_after_step(sol, wav_coeff, level_start - 1) transforms the free surface
  // (sol(S_MASS, zlevels+1)) with the layers: its wavelets on every level above
  // level_start, compress_scalar with the node masks, inverse_scalar_transform
  if (int r2 = eta_after_step(h, E)) return r2;
  return rc;
}

// RK4_split (src/time_integr.f90:360-382): the flux divergence of the previous
// step when theta2 != 1, RK_split four times and free_surface_update.
// The free surface's part of adapt's compress_wavelets and of the inverse
// transform after it (src/adapt.f90:79-103, src/main.f90:441): its wavelets
// from the last free_surface_update, compressed under the current masks, then
// the inverse transform.  Call after wt_mask_build.
int wt_free_surface_adapt(wt_handle* h) {
  if (!h || !h->ell || !h->wav) return WT_ERR_STATE;
  Ell& E = *static_cast<Ell*>(h->ell);
  if (E.ls != h->level_start || E.le != h->level_end || !E.eta_wc_valid) return WT_ERR_STATE;
  std::vector<double*> eta;
  if (int rc = eta_fields(h, E, eta)) return rc;
  return eta_inverse(h, E, eta);
}

int wt_rk4_split(wt_handle* h, double dt, double theta1, double theta2, const wt_solver_opts* opts,
                 wt_solver_report* rep) {
  if (!h || !opts || !rep || dt <= 0) return WT_ERR_ARG;
  if (!h->ell || !h->wav || h->flux_bits != 64) return WT_ERR_STATE;
  if (theta2 != 1.0) {
    if (int rc = wt_rhs_elliptic_multi(h, dt, theta2)) return rc;  // flux_divergence of the current state
    for (int l = h->level_start; l <= h->level_end; ++l) {
      double *div, *div_old;
      if (int rc = wt_level_baro_fields(h, l, nullptr, nullptr, &div, &div_old)) return rc;
      CKE(cudaMemcpyAsync(div_old, div, 8 * h->at(l).NN, cudaMemcpyDeviceToDevice, h->stream));
    }
  }
  if (int rc = wt_rk4_split_explicit(h, dt, theta1)) return rc;
  return wt_free_surface_update(h, dt, theta1, theta2, opts, rep);
}

}  // extern "C"
