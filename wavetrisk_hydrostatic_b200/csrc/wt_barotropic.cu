// C-ABI of the barotropic pieces of the mode-split step on the stepper's level
// (level_end): flux_divergence + rhs_elliptic, grad_eta + u_update
// (src/barotropic_2d.f90:118-185, 326-366, 131-149, 455-474).
#include <cuda_runtime.h>

#include <vector>

#include "../../include/wavetrisk_gpu.h"
#include "barotropic_kernels.cuh"
#include "wt_handle.cuh"

namespace {

constexpr int TPB = 256;
inline unsigned nb(int64_t n) { return (unsigned)((n + TPB - 1) / TPB); }

// Free-surface fields of one level of the hierarchy.
struct BaroLevel {
  double *eta = nullptr, *eta_w = nullptr, *div_old = nullptr, *div = nullptr, *rhs = nullptr, *flux = nullptr,
         *grad = nullptr;
};

struct BaroCtx {
  double *eta = nullptr, *div_old = nullptr, *div = nullptr, *rhs = nullptr, *flux = nullptr, *grad = nullptr;
  std::vector<BaroLevel> L;  // every level, on first use of the hierarchy entry points
  std::vector<void*> allocs;
};

#define CKB(x)                                             \
  do {                                                     \
    cudaError_t e_ = (x);                                  \
    if (e_ != cudaSuccess) return wt_handle_fail(#x, e_);  \
  } while (0)

int ensure(wt_handle* h) {
  if (h->baro) return WT_OK;
  BaroCtx* B = new BaroCtx();
  h->baro = B;
  const size_t NN = (size_t)h->top().NN;
  double** node[] = {&B->eta, &B->div_old, &B->div, &B->rhs};
  for (double** p : node) {
    CKB(cudaMalloc(p, NN * 8));
    CKB(cudaMemsetAsync(*p, 0, NN * 8, h->stream));
  }
  CKB(cudaMalloc(&B->flux, 3 * NN * 8));
  CKB(cudaMalloc(&B->grad, 3 * NN * 8));
  CKB(cudaMemsetAsync(B->flux, 0, 3 * NN * 8, h->stream));
  CKB(cudaMemsetAsync(B->grad, 0, 3 * NN * 8, h->stream));
  return WT_OK;
}

// Per-level free-surface fields of the hierarchy (zeroed on first use).
int ensure_levels(wt_handle* h) {
  if (int rc = ensure(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  if (!B->L.empty()) return WT_OK;
  B->L.resize(h->level_end - h->level_start + 1);
  for (int l = h->level_start; l <= h->level_end; ++l) {
    BaroLevel& V = B->L[l - h->level_start];
    const size_t NN = (size_t)h->at(l).NN;
    double** node[] = {&V.eta, &V.eta_w, &V.div_old, &V.div, &V.rhs};
    for (double** p : node) {
      CKB(cudaMalloc(p, NN * 8));
      B->allocs.push_back(*p);
      CKB(cudaMemsetAsync(*p, 0, NN * 8, h->stream));
    }
    double** edge[] = {&V.flux, &V.grad};
    for (double** p : edge) {
      CKB(cudaMalloc(p, 3 * NN * 8));
      B->allocs.push_back(*p);
      CKB(cudaMemsetAsync(*p, 0, 3 * NN * 8, h->stream));
    }
  }
  return WT_OK;
}

// State (mass, velocity) and mean mass of a level.
void level_state(wt_handle* h, int l, double** m, double** v, double** mm) {
  double* t;
  if (l == h->level_end) {
    *m = h->mass;
    *v = h->velo;
  } else {
    wt_level_state(h, l, m, &t, v);
  }
  wt_level_mean(h, l, WT_FIELD_MEAN_MASS, mm);
}

}  // namespace

void wt_barotropic_release(wt_handle* h) {
  if (!h || !h->baro) return;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  double* a[] = {B->eta, B->div_old, B->div, B->rhs, B->flux, B->grad};
  for (double* p : a)
    if (p) cudaFree(p);
  for (void* p : B->allocs) cudaFree(p);
  delete B;
  h->baro = nullptr;
}

extern "C" {

int wt_barotropic_upload(wt_handle* h, const double* eta, const double* div_old) {
  if (!h) return WT_ERR_ARG;
  if (int rc = ensure(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  const size_t NN = (size_t)h->top().NN;
  if (eta) CKB(cudaMemcpyAsync(B->eta, eta, NN * 8, cudaMemcpyHostToDevice, h->stream));
  if (div_old) CKB(cudaMemcpyAsync(B->div_old, div_old, NN * 8, cudaMemcpyHostToDevice, h->stream));
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_rhs_elliptic(wt_handle* h, double dt, double theta2) {
  if (!h) return WT_ERR_ARG;
  if (int rc = ensure(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  const DevLevel& D = h->top();
  const wtk::LevelDev L = D.view();
  const int m = D.n + 1;
  wtb::k_flux_sum<<<nb(10 * m * m), TPB, 0, h->stream>>>(L, h->nz, h->mass, h->mean_m, h->velo, B->flux);
  wtb::k_div<<<nb(10 * m * m), TPB, 0, h->stream>>>(L, B->flux, B->div);
  wtb::k_rhs<<<nb(10 * m * m), TPB, 0, h->stream>>>(L, B->div, B->eta, B->div_old, dt, theta2, h->ph.ref_density,
                                                     B->rhs);
  CKB(cudaGetLastError());
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_u_update(wt_handle* h, double dt, double theta1) {
  if (!h) return WT_ERR_ARG;
  if (int rc = ensure(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  const DevLevel& D = h->top();
  const int m = D.n + 1;
  wtb::k_grad_eta_update<false><<<nb(10 * m * m), TPB, 0, h->stream>>>(D.view(), h->nz, h->ph.grav, B->eta, theta1 * dt,
                                                                 B->grad, h->velo);
  CKB(cudaGetLastError());
  CKB(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

int wt_step1_flux(wt_handle* h, int itype, int layer, const double* scalar, double* flux) {
  if (!h || !flux || layer < 0 || layer >= h->nz) return WT_ERR_ARG;
  if (itype != 1 && itype != 5 && itype != 6 && itype != 7) return WT_ERR_ARG;
  if ((itype == 1 || itype == 6) && !scalar) return WT_ERR_ARG;
  if (int rc = ensure(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  const DevLevel& D = h->top();
  const wtk::LevelDev L = D.view();
  const size_t NN = (size_t)D.NN;
  const int64_t ko = (int64_t)layer * D.NN;
  if (scalar) CKB(cudaMemcpyAsync(B->rhs, scalar, NN * 8, cudaMemcpyHostToDevice, h->stream));
  CKB(cudaMemsetAsync(B->grad, 0, 3 * NN * 8, h->stream));
  const int m = D.n + 1;
  const double* v = h->velo + 3 * ko;
  const double* ms = h->mass + ko;
  const double* mm = h->mean_m + ko;
  switch (itype) {
    case 1: wtb::k_step1_flux<1><<<nb(10 * m * m), TPB, 0, h->stream>>>(L, B->rhs, v, ms, mm, B->grad); break;
    case 5: wtb::k_step1_flux<5><<<nb(10 * m * m), TPB, 0, h->stream>>>(L, B->rhs, v, ms, mm, B->grad); break;
    case 6: wtb::k_step1_flux<6><<<nb(10 * m * m), TPB, 0, h->stream>>>(L, B->rhs, v, ms, mm, B->grad); break;
    default: wtb::k_step1_flux<7><<<nb(10 * m * m), TPB, 0, h->stream>>>(L, B->rhs, v, ms, mm, B->grad); break;
  }
  CKB(cudaGetLastError());
  CKB(cudaMemcpyAsync(flux, B->grad, 3 * NN * 8, cudaMemcpyDeviceToHost, h->stream));
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_step1_vort(wt_handle* h, int layer, double* vort) {
  if (!h || !vort || layer < 0 || layer >= h->nz) return WT_ERR_ARG;
  if (int rc = ensure(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  const DevLevel& D = h->top();
  const size_t NN = (size_t)D.NN;
  CKB(cudaMemsetAsync(B->grad, 0, 2 * NN * 8, h->stream));
  const int m = D.n + 1;
  wtb::k_step1_vort<<<nb(10 * m * m), TPB, 0, h->stream>>>(D.view(), h->velo + 3 * (int64_t)layer * D.NN, B->grad);
  CKB(cudaGetLastError());
  CKB(cudaMemcpyAsync(vort, B->grad, 2 * NN * 8, cudaMemcpyDeviceToHost, h->stream));
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_barotropic_upload_level(wt_handle* h, int level, const double* eta, const double* div_old) {
  if (!h || level < h->level_start || level > h->level_end) return WT_ERR_ARG;
  if (!h->wav) return WT_ERR_STATE;
  if (int rc = ensure_levels(h)) return rc;
  BaroLevel& V = static_cast<BaroCtx*>(h->baro)->L[level - h->level_start];
  const size_t NN = (size_t)h->at(level).NN;
  if (eta) CKB(cudaMemcpyAsync(V.eta, eta, NN * 8, cudaMemcpyHostToDevice, h->stream));
  if (div_old) CKB(cudaMemcpyAsync(V.div_old, div_old, NN * 8, cudaMemcpyHostToDevice, h->stream));
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

// flux_divergence over the hierarchy (src/barotropic_2d.f90:326-366): per level
// from level_end down, the vertically summed mass flux, on coarser levels the
// compute-or-restrict of that flux with the child's divergence as dscalar
// (cpt_or_restr_flux), and the divergence; then rhs_elliptic on every level.
int wt_rhs_elliptic_multi(wt_handle* h, double dt, double theta2) {
  if (!h) return WT_ERR_ARG;
  if (!h->wav) return WT_ERR_STATE;
  if (int rc = ensure_levels(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  for (int l = h->level_end; l >= h->level_start; --l) {
    BaroLevel& V = B->L[l - h->level_start];
    const DevLevel& D = h->at(l);
    const wtk::LevelDev L = D.view();
    const int m = D.n + 1;
    double *ms, *v, *mm;
    level_state(h, l, &ms, &v, &mm);
    wtb::k_flux_sum<<<nb(10 * m * m), TPB, 0, h->stream>>>(L, h->nz, ms, mm, v, V.flux);
    if (l < h->level_end) {
      BaroLevel& C = B->L[l + 1 - h->level_start];
      if (int rc = wt_level_restrict_flux(h, l, V.flux, nullptr, C.flux, nullptr, C.div, nullptr, 1)) return rc;
    }
    wtb::k_div<<<nb(10 * m * m), TPB, 0, h->stream>>>(L, V.flux, V.div);
    wtb::k_rhs<<<nb(10 * m * m), TPB, 0, h->stream>>>(L, V.div, V.eta, V.div_old, dt, theta2, h->ph.ref_density,
                                                       V.rhs);
  }
  CKB(cudaGetLastError());
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

// grad_eta over the hierarchy (src/barotropic_2d.f90:455-474) with
// cpt_or_restr_eta (:414-453), and u_update (:131-149) on every level.  The
// free surface is ghost-copied once into a work copy; coarser levels restrict
// that copy (parents [0, n]^2 with mask_n >= RESTRCT) and read it as stored.
int wt_u_update_multi(wt_handle* h, double dt, double theta1) {
  if (!h) return WT_ERR_ARG;
  if (!h->wav) return WT_ERR_STATE;
  if (int rc = ensure_levels(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  for (int l = h->level_start; l <= h->level_end; ++l) {
    BaroLevel& V = B->L[l - h->level_start];
    const DevLevel& D = h->at(l);
    CKB(cudaMemcpyAsync(V.eta_w, V.eta, (size_t)D.NN * 8, cudaMemcpyDeviceToDevice, h->stream));
    if (D.n_hn > 0) wtb::k_halo_nodes<<<nb(D.n_hn), TPB, 0, h->stream>>>(D.hn, D.n_hn, V.eta_w);
  }
  for (int l = h->level_end; l >= h->level_start; --l) {
    BaroLevel& V = B->L[l - h->level_start];
    const DevLevel& D = h->at(l);
    const int m = D.n + 1;
    if (l < h->level_end)
      if (int rc = wt_level_restrict_scalar(h, l, V.eta_w, B->L[l + 1 - h->level_start].eta_w, 1)) return rc;
    double *ms, *v, *mm;
    level_state(h, l, &ms, &v, &mm);
    wtb::k_grad_eta_update<true><<<nb(10 * m * m), TPB, 0, h->stream>>>(D.view(), h->nz, h->ph.grav, V.eta_w,
                                                                       theta1 * dt, V.grad, v);
  }
  CKB(cudaGetLastError());
  CKB(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

}  // extern "C"

// barotropic_correction (src/barotropic_2d.f90:52-116) of the scaling fields
// m[q], t[q] of level level_start+q (the hierarchy's own when m is null), from
// each level's free surface; stream-ordered.
int wt_level_barotropic_correction(wt_handle* h, double* const* m, double* const* t) {
  if (int rc = ensure_levels(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  for (int l = h->level_end; l >= h->level_start; --l) {
    const int q = l - h->level_start;
    const DevLevel& D = h->at(l);
    double *ms, *ts, *vs, *mm, *mt;
    if (l == h->level_end) {
      ms = h->mass;
      ts = h->temp;
    } else {
      wt_level_state(h, l, &ms, &ts, &vs);
    }
    if (m) {
      ms = m[q];
      ts = t[q];
    }
    if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_MASS, &mm)) return rc;
    if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_TEMP, &mt)) return rc;
    wtb::k_barotropic_correction<<<nb(10 * (D.n + 1) * (D.n + 1)), TPB, 0, h->stream>>>(D.view(), h->nz, h->ph.ref_density,
                                                                            B->L[q].eta, mm, mt, ms, ts);
  }
  CKB(cudaGetLastError());
  return WT_OK;
}

// The free-surface fields of level l: eta (sol(S_MASS, zlevels+1)), the
// elliptic right-hand side, the flux divergence and the previous one.
int wt_level_baro_fields(wt_handle* h, int l, double** eta, double** rhs, double** div, double** div_old) {
  if (int rc = ensure_levels(h)) return rc;
  BaroLevel& V = static_cast<BaroCtx*>(h->baro)->L[l - h->level_start];
  if (eta) *eta = V.eta;
  if (rhs) *rhs = V.rhs;
  if (div) *div = V.div;
  if (div_old) *div_old = V.div_old;
  return WT_OK;
}

// grad_eta over the hierarchy (src/barotropic_2d.f90:455-474, with
// cpt_or_restr_eta) into each level's gradient field, without the velocity
// update; grad[q] receives level level_start+q's [3][NN] field.  Stream-ordered.
int wt_level_grad_eta(wt_handle* h, const double** grad) {
  if (int rc = ensure_levels(h)) return rc;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  for (int l = h->level_start; l <= h->level_end; ++l) {
    BaroLevel& V = B->L[l - h->level_start];
    const DevLevel& D = h->at(l);
    CKB(cudaMemcpyAsync(V.eta_w, V.eta, (size_t)D.NN * 8, cudaMemcpyDeviceToDevice, h->stream));
    if (D.n_hn > 0) wtb::k_halo_nodes<<<nb(D.n_hn), TPB, 0, h->stream>>>(D.hn, D.n_hn, V.eta_w);
  }
  for (int l = h->level_end; l >= h->level_start; --l) {
    BaroLevel& V = B->L[l - h->level_start];
    const DevLevel& D = h->at(l);
    const int m = D.n + 1;
    if (l < h->level_end)
      if (int rc = wt_level_restrict_scalar(h, l, V.eta_w, B->L[l + 1 - h->level_start].eta_w, 1)) return rc;
    wtb::k_grad_eta_update<true><<<nb(10 * m * m), TPB, 0, h->stream>>>(D.view(), 0, h->ph.grav, V.eta_w, 0.0,
                                                                       V.grad, nullptr);
    grad[l - h->level_start] = V.grad;
  }
  CKB(cudaGetLastError());
  return WT_OK;
}

extern "C" {

// barotropic_correction of the hierarchy's scaling fields from the free surface
// of each level (wt_barotropic_upload_level).
int wt_barotropic_correction_multi(wt_handle* h) {
  if (!h) return WT_ERR_ARG;
  if (!h->wav) return WT_ERR_STATE;
  if (int rc = wt_level_barotropic_correction(h, nullptr, nullptr)) return rc;
  CKB(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

int wt_barotropic_download_level(wt_handle* h, int level, double* div_flux, double* rhs, double* grad) {
  if (!h || level < h->level_start || level > h->level_end) return WT_ERR_ARG;
  if (!h->baro || static_cast<BaroCtx*>(h->baro)->L.empty()) return WT_ERR_STATE;
  BaroLevel& V = static_cast<BaroCtx*>(h->baro)->L[level - h->level_start];
  const size_t NN = (size_t)h->at(level).NN;
  if (div_flux) CKB(cudaMemcpyAsync(div_flux, V.div, NN * 8, cudaMemcpyDeviceToHost, h->stream));
  if (rhs) CKB(cudaMemcpyAsync(rhs, V.rhs, NN * 8, cudaMemcpyDeviceToHost, h->stream));
  if (grad) CKB(cudaMemcpyAsync(grad, V.grad, 3 * NN * 8, cudaMemcpyDeviceToHost, h->stream));
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_free_surface_download(wt_handle* h, int level, double* eta) {
  if (!h || !eta || level < h->level_start || level > h->level_end) return WT_ERR_ARG;
  if (!h->baro || static_cast<BaroCtx*>(h->baro)->L.empty()) return WT_ERR_STATE;
  BaroLevel& V = static_cast<BaroCtx*>(h->baro)->L[level - h->level_start];
  CKB(cudaMemcpyAsync(eta, V.eta, (size_t)h->at(level).NN * 8, cudaMemcpyDeviceToHost, h->stream));
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_barotropic_download(wt_handle* h, double* div_flux, double* rhs, double* grad) {
  if (!h) return WT_ERR_ARG;
  if (!h->baro) return WT_ERR_STATE;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  const size_t NN = (size_t)h->top().NN;
  if (div_flux) CKB(cudaMemcpyAsync(div_flux, B->div, NN * 8, cudaMemcpyDeviceToHost, h->stream));
  if (rhs) CKB(cudaMemcpyAsync(rhs, B->rhs, NN * 8, cudaMemcpyDeviceToHost, h->stream));
  if (grad) CKB(cudaMemcpyAsync(grad, B->grad, 3 * NN * 8, cudaMemcpyDeviceToHost, h->stream));
  CKB(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"
