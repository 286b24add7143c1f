// C-ABI of the barotropic pieces of the mode-split step on the stepper's level
// (level_end): flux_divergence + rhs_elliptic, grad_eta + u_update
// (src/barotropic_2d.f90:118-185, 326-366, 131-149, 455-474).
#include <cuda_runtime.h>

#include "../../include/wavetrisk_gpu.h"
#include "barotropic_kernels.cuh"
#include "wt_handle.cuh"

namespace {

constexpr int TPB = 256;
inline unsigned nb(int64_t n) { return (unsigned)((n + TPB - 1) / TPB); }

struct BaroCtx {
  double *eta = nullptr, *div_old = nullptr, *div = nullptr, *rhs = nullptr, *flux = nullptr, *grad = nullptr;
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

}  // namespace

void wt_barotropic_release(wt_handle* h) {
  if (!h || !h->baro) return;
  BaroCtx* B = static_cast<BaroCtx*>(h->baro);
  double* a[] = {B->eta, B->div_old, B->div, B->rhs, B->flux, B->grad};
  for (double* p : a)
    if (p) cudaFree(p);
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
  wtb::k_grad_eta_update<<<nb(10 * m * m), TPB, 0, h->stream>>>(D.view(), h->nz, h->ph.grav, B->eta, theta1 * dt,
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
