// C-ABI implementation: device context, state upload/download, the trend and
// the RK4 stepper (one captured CUDA graph per step).
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/wavetrisk_gpu.h"
#include "trisk_kernels.cuh"
#include "trisk_mixed.cuh"
#include "trisk_tma.cuh"
#include "wt_handle.cuh"

using namespace wtk;

namespace {

constexpr int TPB = 256;

inline unsigned blocks_for(int64_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

}  // namespace


int wt_handle_fail(const char* where, cudaError_t e) {
  std::fprintf(stderr, "wavetrisk_gpu: %s: %s\n", where, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? WT_ERR_ALLOC : WT_ERR_CUDA;
}

#define CK(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return wt_handle_fail(#x, e_); \
  } while (0)

static int dev_copy(double** dst, const double* src, int64_t count) {
  CK(cudaMalloc(dst, count * sizeof(double)));
  if (src)
    CK(cudaMemcpy(*dst, src, count * sizeof(double), cudaMemcpyHostToDevice));
  else
    CK(cudaMemset(*dst, 0, count * sizeof(double)));
  return WT_OK;
}

static int dev_zero(double** dst, int64_t count) { return dev_copy(dst, nullptr, count); }

// Tensor maps of the trend inputs on the top level: dims (P, P, 10 lozenges,
// planes), boxes of TB_X x TB_Y nodes.  The encoder is taken from the driver
// through the runtime, so the library does not link libcuda directly.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
      std::fprintf(stderr, "wavetrisk_gpu: cuTensorMapEncodeTiled unavailable\n");
      return nullptr;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return encode;
}

// Tensor map of a top-level field of `planes` planes of NN doubles.
static bool top_map(wt_handle* h, CUtensorMap* m, const double* base, int planes) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return false;
  const DevLevel& D = h->top();
  const cuuint64_t dims[4] = {(cuuint64_t)D.P, (cuuint64_t)D.P, 10, (cuuint64_t)planes};
  const cuuint64_t strides[3] = {(cuuint64_t)D.P * 8, (cuuint64_t)D.P * D.P * 8, (cuuint64_t)D.NN * 8};
  const cuuint32_t box[4] = {(cuuint32_t)TB_X, (cuuint32_t)TB_Y, 1, 1};
  const cuuint32_t elem[4] = {1, 1, 1, 1};
  return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The step1 input maps of a top-level state (m, t, v) with the top level's means and geometry.
static bool step1_maps(wt_handle* h, const double* m, const double* t, const double* v, Step1Maps* S) {
  const DevLevel& D = h->top();
  const int nz = h->nz;
  return top_map(h, &S->mass, m, nz) && top_map(h, &S->temp, t, nz) && top_map(h, &S->velo, v, 3 * nz) &&
         top_map(h, &S->mean_m, h->mean_m, nz) && top_map(h, &S->mean_t, h->mean_t, nz) &&
         top_map(h, &S->len, D.len, 3) && top_map(h, &S->ped, D.pedlen, 3) && top_map(h, &S->part, D.part, 6) &&
         top_map(h, &S->cor, D.coriolis, 2);
}

int wt_make_step1_maps(wt_handle* h, const double* m, const double* t, const double* v, wtk::Step1Maps* out) {
  if (h->trend_variant != 0) return WT_ERR_STATE;
  return step1_maps(h, m, t, v, out) ? WT_OK : WT_ERR_CUDA;
}

int wt_make_trend_maps(wt_handle* h, const double* hfm, const double* hft, const double* qe, const double* theta,
                       const double* bern, const double* phik, wtk::TrendMaps* M) {
  if (h->trend_variant != 0) return WT_ERR_STATE;
  const DevLevel& D = h->top();
  const int nz = h->nz;
  const bool ok = top_map(h, &M->hfm, hfm, 3 * nz) && top_map(h, &M->hft, hft, 3 * nz) &&
                  top_map(h, &M->qe, qe, 3 * nz) && top_map(h, &M->theta, theta, nz) &&
                  top_map(h, &M->bern, bern, nz) && top_map(h, &M->phik, phik, nz) &&
                  top_map(h, &M->part, D.part, 6) && top_map(h, &M->hinv, D.hex_inv, 1);
  return ok ? WT_OK : WT_ERR_CUDA;
}

static int make_trend_maps(wt_handle* h) {
  const DevLevel& D = h->top();
  auto mk = [&](CUtensorMap* m, const double* base, int planes) { return top_map(h, m, base, planes); };
  TrendMaps& M = h->maps;
  const int nz = h->nz;
  bool ok = mk(&M.hfm, h->hfm, 3 * nz) && mk(&M.hft, h->hft, 3 * nz) && mk(&M.qe, h->qe, 3 * nz) &&
                  mk(&M.theta, h->theta, nz) && mk(&M.bern, h->bern, nz) && mk(&M.phik, h->phik, nz) &&
                  mk(&M.part, D.part, 6) && mk(&M.hinv, D.hex_inv, 1);
  double* SM[3] = {h->mass, h->m1, h->m2};
  double* ST[3] = {h->temp, h->t1, h->t2};
  double* SV[3] = {h->velo, h->v1, h->v2};
  for (int b = 0; b < 3 && ok; ++b) ok = step1_maps(h, SM[b], ST[b], SV[b], &h->s1maps[b]);
  if (!ok) {
    std::fprintf(stderr, "wavetrisk_gpu: tensor map encoding failed\n");
    return WT_ERR_CUDA;
  }
  CK(cudaFuncSetAttribute(k_step1_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, STEP1_TMA_SMEM));
  CK(cudaFuncSetAttribute(k_trend_tma<MODE_RK>, cudaFuncAttributeMaxDynamicSharedMemorySize, TREND_TMA_SMEM));
  CK(cudaFuncSetAttribute(k_trend_tma<MODE_TREND>, cudaFuncAttributeMaxDynamicSharedMemorySize, TREND_TMA_SMEM));
  CK(cudaFuncSetAttribute(k_trend_tma<MODE_ML>, cudaFuncAttributeMaxDynamicSharedMemorySize, TREND_TMA_SMEM));
  return WT_OK;
}

extern "C" {

int wt_create(const wt_grid_desc* desc, wt_handle** out) {
  if (!desc || !out || !desc->levels || desc->nz < 1 || desc->level_end < desc->level_start) return WT_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return WT_ERR_NO_DEVICE;
  wt_handle* h = new wt_handle();
  h->nz = desc->nz;
  h->ph = Phys{desc->grav, desc->ref_density, desc->p_top};
  h->level_start = desc->level_start;
  h->level_end = desc->level_end;
  const int nlev = desc->level_end - desc->level_start + 1;
  h->lev.resize(nlev);
  int rc = WT_OK;
  for (int q = 0; q < nlev && rc == WT_OK; ++q) {
    const wt_level_desc& ld = desc->levels[q];
    DevLevel& D = h->lev[q];
    if (ld.n != (1 << ld.level) || ld.P != ld.n + 4 || ld.NN != (int64_t)10 * ld.P * ld.P) { rc = WT_ERR_ARG; break; }
    if (6 * ld.NN >= (int64_t)1 << 31) { rc = WT_ERR_ARG; break; }  // 32-bit offsets inside one layer
    D.level = ld.level;
    D.n = ld.n;
    D.P = ld.P;
    D.NN = ld.NN;
    const int64_t NN = ld.NN;
    if ((rc = dev_copy(&D.len, ld.len, 3 * NN))) break;
    if ((rc = dev_copy(&D.pedlen, ld.pedlen, 3 * NN))) break;
    if ((rc = dev_copy(&D.part, ld.part, 6 * NN))) break;
    if ((rc = dev_copy(&D.hex_inv, ld.hex_inv, NN))) break;
    if ((rc = dev_copy(&D.triarea, ld.triarea, 2 * NN))) break;
    if ((rc = dev_copy(&D.coriolis, ld.coriolis, 2 * NN))) break;
    if ((rc = dev_copy(&D.overl_a, ld.overl_a, 4 * NN))) break;
    if ((rc = dev_copy(&D.topo, ld.topo, NN))) break;
    if (ld.iu_wgt && (rc = dev_copy(&D.iu_wgt, ld.iu_wgt, 9 * NN))) break;
    if (ld.overl_split && (rc = dev_copy(&D.overl_split, ld.overl_split, 2 * NN))) break;
    if (ld.rf_wgt && (rc = dev_copy(&D.rf_wgt, ld.rf_wgt, 3 * NN))) break;
    std::vector<int2> hn(ld.n_halo_node);
    for (int64_t k = 0; k < ld.n_halo_node; ++k) {
      int64_t a = ld.halo_node[2 * k], b = ld.halo_node[2 * k + 1];
      if (a < 0 || b < 0 || a >= NN || b >= NN) { rc = WT_ERR_ARG; break; }
      hn[k] = make_int2((int)a, (int)b);
    }
    if (rc) break;
    std::vector<int3> he(ld.n_halo_edge);
    for (int64_t k = 0; k < ld.n_halo_edge; ++k) {
      int64_t a = ld.halo_edge[3 * k], b = ld.halo_edge[3 * k + 1], s = ld.halo_edge[3 * k + 2];
      if (a < 0 || b < 0 || a >= 3 * NN || b >= 3 * NN) { rc = WT_ERR_ARG; break; }
      he[k] = make_int3((int)a, (int)b, (int)s);
    }
    if (rc) break;
    D.n_hn = (int)hn.size();
    D.n_he = (int)he.size();
    cudaError_t e;
    if ((e = cudaMalloc(&D.hn, sizeof(int2) * std::max<size_t>(1, hn.size()))) != cudaSuccess) { rc = wt_handle_fail("halo", e); break; }
    if ((e = cudaMalloc(&D.he, sizeof(int3) * std::max<size_t>(1, he.size()))) != cudaSuccess) { rc = wt_handle_fail("halo", e); break; }
    cudaMemcpy(D.hn, hn.data(), sizeof(int2) * hn.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(D.he, he.data(), sizeof(int3) * he.size(), cudaMemcpyHostToDevice);
    // read remaps: a ghost reads the node / signed edge its copy entry names
    std::vector<int> nsrc(NN), esrc(3 * NN);
    for (int64_t k = 0; k < NN; ++k) nsrc[k] = (int)k;
    for (auto& x : hn) nsrc[x.x] = x.y;
    for (int64_t k = 0; k < 3 * NN; ++k) esrc[k] = (int)(2 * k);
    for (auto& x : he) esrc[x.x] = 2 * x.y + (x.z < 0 ? 1 : 0);
    if ((e = cudaMalloc(&D.nsrc, sizeof(int) * NN)) != cudaSuccess) { rc = wt_handle_fail("remap", e); break; }
    if ((e = cudaMalloc(&D.esrc, sizeof(int) * 3 * NN)) != cudaSuccess) { rc = wt_handle_fail("remap", e); break; }
    cudaMemcpy(D.nsrc, nsrc.data(), sizeof(int) * NN, cudaMemcpyHostToDevice);
    cudaMemcpy(D.esrc, esrc.data(), sizeof(int) * 3 * NN, cudaMemcpyHostToDevice);
  }
  if (rc == WT_OK) {
    // Kernel pair: TMA-staged tiles from n = 64 up; below that the 32-wide tiles
    // are mostly empty (n + 1 = 33 nodes per row at J5) and the L1 kernels are
    // faster.  WAVETRISK_TREND_KERNEL=tma|plain forces either pair.
    h->trend_variant = (h->top().n >= 64) ? 0 : 1;
    if (const char* tv = std::getenv("WAVETRISK_TREND_KERNEL")) {
      if (std::strcmp(tv, "tma") == 0) h->trend_variant = 0;
      if (std::strcmp(tv, "plain") == 0) h->trend_variant = 1;
    }
  }
  if (rc == WT_OK) {
    // Prognostic state and RK/trend work arrays on level_end.
    DevLevel& D = h->top();
    const int64_t NN = D.NN, nn = (int64_t)h->nz * NN, ne = 3 * nn;
    double** node_arrays[] = {&h->mass, &h->temp, &h->mean_m, &h->mean_t, &h->m1, &h->t1, &h->m2, &h->t2,
                              &h->dm, &h->dt, &h->bern, &h->phik, &h->pterm, &h->theta};
    for (double** p : node_arrays)
      if ((rc = dev_zero(p, nn))) break;
    double** edge_arrays[] = {&h->velo, &h->v1, &h->v2, &h->dv, &h->qe, &h->hfm, &h->hft};
    if (rc == WT_OK)
      for (double** p : edge_arrays)
        if ((rc = dev_zero(p, ne))) break;
    if (rc == WT_OK) {
      // The handle's stream carries the critical path of a step (the finest
      // level's step1 and trend, the restrictions, the coarser trends, the
      // velocity reconstruction); the side streams that run beside it (coarser
      // levels' step1, forward wavelets, scalar reconstruction) keep the default
      // priority, so the block scheduler serves this stream's blocks first.
      int least = 0, greatest = 0;
      cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
      if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, greatest);
      if (e != cudaSuccess) rc = wt_handle_fail("stream", e);
    }
    if (rc == WT_OK) {
      cudaError_t e = cudaMalloc(&h->dflag, sizeof(int));
      if (e == cudaSuccess) e = cudaMemset(h->dflag, 0, sizeof(int));
      if (e != cudaSuccess) rc = wt_handle_fail("flag", e);
    }
    if (rc == WT_OK) rc = make_trend_maps(h);
  }
  if (rc != WT_OK) {
    wt_destroy(h);
    return rc;
  }
  *out = h;
  return WT_OK;
}

int wt_destroy(wt_handle* h) {
  if (!h) return WT_OK;
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  for (auto& D : h->lev) D.release();
  double* arrays[] = {h->mass, h->temp, h->velo, h->mean_m, h->mean_t, h->m1, h->t1, h->v1, h->m2, h->t2, h->v2,
                      h->dm, h->dt, h->dv, h->qe, h->hfm, h->hft, h->bern, h->phik, h->pterm, h->theta};
  for (double* p : arrays)
    if (p) cudaFree(p);
  float* arrays32[] = {h->qe32, h->hfm32, h->hft32, h->ke32, h->theta32};
  for (float* p : arrays32)
    if (p) cudaFree(p);
  h->release_extra();
  if (h->dflag) cudaFree(h->dflag);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return WT_OK;
}

void* wt_stream(wt_handle* h) { return h ? (void*)h->stream : nullptr; }

// WT_TUNE_FLUX_PRECISION (wt_tune): the single-level stepper's flux stencils
// in FP64 (64) or FP32 (32).  The FP32 work arrays are allocated on the first
// switch to 32; the captured step graph is dropped so the next step records
// the other kernels.
int wt_set_flux_precision(wt_handle* h, int bits) {
  if (!h || (bits != 64 && bits != 32)) return WT_ERR_ARG;
  if (bits == h->flux_bits) return WT_OK;
  if (bits == 32 && !h->qe32) {
    const int64_t nn = (int64_t)h->nz * h->top().NN;
    float** arrays[] = {&h->qe32, &h->hfm32, &h->hft32, &h->ke32, &h->theta32};
    const int64_t sizes[] = {3 * nn, 3 * nn, 3 * nn, nn, nn};
    for (int q = 0; q < 5; ++q) {
      cudaError_t e = cudaMalloc(arrays[q], sizeof(float) * sizes[q]);
      if (e == cudaSuccess) e = cudaMemset(*arrays[q], 0, sizeof(float) * sizes[q]);
      if (e != cudaSuccess) return wt_handle_fail("flux fp32 arrays", e);
    }
  }
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
  }
  h->flux_bits = bits;
  return WT_OK;
}

int wt_synchronize(wt_handle* h) {
  if (!h) return WT_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_clear_status(wt_handle* h) {
  if (!h) return WT_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  if (h->dflag) CK(cudaMemset(h->dflag, 0, sizeof(int)));
  h->sticky = WT_OK;
  return WT_OK;
}

// Test-only: the TMA kernels of the next steps declare more bytes than their
// copies deliver and take their wait-timeout path (value 1), or run normally
// (0).  The captured step graphs hold the flag, so they are dropped here.
int wt_set_tma_inject(wt_handle* h, int value) {
  if (!h) return WT_ERR_ARG;
  if (value != 0 && value != 1) return WT_ERR_ARG;
  if (h->tma_inject == value) return WT_OK;
  CK(cudaStreamSynchronize(h->stream));
  h->tma_inject = value;
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
  }
  return WT_OK;
}

int wt_status(wt_handle* h) {
  if (!h) return WT_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaGetLastError());
  if (h->dflag && h->sticky == WT_OK) {
    int f = 0;
    CK(cudaMemcpy(&f, h->dflag, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) h->sticky = WT_ERR_TIMEOUT;
  }
  return h->sticky;
}

int wt_upload_state(wt_handle* h, const double* mass, const double* temp, const double* velo, const double* mean_m,
                    const double* mean_t) {
  if (!h || !mass || !temp || !velo) return WT_ERR_ARG;
  const int64_t nn = (int64_t)h->nz * h->top().NN;
  CK(cudaMemcpyAsync(h->mass, mass, nn * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->temp, temp, nn * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->velo, velo, 3 * nn * 8, cudaMemcpyHostToDevice, h->stream));
  if (mean_m) CK(cudaMemcpyAsync(h->mean_m, mean_m, nn * 8, cudaMemcpyHostToDevice, h->stream));
  if (mean_t) CK(cudaMemcpyAsync(h->mean_t, mean_t, nn * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

int wt_download_state(wt_handle* h, double* mass, double* temp, double* velo) {
  if (!h || !mass || !temp || !velo) return WT_ERR_ARG;
  const int64_t nn = (int64_t)h->nz * h->top().NN;
  {
    // ghosts are read through remaps on the device; fill them for the host
    DevLevel& D = h->top();
    int64_t nt = (int64_t)(2 * D.n_hn + D.n_he) * h->nz;
    k_halo_state<<<blocks_for(nt), TPB, 0, h->stream>>>(h->nz, D.NN, D.hn, D.n_hn, D.he, D.n_he, h->mass, h->temp, h->velo);
  }
  CK(cudaMemcpyAsync(mass, h->mass, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(temp, h->temp, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(velo, h->velo, 3 * nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"

// Optional per-launch timing (wt_profile_rk4): events recorded around each
// kernel on the handle's stream.
struct KTimer {
  std::vector<cudaEvent_t> ev;
  std::vector<int> ids;
  cudaStream_t s = nullptr;
  void begin(int) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    ev.push_back(e);
  }
  void end(int id) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    ev.push_back(e);
    ids.push_back(id);
  }
  ~KTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};
#define TB(id) \
  if (tm) tm->begin(id)
#define TE(id) \
  if (tm) tm->end(id)

// Launch sequence of one trend evaluation of state (m, t, v); MODE_RK writes
// dst = base + hstep * trend, MODE_TREND writes the trends into h->dm/dt/dv.
static int launch_trend(wt_handle* h, double* m, double* t, double* v, int mode, const double* bm, const double* bt,
                        const double* bv, double* om, double* ot, double* ov, double hstep, bool halo_first,
                        KTimer* tm = nullptr) {
  DevLevel& D = h->top();
  LevelDev L = D.view();
  const int nz = h->nz;
  cudaStream_t s = h->stream;
  (void)halo_first;
  // block b: layer b % nz of node chunk b / nz (layer_node in trisk_kernels.cuh)
  const unsigned chunks = blocks_for(D.NN, NODE_TILE);
  TB(1);
  k_column<<<chunks, NODE_TILE, 0, s>>>(L, h->ph, nz, m, t, h->mean_m, h->mean_t, h->phik, h->pterm, nullptr);
  TE(1);
  if (h->flux_bits == 32) {  // FP32 flux stencils, FP64 trends and sub-step (trisk_mixed.cuh)
    TB(2);
    k_step1_f32<<<chunks * nz, NODE_TILE, 0, s>>>(L, nz, m, t, v, h->mean_m, h->mean_t,
                                                   Step1OutF{h->qe32, h->hfm32, h->hft32, h->ke32, h->theta32});
    TE(2);
    TrendIOF io{};
    io.theta = h->theta32; io.qe = h->qe32; io.hfm = h->hfm32; io.hft = h->hft32; io.ke = h->ke32;
    io.phik = h->phik; io.pterm = h->pterm;
    io.base_m = bm; io.base_t = bt; io.base_v = bv; io.dst_m = om; io.dst_t = ot; io.dst_v = ov; io.h = hstep;
    io.dm = h->dm; io.dtt = h->dt; io.dv = h->dv;
    TB(5);
    if (mode == MODE_RK)
      k_trend_mixed<MODE_RK><<<chunks * nz, NODE_TILE, 0, s>>>(L, nz, io);
    else
      k_trend_mixed<MODE_TREND><<<chunks * nz, NODE_TILE, 0, s>>>(L, nz, io);
    TE(5);
    CK(cudaGetLastError());
    return WT_OK;
  }
  Step1Out so{h->qe, h->hfm, h->hft, h->bern, h->theta};
  TB(2);
  if (h->trend_variant == 0) {
    const int sb = (m == h->m1) ? 1 : (m == h->m2) ? 2 : 0;  // which state buffer the stage reads
    const int nbx = (D.n + 1 + TT_X - 1) / TT_X, nby = (D.n + 1 + TT_Y - 1) / TT_Y;
    const unsigned nblk = (unsigned)(nz * nbx * nby * 10);
    k_step1_tma<<<nblk, TT_X * TT_Y, STEP1_TMA_SMEM, s>>>(L, nz, nbx, nby, m, t, v, h->mean_m, h->phik, h->pterm, so,
                                                           h->dflag, h->tma_inject, h->s1maps[sb], nullptr);
  } else {
    k_step1<<<chunks * nz, NODE_TILE, 0, s>>>(L, nz, m, t, v, h->mean_m, h->mean_t, h->phik, h->pterm, so, nullptr);
  }
  TE(2);
  TrendIO io{};
  io.theta = h->theta; io.qe = h->qe; io.hfm = h->hfm; io.hft = h->hft; io.bern = h->bern; io.phik = h->phik;
  io.base_m = bm; io.base_t = bt; io.base_v = bv; io.dst_m = om; io.dst_t = ot; io.dst_v = ov; io.h = hstep;
  io.dm = h->dm; io.dtt = h->dt; io.dv = h->dv;
  TB(5);
  if (h->trend_variant == 0) {
    const int nbx = (D.P + TT_X - 1) / TT_X, nby = (D.P + TT_Y - 1) / TT_Y;
    const unsigned nblk = (unsigned)(nz * nbx * nby * 10);
    if (mode == MODE_RK)
      k_trend_tma<MODE_RK><<<nblk, TT_X * TT_Y, TREND_TMA_SMEM, s>>>(L, nz, nbx, nby, io, h->dflag, h->tma_inject,
                                                                     h->maps);
    else
      k_trend_tma<MODE_TREND><<<nblk, TT_X * TT_Y, TREND_TMA_SMEM, s>>>(L, nz, nbx, nby, io, h->dflag, h->tma_inject,
                                                                        h->maps);
  } else {
    if (mode == MODE_RK)
      k_trend<MODE_RK><<<chunks * nz, NODE_TILE, 0, s>>>(L, nz, io);
    else
      k_trend<MODE_TREND><<<chunks * nz, NODE_TILE, 0, s>>>(L, nz, io);
  }
  TE(5);
  CK(cudaGetLastError());
  return WT_OK;
}

// k_trend_tma<MODE_ML> on the top level: the multi-level trend of the finest
// level with the RK sub-step, its inputs read through the maps M.
int wt_level_trend_ml_tma(wt_handle* h, const wtk::TrendIO& io, const wtk::TrendMaps& M, cudaStream_t stream) {
  const DevLevel& D = h->top();
  const int nz = h->nz;
  const int nbx = (D.P + TT_X - 1) / TT_X, nby = (D.P + TT_Y - 1) / TT_Y;
  const unsigned nblk = (unsigned)(nz * nbx * nby * 10);
  k_trend_tma<MODE_ML><<<nblk, TT_X * TT_Y, TREND_TMA_SMEM, stream ? stream : h->stream>>>(D.view(), nz, nbx, nby, io,
                                                                                           h->dflag, h->tma_inject, M);
  CK(cudaGetLastError());
  return WT_OK;
}

int wt_level_step1(wt_handle* h, int level, const double* m, const double* t, const double* v, const double* mean_m,
                   const double* mean_t, double* phik, double* pterm, double* qe, double* hfm, double* hft,
                   double* bern, double* theta, const wtk::Step1Maps* maps, cudaStream_t stream,
                   const unsigned char* need, const wtk::NodeList* list) {
  const DevLevel& D = h->at(level);
  const LevelDev L = D.view();
  const int nz = h->nz;
  cudaStream_t s = stream ? stream : h->stream;
  const unsigned chunks = blocks_for(D.NN, NODE_TILE);
  Step1Out so{qe, hfm, hft, bern, theta};
  if (list && list->ids) {  // the needed slots only, persistent blocks over the level's work list
    k_column_list<<<persistent_grid(k_column_list, chunks), NODE_TILE, 0, s>>>(L, h->ph, nz, m, t, mean_m, mean_t,
                                                                               phik, pterm, *list);
    k_step1_list<<<persistent_grid(k_step1_list, chunks * nz), NODE_TILE, 0, s>>>(L, nz, m, t, v, mean_m, mean_t,
                                                                                  phik, pterm, so, *list);
    CK(cudaGetLastError());
    return WT_OK;
  }
  k_column<<<chunks, NODE_TILE, 0, s>>>(L, h->ph, nz, m, t, mean_m, mean_t, phik, pterm, need);
  if (maps && level == h->level_end && h->trend_variant == 0) {
    const int nbx = (D.n + 1 + TT_X - 1) / TT_X, nby = (D.n + 1 + TT_Y - 1) / TT_Y;
    const unsigned nblk = (unsigned)(nz * nbx * nby * 10);
    k_step1_tma<<<nblk, TT_X * TT_Y, STEP1_TMA_SMEM, s>>>(L, nz, nbx, nby, m, t, v, mean_m, phik, pterm, so,
                                                           h->dflag, h->tma_inject, *maps, need);
  } else {
    k_step1<<<chunks * nz, NODE_TILE, 0, s>>>(L, nz, m, t, v, mean_m, mean_t, phik, pterm, so, need);
  }
  CK(cudaGetLastError());
  return WT_OK;
}

extern "C" {

int wt_trend(wt_handle* h) {
  if (!h) return WT_ERR_ARG;
  int rc = launch_trend(h, h->mass, h->temp, h->velo, MODE_TREND, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                        0.0, true);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_download_trend(wt_handle* h, double* dmass, double* dtemp, double* dvelo) {
  if (!h || !dmass || !dtemp || !dvelo) return WT_ERR_ARG;
  const int64_t nn = (int64_t)h->nz * h->top().NN;
  CK(cudaMemcpyAsync(dmass, h->dm, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(dtemp, h->dt, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(dvelo, h->dv, 3 * nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

// One RK4 step (src/time_integr.f90:78-103): four trend evaluations, each
// fused with its sub-step.  WT_after_step on a uniform level is the ghost copy,
// which the kernels replace by reading ghosts through the remap tables.
static int record_rk4(wt_handle* h, double dt, KTimer* tm = nullptr) {
  const double hs[4] = {dt / 4.0, dt / 3.0, dt / 2.0, dt};
  // Stage states ping-pong between two buffers: k_trend reads the stage state at
  // neighbouring nodes while it writes the next one, so they must differ (the
  // reference finishes the whole trend before RK_sub_step).  The last stage
  // writes the solution in place, which it reads only at each thread's own node.
  double* SM[3] = {h->mass, h->m1, h->m2};
  double* ST[3] = {h->temp, h->t1, h->t2};
  double* SV[3] = {h->velo, h->v1, h->v2};
  const int qi[4] = {0, 1, 2, 1}, oi[4] = {1, 2, 1, 0};
  for (int stage = 0; stage < 4; ++stage) {
    double* qm = SM[qi[stage]];
    double* qt = ST[qi[stage]];
    double* qv = SV[qi[stage]];
    double* om = SM[oi[stage]];
    double* ot = ST[oi[stage]];
    double* ov = SV[oi[stage]];
    int rc = launch_trend(h, qm, qt, qv, MODE_RK, h->mass, h->temp, h->velo, om, ot, ov, hs[stage], false, tm);
    if (rc) return rc;
  }
  CK(cudaGetLastError());
  return WT_OK;
}

int wt_rk4_step(wt_handle* h, double dt, int nsteps) {
  if (!h || nsteps < 0) return WT_ERR_ARG;
  if (nsteps == 0) return WT_OK;
  if (!h->graph_exec || h->graph_dt != dt) {
    if (h->graph_exec) { cudaGraphExecDestroy(h->graph_exec); h->graph_exec = nullptr; }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = record_rk4(h, dt);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return wt_handle_fail("capture", e);
    CK(cudaGraphInstantiate(&h->graph_exec, g, 0));
    cudaGraphDestroy(g);
    h->graph_dt = dt;
  }
  for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(h->graph_exec, h->stream));
  CK(cudaGetLastError());
  return WT_OK;
}

// Same steps as wt_rk4_step, launched kernel by kernel (no graph) with CUDA
// events around every launch; ms_per_launch[k] receives the average duration
// of kernel k (0 halo_state, 1 column, 2 step1, 3 post_step1, 4 halo_flux,
// 5 trend_rk) and *nkernels the number of kernel kinds.
int wt_profile_rk4(wt_handle* h, double dt, int nsteps, double* ms_per_launch, int* nkernels) {
  if (!h || nsteps < 1 || !ms_per_launch || !nkernels) return WT_ERR_ARG;
  KTimer tm;
  tm.s = h->stream;
  for (int s = 0; s < nsteps; ++s) {
    int rc = record_rk4(h, dt, &tm);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(h->stream));
  double tot[8] = {0};
  int cnt[8] = {0};
  for (size_t q = 0; q < tm.ids.size(); ++q) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, tm.ev[2 * q], tm.ev[2 * q + 1]));
    tot[tm.ids[q]] += ms;
    cnt[tm.ids[q]] += 1;
  }
  for (int k = 0; k < 6; ++k) ms_per_launch[k] = cnt[k] ? tot[k] / cnt[k] : 0.0;
  *nkernels = 6;   // kinds 0 (ghost copy), 3, 4 are no longer launched by the stepper
  return WT_OK;
}

int wt_rk4_step_host(wt_handle* h, double dt, int nsteps, double* mass, double* temp, double* velo) {
  if (!h || !mass || !temp || !velo) return WT_ERR_ARG;
  const int64_t nn = (int64_t)h->nz * h->top().NN;
  CK(cudaMemcpyAsync(h->mass, mass, nn * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->temp, temp, nn * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->velo, velo, 3 * nn * 8, cudaMemcpyHostToDevice, h->stream));
  h->state_halo_done = false;
  int rc = wt_rk4_step(h, dt, nsteps);
  if (rc) return rc;
  {
    DevLevel& D = h->top();
    int64_t nt = (int64_t)(2 * D.n_hn + D.n_he) * h->nz;
    k_halo_state<<<blocks_for(nt), TPB, 0, h->stream>>>(h->nz, D.NN, D.hn, D.n_hn, D.he, D.n_he, h->mass, h->temp, h->velo);
  }
  CK(cudaMemcpyAsync(mass, h->mass, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(temp, h->temp, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(velo, h->velo, 3 * nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"
