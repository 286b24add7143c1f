// Device context behind the opaque wt_handle of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "trisk_types.cuh"

struct DevLevel {
  int level = 0, n = 0, P = 0;
  int64_t NN = 0;
  double *len = nullptr, *pedlen = nullptr, *part = nullptr, *hex_inv = nullptr, *triarea = nullptr,
         *coriolis = nullptr, *overl_a = nullptr, *topo = nullptr;
  double* iu_wgt = nullptr;  // 9*NN outer velocity weights (levels above level_start)
  double* overl_split = nullptr;  // 2*NN Overl_Area%split
  double* rf_wgt = nullptr;       // 3*NN flux-restriction weights (levels above level_start)
  int2* hn = nullptr;
  int3* he = nullptr;
  int n_hn = 0, n_he = 0;
  int* nsrc = nullptr;  // node read remap (ghost -> source node)
  int* esrc = nullptr;  // signed edge read remap: source slot * 2 + negate
  wtk::LevelDev view() const {
    return wtk::LevelDev{n, P, (int)NN, len, pedlen, part, hex_inv, triarea, coriolis, topo, nsrc, esrc};
  }
  void release() {
    double* a[] = {len, pedlen, part, hex_inv, triarea, coriolis, overl_a, topo, iu_wgt, overl_split, rf_wgt};
    for (double* p : a)
      if (p) cudaFree(p);
    if (hn) cudaFree(hn);
    if (he) cudaFree(he);
    if (nsrc) cudaFree(nsrc);
    if (esrc) cudaFree(esrc);
    nsrc = esrc = nullptr;
    len = pedlen = part = hex_inv = triarea = coriolis = overl_a = topo = iu_wgt = overl_split = rf_wgt = nullptr;
    hn = nullptr;
    he = nullptr;
  }
};

struct wt_handle {
  int nz = 0, level_start = 0, level_end = 0;
  wtk::Phys ph{};
  std::vector<DevLevel> lev;
  cudaStream_t stream = nullptr;
  // prognostic state (level_end) and RK4 stage copy
  double *mass = nullptr, *temp = nullptr, *velo = nullptr, *mean_m = nullptr, *mean_t = nullptr;
  double *m1 = nullptr, *t1 = nullptr, *v1 = nullptr;
  double *m2 = nullptr, *t2 = nullptr, *v2 = nullptr;  // second stage buffer: a stage never writes what it reads
  // trend output (wt_trend) and operator work arrays
  double *dm = nullptr, *dt = nullptr, *dv = nullptr;
  double *qe = nullptr, *hfm = nullptr, *hft = nullptr, *bern = nullptr, *phik = nullptr, *pterm = nullptr;
  double* theta = nullptr;  // Theta/rho of the stage state, written by k_step1
  wtk::TrendMaps maps{};    // tensor maps of the trend inputs (TMA-staged trend kernel)
  wtk::Step1Maps s1maps[3]{};  // step1 input maps for the state buffers (mass,temp,velo), (m1,t1,v1), (m2,t2,v2)
  int* dflag = nullptr;     // device error flag: 1 = a kernel's staged copies did not complete
  int tma_inject = 0;       // test only: the TMA kernels take their wait-timeout path
  int trend_variant = 0;    // 0: TMA-staged k_step1_tma/k_trend_tma, 1: k_step1/k_trend (loads through L1)
  // WT_TUNE_FLUX_PRECISION: 64 (default) or 32, the FP32 step1 of the
  // single-level stepper (trisk_mixed.cuh) with its FP32 results below
  int flux_bits = 64;
  float *qe32 = nullptr, *hfm32 = nullptr, *hft32 = nullptr, *ke32 = nullptr, *theta32 = nullptr;
  bool state_halo_done = false;
  cudaGraphExec_t graph_exec = nullptr;
  double graph_dt = 0.0;
  int sticky = 0;  // WT_OK or the first error seen by a device-side check

  // elliptic solver state (allocated by wt_elliptic_setup)
  void* ell = nullptr;
  // multi-level wavelet fields and masks (allocated by wt_wavelet_setup)
  void* wav = nullptr;
  // free-surface fields of the barotropic step (allocated on first use)
  void* baro = nullptr;
  // per-level operator arrays of the multi-level trend (allocated on first use)
  void* ml = nullptr;
  void release_extra();

  DevLevel& top() { return lev.back(); }
  DevLevel& at(int l) { return lev[l - level_start]; }
};

int wt_handle_fail(const char* where, cudaError_t e);
void wt_wavelet_release(wt_handle* h);
void wt_barotropic_release(wt_handle* h);
void wt_trend_ml_release(wt_handle* h);

// Launchers shared between translation units (stream-ordered, no sync).
// integrate_pressure_up + step1 (itype 0) + post_step1 of every layer of `level`
// on the given state, into the given operator arrays (wt_api.cu).
// With maps (the top level's step1 input maps of this state) the top level runs
// the TMA-staged step1 when the handle selected it.
// stream: the handle's when null.  need: the column and the L1 step1 leave out
// the nodes outside this needed-node map (need_map.cuh), the TMA step1 the tiles
// with none of them; step1 reads the column's results only at its own node.
// Tensor maps of the top level's trend inputs held in the given arrays (with the
// level's geometry), for k_trend_tma; WT_ERR_STATE unless the TMA variant is on.
int wt_make_trend_maps(wt_handle* h, const double* hfm, const double* hft, const double* qe, const double* theta,
                       const double* bern, const double* phik, wtk::TrendMaps* M);
// k_trend_tma<MODE_ML> on the top level (stream: the handle's when null).
int wt_level_trend_ml_tma(wt_handle* h, const wtk::TrendIO& io, const wtk::TrendMaps& M, cudaStream_t stream);
int wt_level_step1(wt_handle* h, int level, const double* m, const double* t, const double* v, const double* mean_m,
                   const double* mean_t, double* phik, double* pterm, double* qe, double* hfm, double* hft,
                   double* bern, double* theta, const wtk::Step1Maps* maps, cudaStream_t stream,
                   const unsigned char* need = nullptr, const wtk::NodeList* list = nullptr);
// The step1 input maps of a top-level state (WT_ERR_STATE when the handle runs the L1 kernels) (wt_api.cu).
int wt_make_step1_maps(wt_handle* h, const double* m, const double* t, const double* v, wtk::Step1Maps* out);
// scalar_cpt_restr / flux_cpt_restr of the nz layers of the given fields from
// level+1 to `level` with the masks of the hierarchy (wt_wavelet.cu).
int wt_level_restrict_scalar(wt_handle* h, int level, double* par, const double* chd, int nz,
                             cudaStream_t stream = nullptr);
// flux_cpt_restr of two fluxes (par1/chd1/dsc1 may be null) in one launch.
int wt_level_restrict_flux(wt_handle* h, int level, double* par0, double* par1, const double* chd0,
                           const double* chd1, const double* dsc0, const double* dsc1, int nz);
// The layer mean WT_FIELD_MEAN_MASS/TEMP of a level (wt_wavelet.cu).
int wt_level_mean(wt_handle* h, int level, int field, double** out);
// The masks of a level, or null before wt_wavelet_setup (wt_wavelet.cu).
void wt_level_masks(wt_handle* h, int level, const int** mask_n, const int** mask_e);
// WT_after_step on the given per-level scaling fields (level_start first), or on
// the hierarchy's own when the arrays are null; stream-ordered (wt_wavelet.cu).
// mode selects the parents the inverse transform rebuilds, as in
// wt_level_wav_finish.
int wt_level_after_step(wt_handle* h, double* const* m, double* const* t, double* const* v, int mode = 0);
// WT_after_step in pieces, for callers that launch each level pair's forward
// wavelets as soon as both levels' fields are written: bind the stage's scaling
// fields, wt_level_clean_wavelets, wt_level_wav_forward_pair for every l in
// [level_start, level_end), wt_level_wav_finish, unbind.
void wt_level_wav_bind(wt_handle* h, double* const* m, double* const* t, double* const* v);
void wt_level_wav_unbind(wt_handle* h);
int wt_level_wav_forward_pair(wt_handle* h, int level);
// mode 0: the inverse rebuilds every parent; 1: only the parents of
// wt_level_rec (an intermediate RK stage, whose state the next stage reads only
// where needed); 2: those of wt_level_rec_final (the step's last inverse).
// rebuild false: join the forward wavelets and leave the inverse out (its result
// would be overwritten before anything reads it)
int wt_level_wav_finish(wt_handle* h, int mode = 0, bool rebuild = true);
const unsigned char* wt_level_rec(wt_handle* h, int level);
// the parents the inverse after adapt rebuilds (patch tree), or null: every parent
const unsigned char* wt_level_rec_final(wt_handle* h, int level);
// adapt's mask sequence without host synchronisation (capturable), compression
// and inverse transform of the hierarchy, and the threshold upload (wt_wavelet.cu).
int wt_level_mask_sequence(wt_handle* h, int level_fill, int max_level, int patch_size, unsigned char* dreq);
void wt_level_compress(wt_handle* h);
int wt_level_mask_snapshot_alloc(wt_handle* h);
void wt_level_mask_snapshot(wt_handle* h);
void wt_level_compress_delta(wt_handle* h);
// zero every wavelet array if a host upload wrote wavelets since the last
// zeroing (stream-ordered; WT_after_step then writes only the slots it computes)
void wt_level_clean_wavelets(wt_handle* h);
// whether every wavelet slot that WT_after_step sets to 0 under the current
// masks holds 0 already (then the forward wavelets write only the kept slots)
bool wt_level_zero_ok(wt_handle* h);
// The needed-node maps of the levels above level_start (need_map.cuh): build
// them from the current masks (stream-ordered; the mask sequence does so at its
// end); the map a level's RK-stage kernels may skip by, or null; the count of
// changes to WT_TUNE_SKIP_INACTIVE.
int wt_level_need_build(wt_handle* h);
const unsigned char* wt_level_need(wt_handle* h, int level);
// the work list of a level's needed-node map ({null, null} without a map)
wtk::NodeList wt_level_list(wt_handle* h, int level);
int wt_level_skip_epoch(wt_handle* h);
// barotropic_correction of the given per-level scaling fields (hierarchy's own
// when m is null) and grad_eta per level, without the velocity update
// (wt_barotropic.cu); stream-ordered.
int wt_level_barotropic_correction(wt_handle* h, double* const* m, double* const* t);
int wt_level_grad_eta(wt_handle* h, const double** grad);
// make stream st wait until the last inverse transform (wt_level_inverse or
// WT_after_step) has completed level's state; only valid when that transform was
// issued after every other write of the state (stream-ordered)
int wt_level_ready_wait(wt_handle* h, int level, cudaStream_t st);
// build the map if skipping is on and the masks changed since the last build
int wt_level_need_refresh(wt_handle* h);
// The inverse transform after adapt (stream-ordered): with a patch tree it
// rebuilds the parents the next step reads and those of the tree's nodes, so
// that the state is complete on the tree; without one every parent.
void wt_level_inverse(wt_handle* h);
int wt_level_set_thresholds(wt_handle* h, const double* threshold);
// The scaling fields (mass, Theta, velocity) of a level (wt_wavelet.cu).
void wt_level_state(wt_handle* h, int level, double** m, double** t, double** v);
