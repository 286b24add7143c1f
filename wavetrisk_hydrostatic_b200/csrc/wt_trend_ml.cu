// C-ABI of trend_ml over the handle's whole hierarchy (src/multi_level.f90:5-188):
// per level, fine to coarse, the level's operator arrays are computed by the
// single-level column and step1 kernels, the coarse ones are then restricted
// from the level above, and k_trend_ml finishes the level (scalar trends,
// velocity source computed or restricted, gradient terms).  All layers of a
// level are processed per launch: the layers interact only through the
// pressure column, which k_column integrates bottom-up.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/wavetrisk_gpu.h"
#include "trisk_ml.cuh"
#include "wt_handle.cuh"

namespace {

struct MLLevel {
  double *phik = nullptr, *pterm = nullptr, *qe = nullptr, *hfm = nullptr, *hft = nullptr, *bern = nullptr,
         *theta = nullptr, *dm = nullptr, *dt = nullptr, *dv = nullptr, *src = nullptr;
  double *m1 = nullptr, *t1 = nullptr, *v1 = nullptr;  // RK stage state q1
};

struct MLCtx {
  std::vector<MLLevel> L;
  std::vector<void*> allocs;
  // step1 input maps of the top level's RK stage state (TMA-staged step1)
  wtk::Step1Maps q1maps{};
  bool q1maps_ok = false;
  // trend input maps of the top level's work arrays (TMA-staged trend)
  wtk::TrendMaps tmaps{};
  bool tmaps_ok = false;
  // graph of one adaptive step and the parameters it was captured with
  cudaGraphExec_t step_graph = nullptr;
  double g_dt = 0.0;
  int g_fill = -1, g_max = -1, g_epoch = -1;
  // column + step1 of the coarser levels run on side streams, forked from the
  // handle's stream and joined before each level's restriction
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> done;
  cudaEvent_t fork = nullptr;
  // the Bernoulli and Exner restrictions, level by level on their own stream
  // (they need both levels' step1 and the finer restriction, not the trends)
  cudaStream_t rs = nullptr;
  std::vector<cudaEvent_t> rsd;
  cudaEvent_t s1top = nullptr;
};

#define CKM(x)                                            \
  do {                                                    \
    cudaError_t e_ = (x);                                 \
    if (e_ != cudaSuccess) return wt_handle_fail(#x, e_); \
  } while (0)

int ensure(wt_handle* h) {
  if (h->ml) return WT_OK;
  MLCtx* M = new MLCtx();
  h->ml = M;
  M->L.resize(h->level_end - h->level_start + 1);
  for (int l = h->level_start; l <= h->level_end; ++l) {
    MLLevel& V = M->L[l - h->level_start];
    const size_t nn = (size_t)h->nz * h->at(l).NN;
    double** node[] = {&V.phik, &V.pterm, &V.bern, &V.theta, &V.dm, &V.dt, &V.m1, &V.t1};
    double** edge[] = {&V.qe, &V.hfm, &V.hft, &V.dv, &V.src, &V.v1};
    for (double** p : node) {
      CKM(cudaMalloc(p, nn * 8));
      M->allocs.push_back(*p);
      CKM(cudaMemsetAsync(*p, 0, nn * 8, h->stream));
    }
    for (double** p : edge) {
      CKM(cudaMalloc(p, 3 * nn * 8));
      M->allocs.push_back(*p);
      CKM(cudaMemsetAsync(*p, 0, 3 * nn * 8, h->stream));
    }
  }
  if (h->trend_variant == 0) {
    const MLLevel& T = M->L.back();
    M->tmaps_ok = wt_make_trend_maps(h, T.hfm, T.hft, T.qe, T.theta, T.bern, T.phik, &M->tmaps) == WT_OK;
  }
  CKM(cudaEventCreateWithFlags(&M->fork, cudaEventDisableTiming));
  CKM(cudaEventCreateWithFlags(&M->s1top, cudaEventDisableTiming));
  // The restriction chain feeds the critical path (top priority); the coarser
  // levels' column and step1 run in the slack of the inverse transform and of
  // the finest level's kernels, above the forward wavelets (lowest).
  int least = 0, greatest = 0;
  CKM(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  const int medium = greatest < least ? greatest + 1 : greatest;
  CKM(cudaStreamCreateWithPriority(&M->rs, cudaStreamNonBlocking, greatest));
  for (int l = h->level_start; l < h->level_end; ++l) {
    cudaStream_t s;
    cudaEvent_t e, r;
    CKM(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, medium));
    M->side.push_back(s);
    CKM(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    M->done.push_back(e);
    CKM(cudaEventCreateWithFlags(&r, cudaEventDisableTiming));
    M->rsd.push_back(r);
  }
  return WT_OK;
}

}  // namespace

void wt_trend_ml_release(wt_handle* h) {
  if (!h || !h->ml) return;
  MLCtx* M = static_cast<MLCtx*>(h->ml);
  if (M->step_graph) cudaGraphExecDestroy(M->step_graph);
  for (cudaEvent_t e : M->done) cudaEventDestroy(e);
  for (cudaEvent_t e : M->rsd) cudaEventDestroy(e);
  for (cudaStream_t s : M->side) cudaStreamDestroy(s);
  if (M->rs) cudaStreamDestroy(M->rs);
  if (M->fork) cudaEventDestroy(M->fork);
  if (M->s1top) cudaEventDestroy(M->s1top);
  for (void* p : M->allocs) cudaFree(p);
  delete M;
  h->ml = nullptr;
}

namespace {

// Phase timer of the profiling entry point: CUDA events on the handle's stream
// around each phase, accumulated per phase id.
struct PhaseTimer {
  cudaStream_t s;
  std::vector<cudaEvent_t> ev;
  std::vector<int> ids;
  void mark(int id) {  // begin (id < 0) or end of phase id
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    ev.push_back(e);
    if (id >= 0) ids.push_back(id);
  }
  ~PhaseTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};
enum { PH_STEP1_TOP = 0, PH_STEP1_COARSE, PH_RESTRICT, PH_TREND_TOP, PH_TREND_COARSE, PH_RK_SUB, PH_AFTER_STEP, NPH };
#define PB(t) \
  if (t) (t)->mark(-1)
#define PE(t, id) \
  if (t) (t)->mark(id)

// The scaling fields of every level (level_start first).
struct States {
  std::vector<double*> m, t, v;
};

States hierarchy_state(wt_handle* h) {
  States S;
  for (int l = h->level_start; l <= h->level_end; ++l) {
    double *m, *t, *v;
    if (l == h->level_end) {
      m = h->mass;
      t = h->temp;
      v = h->velo;
    } else {
      wt_level_state(h, l, &m, &t, &v);
    }
    S.m.push_back(m);
    S.t.push_back(t);
    S.v.push_back(v);
  }
  return S;
}

// trend_ml of the state S into each level's dm, dt, dv (stream-ordered).  With
// base and dest, each level's k_trend_ml also takes the RK sub-step
// dest = base + hs * trend (RK_sub_step, src/time_integr.f90:206-225) instead of
// writing dv: a level's state is not read after its step1, so dest may be S.
// With wav (and dest), the forward wavelets of WT_after_step for the level
// pair (l, l+1) are launched as soon as level l's sub-step is written, beside
// the coarser levels' trend; the caller binds dest to the wavelet context
// before and finishes WT_after_step after.
// With after_inverse, the state S was completed by the inverse transform issued
// last (the previous RK stage's WT_after_step): a coarser level's column and
// step1 start as soon as that transform has rebuilt the level, beside the finer
// levels' reconstruction.
// With grad (per level), the velocity sub-step is u_star's base + hs * (trend +
// th1 * grad) (src/barotropic_2d.f90:29-50).
int trend_multi(wt_handle* h, const States& S, PhaseTimer* tm = nullptr, const States* base = nullptr,
                const States* dest = nullptr, double hs = 0.0, bool wav = false, bool after_inverse = false,
                const double* const* grad = nullptr, double th1 = 0.0) {
  MLCtx* M = static_cast<MLCtx*>(h->ml);
  const int nz = h->nz;
  // With WT_after_step following (wav), a level's results above level_start are
  // read only where its needed-node map says so (need_map.cuh).
  // The phase profile (tm) takes the same maps, so that its times are those of the steps.  The
  // mode-split stages (grad) take them too: their extra terms (barotropic_correction, grad_eta) run on
  // every node and read the stage's values only where the next trend does.
  auto need = [&](int l) -> const unsigned char* { return ((wav || tm) && dest) ? wt_level_need(h, l) : nullptr; };
  // and then over the level's work list, the needed slots only (persistent blocks)
  auto list = [&](int l) { return need(l) ? wt_level_list(h, l) : wtk::NodeList{nullptr, nullptr}; };
  // Column + step1 of a level read only that level's state and write only its
  // own work fields, so the coarser levels' run beside the finest level's on
  // side streams (parallel branches of a captured graph).  The phase timer
  // keeps them on the handle's stream so that its events bracket them.
  const bool concurrent = tm == nullptr && h->level_end > h->level_start;
  if (concurrent) {
    CKM(cudaEventRecord(M->fork, h->stream));
    for (int l = h->level_start; l < h->level_end; ++l) {
      const int q = l - h->level_start;
      MLLevel& V = M->L[q];
      double *mm, *mt;
      if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_MASS, &mm)) return rc;
      if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_TEMP, &mt)) return rc;
      if (after_inverse) {
        if (int rc = wt_level_ready_wait(h, l, M->side[q])) return rc;
      } else {
        CKM(cudaStreamWaitEvent(M->side[q], M->fork, 0));
      }
      const wtk::NodeList wl = list(l);
      if (int rc = wt_level_step1(h, l, S.m[q], S.t[q], S.v[q], mm, mt, V.phik, V.pterm, V.qe, V.hfm, V.hft, V.bern,
                                  V.theta, nullptr, M->side[q], need(l), &wl))
        return rc;
      CKM(cudaEventRecord(M->done[q], M->side[q]));
    }
  }
  for (int l = h->level_end; l >= h->level_start; --l) {
    const int q = l - h->level_start;
    MLLevel& V = M->L[q];
    const DevLevel& D = h->at(l);
    if (concurrent && l < h->level_end) {
      CKM(cudaStreamWaitEvent(h->stream, M->done[q], 0));
    } else {
      double *mm, *mt;
      if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_MASS, &mm)) return rc;
      if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_TEMP, &mt)) return rc;
      PB(tm);
      const wtk::Step1Maps* maps = nullptr;
      if (l == h->level_end && h->trend_variant == 0) {
        if (S.m[q] == h->mass && S.t[q] == h->temp && S.v[q] == h->velo) {
          maps = &h->s1maps[0];
        } else if (S.m[q] == V.m1 && S.t[q] == V.t1 && S.v[q] == V.v1) {
          if (!M->q1maps_ok) {
            if (int rc = wt_make_step1_maps(h, V.m1, V.t1, V.v1, &M->q1maps)) return rc;
            M->q1maps_ok = true;
          }
          maps = &M->q1maps;
        }
      }
      const wtk::NodeList wl = list(l);
      if (int rc = wt_level_step1(h, l, S.m[q], S.t[q], S.v[q], mm, mt, V.phik, V.pterm, V.qe, V.hfm, V.hft,
                                  V.bern, V.theta, maps, nullptr, need(l), &wl))
        return rc;
      PE(tm, l == h->level_end ? PH_STEP1_TOP : PH_STEP1_COARSE);
      if (concurrent) CKM(cudaEventRecord(M->s1top, h->stream));
    }
    wtk::TrendML io{};
    const int *mask_n, *mask_e;
    wt_level_masks(h, l, &mask_n, &mask_e);
    io.mask_n = mask_n;
    if (l < h->level_end) {
      MLLevel& C = M->L[q + 1];
      PB(tm);
      cudaStream_t rs = h->stream;
      if (concurrent) {  // after this level's and the child's step1; the finer restriction precedes on rs
        rs = M->rs;
        CKM(cudaStreamWaitEvent(rs, M->done[q], 0));
        CKM(cudaStreamWaitEvent(rs, l + 1 == h->level_end ? M->s1top : M->done[q + 1], 0));
      }
      if (int rc = wt_level_restrict_scalar(h, l, V.bern, C.bern, nz, rs)) return rc;
      if (int rc = wt_level_restrict_scalar(h, l, V.phik, C.phik, nz, rs)) return rc;  // exner = -Phi_k
      if (int rc = wt_level_restrict_flux(h, l, V.hfm, V.hft, C.hfm, C.hft, C.dm, C.dt, nz)) return rc;
      if (concurrent) {
        CKM(cudaEventRecord(M->rsd[q], rs));
        CKM(cudaStreamWaitEvent(h->stream, M->rsd[q], 0));
      }
      PE(tm, PH_RESTRICT);
      const int *mask_n_c, *mask_e_c;
      wt_level_masks(h, l + 1, &mask_n_c, &mask_e_c);
      io.mask_e_chd = mask_e_c;
      io.src_chd = C.src;
      io.P_chd = h->at(l + 1).P;
      io.NN_chd = (int)h->at(l + 1).NN;
    }
    io.theta = V.theta; io.qe = V.qe; io.hfm = V.hfm; io.hft = V.hft; io.bern = V.bern; io.phik = V.phik;
    io.dm = V.dm; io.dtt = V.dt; io.dv = V.dv; io.src = V.src;
    if (base && dest) {
      io.dv = nullptr;
      io.base_m = base->m[q]; io.base_t = base->t[q]; io.base_v = base->v[q];
      io.dst_m = dest->m[q]; io.dst_t = dest->t[q]; io.dst_v = dest->v[q];
      io.h = hs;
      io.grad = grad ? grad[q] : nullptr;
      io.th1 = th1;
    }
    io.need = need(l);
    const unsigned chunks = (unsigned)((D.NN + wtk::NODE_TILE - 1) / wtk::NODE_TILE);
    PB(tm);
    const wtk::NodeList wl = list(l);
    if (wl.ids) {  // the needed slots only, persistent blocks over the level's work list
      wtk::k_trend_ml_list<<<wtk::persistent_grid(wtk::k_trend_ml_list, chunks * nz), wtk::NODE_TILE, 0,
                             h->stream>>>(D.view(), nz, io, wl);
    } else if (l == h->level_end && M->tmaps_ok && base && dest) {  // TMA-staged, the same arithmetic
      wtk::TrendIO t{};
      t.theta = V.theta; t.qe = V.qe; t.hfm = V.hfm; t.hft = V.hft; t.bern = V.bern; t.phik = V.phik;
      t.base_m = io.base_m; t.base_t = io.base_t; t.base_v = io.base_v;
      t.dst_m = io.dst_m; t.dst_t = io.dst_t; t.dst_v = io.dst_v; t.h = io.h;
      t.dm = V.dm; t.dtt = V.dt; t.mask_n = mask_n; t.src = V.src; t.need = io.need;
      t.grad = io.grad; t.th1 = io.th1;
      if (int rc = wt_level_trend_ml_tma(h, t, M->tmaps, nullptr)) return rc;
    } else {
      wtk::k_trend_ml<<<chunks * nz, wtk::NODE_TILE, 0, h->stream>>>(D.view(), nz, io);
    }
    PE(tm, l == h->level_end ? PH_TREND_TOP : PH_TREND_COARSE);
    CKM(cudaGetLastError());
    if (wav && dest && l < h->level_end)
      if (int rc = wt_level_wav_forward_pair(h, l)) return rc;
  }
  return WT_OK;
}

}  // namespace

extern "C" {

int wt_trend_multi(wt_handle* h) {
  if (!h) return WT_ERR_ARG;
  if (!h->wav || h->flux_bits != 64) return WT_ERR_STATE;  // the hierarchy's steps are FP64 only
  if (int rc = ensure(h)) return rc;
  if (int rc = trend_multi(h, hierarchy_state(h))) return rc;
  CKM(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"

namespace {
// last_inverse false: the last stage's WT_after_step computes its wavelets but
// not the inverse transform, for a caller that rebuilds the hierarchy from
// them next (adapt, then inverse_wavelet_transform) without reading the state.
int rk4_multi(wt_handle* h, double dt, int nsteps, PhaseTimer* tm, bool last_inverse = true) {
  MLCtx* M = static_cast<MLCtx*>(h->ml);
  const States q = hierarchy_state(h);
  States q1;
  for (auto& V : M->L) {
    q1.m.push_back(V.m1);
    q1.t.push_back(V.t1);
    q1.v.push_back(V.v1);
  }
  const double hs[4] = {dt / 4.0, dt / 3.0, dt / 2.0, dt};
  if (int rc = wt_level_need_refresh(h)) return rc;
  for (int s = 0; s < nsteps; ++s)
    for (int stage = 0; stage < 4; ++stage) {
      const States& src = stage == 0 ? q : q1;
      const States& dest = stage == 3 ? q : q1;
      if (tm) {  // phase by phase, each stage's inverse over the parents the timed step rebuilds
        if (int rc = trend_multi(h, src, tm, &q, &dest, hs[stage])) return rc;
        PB(tm);
        if (int rc = wt_level_after_step(h, dest.m.data(), dest.t.data(), dest.v.data(), stage < 3 ? 1 : 2))
          return rc;
        PE(tm, PH_AFTER_STEP);
        continue;
      }
      // WT_after_step's forward wavelets start inside the trend, level pair by level pair
      wt_level_wav_bind(h, dest.m.data(), dest.t.data(), dest.v.data());
      wt_level_clean_wavelets(h);
      int rc = trend_multi(h, src, nullptr, &q, &dest, hs[stage], true, stage > 0);
      // the last stage's state is the step's result: rebuilt completely, unless the caller rebuilds it
      if (!rc) rc = wt_level_wav_finish(h, stage < 3, stage < 3 || s < nsteps - 1 || last_inverse);
      wt_level_wav_unbind(h);
      if (rc) return rc;
    }
  return WT_OK;
}
}  // namespace

namespace {
// The four RK_split calls of RK4_split (src/time_integr.f90:360-382, 444-463)
// over the hierarchy, without free_surface_update: per stage
// barotropic_correction of the stage's source state, trend_ml, scalar_star and
// u_star (src/barotropic_2d.f90:9-50; the base is always the solution, as the
// reference's sol), and WT_after_step of the stage state.  The trends run over
// the levels' work lists (needed-node maps); the first three stages' inverse
// transforms rebuild the parents the next stage reads, the last one every
// parent.
int rk4_split_explicit(wt_handle* h, double dt, double theta1) {
  MLCtx* M = static_cast<MLCtx*>(h->ml);
  const States q = hierarchy_state(h);
  States q1;
  for (auto& V : M->L) {
    q1.m.push_back(V.m1);
    q1.t.push_back(V.t1);
    q1.v.push_back(V.v1);
  }
  const double hs[4] = {dt / 4.0, dt / 3.0, dt / 2.0, dt};
  std::vector<const double*> grad(M->L.size(), nullptr);
  for (int stage = 0; stage < 4; ++stage) {
    const States& src = stage == 0 ? q : q1;
    const States& dest = stage == 3 ? q : q1;
    if (int rc = wt_level_barotropic_correction(h, src.m.data(), src.t.data())) return rc;
    if (int rc = wt_level_grad_eta(h, grad.data())) return rc;
    wt_level_wav_bind(h, dest.m.data(), dest.t.data(), dest.v.data());
    wt_level_clean_wavelets(h);
    int rc = trend_multi(h, src, nullptr, &q, &dest, hs[stage], true, false, grad.data(), theta1);
    // the intermediate stages' inverse rebuilds the parents the next stage reads; the last stage's every one
    // (free_surface_update reads the whole state)
    if (!rc) rc = wt_level_wav_finish(h, stage < 3);
    wt_level_wav_unbind(h);
    if (rc) return rc;
  }
  return WT_OK;
}
}  // namespace

extern "C" {

// The explicit part of RK4_split over the hierarchy (RK_split four times: see
// rk4_split_explicit); the host then takes free_surface_update (eta_update,
// barotropic_correction, u_update, WT_after_step).  Uses each level's free
// surface (wt_barotropic_upload_level) and the masks as they are.
int wt_rk4_split_explicit(wt_handle* h, double dt, double theta1) {
  if (!h) return WT_ERR_ARG;
  if (!h->wav || h->flux_bits != 64) return WT_ERR_STATE;  // the hierarchy's steps are FP64 only
  if (int rc = ensure(h)) return rc;
  if (int rc = rk4_split_explicit(h, dt, theta1)) return rc;
  CKM(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

// RK4 (src/time_integr.f90:78-103) over the hierarchy: each stage evaluates
// trend_ml on every level, takes the RK sub-step on every level and runs
// WT_after_step on the new stage state, with the masks held fixed.
int wt_rk4_multi(wt_handle* h, double dt, int nsteps) {
  if (!h || nsteps < 0) return WT_ERR_ARG;
  if (!h->wav || h->flux_bits != 64) return WT_ERR_STATE;  // the hierarchy's steps are FP64 only
  if (int rc = ensure(h)) return rc;
  if (int rc = rk4_multi(h, dt, nsteps, nullptr)) return rc;
  CKM(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

// One adaptive time step of the fully refined hierarchy, as the reference's
// time_step (src/main.f90:405-444) with fixed thresholds: RK4 of the hierarchy
// (trend_ml, RK_sub_step, WT_after_step per stage), adapt's mask sequence and
// compression, and the inverse wavelet transform.  The ~280 launches of a step
// are captured once into a CUDA graph (re-captured when dt, level_fill or
// max_level change) and replayed; the thresholds are uploaded before each call.
int wt_adaptive_step(wt_handle* h, double dt, const double* threshold, int level_fill, int max_level, int nsteps) {
  if (!h || !threshold || nsteps < 0) return WT_ERR_ARG;
  if (!h->wav || h->flux_bits != 64) return WT_ERR_STATE;  // the hierarchy's steps are FP64 only
  if (int rc = ensure(h)) return rc;
  MLCtx* M = static_cast<MLCtx*>(h->ml);
  for (int l = h->level_start; l <= h->level_end; ++l) {  // allocate before any capture
    double* p;
    if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_MASS, &p)) return rc;
    if (int rc = wt_level_mean(h, l, WT_FIELD_MEAN_TEMP, &p)) return rc;
  }
  if (int rc = wt_level_set_thresholds(h, threshold)) return rc;
  wt_level_clean_wavelets(h);  // outside the graph, which assumes clean wavelet arrays
  // and wavelets compressed under the current masks: the graph's first stage
  // writes only the kept slots (the wavelets on entry are not read otherwise)
  if (!wt_level_zero_ok(h)) wt_level_compress(h);
  if (int rc = wt_level_need_refresh(h)) return rc;  // likewise a current needed-node map
  if (int rc = wt_level_mask_snapshot_alloc(h)) return rc;
  if (!M->step_graph || M->g_dt != dt || M->g_fill != level_fill || M->g_max != max_level ||
      M->g_epoch != wt_level_skip_epoch(h)) {
    if (M->step_graph) {
      cudaGraphExecDestroy(M->step_graph);
      M->step_graph = nullptr;
    }
    cudaGraph_t g;
    CKM(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    // adapt reads wavelets and masks only, and the inverse transform after it
    // rebuilds every level above level_start: the last stage's own inverse is
    // left out
    // the last stage's WT_after_step leaves the wavelets compressed under the
    // masks of this step, so compress_wavelets under the new masks only has to
    // zero the slots the new masks drop (the masks are kept before adapt)
    int rc = rk4_multi(h, dt, 1, nullptr, false);
    if (!rc) {
      wt_level_mask_snapshot(h);
      rc = wt_level_mask_sequence(h, level_fill, max_level, 0, nullptr);
    }
    if (!rc) {
      wt_level_compress_delta(h);
      wt_level_inverse(h);
    }
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return wt_handle_fail("capture", e);
    // the nodes keep the priorities of the streams they were captured from
    e = cudaGraphInstantiate(&M->step_graph, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return wt_handle_fail("instantiate", e);
    M->g_dt = dt;
    M->g_fill = level_fill;
    M->g_max = max_level;
    M->g_epoch = wt_level_skip_epoch(h);
  }
  for (int s = 0; s < nsteps; ++s) CKM(cudaGraphLaunch(M->step_graph, h->stream));
  CKM(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

// wt_rk4_multi with CUDA events around its phases: ms[p] = mean time of one
// occurrence of phase p (0 column+step1 of level_end, 1 column+step1 of one
// coarser level, 2 restrictions into one level, 3 k_trend_ml of level_end with
// the fused RK sub-step, 4 the same on one coarser level, 5 unused (the RK
// sub-step is fused), 6 WT_after_step); count[p] = occurrences per step.
int wt_profile_rk4_multi(wt_handle* h, double dt, int nsteps, double* ms, int* count) {
  if (!h || nsteps < 1 || !ms || !count) return WT_ERR_ARG;
  if (!h->wav || h->flux_bits != 64) return WT_ERR_STATE;  // the hierarchy's steps are FP64 only
  if (int rc = ensure(h)) return rc;
  PhaseTimer tm{h->stream, {}, {}};
  if (int rc = rk4_multi(h, dt, nsteps, &tm)) return rc;
  CKM(cudaStreamSynchronize(h->stream));
  double tot[NPH] = {0};
  int cnt[NPH] = {0};
  for (size_t q = 0; q < tm.ids.size(); ++q) {
    float t = 0.f;
    CKM(cudaEventElapsedTime(&t, tm.ev[2 * q], tm.ev[2 * q + 1]));
    tot[tm.ids[q]] += t;
    cnt[tm.ids[q]] += 1;
  }
  for (int p = 0; p < NPH; ++p) {
    ms[p] = cnt[p] ? tot[p] / cnt[p] : 0.0;
    count[p] = cnt[p] / nsteps;
  }
  h->state_halo_done = false;
  return WT_OK;
}

int wt_download_trend_level(wt_handle* h, int level, double* dmass, double* dtemp, double* dvelo) {
  if (!h || level < h->level_start || level > h->level_end) return WT_ERR_ARG;
  if (!h->ml) return WT_ERR_STATE;
  MLLevel& V = static_cast<MLCtx*>(h->ml)->L[level - h->level_start];
  const size_t nn = (size_t)h->nz * h->at(level).NN;
  if (dmass) CKM(cudaMemcpyAsync(dmass, V.dm, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  if (dtemp) CKM(cudaMemcpyAsync(dtemp, V.dt, nn * 8, cudaMemcpyDeviceToHost, h->stream));
  if (dvelo) CKM(cudaMemcpyAsync(dvelo, V.dv, 3 * nn * 8, cudaMemcpyDeviceToHost, h->stream));
  CKM(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"
