// C-ABI of the wavelet transforms, threshold mask and compression of the
// prognostic variables on the handle's uniform hierarchy.  The launch order of
// each entry point follows the reference driver named in its comment; ghost
// copies (update_bdry) are replaced by the kernels' remapped reads.
#include <cuda_runtime.h>

#include <algorithm>
#include <initializer_list>
#include <cstdio>
#include <vector>

#include "../../include/wavetrisk_gpu.h"
#include "restrict_kernels.cuh"
#include "wavelet_kernels.cuh"
#include "wavelet_layers.cuh"
#include "need_map.cuh"
#include "tree_kernels.cuh"
#include "wt_handle.cuh"
#include "wt_wavctx.cuh"

using namespace wtw;

namespace {

constexpr int TPB = 256;
inline unsigned nb(int64_t n) { return (unsigned)((n + TPB - 1) / TPB); }
constexpr int TPBL = 128;  // the layer-group kernels (wavelet_layers.cuh)
int g_lpt_set = 0;         // layers per thread of those kernels (wt_tune); 0: by layer count
// Measured on B200 (J5..J7 x 16 and J6..J8 x 32): 2 layers per thread up to
// 16 layers, 4 beyond.
inline int lpt_for(int nz) { return g_lpt_set > 0 ? g_lpt_set : (nz > 16 ? 4 : 2); }
// blocks for n parents per layer group
inline unsigned nbl(int64_t n, int nz) {
  const int lpt = lpt_for(nz);
  return (unsigned)((n * ((nz + lpt - 1) / lpt) + TPBL - 1) / TPBL);
}

int fail(const char* where, cudaError_t e) { return wt_handle_fail(where, e); }

// Grid of a persistent kernel over a work list: the blocks of `threads`
// threads the device keeps resident at once, at most `dense`.
template <class K>
unsigned pgrid(K kernel, int threads, unsigned dense) {
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0) != cudaSuccess || per < 1)
    return dense;
  const unsigned g = (unsigned)sms * (unsigned)per;
  return g < dense ? g : dense;
}
const ParentList kNoList{nullptr, nullptr};

// Blocks of LIST_B candidates of the largest level (the list compaction's scratch).
size_t mx_nn_blocks(wt_handle* h) {
  size_t mx = 0;
  for (int l = h->level_start; l <= h->level_end; ++l) mx = std::max(mx, (size_t)h->at(l).NN);
  return (mx + LIST_B - 1) / LIST_B;
}

// An ascending work list of the candidates c into ids, its count into *count
// (stream-ordered; scratch: the context's block counts and offsets).
template <class Cand>
void build_list(wt_handle* h, const Cand& c, int n, int* ids, int* count) {
  WavCtx* W = ctx(h);
  const int nb = (n + LIST_B - 1) / LIST_B;
  int* bcnt = W->lscr;
  int* boff = W->lscr + W->lscr_n / 2;
  cudaStream_t s = h->stream;
  k_list_count<<<nb, LIST_B, 0, s>>>(c, bcnt);
  k_list_scan<<<1, LIST_B, 0, s>>>(nb, bcnt, boff, count);
  k_list_write<<<nb, LIST_B, 0, s>>>(c, boff, ids);
}

#define CKW(x)                                  \
  do {                                          \
    cudaError_t e_ = (x);                       \
    if (e_ != cudaSuccess) return fail(#x, e_); \
  } while (0)

int ready(wt_handle* h) {
  if (!h) return WT_ERR_ARG;
  if (!h->wav) return WT_ERR_STATE;
  return WT_OK;
}

// The work field `field` (WT_WORK_*) of level l, allocated and zeroed on first use.
int work_field(wt_handle* h, int l, int field, double** out, size_t* bytes) {
  WavLevel& V = ctx(h)->L[l - h->level_start];
  const size_t nn = (size_t)h->nz * h->at(l).NN;
  double** slot = field == WT_WORK_SCALAR ? &V.scal : field == WT_WORK_DSCALAR ? &V.dscal
                : field == WT_WORK_FLUX ? &V.flux : &V.dvelo;
  const size_t n = (field == WT_WORK_FLUX || field == WT_WORK_DVELO) ? 3 * nn : nn;
  if (!*slot) {
    CKW(ctx(h)->alloc(slot, n));
    CKW(cudaMemsetAsync(*slot, 0, n * 8, h->stream));
  }
  *out = *slot;
  if (bytes) *bytes = n * 8;
  return WT_OK;
}

}  // namespace

// The layer mean of mass or Theta (WT_FIELD_MEAN_*) of level l: the stepper's
// on level_end, allocated (zero) on first use below it.
int wt_level_mean(wt_handle* h, int l, int field, double** out) {
  if (l == h->level_end) {
    *out = field == WT_FIELD_MEAN_MASS ? h->mean_m : h->mean_t;
    return WT_OK;
  }
  WavLevel& V = ctx(h)->L[l - h->level_start];
  double** slot = field == WT_FIELD_MEAN_MASS ? &V.mean_m : &V.mean_t;
  const size_t n = (size_t)h->nz * h->at(l).NN;
  if (!*slot) {
    CKW(ctx(h)->alloc(slot, n));
    CKW(cudaMemsetAsync(*slot, 0, n * 8, h->stream));
  }
  *out = *slot;
  return WT_OK;
}

void wt_level_masks(wt_handle* h, int l, const int** mask_n, const int** mask_e) {
  if (!h->wav) { *mask_n = *mask_e = nullptr; return; }
  WavLevel& V = ctx(h)->L[l - h->level_start];
  *mask_n = V.mask_n;
  *mask_e = V.mask_e;
}

void wt_level_state(wt_handle* h, int l, double** m, double** t, double** v) {
  WavLevel& V = ctx(h)->L[l - h->level_start];
  *m = V.sm;
  *t = V.st;
  *v = V.sv;
}

namespace {

void zero_wavelets(wt_handle* h) {
  for (int l = h->level_start; l <= h->level_end; ++l) {
    const DevLevel& D = h->at(l);
    WavLevel& W = ctx(h)->L[l - h->level_start];
    const size_t nn = (size_t)h->nz * D.NN * sizeof(double);
    cudaMemsetAsync(W.wm, 0, nn, h->stream);
    cudaMemsetAsync(W.wt, 0, nn, h->stream);
    cudaMemsetAsync(W.wv, 0, 3 * nn, h->stream);
  }
}

}  // namespace
ParentList wt_level_plist(wt_handle* h, int level);
namespace {

// Scalar wavelets of level l+1 (Compute_scalar_wavelets over parents [0, n_l)).
// With CMP 2 (only the kept slots written) and a parent work list, the listed
// parents only, persistent threads.
template <int CMP>
void launch_scalar_wc(wt_handle* h, int l, cudaStream_t s) {
  const int np = h->at(l).n, nz = h->nz;
  const ParentList PL = CMP == 2 ? wt_level_plist(h, l) : kNoList;
  const unsigned dense = nbl((int64_t)10 * np * np, nz);
  k_scalar_wc_l<CMP><<<PL.ids ? pgrid(k_scalar_wc_l<CMP>, TPBL, dense) : dense, TPBL, 0, s>>>(view(h, l + 1), np, nz,
                                                                                             lpt_for(nz), PL);
}

// Blocks of 32 plan rows by min(nz, 8) layer threads (the plan kernels).
inline dim3 plan_block(int nz) { return dim3(32, std::min(nz, 8)); }
inline unsigned plan_grid(int64_t rows) { return (unsigned)((rows + 31) / 32); }
// Velocity wavelets of level l+1 (pentagon corrections included): outer edges
// on s, inner edges on si (they read only the scaling fields).
template <int CMP>
void launch_velo_wc(wt_handle* h, int l, cudaStream_t s, cudaStream_t si) {
  const int np = h->at(l).n, nz = h->nz;
  const unsigned g = nbl((int64_t)10 * np * np, nz);
  const ParentList PL = CMP == 2 ? wt_level_plist(h, l) : kNoList;
  k_velo_wc_outer_l<CMP><<<PL.ids ? pgrid(k_velo_wc_outer_l<CMP>, TPBL, g) : g, TPBL, 0, s>>>(
      view(h, l), view(h, l + 1), nz, lpt_for(nz), PL);
  k_velo_wc_inner_l<CMP><<<PL.ids ? pgrid(k_velo_wc_inner_l<CMP>, TPBL, g) : g, TPBL, 0, si>>>(
      view(h, l), view(h, l + 1), nz, lpt_for(nz), PL);
}

// inverse_wavelet_transform (src/wavelet.f90:208-296) from level_start.  The
// scalars and the velocity reconstruct independently of each other, so the
// scalar chain (Prolong_scalar, Reconstruct_scalar per level) runs on a side
// stream beside the velocity chain (outer, then inner edges per level).
// partial 0: every parent; 1: those of wt_level_rec (an intermediate RK
// stage); 2: those of wt_level_rec_final (after adapt, with a patch tree)
void inverse(wt_handle* h, int partial = 0) {
  const int nz = h->nz;
  WavCtx* W = ctx(h);
  cudaStream_t s = h->stream, sa = W->side[0];
  cudaEventRecord(W->ev[0], s);
  cudaStreamWaitEvent(sa, W->ev[0], 0);
  cudaEventRecord(W->ready_v[0], s);  // level_start is not rebuilt
  for (int l = h->level_start; l <= h->level_end - 1; ++l) {
    const int np = h->at(l).n, q = l + 1 - h->level_start;
    const WLev P = view(h, l), C = view(h, l + 1);
    const int64_t par1 = (int64_t)10 * (np + 1) * (np + 1), par0 = (int64_t)10 * np * np;
    const unsigned char* rec = partial == 1 ? wt_level_rec(h, l) : partial == 2 ? wt_level_rec_final(h, l) : nullptr;
    // a partial rebuild over the parent work list (its parents include every rebuilt one)
    const ParentList PL = rec ? wt_level_plist(h, l) : kNoList;
    const dim3 pb = plan_block(nz);
    const int pt = (int)(pb.x * pb.y);
    k_prolong_l<<<PL.ids ? pgrid(k_prolong_l, TPBL, nbl(par1, nz)) : nbl(par1, nz), TPBL, 0, sa>>>(P, C, nz, lpt_for(nz),
                                                                                                  rec, PL);
    k_recon_scalar_l<<<PL.ids ? pgrid(k_recon_scalar_l, TPBL, nbl(par0, nz)) : nbl(par0, nz), TPBL, 0, sa>>>(
        P, C, np, nz, lpt_for(nz), rec, PL);
    cudaEventRecord(W->ready_s[q], sa);
    const WavLevel& V = W->L[l - h->level_start];
    k_recon_outer_p<<<PL.ids ? pgrid(k_recon_outer_p, pt, plan_grid(par1)) : plan_grid(par1), pb, 0, s>>>(
        P, C, nz, V.op_i, V.op_d, rec, PL);
    k_recon_inner_p<<<PL.ids ? pgrid(k_recon_inner_p, pt, plan_grid(par0)) : plan_grid(par0), pb, 0, s>>>(
        P, C, nz, V.ip_i, V.ip_d, rec, PL);
    cudaEventRecord(W->ready_v[q], s);
  }
  cudaEventRecord(W->ev[1], sa);
  cudaStreamWaitEvent(s, W->ev[1], 0);
}

void compress(wt_handle* h) {
  const int nz = h->nz;
  for (int l = h->level_start + 1; l <= h->level_end; ++l) {
    const int n = h->at(l).n;
    k_compress<<<nb((int64_t)nz * 10 * (n + 1) * (n + 1)), TPB, 0, h->stream>>>(view(h, l), nz);
  }
  ctx(h)->zero_ok = true;
}

}  // namespace

// WT_after_step's scaling fields: m[q], t[q], v[q] of level level_start+q
// replace the hierarchy's own until wt_level_wav_unbind.  Launches read the
// pointers when they are made.
void wt_level_wav_bind(wt_handle* h, double* const* m, double* const* t, double* const* v) {
  WavCtx* W = ctx(h);
  W->bound_saved = W->L;
  for (size_t q = 0; q < W->L.size(); ++q) {
    W->L[q].sm = m[q];
    W->L[q].st = t[q];
    W->L[q].sv = v[q];
  }
}
void wt_level_wav_unbind(wt_handle* h) {
  WavCtx* W = ctx(h);
  for (size_t q = 0; q < W->L.size(); ++q) {
    W->L[q].sm = W->bound_saved[q].sm;
    W->L[q].st = W->bound_saved[q].st;
    W->L[q].sv = W->bound_saved[q].sv;
  }
}

// The wavelets of level l+1 from the scaling fields of levels l and l+1, with
// zero_float and compress_wavelets folded in (CMP), once both levels' fields
// are written on the handle's stream: the scalar, inner and outer velocity
// wavelets run on three side streams forked here.  The arrays must be clean
// (wt_level_clean_wavelets) before the first pair of a WT_after_step.
int wt_level_wav_forward_pair(wt_handle* h, int l) {
  WavCtx* W = ctx(h);
  cudaEvent_t f = W->fork[l - h->level_start];
  CKW(cudaEventRecord(f, h->stream));
  for (int k = 1; k < 4; ++k) CKW(cudaStreamWaitEvent(W->side[k], f, 0));
  if (W->zero_ok) {
    launch_scalar_wc<2>(h, l, W->side[3]);
    launch_velo_wc<2>(h, l, W->side[2], W->side[1]);
  } else {
    launch_scalar_wc<1>(h, l, W->side[3]);
    launch_velo_wc<1>(h, l, W->side[2], W->side[1]);
  }
  CKW(cudaGetLastError());
  return WT_OK;
}

// The end of WT_after_step once every level pair's forward wavelets are
// launched: join the side streams, then the inverse transform.
int wt_level_wav_finish(wt_handle* h, int mode, bool rebuild) {
  WavCtx* W = ctx(h);
  for (int k = 1; k < 4; ++k) {
    CKW(cudaEventRecord(W->ev[1 + k], W->side[k]));
    CKW(cudaStreamWaitEvent(h->stream, W->ev[1 + k], 0));
  }
  W->zero_ok = true;  // every level pair's forward wavelets are launched
  if (rebuild) inverse(h, mode);
  CKW(cudaGetLastError());
  return WT_OK;
}

// WT_after_step (src/adapt.f90:192-237) on the scaling fields m[q], t[q], v[q]
// of level level_start+q (the hierarchy's own scaling fields when the arrays
// are null).
int wt_level_after_step(wt_handle* h, double* const* m, double* const* t, double* const* v, int mode) {
  if (m) wt_level_wav_bind(h, m, t, v);
  wt_level_clean_wavelets(h);
  int rc = WT_OK;
  for (int l = h->level_start; l <= h->level_end - 1 && !rc; ++l) rc = wt_level_wav_forward_pair(h, l);
  if (!rc) rc = wt_level_wav_finish(h, mode);
  if (m) wt_level_wav_unbind(h);
  return rc;
}

void wt_wavelet_release(wt_handle* h) {
  if (!h || !h->wav) return;
  for (cudaEvent_t e : ctx(h)->ev)
    if (e) cudaEventDestroy(e);
  for (auto* v : {&ctx(h)->fork, &ctx(h)->ready_v, &ctx(h)->ready_s})
    for (cudaEvent_t e : *v)
      if (e) cudaEventDestroy(e);
  for (cudaStream_t s : ctx(h)->side)
    if (s) cudaStreamDestroy(s);
  for (void* p : ctx(h)->allocs) cudaFree(p);
  delete ctx(h);
  h->wav = nullptr;
}

extern "C" {

int wt_wavelet_setup(wt_handle* h) {
  if (!h || h->lev.empty()) return WT_ERR_ARG;
  for (int l = h->level_start + 1; l <= h->level_end; ++l)
    if (!h->at(l).iu_wgt) return WT_ERR_ARG;
  wt_wavelet_release(h);
  WavCtx* W = new WavCtx();
  h->wav = W;
  const int nz = h->nz;
  W->L.resize(h->level_end - h->level_start + 1);
  for (int l = h->level_start; l <= h->level_end; ++l) {
    const DevLevel& D = h->at(l);
    WavLevel& V = W->L[l - h->level_start];
    const size_t nn = (size_t)nz * D.NN;
    if (l == h->level_end) {
      V.sm = h->mass;
      V.st = h->temp;
      V.sv = h->velo;
    } else {
      V.own_scaling = true;
      CKW(W->alloc(&V.sm, nn));
      CKW(W->alloc(&V.st, nn));
      CKW(W->alloc(&V.sv, 3 * nn));
      CKW(cudaMemsetAsync(V.sm, 0, nn * 8, h->stream));
      CKW(cudaMemsetAsync(V.st, 0, nn * 8, h->stream));
      CKW(cudaMemsetAsync(V.sv, 0, 3 * nn * 8, h->stream));
    }
    CKW(W->alloc(&V.wm, nn));
    CKW(W->alloc(&V.wt, nn));
    CKW(W->alloc(&V.wv, 3 * nn));
    CKW(W->alloc(&V.mask_n, (size_t)D.NN));
    CKW(W->alloc(&V.mask_e, (size_t)3 * D.NN));
    std::vector<int> tol(3 * D.NN, WT_MASK_TOLRNZ);
    CKW(cudaMemcpy(V.mask_n, tol.data(), D.NN * sizeof(int), cudaMemcpyHostToDevice));
    CKW(cudaMemcpy(V.mask_e, tol.data(), 3 * D.NN * sizeof(int), cudaMemcpyHostToDevice));
  }
  CKW(W->alloc(&W->thr, (size_t)3 * nz));
  // needed-node maps of the levels above level_start and their dilation scratch
  if (h->level_end > h->level_start && h->level_end - h->level_start < NEED_MAXL) {
    size_t tot = 0;
    W->need_off.assign(W->L.size(), 0);
    for (int l = h->level_start + 1; l <= h->level_end; ++l) {
      W->need_off[l - h->level_start] = tot;
      tot += (size_t)h->at(l).NN;
    }
    CKW(W->alloc(&W->need[0], tot));
    CKW(W->alloc(&W->need[1], tot));
    CKW(W->alloc(&W->list, tot));
    CKW(W->alloc(&W->list_cnt, W->L.size()));
    W->lscr_n = 2 * (mx_nn_blocks(h) + 1);
    CKW(W->alloc(&W->lscr, W->lscr_n));
    size_t ptot = 0, mx = 0;
    W->rec_off.assign(W->L.size(), 0);
    for (int l = h->level_start; l <= h->level_end; ++l) {
      if (l < h->level_end) {
        W->rec_off[l - h->level_start] = ptot;
        ptot += (size_t)h->at(l).NN;
      }
      mx = std::max(mx, (size_t)h->at(l).NN);
    }
    CKW(W->alloc(&W->recpar, ptot));
    W->rec_tot = ptot;
    CKW(W->alloc(&W->rscr[0], mx));
    CKW(W->alloc(&W->rscr[1], mx));
  }
  // velocity-wavelet plans of every parent level
  for (int l = h->level_start; l < h->level_end; ++l) {
    WavLevel& V = W->L[l - h->level_start];
    const int m = h->at(l).n;
    const int64_t n1 = (int64_t)10 * (m + 1) * (m + 1), n0 = (int64_t)10 * m * m;
    CKW(W->alloc(&V.op_i, (size_t)OP_NI * n1));
    CKW(W->alloc(&V.op_d, (size_t)OP_ND * n1));
    CKW(W->alloc(&V.ip_i, (size_t)IP_NI * n0));
    CKW(W->alloc(&V.ip_d, (size_t)IP_ND * n0));
    k_outer_plan<<<nb(n1), TPB, 0, h->stream>>>(view(h, l), view(h, l + 1), V.op_i, V.op_d);
    k_inner_plan<<<nb(n0), TPB, 0, h->stream>>>(view(h, l), view(h, l + 1), V.ip_i, V.ip_d);
    CKW(cudaGetLastError());
  }
  // flux-restriction plans of every parent level whose child has R_F_wgt
  for (int l = h->level_start; l < h->level_end; ++l) {
    const DevLevel& Dc = h->at(l + 1);
    if (!Dc.rf_wgt || !Dc.overl_split) continue;
    WavLevel& V = W->L[l - h->level_start];
    const int m = h->at(l).n;
    const int64_t ne = (int64_t)3 * 10 * m * m;
    CKW(W->alloc(&V.rf_pi, (size_t)RF_NI * ne));
    CKW(W->alloc(&V.rf_pd, (size_t)RF_ND * ne));
    k_rf_plan<<<nb(ne), TPB, 0, h->stream>>>(view(h, l), view(h, l + 1), V.rf_pi, V.rf_pd);
    CKW(cudaGetLastError());
  }
  int least = 0, greatest = 0;
  CKW(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  CKW(cudaStreamCreateWithPriority(&W->side[0], cudaStreamNonBlocking, greatest));
  for (int k = 1; k < 4; ++k) CKW(cudaStreamCreateWithPriority(&W->side[k], cudaStreamNonBlocking, least));
  for (cudaEvent_t& e : W->ev) CKW(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  W->fork.assign(W->L.size(), nullptr);
  W->ready_v.assign(W->L.size(), nullptr);
  W->ready_s.assign(W->L.size(), nullptr);
  for (auto* v : {&W->fork, &W->ready_v, &W->ready_s})
    for (cudaEvent_t& e : *v) CKW(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  zero_wavelets(h);
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"

namespace {

bool field_ok(wt_handle* h, int level, int field) {
  return level >= h->level_start && level <= h->level_end && field >= 0 && field <= WT_FIELD_MEAN_TEMP;
}

// Queue the host-to-device copy of one field of one level (no synchronisation).
int enqueue_upload(wt_handle* h, int level, int field, const void* src) {
  if (field >= WT_FIELD_MEAN_MASS) {
    double* p;
    if (int rc = wt_level_mean(h, level, field, &p)) return rc;
    CKW(cudaMemcpyAsync(p, src, (size_t)h->nz * h->at(level).NN * 8, cudaMemcpyHostToDevice, h->stream));
    return WT_OK;
  }
  if (field >= WT_WORK_SCALAR) {
    double* p;
    size_t bytes;
    if (int rc = work_field(h, level, field, &p, &bytes)) return rc;
    CKW(cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, h->stream));
    return WT_OK;
  }
  const DevLevel& D = h->at(level);
  WavLevel& V = ctx(h)->L[level - h->level_start];
  const size_t nn = (size_t)h->nz * D.NN;
  void* dst[8] = {V.sm, V.st, V.sv, V.wm, V.wt, V.wv, V.mask_n, V.mask_e};
  const size_t bytes[8] = {nn * 8, nn * 8, 3 * nn * 8, nn * 8, nn * 8, 3 * nn * 8, (size_t)D.NN * 4, (size_t)3 * D.NN * 4};
  CKW(cudaMemcpyAsync(dst[field], src, bytes[field], cudaMemcpyHostToDevice, h->stream));
  if (level == h->level_end && field <= WT_FIELD_VELO) h->state_halo_done = false;
  if (field >= WT_WAVE_MASS && field <= WT_WAVE_VELO) ctx(h)->wav_dirty = true;
  if (field == WT_MASK_NODE || field == WT_MASK_EDGE) ctx(h)->need_ok = false;
  if (field >= WT_WAVE_MASS && field <= WT_MASK_EDGE) ctx(h)->zero_ok = false;
  return WT_OK;
}

// Queue the ghost copy of level's scaling (wav false) or wavelet fields.
int enqueue_halo(wt_handle* h, int level, bool wav) {
  const DevLevel& D = h->at(level);
  WavLevel& V = ctx(h)->L[level - h->level_start];
  const int64_t nt = (int64_t)(2 * D.n_hn + D.n_he) * h->nz;
  k_halo_level<<<nb(nt), TPB, 0, h->stream>>>(h->nz, (int)D.NN, D.hn, D.n_hn, D.he, D.n_he, wav ? V.wm : V.sm,
                                               wav ? V.wt : V.st, wav ? V.wv : V.sv);
  CKW(cudaGetLastError());
  return WT_OK;
}

// Queue the device-to-host copy of one field of one level (ghosts as they are).
int enqueue_download(wt_handle* h, int level, int field, void* dst) {
  if (field >= WT_FIELD_MEAN_MASS) {
    double* p;
    if (int rc = wt_level_mean(h, level, field, &p)) return rc;
    CKW(cudaMemcpyAsync(dst, p, (size_t)h->nz * h->at(level).NN * 8, cudaMemcpyDeviceToHost, h->stream));
    return WT_OK;
  }
  if (field >= WT_WORK_SCALAR) {
    double* p;
    size_t bytes;
    if (int rc = work_field(h, level, field, &p, &bytes)) return rc;
    CKW(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyDeviceToHost, h->stream));
    return WT_OK;
  }
  const DevLevel& D = h->at(level);
  WavLevel& V = ctx(h)->L[level - h->level_start];
  const size_t nn = (size_t)h->nz * D.NN;
  const void* src[8] = {V.sm, V.st, V.sv, V.wm, V.wt, V.wv, V.mask_n, V.mask_e};
  const size_t bytes[8] = {nn * 8, nn * 8, 3 * nn * 8, nn * 8, nn * 8, 3 * nn * 8, (size_t)D.NN * 4, (size_t)3 * D.NN * 4};
  CKW(cudaMemcpyAsync(dst, src[field], bytes[field], cudaMemcpyDeviceToHost, h->stream));
  return WT_OK;
}

}  // namespace

extern "C" {

int wt_upload_field(wt_handle* h, int level, int field, const void* src) {
  if (int rc = ready(h)) return rc;
  if (!src || !field_ok(h, level, field)) return WT_ERR_ARG;
  if (int rc = enqueue_upload(h, level, field, src)) return rc;
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_download_field(wt_handle* h, int level, int field, void* dst) {
  if (int rc = ready(h)) return rc;
  if (!dst || !field_ok(h, level, field)) return WT_ERR_ARG;
  if (field <= WT_WAVE_VELO)
    if (int rc = enqueue_halo(h, level, field >= WT_WAVE_MASS)) return rc;
  if (int rc = enqueue_download(h, level, field, dst)) return rc;
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_upload_fields(wt_handle* h, int n, const int* levels, const int* fields, const void* const* src) {
  if (int rc = ready(h)) return rc;
  if (n < 0 || (n > 0 && (!levels || !fields || !src))) return WT_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (!src[i] || !field_ok(h, levels[i], fields[i])) return WT_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (int rc = enqueue_upload(h, levels[i], fields[i], src[i])) return rc;
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_download_fields(wt_handle* h, int n, const int* levels, const int* fields, void* const* dst) {
  if (int rc = ready(h)) return rc;
  if (n < 0 || (n > 0 && (!levels || !fields || !dst))) return WT_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (!dst[i] || !field_ok(h, levels[i], fields[i])) return WT_ERR_ARG;
  std::vector<char> done(2 * (h->level_end - h->level_start + 1), 0);  // ghost copy per (level, kind)
  for (int i = 0; i < n; ++i)
    if (fields[i] <= WT_WAVE_VELO) {
      const int k = 2 * (levels[i] - h->level_start) + (fields[i] >= WT_WAVE_MASS ? 1 : 0);
      if (!done[k]) {
        done[k] = 1;
        if (int rc = enqueue_halo(h, levels[i], fields[i] >= WT_WAVE_MASS)) return rc;
      }
    }
  for (int i = 0; i < n; ++i)
    if (int rc = enqueue_download(h, levels[i], fields[i], dst[i])) return rc;
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

// forward_wavelet_transform (src/wavelet.f90:20-98) with jmin_in = level_start+1.
int wt_forward_wt(wt_handle* h) {
  if (int rc = ready(h)) return rc;
  const int nz = h->nz;
  zero_wavelets(h);
  ctx(h)->wav_dirty = false;
  ctx(h)->zero_ok = false;  // the forward transform keeps what compress_wavelets would zero
  for (int l = h->level_end - 1; l >= h->level_start; --l) {
    const int np = h->at(l).n;
    launch_scalar_wc<0>(h, l, h->stream);
    k_restrict<<<nb((int64_t)nz * 10 * (np + 1) * (np + 1)), TPB, 0, h->stream>>>(view(h, l), view(h, l + 1), nz);
  }
  for (int l = h->level_end - 1; l >= h->level_start; --l) launch_velo_wc<0>(h, l, h->stream, h->stream);
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_inverse_wt(wt_handle* h) {
  if (int rc = ready(h)) return rc;
  inverse(h);
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"

namespace {
void comm_masks(wt_handle* h) {
  MaskHaloSet S{};
  S.nl = h->level_end - h->level_start + 1;
  for (int q = 0; q < S.nl; ++q) {
    const DevLevel& D = h->at(h->level_start + q);
    const WavLevel& V = ctx(h)->L[q];
    S.n_hn[q] = D.n_hn;
    S.mask_n[q] = V.mask_n;
    S.mask_e[q] = V.mask_e;
    S.hn[q] = D.hn;
    S.he[q] = D.he;
    S.start[q + 1] = S.start[q] + D.n_hn + D.n_he;
  }
  k_mask_halo_all<<<nb(S.start[S.nl]), TPB, 0, h->stream>>>(S);
}
// mask_tol_vars of level l on nodes [st, n-1+en]^2
void mask_tol(wt_handle* h, int l, int st, int en, int level_fill) {
  const int m = h->at(l).n + en - st;
  const dim3 blk(32, std::min(h->nz, 8));
  WavCtx* W = ctx(h);
  // with a patch tree, the nodes outside it are left out (levels above level_start)
  const unsigned char* ex = (W->tree_ps > 0 && l > h->level_start) ? W->tree + W->tree_off[l - h->level_start] : nullptr;
  k_mask_tol_y<<<(unsigned)(((int64_t)10 * m * m + 31) / 32), blk, 0, h->stream>>>(view(h, l), h->nz, st, en, W->thr,
                                                                                     l < level_fill ? 1 : 0, ex,
                                                                                     W->tree_ps);
}
inline unsigned nodes_blocks(int m) { return nb((int64_t)10 * m * m); }
}  // namespace

extern "C" {

int wt_mask_tol_vars(wt_handle* h, const double* threshold, int level_fill) {
  if (int rc = ready(h)) return rc;
  if (!threshold) return WT_ERR_ARG;
  const int nz = h->nz;
  WavCtx* W = ctx(h);
  CKW(cudaMemcpyAsync(W->thr, threshold, 3 * nz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  for (int l = h->level_end; l >= h->level_start; --l) {
    const int st = (l == h->level_end) ? 0 : -1, en = (l == h->level_end) ? 1 : 2;
    mask_tol(h, l, st, en, level_fill);
  }
  W->zero_ok = false;
  W->need_ok = false;
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}


// adapt (src/adapt.f90:14-65) without tree surgery, on the dense hierarchy.
}  // extern "C"

// adapt's mask sequence (src/adapt.f90:14-65) up to refine(), stream-ordered
// and without host synchronisation (capturable), on levels level_start .. le:
// init_masks_zero, mask_active (le is level_end: nodes [0, n] there, [-1, n+1]
// below), mask_adj_same_scale and mask_restrict_same_scale; then, with dreq
// non-null, check_child_required of the parent levels level_start .. req_hi
// into dreq (patch_size > 0).  The thresholds are already in the context's
// device buffer.  Levels above le are the tree's missing levels: their masks
// stay ZERO.
static int mask_phase1(wt_handle* h, int level_fill, int max_level, int patch_size, unsigned char* dreq, int le,
                int req_hi) {
  const int ls = h->level_start;
  cudaStream_t s = h->stream;
  const bool child_required = dreq != nullptr;
  for (int l = ls + 1; l <= le; ++l) k_mask_zero<<<nb(3 * h->at(l).NN), TPB, 0, s>>>(view(h, l));
  // mask_active
  auto tol = [&](int l, int st, int en) { mask_tol(h, l, st, en, level_fill); };
  tol(le, 0, 1);
  comm_masks(h);
  for (int l = le - 1; l >= ls; --l) {
    tol(l, -1, 2);
    k_mask_parent<<<nodes_blocks(h->at(l).n + 1), TPB, 0, s>>>(view(h, l), view(h, l + 1));
    comm_masks(h);
  }
  comm_masks(h);
  for (int l = ls; l <= le; ++l) k_mask_adj_same<<<nodes_blocks(h->at(l).n + 1), TPB, 0, s>>>(view(h, l));
  comm_masks(h);
  for (int l = ls; l <= std::min(le, max_level - 1); ++l)
    k_mask_restrict_flux<<<nodes_blocks(h->at(l).n), TPB, 0, s>>>(view(h, l));
  comm_masks(h);
  if (child_required) {
    int64_t o = 0;
    for (int l = ls; l <= req_hi; ++l) {
      const int64_t cnt = (int64_t)10 * (h->at(l).n / patch_size) * (h->at(l).n / patch_size) * 4;
      k_child_required<<<nb(cnt), TPB, 0, s>>>(view(h, l), patch_size, dreq + o);
      o += cnt;
    }
  }
  CKW(cudaGetLastError());
  return WT_OK;
}

// refine() on the device tree from the flags in W->treq (tree_kernels.cuh):
// parent levels req_hi down to level_start, so that every launch reads parent
// bytes no earlier launch of this refine wrote; clears the new-patch marks
// first.  Stream-ordered.
static void tree_refine(wt_handle* h, int req_hi) {
  WavCtx* W = ctx(h);
  const int ls = h->level_start, ps = W->tree_ps;
  cudaStream_t s = h->stream;
  cudaMemsetAsync(W->fresh, 0, W->tree_off.back(), s);
  for (int l = req_hi; l >= ls; --l) {
    const int q = l - ls, np = h->at(l).n / ps;
    k_tree_refine<<<nb((int64_t)10 * np * np * 4), TPB, 0, s>>>(W->treq + W->treq_off[q], W->tree + W->tree_off[q],
                                                               W->tree + W->tree_off[q + 1],
                                                               W->fresh + W->tree_off[q + 1], np, l, W->tree_le);
  }
}

// adapt's mask sequence after refine() on levels level_start .. le (the
// level_end refine left): post_refine's comm_masks, mask_adj_finer_scale,
// complete_masks and mask_trsk; then the needed-node maps of the new masks.
static int mask_phase2(wt_handle* h, int le) {
  const int ls = h->level_start;
  cudaStream_t s = h->stream;
  comm_masks(h);  // post_refine
  for (int l = le - 1; l >= ls; --l) {
    k_mask_adj_child<<<nodes_blocks(h->at(l).n + 1), TPB, 0, s>>>(view(h, l), view(h, l + 1));
    k_mask_edges_both<<<nodes_blocks(h->at(l + 1).n), TPB, 0, s>>>(view(h, l + 1));
  }
  comm_masks(h);
  // complete_masks
  for (int l = le - 1; l >= ls + 1; --l) {
    k_mask_edges_consist<<<nodes_blocks(h->at(l).n + 1), TPB, 0, s>>>(view(h, l), view(h, l + 1));
    comm_masks(h);
    k_mask_edges_consist2<<<nodes_blocks(h->at(l).n), TPB, 0, s>>>(view(h, l), view(h, l + 1));
    comm_masks(h);
  }
  if (ls < le) {
    k_mask_edges_consist<<<nodes_blocks(h->at(ls).n + 1), TPB, 0, s>>>(view(h, ls), view(h, ls + 1));
    comm_masks(h);
  }
  for (int l = le - 1; l >= ls + 1; --l) {
    k_mask_nodes_all<<<nodes_blocks(h->at(l + 1).n + 1), TPB, 0, s>>>(view(h, l + 1));
    k_mask_prolong_adj<<<nodes_blocks(h->at(l).n + 1), TPB, 0, s>>>(view(h, l), view(h, l + 1));
  }
  if (ls + 1 <= le) k_mask_nodes_all<<<nodes_blocks(h->at(ls + 1).n + 1), TPB, 0, s>>>(view(h, ls + 1));
  comm_masks(h);
  // mask_trsk
  for (int l = ls; l <= le; ++l) k_mask_trsk<<<nodes_blocks(h->at(l).n + 4), TPB, 0, s>>>(view(h, l));
  CKW(cudaGetLastError());
  ctx(h)->zero_ok = false;  // new masks: compress_wavelets has not run under them
  return wt_level_need_build(h);
}

// adapt's mask sequence (src/adapt.f90:14-65) on every level of the hierarchy,
// stream-ordered and without host synchronisation (so that it can be captured
// in a graph).  With dreq non-null, check_child_required flags of parent
// levels level_start .. level_end-1 go there (patch_size > 0).  With a patch
// tree whose level_end is the hierarchy's, refine() runs on the device between
// the two halves, as in the reference (the flags then go to the tree's own
// buffer when dreq is null).
int wt_level_mask_sequence(wt_handle* h, int level_fill, int max_level, int patch_size, unsigned char* dreq) {
  const int le = h->level_end;
  WavCtx* W = ctx(h);
  const bool tree = W->tree_ps > 0 && W->tree_level_end == le && !dreq;
  const int req_hi = std::min(le, max_level) - 1;
  if (tree) {
    if (int rc = mask_phase1(h, level_fill, max_level, W->tree_ps, W->treq, le, req_hi)) return rc;
    tree_refine(h, req_hi);
  } else if (int rc = mask_phase1(h, level_fill, max_level, patch_size, dreq, le, le - 1)) {
    return rc;
  }
  return mask_phase2(h, le);
}

// The needed-node maps of the levels above level_start from the current masks
// (stream-ordered).
int wt_level_need_build(wt_handle* h) {
  WavCtx* W = ctx(h);
  if (!W->need[0]) return WT_OK;
  NeedSet S{};
  S.nl = h->level_end - h->level_start + 1;
  for (int q = 0; q < S.nl; ++q) {
    const DevLevel& D = h->at(h->level_start + q);
    NeedLev& E = S.L[q];
    E.n = D.n;
    E.P = D.P;
    E.NN = (int)D.NN;
    E.nsrc = D.nsrc;
    E.mask_n = W->L[q].mask_n;
    E.mask_e = W->L[q].mask_e;
    if (q > 0) {
      E.buf[0] = W->need[0] + W->need_off[q];
      E.buf[1] = W->need[1] + W->need_off[q];
      S.start[q + 1] = S.start[q] + E.NN;
    }
  }
  const unsigned g = nb(S.start[S.nl]);
  cudaStream_t s = h->stream;
  k_need_seed<<<g, TPB, 0, s>>>(S);
  for (int r = 0; r < NEED_R; ++r) k_need_dilate<<<g, TPB, 0, s>>>(S, r);
  // with a patch tree: only the nodes of existing patches and their 2-node ring
  const bool tree = W->tree_ps > 0;
  auto tl = [&](int l) {
    const DevLevel& D = h->at(l);
    return TreeLev{D.n, D.P, (int)D.NN, D.nsrc, W->tree + W->tree_off[l - h->level_start]};
  };
  if (tree)
    for (int l = h->level_start + 1; l <= h->level_end; ++l)
      k_need_tree<<<nb(h->at(l).NN), TPB, 0, s>>>(tl(l), W->tree_ps,
                                                  W->need[NEED_R & 1] + W->need_off[l - h->level_start]);
  // parents rebuilt by the intermediate stages' inverse transforms, finest first
  auto ml = [&](int l) {
    const DevLevel& D = h->at(l);
    return MapLev{D.n, D.P, (int)D.NN, D.nsrc};
  };
  unsigned char *A = W->rscr[0], *B = W->rscr[1];
  for (int l = h->level_end - 1; l >= h->level_start; --l) {
    const int c = l + 1;
    const MapLev Lc = ml(c), Lp = ml(l);
    const unsigned char* nc = W->need[NEED_R & 1] + W->need_off[c - h->level_start];
    const unsigned char* rc = c < h->level_end ? W->recpar + W->rec_off[c - h->level_start] : nullptr;
    unsigned char* rp = W->recpar + W->rec_off[l - h->level_start];
    k_map_or<<<nb(Lc.NN), TPB, 0, s>>>(Lc.NN, nc, rc, A);
    k_map_dilate<<<nb(Lc.NN), TPB, 0, s>>>(Lc, A, B);
    k_map_dilate<<<nb(Lc.NN), TPB, 0, s>>>(Lc, B, A);  // rec(c)
    k_map_up<<<nb(Lp.NN), TPB, 0, s>>>(Lc, Lp, A, B);
    k_map_dilate<<<nb(Lp.NN), TPB, 0, s>>>(Lp, B, A);
    k_map_dilate<<<nb(Lp.NN), TPB, 0, s>>>(Lp, A, rp);  // recpar(l)
    if (tree && W->recfin)
      k_map_tree_par<<<nb(Lp.NN), TPB, 0, s>>>(Lp, tl(c), W->tree_ps, rp, W->recfin + W->rec_off[l - h->level_start]);
  }
  // with a patch tree, the parent levels' work lists from recfin
  if (tree && W->recfin)
    for (int l = h->level_start; l < h->level_end; ++l) {
      const int q = l - h->level_start, m = h->at(l).n + 1;
      const DevLevel& D = h->at(l);
      build_list(h, ParentCand{D.n, D.P, D.nsrc, W->recfin + W->rec_off[q]}, 10 * m * m, W->plist_par + W->rec_off[q],
                 W->plist_cnt + q);
    }
  // work lists of the levels above level_start
  for (int l = h->level_start + 1; l <= h->level_end; ++l) {
    const int q = l - h->level_start;
    const DevLevel& D = h->at(l);
    build_list(h, NodeCand{(int)D.NN, D.nsrc, W->need[NEED_R & 1] + W->need_off[q]}, (int)D.NN,
               W->list + W->need_off[q], W->list_cnt + q);
  }
  CKW(cudaGetLastError());
  W->need_ok = true;
  W->recfin_ok = tree && W->recfin;
  return WT_OK;
}

// The parents of level that the inverse transform of an intermediate RK stage
// rebuilds, or null (rebuild every parent).
const unsigned char* wt_level_rec(wt_handle* h, int level) {
  WavCtx* W = ctx(h);
  if (level >= h->level_end || !W->recpar || !W->skip_inactive || !W->need_ok) return nullptr;
  return W->recpar + W->rec_off[level - h->level_start];
}
// The work list of parent level `level` (a patch tree and current maps), else
// {null, null}: the interscale kernels then launch over every parent.
ParentList wt_level_plist(wt_handle* h, int level) {
  WavCtx* W = ctx(h);
  if (level >= h->level_end || !W->plist_par || !W->recfin_ok || !W->skip_inactive || !W->need_ok)
    return ParentList{nullptr, nullptr};
  const int q = level - h->level_start;
  return ParentList{W->plist_par + W->rec_off[q], W->plist_cnt + q};
}

// The parents of level that the inverse transform after adapt rebuilds: with a
// patch tree those the next step reads and those of the tree's nodes (recfin),
// else null (every parent).
const unsigned char* wt_level_rec_final(wt_handle* h, int level) {
  WavCtx* W = ctx(h);
  if (level >= h->level_end || !W->recfin || !W->recfin_ok || !W->skip_inactive || !W->need_ok) return nullptr;
  return W->recfin + W->rec_off[level - h->level_start];
}

// The map level's step1 and trend may skip by, or null (level_start, no map,
// skipping turned off, or masks uploaded since the last build).
const unsigned char* wt_level_need(wt_handle* h, int level) {
  WavCtx* W = ctx(h);
  if (level <= h->level_start || !W->need[0] || !W->skip_inactive || !W->need_ok) return nullptr;
  return W->need[NEED_R & 1] + W->need_off[level - h->level_start];  // the last dilation's output
}
int wt_level_skip_epoch(wt_handle* h) { return ctx(h)->skip_epoch; }
// The work list of level (the slots of its needed-node map), or {null, null}
// when wt_level_need gives no map.
wtk::NodeList wt_level_list(wt_handle* h, int level) {
  WavCtx* W = ctx(h);
  if (!wt_level_need(h, level) || !W->list) return wtk::NodeList{nullptr, nullptr};
  const int q = level - h->level_start;
  return wtk::NodeList{W->list + W->need_off[q], W->list_cnt + q};
}

// Make stream st wait until the last inverse transform has completed level's state.
int wt_level_ready_wait(wt_handle* h, int level, cudaStream_t st) {
  WavCtx* W = ctx(h);
  const int q = level - h->level_start;
  CKW(cudaStreamWaitEvent(st, W->ready_v[q], 0));
  if (q > 0) CKW(cudaStreamWaitEvent(st, W->ready_s[q], 0));
  return WT_OK;
}
int wt_level_need_refresh(wt_handle* h) {
  WavCtx* W = ctx(h);
  if (W->need[0] && W->skip_inactive && !W->need_ok) return wt_level_need_build(h);
  return WT_OK;
}

void wt_level_compress(wt_handle* h) { compress(h); }

// Arrays for the masks before a mask sequence, levels above level_start.
int wt_level_mask_snapshot_alloc(wt_handle* h) {
  WavCtx* W = ctx(h);
  for (int l = h->level_start + 1; l <= h->level_end; ++l) {
    WavLevel& V = W->L[l - h->level_start];
    if (V.old_n) continue;
    CKW(W->alloc(&V.old_n, (size_t)h->at(l).NN));
    CKW(W->alloc(&V.old_e, (size_t)3 * h->at(l).NN));
  }
  return WT_OK;
}

// The masks now, kept for wt_level_compress_delta (stream-ordered).
void wt_level_mask_snapshot(wt_handle* h) {
  WavCtx* W = ctx(h);
  for (int l = h->level_start + 1; l <= h->level_end; ++l) {
    WavLevel& V = W->L[l - h->level_start];
    const size_t nn = (size_t)h->at(l).NN;
    cudaMemcpyAsync(V.old_n, V.mask_n, 4 * nn, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(V.old_e, V.mask_e, 12 * nn, cudaMemcpyDeviceToDevice, h->stream);
  }
}

// compress_wavelets when the wavelets were compressed under the snapshot's
// masks: zero only the slots those masks kept and the current ones drop.
void wt_level_compress_delta(wt_handle* h) {
  WavCtx* W = ctx(h);
  for (int l = h->level_start + 1; l <= h->level_end; ++l) {
    const WavLevel& V = W->L[l - h->level_start];
    const int n = h->at(l).n;
    k_compress_delta<<<nb((int64_t)10 * (n + 1) * (n + 1)), TPB, 0, h->stream>>>(view(h, l), V.old_n, V.old_e,
                                                                                   h->nz);
  }
  W->zero_ok = true;
}
void wt_level_clean_wavelets(wt_handle* h) {
  if (!ctx(h)->wav_dirty) return;
  zero_wavelets(h);
  ctx(h)->wav_dirty = false;
  ctx(h)->zero_ok = true;  // every slot is 0
}
bool wt_level_zero_ok(wt_handle* h) { return ctx(h)->zero_ok; }
void wt_level_inverse(wt_handle* h) { inverse(h, 2); }
int wt_level_set_thresholds(wt_handle* h, const double* threshold) {
  CKW(cudaMemcpyAsync(ctx(h)->thr, threshold, 3 * h->nz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return WT_OK;
}

extern "C" {

int wt_mask_build(wt_handle* h, const double* threshold, int level_fill, int max_level, int patch_size,
                  unsigned char* child_required) {
  if (int rc = ready(h)) return rc;
  const int ls = h->level_start, le = h->level_end, nz = h->nz;
  if (!threshold) return WT_ERR_ARG;
  if (child_required && (patch_size < 2 || (patch_size & 1) || h->at(ls).n % patch_size)) return WT_ERR_ARG;
  WavCtx* W = ctx(h);
  cudaStream_t s = h->stream;
  CKW(cudaMemcpyAsync(W->thr, threshold, 3 * nz * sizeof(double), cudaMemcpyHostToDevice, s));
  unsigned char* dreq = nullptr;
  int64_t nreq = 0;
  if (child_required) {
    for (int l = ls; l <= le - 1; ++l) nreq += (int64_t)10 * (h->at(l).n / patch_size) * (h->at(l).n / patch_size) * 4;
    if (nreq > 0) CKW(cudaMalloc(&dreq, nreq));
  }
  int rc = wt_level_mask_sequence(h, level_fill, max_level, patch_size, dreq);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && dreq) e = cudaMemcpy(child_required, dreq, nreq, cudaMemcpyDeviceToHost);
  if (dreq) cudaFree(dreq);
  if (rc) return rc;
  if (e != cudaSuccess) return fail("mask_build", e);
  return WT_OK;
}

int wt_compress(wt_handle* h) {
  if (int rc = ready(h)) return rc;
  compress(h);
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_wt_after_step(wt_handle* h) {
  if (int rc = ready(h)) return rc;
  if (int rc = wt_level_after_step(h, nullptr, nullptr, nullptr)) return rc;
  CKW(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

// ---- compute-or-restrict of the multi-level trend (src/multi_level.f90:311-659)

}  // extern "C"

int wt_level_restrict_scalar(wt_handle* h, int level, double* par, const double* chd, int nz, cudaStream_t stream) {
  WLev P = view(h, level), C = view(h, level + 1);
  P.scal = par;
  C.scal = const_cast<double*>(chd);
  const int m = h->at(level).n + 1;
  const ParentList PL = wt_level_plist(h, level);
  const unsigned dense = nb((int64_t)nz * 10 * m * m);
  k_restr_scalar<<<PL.ids ? pgrid(k_restr_scalar, TPB, dense) : dense, TPB, 0, stream ? stream : h->stream>>>(P, C, nz,
                                                                                                              PL);
  CKW(cudaGetLastError());
  return WT_OK;
}

namespace {
// flux_cpt_restr of parent `level` from the plan built at setup (k_rf_plan).
int restrict_flux(wt_handle* h, int level, double* par0, double* par1, const double* chd0, const double* chd1,
                  const double* dsc0, const double* dsc1, int nz) {
  const WavLevel& V = ctx(h)->L[level - h->level_start];
  if (!V.rf_pi) return WT_ERR_ARG;
  const int m = h->at(level).n;
  const int64_t ne = (int64_t)3 * 10 * m * m;
  const dim3 blk(32, std::min(nz, 8));
  const ParentList PL = wt_level_plist(h, level);
  const unsigned dense = (unsigned)((ne + 31) / 32);
  k_restr_flux3<<<PL.ids ? pgrid(k_restr_flux3, (int)(blk.x * blk.y), dense) : dense, blk, 0, h->stream>>>(
      view(h, level), m, nz, V.rf_pi, V.rf_pd, par0, par1, chd0, chd1, dsc0, dsc1, (int)h->at(level + 1).NN, PL);
  CKW(cudaGetLastError());
  return WT_OK;
}
}  // namespace

int wt_level_restrict_flux(wt_handle* h, int level, double* par0, double* par1, const double* chd0,
                           const double* chd1, const double* dsc0, const double* dsc1, int nz) {
  return restrict_flux(h, level, par0, par1, chd0, chd1, dsc0, dsc1, nz);
}

extern "C" {

namespace {
// Parent `level` and child level+1 with the given work fields allocated on both.
int restrict_pair(wt_handle* h, int level, std::initializer_list<int> fields) {
  if (int rc = ready(h)) return rc;
  if (level < h->level_start || level >= h->level_end) return WT_ERR_ARG;
  for (int f : fields)
    for (int l = level; l <= level + 1; ++l) {
      double* p;
      if (int rc = work_field(h, l, f, &p, nullptr)) return rc;
    }
  return WT_OK;
}
}  // namespace

int wt_restrict_scalar(wt_handle* h, int level) {
  if (int rc = restrict_pair(h, level, {WT_WORK_SCALAR})) return rc;
  const int m = h->at(level).n + 1;
  k_restr_scalar<<<nb((int64_t)h->nz * 10 * m * m), TPB, 0, h->stream>>>(view(h, level), view(h, level + 1), h->nz,
                                                                          kNoList);
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_restrict_flux(wt_handle* h, int level) {
  if (int rc = restrict_pair(h, level, {WT_WORK_FLUX, WT_WORK_DSCALAR})) return rc;
  const WLev P = view(h, level), C = view(h, level + 1);
  if (int rc = restrict_flux(h, level, P.flux, nullptr, C.flux, nullptr, C.dscal, nullptr, h->nz)) return rc;
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_restrict_u_source(wt_handle* h, int level) {
  if (int rc = restrict_pair(h, level, {WT_WORK_DVELO})) return rc;
  const int m = h->at(level).n;
  k_restr_u_source<<<nb((int64_t)h->nz * 10 * m * m), TPB, 0, h->stream>>>(view(h, level), view(h, level + 1),
                                                                            h->nz);
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

// cal_lnorm (src/lnorms.f90:7-58) of the hierarchy's scaling fields: out[v][k]
// for v = mass, Theta, velocity.
int wt_lnorm(wt_handle* h, int order, double* out) {
  if (int rc = ready(h)) return rc;
  if (!out || order < 0 || order > 3) return WT_ERR_ARG;
  const int nz = h->nz, nl = h->level_end - h->level_start + 1;
  std::vector<int> nparts(nl);
  int64_t np_tot = 0;
  for (int q = 0; q < nl; ++q) {
    nparts[q] = (int)nb(h->at(h->level_start + q).NN);
    np_tot += nparts[q];
  }
  double *part = nullptr, *dout = nullptr;
  int *cnt = nullptr, *dn = nullptr;
  cudaError_t e = cudaMalloc(&part, np_tot * nz * 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&cnt, np_tot * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&dn, nl * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&dout, 3 * nz * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dn, nparts.data(), nl * sizeof(int), cudaMemcpyHostToDevice, h->stream);
  int64_t base = 0, cbase = 0;
  for (int q = 0; q < nl && e == cudaSuccess; ++q) {
    const int l = h->level_start + q;
    double *mm, *mt;
    int rc = wt_level_mean(h, l, WT_FIELD_MEAN_MASS, &mm);
    if (!rc) rc = wt_level_mean(h, l, WT_FIELD_MEAN_TEMP, &mt);
    if (rc) { e = cudaErrorMemoryAllocation; break; }
    k_lnorm_part<<<dim3(nparts[q], nz), TPB, 0, h->stream>>>(view(h, l), mm, mt, order, part + base, cnt + cbase);
    base += (int64_t)nz * nparts[q] * 3;
    cbase += nparts[q];
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_lnorm_final<<<nz, 32, 0, h->stream>>>(part, dn, nl, cnt, order, nz, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, 3 * nz * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(part);
  cudaFree(cnt);
  cudaFree(dn);
  cudaFree(dout);
  if (e != cudaSuccess) return fail("lnorm", e);
  return WT_OK;
}

// Launch-shape tuning of the wavelet kernels: WT_TUNE_WAVELET_LAYERS = layers
// per thread of the layer-group kernels (1 .. 64; 0 restores the default
// chosen from the layer count).  Process-wide.
int wt_set_flux_precision(wt_handle* h, int bits);
int wt_set_tma_inject(wt_handle* h, int value);

int wt_tune(wt_handle* h, int param, int value) {
  if (param == WT_TUNE_FLUX_PRECISION) return wt_set_flux_precision(h, value);
  if (param == WT_TUNE_TEST_TMA_TIMEOUT) {
    const int rc = wt_set_tma_inject(h, value);
    if (rc == WT_OK && h->wav) ++ctx(h)->skip_epoch;  // the hierarchy's step graph re-records
    return rc;
  }
  if (param == WT_TUNE_WAVELET_LAYERS) {
    if (value < 0 || value > 64) return WT_ERR_ARG;
    g_lpt_set = value;
    return WT_OK;
  }
  if (param == WT_TUNE_SKIP_INACTIVE) {
    if (!h) return WT_ERR_ARG;
    if (!h->wav) return WT_ERR_STATE;
    if (value != 0 && value != 1) return WT_ERR_ARG;
    if (ctx(h)->skip_inactive != (value == 1)) {
      ctx(h)->skip_inactive = value == 1;
      ++ctx(h)->skip_epoch;
    }
    return WT_OK;
  }
  return WT_ERR_ARG;
}

}  // extern "C"

// ---- the patch tree of a partially refined hierarchy (src/refine_patch.f90)

extern "C" {

int wt_tree_init(wt_handle* h, int patch_size) {
  if (int rc = ready(h)) return rc;
  const int ls = h->level_start, le = h->level_end;
  if (patch_size < 2 || (patch_size & 1) || h->at(ls).n % patch_size) return WT_ERR_ARG;
  WavCtx* W = ctx(h);
  if (W->tree && W->tree_ps != patch_size) return WT_ERR_STATE;  // one patch size per handle
  if (!W->tree) {
    const size_t nl = W->L.size();
    W->tree_off.assign(nl + 1, 0);
    W->treq_off.assign(nl, 0);
    size_t t = 0, r = 0;
    for (int l = ls; l <= le; ++l) {
      const size_t np = (size_t)(h->at(l).n / patch_size);
      W->tree_off[l - ls] = t;
      W->treq_off[l - ls] = r;
      t += 10 * np * np;
      r += 10 * np * np * 4;
    }
    W->tree_off[nl] = t;
    CKW(W->alloc(&W->tree, t));
    CKW(W->alloc(&W->fresh, t));
    CKW(W->alloc(&W->treq, r));
    CKW(W->alloc(&W->tree_le, 1));
    CKW(W->alloc(&W->tree_cnt, 2));
    if (W->recpar) {
      CKW(W->alloc(&W->recfin, W->rec_tot));
      CKW(W->alloc(&W->plist_par, W->rec_tot));
      CKW(W->alloc(&W->plist_cnt, W->L.size()));
    }
  }
  W->tree_ps = patch_size;
  // add_second_level: every patch of level_start; none above
  CKW(cudaMemsetAsync(W->tree, 0, W->tree_off.back(), h->stream));
  CKW(cudaMemsetAsync(W->tree, 1, W->tree_off[1], h->stream));
  CKW(cudaMemsetAsync(W->fresh, 0, W->tree_off.back(), h->stream));
  CKW(cudaMemcpyAsync(W->tree_le, &h->level_start, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  W->tree_level_end = ls;
  ++W->skip_epoch;  // the hierarchy's step graph re-records (refine inside it or not)
  W->need_ok = false;  // the maps are limited to the tree
  return WT_OK;
}

int wt_tree_level_end(wt_handle* h, int* level_end) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps || !level_end) return W->tree_ps ? WT_ERR_ARG : WT_ERR_STATE;
  CKW(cudaMemcpyAsync(level_end, W->tree_le, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  if (W->tree_level_end != *level_end) {
    W->tree_level_end = *level_end;
    ++W->skip_epoch;
  }
  return WT_OK;
}

int wt_tree_download(wt_handle* h, int level, unsigned char* exist, unsigned char* fresh) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps) return WT_ERR_STATE;
  if (level < h->level_start || level > h->level_end) return WT_ERR_ARG;
  const int q = level - h->level_start;
  const size_t n = W->tree_off[q + 1] - W->tree_off[q];
  if (exist) CKW(cudaMemcpyAsync(exist, W->tree + W->tree_off[q], n, cudaMemcpyDeviceToHost, h->stream));
  if (fresh) CKW(cudaMemcpyAsync(fresh, W->fresh + W->tree_off[q], n, cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_grid_sync(wt_handle* h, const unsigned char* exist, int level_end) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps) return WT_ERR_STATE;
  if (!exist || level_end < h->level_start || level_end > h->level_end) return WT_ERR_ARG;
  for (size_t x = 0; x < W->tree_off[1]; ++x)
    if (!exist[x]) return WT_ERR_ARG;  // level_start is complete
  CKW(cudaMemcpyAsync(W->tree, exist, W->tree_off.back(), cudaMemcpyHostToDevice, h->stream));
  CKW(cudaMemsetAsync(W->fresh, 0, W->tree_off.back(), h->stream));
  CKW(cudaMemcpyAsync(W->tree_le, &level_end, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  if (W->tree_level_end != level_end) ++W->skip_epoch;
  W->tree_level_end = level_end;
  W->need_ok = false;
  return WT_OK;
}

int wt_adapt(wt_handle* h, const double* threshold, int level_fill, int max_level, int* level_end, int* refined) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps) return WT_ERR_STATE;
  if (!threshold) return WT_ERR_ARG;
  const int ls = h->level_start, le1 = W->tree_level_end;
  const int req_hi = std::min(std::min(le1, max_level - 1), h->level_end - 1);
  // wavelets already compressed under the masks now (as after an RK stage's
  // WT_after_step): compress_wavelets only has to zero the slots the new masks
  // drop, as in the step graph
  const bool delta = W->zero_ok;
  if (delta) {
    if (int rc = wt_level_mask_snapshot_alloc(h)) return rc;
    wt_level_mask_snapshot(h);
  }
  CKW(cudaMemcpyAsync(W->thr, threshold, 3 * h->nz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (int rc = mask_phase1(h, level_fill, max_level, W->tree_ps, W->treq, le1, req_hi)) return rc;
  if (req_hi >= ls) {
    tree_refine(h, req_hi);
  } else {
    CKW(cudaMemsetAsync(W->fresh, 0, W->tree_off.back(), h->stream));
  }
  int le2 = le1;
  CKW(cudaMemcpyAsync(&le2, W->tree_le, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  std::vector<unsigned char> fr(W->tree_off.back());
  CKW(cudaMemcpyAsync(fr.data(), W->fresh, fr.size(), cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  if (le2 != le1) ++W->skip_epoch;
  W->tree_level_end = le2;
  if (int rc = mask_phase2(h, le2)) return rc;
  if (delta)
    wt_level_compress_delta(h);
  else
    compress(h);
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  if (level_end) *level_end = le2;
  if (refined) *refined = std::any_of(fr.begin(), fr.end(), [](unsigned char c) { return c != 0; }) ? 1 : 0;
  return WT_OK;
}

int wt_inverse_tree(wt_handle* h) {
  if (int rc = ready(h)) return rc;
  if (int rc = wt_level_need_refresh(h)) return rc;  // maps of the current masks (wt_adapt leaves them built)
  inverse(h, 2);
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_count_active(wt_handle* h, const double* threshold, long long* counts) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps) return WT_ERR_STATE;
  if (!threshold || !counts) return WT_ERR_ARG;
  CKW(cudaMemcpyAsync(W->thr, threshold, 3 * h->nz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CKW(cudaMemsetAsync(W->tree_cnt, 0, 2 * sizeof(unsigned long long), h->stream));
  for (int l = h->level_start + 1; l <= h->level_end; ++l) {
    const int n = h->at(l).n;
    k_tree_count_new<<<nb((int64_t)10 * n * n), TPB, 0, h->stream>>>(
        view(h, l), W->fresh + W->tree_off[l - h->level_start], W->tree_ps, h->nz, W->thr, W->tree_cnt);
  }
  unsigned long long c[2] = {0, 0};
  CKW(cudaMemcpyAsync(c, W->tree_cnt, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  counts[0] = (long long)c[0];
  counts[1] = (long long)c[1];
  return WT_OK;
}

int wt_tree_stats(wt_handle* h, int level, long long* out) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps) return WT_ERR_STATE;
  if (!out || level < h->level_start || level > h->level_end) return WT_ERR_ARG;
  const int q = level - h->level_start, n = h->at(level).n;
  const size_t np2 = W->tree_off[q + 1] - W->tree_off[q];
  std::vector<unsigned char> ex(np2), fr(np2);
  CKW(cudaMemsetAsync(W->tree_cnt, 0, 2 * sizeof(unsigned long long), h->stream));
  k_tree_outside<<<nb((int64_t)10 * n * n), TPB, 0, h->stream>>>(view(h, level), W->tree + W->tree_off[q], W->tree_ps,
                                                                 W->tree_cnt);
  unsigned long long c[2] = {0, 0};
  CKW(cudaMemcpyAsync(ex.data(), W->tree + W->tree_off[q], np2, cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaMemcpyAsync(fr.data(), W->fresh + W->tree_off[q], np2, cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaMemcpyAsync(c, W->tree_cnt, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  out[0] = (long long)std::count(ex.begin(), ex.end(), (unsigned char)1);
  out[1] = (long long)std::count(fr.begin(), fr.end(), (unsigned char)1);
  out[2] = (long long)c[0];
  // owned nodes in the level's needed-node map (-1 without a current map)
  out[3] = -1;
  if (const unsigned char* nd = wt_level_need(h, level)) {
    const DevLevel& D = h->at(level);
    std::vector<unsigned char> m(D.NN);
    CKW(cudaMemcpy(m.data(), nd, D.NN, cudaMemcpyDeviceToHost));
    long long k = 0;
    for (int d = 0; d < 10; ++d)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) k += m[((int64_t)d * D.P + j + 2) * D.P + i + 2] != 0;
    out[3] = k;
  }
  return WT_OK;
}

}  // extern "C"

namespace {
// The patch list of level_end and its count on the host; the packed arrays'
// base pointers (mass, Theta, velocity) in the staging buffer.
int tree_pack_prepare(wt_handle* h, long long* n, double** pm, double** pt, double** pv) {
  WavCtx* W = ctx(h);
  const int le = h->level_end, q = le - h->level_start, ps = W->tree_ps;
  const DevLevel& D = h->at(le);
  const int npatch = (int)(W->tree_off[q + 1] - W->tree_off[q]);
  const size_t per = (size_t)h->nz * ps * ps;  // doubles of one field of one patch
  if (!W->pack) {
    CKW(W->alloc(&W->plist, (size_t)npatch));
    CKW(W->alloc(&W->pcount, 1));
    CKW(W->alloc(&W->pack, (size_t)npatch * per * 5));
  }
  k_patch_list<<<1, TREE_SCAN, 0, h->stream>>>(W->tree + W->tree_off[q], npatch, W->plist, W->pcount);
  int c = 0;
  CKW(cudaMemcpyAsync(&c, W->pcount, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CKW(cudaStreamSynchronize(h->stream));
  *n = c;
  *pm = W->pack;
  *pt = W->pack + (size_t)c * per;
  *pv = W->pack + (size_t)c * per * 2;
  (void)D;
  return WT_OK;
}
}  // namespace

extern "C" {

int wt_download_tree_state(wt_handle* h, double* mass, double* temp, double* velo, long long capacity,
                           long long* n_patches) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps) return WT_ERR_STATE;
  if (!mass || !temp || !velo || !n_patches) return WT_ERR_ARG;
  long long n = 0;
  double *pm, *pt, *pv;
  if (int rc = tree_pack_prepare(h, &n, &pm, &pt, &pv)) return rc;
  *n_patches = n;
  if (n > capacity) return WT_ERR_ARG;
  const DevLevel& D = h->at(h->level_end);
  const int ps = W->tree_ps;
  const size_t per = (size_t)h->nz * ps * ps;
  const int64_t tot = (int64_t)n * per;
  if (tot > 0) {
    k_tree_pack<false><<<nb(tot), TPB, 0, h->stream>>>(D.n, D.P, (int)D.NN, ps, h->nz, W->plist, W->pcount, h->mass,
                                                       h->temp, h->velo, pm, pt, pv);
    CKW(cudaMemcpyAsync(mass, pm, tot * 8, cudaMemcpyDeviceToHost, h->stream));
    CKW(cudaMemcpyAsync(temp, pt, tot * 8, cudaMemcpyDeviceToHost, h->stream));
    CKW(cudaMemcpyAsync(velo, pv, 3 * tot * 8, cudaMemcpyDeviceToHost, h->stream));
  }
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_upload_tree_state(wt_handle* h, const double* mass, const double* temp, const double* velo,
                         long long n_patches) {
  if (int rc = ready(h)) return rc;
  WavCtx* W = ctx(h);
  if (!W->tree_ps) return WT_ERR_STATE;
  if (!mass || !temp || !velo) return WT_ERR_ARG;
  long long n = 0;
  double *pm, *pt, *pv;
  if (int rc = tree_pack_prepare(h, &n, &pm, &pt, &pv)) return rc;
  if (n != n_patches) return WT_ERR_ARG;  // packed for another tree
  const DevLevel& D = h->at(h->level_end);
  const int ps = W->tree_ps;
  const size_t per = (size_t)h->nz * ps * ps;
  const int64_t tot = (int64_t)n * per;
  if (tot > 0) {
    CKW(cudaMemcpyAsync(pm, mass, tot * 8, cudaMemcpyHostToDevice, h->stream));
    CKW(cudaMemcpyAsync(pt, temp, tot * 8, cudaMemcpyHostToDevice, h->stream));
    CKW(cudaMemcpyAsync(pv, velo, 3 * tot * 8, cudaMemcpyHostToDevice, h->stream));
    k_tree_pack<true><<<nb(tot), TPB, 0, h->stream>>>(D.n, D.P, (int)D.NN, ps, h->nz, W->plist, W->pcount, h->mass,
                                                      h->temp, h->velo, pm, pt, pv);
  }
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  h->state_halo_done = false;
  return WT_OK;
}

int wt_mask_adj_child(wt_handle* h, int level) {
  if (int rc = ready(h)) return rc;
  if (level < h->level_start || level >= h->level_end) return WT_ERR_ARG;
  k_mask_adj_child<<<nodes_blocks(h->at(level).n + 1), TPB, 0, h->stream>>>(view(h, level), view(h, level + 1));
  ctx(h)->zero_ok = false;
  ctx(h)->need_ok = false;
  CKW(cudaGetLastError());
  CKW(cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // extern "C"
