// Device storage of the multi-level fields of a handle (h->wav): per level the
// scaling fields below level_end, the wavelet coefficients, the masks, the
// work fields of the compute-or-restrict operators and the layer means; and
// the WLev view that the wavelet, mask and restriction kernels take.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "wavelet_kernels.cuh"
#include "wt_handle.cuh"

namespace wtw {

struct WavLevel {
  double *sm = nullptr, *st = nullptr, *sv = nullptr;  // scaling (owned below level_end)
  double *wm = nullptr, *wt = nullptr, *wv = nullptr;
  int *mask_n = nullptr, *mask_e = nullptr;
  int *old_n = nullptr, *old_e = nullptr;  // the masks before the adaptive step's mask sequence
  double *scal = nullptr, *dscal = nullptr, *flux = nullptr, *dvelo = nullptr;  // work fields, on first use
  double *mean_m = nullptr, *mean_t = nullptr;  // layer means below level_end, on first use
  int* rf_pi = nullptr;     // flux-restriction plan into this level (k_rf_plan), below level_end
  double* rf_pd = nullptr;
  int* op_i = nullptr;      // outer and inner velocity-wavelet plans of this level's parents
  double* op_d = nullptr;   // (k_outer_plan, k_inner_plan), below level_end
  int* ip_i = nullptr;
  double* ip_d = nullptr;
  bool own_scaling = false;
};

struct WavCtx {
  std::vector<WavLevel> L;
  double* thr = nullptr;  // [3][nz] thresholds
  std::vector<void*> allocs;
  // Wavelet slots that no transform kernel writes (parent-coincident nodes,
  // ghost rows, the coarsest level) hold 0 unless a host upload wrote them;
  // WT_after_step re-zeroes the arrays only then.
  bool wav_dirty = false;
  // Every wavelet slot that WT_after_step sets to 0 under the current masks
  // holds 0 already (compress_wavelets ran under them, or a WT_after_step did):
  // the forward kernels then write the kept slots only (CMP 2).
  bool zero_ok = false;
  // side streams of the transforms, forked from and joined back into the
  // handle's stream: the scalar chain of the inverse (0, top priority: it is as
  // long as the velocity chain on the handle's stream), and the forward scalar
  // (3), inner (1) and outer (2) velocity wavelets (lowest priority: they run
  // beside the coarser levels' trend)
  cudaStream_t side[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> fork;  // per level pair: its forward wavelets may start
  // per level: its state is complete in the last inverse transform (velocity
  // chain on the handle's stream, scalar chain on side[0])
  std::vector<cudaEvent_t> ready_v, ready_s;
  // scaling-field pointers put aside while WT_after_step runs on other arrays
  std::vector<WavLevel> bound_saved;
  // needed-node maps of the levels above level_start (need_map.cuh): level
  // level_start + q uses need[NEED_R & 1] + need_off[q], the other buffer is the
  // dilation scratch; need_ok once built from the current masks.  skip_inactive
  // lets the RK stages of the hierarchy leave the finest level's step1 and
  // trend out where the map is 0; skip_epoch counts its changes.
  unsigned char* need[2] = {nullptr, nullptr};
  std::vector<size_t> need_off;
  // parents the inverse transforms of the intermediate RK stages rebuild, per
  // parent level (need_map.cuh), at recpar + rec_off[q]; rscr: scratch maps
  unsigned char* recpar = nullptr;
  std::vector<size_t> rec_off;
  size_t rec_tot = 0;
  // with a patch tree: the parents the inverse transform after adapt rebuilds
  // (recpar and every parent of a node of an existing patch), at recfin +
  // rec_off[q]; recfin_ok once built with the current maps
  unsigned char* recfin = nullptr;
  bool recfin_ok = false;
  // with a patch tree: each parent level's work list (wavelet_kernels.cuh:
  // ParentList) at plist_par + rec_off[q], its count at plist_cnt[q]
  int* plist_par = nullptr;
  int* plist_cnt = nullptr;
  // block counts and offsets of the list compaction (need_map.cuh: k_list_*)
  int* lscr = nullptr;
  size_t lscr_n = 0;
  unsigned char* rscr[2] = {nullptr, nullptr};
  // work lists of the levels above level_start (need_map.cuh: k_list_*):
  // the slots of the needed-node map at list + need_off[q], their count at
  // list_cnt[q], built with the maps
  int* list = nullptr;
  int* list_cnt = nullptr;
  bool need_ok = false;
  bool skip_inactive = true;
  int skip_epoch = 0;
  // patch tree (wt_tree_init; tree_ps = 0: none, every patch exists): per
  // level a byte per patch of tree_ps^2 owned nodes at tree + tree_off[q]
  // (tree_kernels.cuh), the patches the last refine made at fresh +
  // tree_off[q], the check_child_required flags of parent level
  // level_start + q at treq + treq_off[q], and the tree's level_end on the
  // device (tree_le) and as last read by the host (tree_level_end)
  int tree_ps = 0;
  unsigned char* tree = nullptr;
  unsigned char* fresh = nullptr;
  unsigned char* treq = nullptr;
  std::vector<size_t> tree_off, treq_off;
  int* tree_le = nullptr;
  int tree_level_end = 0;
  unsigned long long* tree_cnt = nullptr;  // [2] counters of k_tree_count_new / k_tree_outside
  // packed transfers of level_end's state on its patches (wt_download_tree_state):
  // the patch list, its count and the packed arrays, allocated on first use
  int* plist = nullptr;
  int* pcount = nullptr;
  double* pack = nullptr;
  template <class T>
  cudaError_t alloc(T** p, size_t count) {
    cudaError_t e = cudaMalloc(p, count * sizeof(T));
    if (e == cudaSuccess) allocs.push_back(*p);
    return e;
  }
};

inline WavCtx* ctx(wt_handle* h) { return static_cast<WavCtx*>(h->wav); }

inline WLev view(wt_handle* h, int l) {
  const DevLevel& D = h->at(l);
  WavLevel& W = ctx(h)->L[l - h->level_start];
  WLev v;
  v.n = D.n;
  v.P = D.P;
  v.NN = (int)D.NN;
  v.len = D.len;
  v.tri = D.triarea;
  v.hinv = D.hex_inv;
  v.oa = D.overl_a;
  v.iu = D.iu_wgt;
  v.nsrc = D.nsrc;
  v.esrc = D.esrc;
  v.mask_n = W.mask_n;
  v.mask_e = W.mask_e;
  v.sm = W.sm;
  v.st = W.st;
  v.sv = W.sv;
  v.wm = W.wm;
  v.wt = W.wt;
  v.wv = W.wv;
  v.split = D.overl_split;
  v.rf = D.rf_wgt;
  v.scal = W.scal;
  v.dscal = W.dscal;
  v.flux = W.flux;
  v.dvelo = W.dvelo;
  return v;
}

}  // namespace wtw
