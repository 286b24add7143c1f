// Learned preconditioner of the free-surface solve (network in
// learned_kernels.cuh): node layout and inverse taps, training-pair
// generation with the FP64 multigrid (streamed in batches of right-hand
// sides), Adam training, and flexible CG preconditioned by a V-cycle plus the
// network's correction, with the FP64 V-cycle alone as the fallback.
// Included by wt_elliptic.cu only, after wt_elliptic_mixed.cuh.
#pragma once

#include <functional>
#include <random>

#include "learned_kernels.cuh"

void lp_release(void* p);

namespace {

using namespace wtl;

constexpr int LP_TPB = 128, LP_DOT = 256;

struct LPNet {
  int l = 0, ns = 0;
  int64_t NN = 0;
  int* slot = nullptr;  // ns node slots of the level
  int* tap = nullptr;   // 7*ns compact tap indices
  int *inv_ptr = nullptr, *inv = nullptr;  // inverse taps: (s, t) with tap_t(s) = u, entry 8 s + t
  float* own = nullptr; // ns: 1 on owned nodes, 0 at the pole slots
  float *w = nullptr, *wr = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16* wpk = nullptr;  // W2 packed for the tensor cores
  float *x = nullptr, *y = nullptr, *dy = nullptr, *dz1 = nullptr, *dz2 = nullptr;
  uint4 *h1 = nullptr, *h2 = nullptr;  // BF16 activations, 32 a node
  float slope = 1.0f;                  // hidden activation (1: identity)
  int tensor_cores = 1;                // layer 2 on tcgen05 (0: CUDA cores)
  int l2_grid = 1;                     // persistent CTAs of the tcgen05 layer
  double *rs = nullptr, *fcg = nullptr, *partial = nullptr, *partial2 = nullptr, *losses = nullptr;
  double *rc = nullptr, *ec = nullptr;  // one compact pair (grad / infer)
  double *pr = nullptr, *pe = nullptr, *pscale = nullptr;  // training pairs
  int npairs = 0;
  double *r = nullptr, *z = nullptr, *lz = nullptr, *p = nullptr, *lp = nullptr, *ustar = nullptr,
         *usave = nullptr, *fsave = nullptr, *c = nullptr;
  // level arrays (usave: also u at the start of a learned solve; c: the
  // V-cycle's correction)
  int adam_t = 0;
  double inv_area = 1.0;  // 1 / sum of the node areas 1 / hex_inv
  cudaGraphExec_t it_exec[4] = {nullptr, nullptr, nullptr, nullptr};
  int it_key[4] = {-1, -1, -1, -1};
  std::vector<const void*> it_ptrs[4];  // Ell::rotating() at each graph's capture
  std::vector<void*> allocs, pair_allocs;
  int nbd() const { return (ns + LP_DOT - 1) / LP_DOT; }
};

template <class T>
int lpalloc(std::vector<void*>& A, T** p, int64_t n) {
  cudaError_t e = cudaMalloc(p, sizeof(T) * std::max<int64_t>(1, n));
  if (e != cudaSuccess) return wt_handle_fail("learned alloc", e);
  cudaMemset(*p, 0, sizeof(T) * std::max<int64_t>(1, n));
  A.push_back(*p);
  return WT_OK;
}

void lp_free_pairs(LPNet* N) {
  for (void* q : N->pair_allocs) cudaFree(q);
  N->pair_allocs.clear();
  N->pr = N->pe = N->pscale = nullptr;
  N->npairs = 0;
}

inline unsigned lpg(int64_t n, int tpb = LP_TPB) { return (unsigned)((n + tpb - 1) / tpb); }

// Box-Muller normal deviates from a 64-bit Mersenne twister (same sequence on
// every platform, unlike std::normal_distribution).
struct Normal {
  std::mt19937_64 g;
  explicit Normal(uint64_t s) : g(s) {}
  double u() { return ((g() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double operator()() {
    const double a = u(), b = u();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
  }
};

// BF16 copies of the master weights: rounded floats for the CUDA-core
// kernels, W2 packed in the tensor cores' shared-memory layout.
void lp_round_pack(LPNet& N, cudaStream_t st) {
  k_lp_round<<<lpg(kLpParams, 256), 256, 0, st>>>(N.w, N.wr, kLpParams);
  k_lp_pack_w2<<<lpg(kTaps * kC * kC, 256), 256, 0, st>>>(N.wr, N.wpk);
}

int lp_init_params(LPNet& N, uint64_t seed) {
  std::vector<float> w(kLpParams, 0.f);
  Normal rn(seed);
  auto fill = [&](int off, int cnt, double sd) {
    for (int k = 0; k < cnt; ++k) w[off + k] = (float)(sd * rn());
  };
  // variance-preserving scales for linear layers; a small last layer
  // variance-preserving through the activation, gain sqrt(2 / (1 + slope^2))
  const double gain = std::sqrt(2.0 / (1.0 + (double)N.slope * N.slope));
  fill(kW1, kTaps * kIn * kC, gain * std::sqrt(1.0 / (kTaps * kIn)));
  fill(kW2, kTaps * kC * kC, gain * std::sqrt(1.0 / (kTaps * kC)));
  fill(kW3, kTaps * kC, 0.1 * std::sqrt(1.0 / (kTaps * kC)));
  cudaMemcpy(N.w, w.data(), 4 * kLpParams, cudaMemcpyHostToDevice);
  cudaMemset(N.m, 0, 4 * kLpParams);
  cudaMemset(N.v, 0, 4 * kLpParams);
  N.adam_t = 0;
  lp_round_pack(N, 0);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? WT_OK : wt_handle_fail("learned init", e);
}

int lp_build(Ell& E, uint64_t seed) {
  auto* N = new LPNet();
  DevLevel& D = E.h->at(E.le);
  N->l = E.le;
  N->NN = D.NN;
  const int n = D.n, P = D.P;
  std::vector<int> nsrc(D.NN);
  cudaMemcpy(nsrc.data(), D.nsrc, 4 * D.NN, cudaMemcpyDeviceToHost);
  std::vector<int> slot, cid(D.NN, -1);
  for (int d = 0; d < 10; ++d)
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) {
        const int k = (d * P + j + 2) * P + i + 2;
        if (nsrc[k] == k) {
          cid[k] = (int)slot.size();
          slot.push_back(k);
        }
      }
  const int ns = (int)slot.size();
  N->ns = ns;
  {
    std::vector<double> hinv(D.NN);
    cudaMemcpy(hinv.data(), D.hex_inv, 8 * D.NN, cudaMemcpyDeviceToHost);
    double area = 0.0;
    for (int k : slot) area += 1.0 / hinv[k];
    N->inv_area = 1.0 / area;
  }
  static const int di[kTaps] = {0, 1, 1, 0, -1, -1, 0}, dj[kTaps] = {0, 0, 1, 1, 0, -1, -1};
  std::vector<int> tap((size_t)kTaps * ns);
  std::vector<float> own(ns);
  for (int s = 0; s < ns; ++s) {
    const int k = slot[s], d = k / (P * P), r = k % (P * P), i = r % P - 2, j = r / P - 2;
    own[s] = (i < n && j < n) ? 1.f : 0.f;
    for (int t = 0; t < kTaps; ++t) {
      const int kn = (d * P + j + dj[t] + 2) * P + i + di[t] + 2;
      tap[(size_t)t * ns + s] = cid[nsrc[kn]];
    }
  }
  // inverse taps, each node's list ordered by tap
  std::vector<int> inv_ptr(ns + 1, 0), inv;
  for (int t = 0; t < kTaps; ++t)
    for (int s = 0; s < ns; ++s)
      if (tap[(size_t)t * ns + s] >= 0) ++inv_ptr[tap[(size_t)t * ns + s] + 1];
  for (int u = 0; u < ns; ++u) inv_ptr[u + 1] += inv_ptr[u];
  inv.resize(inv_ptr[ns]);
  {
    std::vector<int> fill(inv_ptr.begin(), inv_ptr.end() - 1);
    for (int t = 0; t < kTaps; ++t)
      for (int s = 0; s < ns; ++s) {
        const int u = tap[(size_t)t * ns + s];
        if (u >= 0) inv[fill[u]++] = 8 * s + t;
      }
  }
  auto& A = N->allocs;
  int rc = WT_OK;
  auto al = [&](auto** p, int64_t cnt) {
    if (rc == WT_OK) rc = lpalloc(A, p, cnt);
  };
  al(&N->slot, ns);
  al(&N->tap, (int64_t)kTaps * ns);
  al(&N->inv_ptr, ns + 1);
  al(&N->inv, std::max<int64_t>(1, (int64_t)inv.size()));
  al(&N->own, ns);
  for (float** p : {&N->w, &N->wr, &N->g, &N->m, &N->v}) al(p, kLpParams);
  al(&N->wpk, (int64_t)kTaps * kC * kC);
  al(&N->x, (int64_t)kIn * ns);
  al(&N->h1, (int64_t)ns * (kC / 8));
  al(&N->h2, (int64_t)ns * (kC / 8));
  al(&N->dz1, (int64_t)kC * ns);
  al(&N->dz2, (int64_t)kC * ns);
  al(&N->y, ns);
  al(&N->dy, ns);
  al(&N->rs, 1);
  al(&N->fcg, FCG_N);
  al(&N->partial, N->nbd());
  al(&N->partial2, N->nbd());
  al(&N->losses, 1);
  al(&N->rc, ns);
  al(&N->ec, ns);
  for (double** p : {&N->r, &N->z, &N->lz, &N->p, &N->lp, &N->ustar, &N->usave, &N->fsave, &N->c})
    al(p, D.NN);
  if (rc == WT_OK) {
    cudaMemcpy(N->slot, slot.data(), 4 * (size_t)ns, cudaMemcpyHostToDevice);
    cudaMemcpy(N->tap, tap.data(), 4 * tap.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(N->own, own.data(), 4 * (size_t)ns, cudaMemcpyHostToDevice);
    cudaMemcpy(N->inv_ptr, inv_ptr.data(), 4 * (size_t)(ns + 1), cudaMemcpyHostToDevice);
    if (!inv.empty()) cudaMemcpy(N->inv, inv.data(), 4 * inv.size(), cudaMemcpyHostToDevice);
    // persistent CTAs of the tensor-core layer: as many as fit on the device at once
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaFuncSetAttribute(k_lp_l2_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, kL2Smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_lp_l2_umma, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lp_l2_umma, kL2Threads, kL2Smem);
    if (e != cudaSuccess) rc = wt_handle_fail("learned l2 attributes", e);
    // three CTAs fit an SM by shared memory (70 KB each) and registers
    const int tiles = (ns + kL2M - 1) / kL2M;
    N->l2_grid = std::max(1, std::min(tiles, std::max(3, per_sm) * std::max(1, nsm)));
    if (rc == WT_OK) rc = lp_init_params(*N, seed);
  }
  if (rc != WT_OK) {
    lp_release(N);
    return rc;
  }
  if (E.lp) lp_release(E.lp);
  E.lp = N;
  return WT_OK;
}

// rs = rms of r over the nodes (r read at slot[s]; nullptr: compact).
void lp_rms(LPNet& N, cudaStream_t st, const int* slot, const double* r, double* rs) {
  k_lp_dot<LP_DOT><<<N.nbd(), LP_DOT, 0, st>>>(N.ns, slot, r, r, nullptr, N.partial);
  k_lp_sum<<<1, 256, 0, st>>>(N.partial, N.nbd(), rs, 1, 1.0 / N.ns);
}

// Layer 2, h2 = act(conv(h1)): tcgen05 or, for comparison, the CUDA cores.
void lp_l2(Ell& E, LPNet& N, cudaStream_t st) {
  if (N.tensor_cores)
    k_lp_l2_umma<<<N.l2_grid, kL2Threads, kL2Smem, st>>>(N.ns, N.tap, N.h1, reinterpret_cast<const uint4*>(N.wpk),
                                                        N.slope, N.h2, E.h->dflag);
  else
    k_lp_l2_simt<<<lpg(N.ns), LP_TPB, 0, st>>>(N.ns, N.tap, N.h1, N.wr + kW2, N.slope, N.h2);
}

// Network output y for input r / *rs (r read at slot[s]; nullptr: compact).
void lp_forward(Ell& E, LPNet& N, const int* slot, const double* r, const double* rs) {
  cudaStream_t st = E.s();
  const int ns = N.ns;
  k_lp_input<<<lpg(ns), LP_TPB, 0, st>>>(ns, slot, N.slot, r, rs, E.h->at(N.l).topo, N.x);
  k_lp_l1<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.tap, N.x, nullptr, nullptr, nullptr, nullptr, N.wr + kW1, N.slope,
                                      N.h1);
  lp_l2(E, N, st);
  k_lp_l3<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.tap, N.h2, N.wr + kW3, N.y, nullptr, nullptr, nullptr, nullptr);
}

// The network's correction z = base + own * rs * net(r/rs), rs = rms(r) (the
// scaling keeps FP32 in range; the network is positively homogeneous).  r read and z written
// at slot[s] (nullptr: compact); base may be nullptr.
void lp_precondition(Ell& E, LPNet& N, const int* slot, const double* r, const double* base, double* z) {
  cudaStream_t st = E.s();
  lp_rms(N, st, slot, r, N.rs);
  lp_forward(E, N, slot, r, N.rs);
  k_lp_output<<<lpg(N.ns), LP_TPB, 0, st>>>(N.ns, slot, N.y, N.rs, N.own, base, z);
}

// Energy-norm loss of the network output against the compact target e (scaled
// by *rs) into *loss, then the parameter gradient into N.g.
void lp_backward(Ell& E, LPNet& N, const double* e, const double* rs, double* loss) {
  cudaStream_t st = E.s();
  const int ns = N.ns;
  k_lp_err<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.slot, N.y, N.own, e, rs, N.z);
  op(E, OP_APPLY, N.l, N.z, nullptr, N.lz);
  k_lp_aloss<LP_DOT><<<N.nbd(), LP_DOT, 0, st>>>(ns, N.slot, N.z, N.lz, E.h->at(N.l).hex_inv, N.own, N.inv_area,
                                                 N.dy, N.partial);
  k_lp_sum<<<1, 256, 0, st>>>(N.partial, N.nbd(), loss, 0, N.inv_area);
  cudaMemsetAsync(N.g, 0, 4 * kLpParams, st);
  const unsigned gw = std::min<unsigned>((ns + kChunk - 1) / kChunk, 148 * 4);
  const auto* h1 = reinterpret_cast<const __nv_bfloat16*>(N.h1);
  const auto* h2 = reinterpret_cast<const __nv_bfloat16*>(N.h2);
  k_lp_wgrad<kC, 1><<<gw, 256, 0, st>>>(ns, N.tap, h2, N.dy, N.g + kW3);
  k_lp_igrad<1><<<lpg(ns), LP_TPB, 0, st>>>(ns, N.inv_ptr, N.inv, N.wr + kW3, N.dy, h2, N.slope, N.dz2);
  k_lp_wgrad<kC, kC><<<gw, 256, 0, st>>>(ns, N.tap, h1, N.dz2, N.g + kW2);
  k_lp_igrad<kC><<<lpg(ns), LP_TPB, 0, st>>>(ns, N.inv_ptr, N.inv, N.wr + kW2, N.dz2, h1, N.slope, N.dz1);
  k_lp_wgrad<kIn, kC><<<gw, 256, 0, st>>>(ns, N.tap, N.x, N.dz1, N.g + kW1);
}

void lp_adam(Ell& E, LPNet& N, float lr) {
  cudaStream_t st = E.s();
  ++N.adam_t;
  k_lp_adam<<<lpg(kLpParams, 256), 256, 0, st>>>(kLpParams, N.w, N.g, N.m, N.v, lr, 0.9f, 0.999f, 1e-8f, N.adam_t);
  lp_round_pack(N, st);
}

// Residual/error pairs from FP64 multigrid: for each seeded right-hand side
// k0 <= k < k1, the solution u* to 1e-11, then from u = 0 the residual
// f - L u and error u* - u after each of `cycles` V-cycles (what a V-cycle
// leaves, which the network learns to correct).  u and f of the level are
// kept.  The pair buffers hold one batch and are reused across batches.
int lp_generate(Ell& E, LPNet& N, const wt_learn_opts& lo, const wt_solver_opts& mg, int k0, int k1) {
  const int q = E.le - E.ls, ns = N.ns, l = E.le;
  const int64_t NN = N.NN;
  cudaStream_t st = E.s();
  const int np = (k1 - k0) * lo.cycles;
  int rc = WT_OK;
  if (N.npairs < np) {
    lp_free_pairs(&N);
    if ((rc = lpalloc(N.pair_allocs, &N.pr, (int64_t)np * ns))) return rc;
    if ((rc = lpalloc(N.pair_allocs, &N.pe, (int64_t)np * ns))) return rc;
    if ((rc = lpalloc(N.pair_allocs, &N.pscale, np))) return rc;
    N.npairs = np;
  }
  cudaMemcpyAsync(N.usave, E.u.lv[q], 8 * NN, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(N.fsave, E.f.lv[q], 8 * NN, cudaMemcpyDeviceToDevice, st);
  std::vector<double> fc(ns);
  wt_solver_opts o = mg;
  o.ir_tol = 1e-11;
  o.ir_max = std::max(o.ir_max, 60);
  for (int k = k0; k < k1; ++k) {
    Normal rn(lo.seed * 1000003ull + 7919ull * (uint64_t)k + 1);
    double mean = 0.0;
    for (double& v : fc) mean += (v = rn());
    mean /= ns;
    for (double& v : fc) v -= mean;
    cudaMemcpyAsync(N.rc, fc.data(), 8 * (size_t)ns, cudaMemcpyHostToDevice, st);
    k_lp_scatter<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.slot, N.rc, E.f.lv[q]);
    zero_level(E, l, E.u.lv[q]);
    wt_solver_report rep{};
    rc = mixed_ir(E, o, rep, true);
    if (rc != WT_OK && rc != WT_ERR_NOT_CONVERGED) break;
    rc = WT_OK;
    cudaMemcpyAsync(N.ustar, E.u.lv[q], 8 * NN, cudaMemcpyDeviceToDevice, st);
    zero_level(E, l, E.u.lv[q]);
    op(E, OP_RESID, l, E.u.lv[q], E.f.lv[q], E.res.lv[q]);
    for (int c = 0; c < lo.cycles; ++c) {
      const int64_t idx = (int64_t)(k - k0) * lo.cycles + c;
      vcycle64(E, o);
      k_axpy_d<<<nb(NN), TPB, 0, st>>>(NN, E.u.lv[q], E.corr.lv[q]);
      op(E, OP_RESID, l, E.u.lv[q], E.f.lv[q], E.res.lv[q]);
      k_lp_gather<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.slot, E.res.lv[q], N.pr + idx * ns);
      k_lp_diff<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.slot, N.ustar, E.u.lv[q], N.pe + idx * ns);
      lp_rms(N, st, nullptr, N.pr + idx * ns, N.pscale + idx);
    }
  }
  cudaMemcpyAsync(E.u.lv[q], N.usave, 8 * NN, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(E.f.lv[q], N.fsave, 8 * NN, cudaMemcpyDeviceToDevice, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return wt_handle_fail("learned generate", e);
  return rc;
}

// `epochs` Adam passes over the np pairs of the current batch, one pair a
// step, in a shuffled order; the step size follows one cosine decay from lr
// to lr / 20 over all `total` steps of the training, of which `step` are done.
// The loss of each step goes to losses[step].
void lp_train_batch(Ell& E, LPNet& N, const wt_learn_opts& lo, int np, std::mt19937_64& g, int& step, int total,
                    double* losses) {
  const int ns = N.ns;
  std::vector<int> perm(np);
  for (int k = 0; k < np; ++k) perm[k] = k;
  const double PI = std::acos(-1.0);
  for (int ep = 0; ep < std::max(1, lo.epochs); ++ep) {
    std::shuffle(perm.begin(), perm.end(), g);
    for (int k : perm) {
      const float lr =
          (float)(lo.lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(PI * step / std::max(1, total - 1)))));
      lp_forward(E, N, nullptr, N.pr + (int64_t)k * ns, N.pscale + k);
      lp_backward(E, N, N.pe + (int64_t)k * ns, N.pscale + k, losses + step);
      lp_adam(E, N, lr);
      ++step;
    }
  }
}

// ------------------------------------------------------- flexible CG ----
enum { PRE_NONE = 0, PRE_NET = 1, PRE_MG = 2, PRE_MG64 = 3 };

// One FCG iteration as a stream sequence (captured once per preconditioner):
// z = M(r); Lz; beta and the new direction; alpha and the update; ||r||.
// M: -1 (PRE_NONE); the FP32 V-cycle V of the mixed solve (PRE_MG); V then the
// network's correction of the residual V leaves, z = c + net(r - L c),
// c = V(r) (PRE_NET); or the FP64 V-cycle, plain multigrid (PRE_MG64, the
// fallback).  The recurrences stay FP64 whatever the preconditioner.
void fcg_iteration(Ell& E, LPNet& N, const wt_solver_opts& o, int pre) {
  cudaStream_t st = E.s();
  const int q = E.le - E.ls, l = E.le, ns = N.ns;
  const double* hinv = E.h->at(l).hex_inv;
  if (pre == PRE_NONE) {
    k_fcg_neg<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.slot, N.r, N.z);
  } else if (pre == PRE_MG64) {
    cudaMemcpyAsync(E.res.lv[q], N.r, 8 * N.NN, cudaMemcpyDeviceToDevice, st);
    vcycle64(E, o);
    cudaMemcpyAsync(N.z, E.corr.lv[q], 8 * N.NN, cudaMemcpyDeviceToDevice, st);
  } else {
    double* c = pre == PRE_NET ? N.c : N.z;
    k_d2f<<<nb(N.NN), TPB, 0, st>>>(N.NN, N.r, E.r32.lvf[q]);
    vcycle32(E, o);
    cudaMemsetAsync(c, 0, 8 * N.NN, st);
    k_axpy_f2d<<<nb(N.NN), TPB, 0, st>>>(N.NN, c, E.c32.lvf[q]);
    if (pre == PRE_NET) {
      // z = c + net(r - L c): the network is positively homogeneous, so it
      // runs on the unscaled residual; its input and output are fused into
      // the first and last layers
      op(E, OP_APPLY, l, N.c, nullptr, N.lz);
      k_lp_l1<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.tap, nullptr, N.slot, N.r, N.lz, E.h->at(l).topo, N.wr + kW1,
                                          N.slope, N.h1);
      lp_l2(E, N, st);
      k_lp_l3<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.tap, N.h2, N.wr + kW3, nullptr, N.slot, N.own, N.c, N.z);
    }
  }
  op(E, OP_APPLY, l, N.z, nullptr, N.lz);
  auto wdot = [&](const double* a, const double* b, int slotv) {
    k_lp_dot<LP_DOT><<<N.nbd(), LP_DOT, 0, st>>>(ns, N.slot, a, b, hinv, N.partial);
    k_lp_sum<<<1, 256, 0, st>>>(N.partial, N.nbd(), N.fcg + slotv, 0, 1.0);
  };
  wdot(N.z, N.lp, FCG_ZLP);
  // the new direction and <p, r>, <p, Lp> in one pass
  k_fcg_dir_dots<LP_DOT><<<N.nbd(), LP_DOT, 0, st>>>(ns, N.slot, N.fcg, N.z, N.lz, N.r, hinv, N.p, N.lp, N.partial,
                                                     N.partial2);
  k_lp_sum2<<<1, 256, 0, st>>>(N.partial, N.partial2, N.nbd(), N.fcg + FCG_PR, N.fcg + FCG_DELTA);
  k_fcg_step<<<lpg(ns), LP_TPB, 0, st>>>(ns, N.slot, N.fcg, N.p, N.lp, E.u.lv[q], N.r);
  EllLev V = E.view(l);
  const unsigned g = nb(10 * E.m(l) * E.m(l));
  k_ell_dot<TPB><<<g, TPB, 0, st>>>(V, N.r, N.r, E.partial);
  k_final_sum<<<1, 256, 0, st>>>(E.partial, (int)g, N.fcg + FCG_RNORM, 1, nullptr);
}

int fcg_launch(Ell& E, LPNet& N, const wt_solver_opts& o, int pre) {
  cudaGraphExec_t& ex = N.it_exec[pre];
  const int key = pre != PRE_NONE ? o.down_iter * 1000000 + o.up_iter * 10000 + o.coarse_iter : 0;
  // re-captured when the schedule changed or a reference-path solver has
  // rotated u, res or the V-cycle's work buffers since the capture
  if (!ex || N.it_key[pre] != key || N.it_ptrs[pre] != E.rotating()) {
    N.it_key[pre] = -1;
    int rc = capture_graph(E, ex, N.it_ptrs[pre], "fcg graph", [&] { fcg_iteration(E, N, o, pre); });
    if (rc != WT_OK) return rc;
    N.it_key[pre] = key;
  }
  cudaError_t le = cudaGraphLaunch(ex, E.s());
  return le == cudaSuccess ? WT_OK : wt_handle_fail("fcg launch", le);
}

// r = f - L u (true residual) and a restart of the recurrences.
void fcg_restart(Ell& E, LPNet& N) {
  const int q = E.le - E.ls;
  op(E, OP_RESID, E.le, E.u.lv[q], E.f.lv[q], N.r);
  cudaMemsetAsync(N.fcg, 0, 8 * FCG_N, E.s());
}

// Flexible CG on level_end to ir_tol (relative to ||f||, the solver's l2).
// With the network (PRE_NET) plain FP64 multigrid takes over when the residual has not
// halved over the last kWin iterations, has grown tenfold above its smallest
// value, or a step breaks down (<p, Lp> not negative or not finite); if the
// residual is then above the initial one, u restarts from the initial guess.
int fcg_solve(Ell& E, const wt_solver_opts& o, wt_solver_report& rep, int pre) {
  if (!E.lp) {
    if (int rc = lp_build(E, 1)) return rc;
  }
  LPNet& N = *static_cast<LPNet*>(E.lp);
  const int q = E.le - E.ls, l = E.le;
  constexpr int kWin = 10;
  double nf = l2(E, l, E.f.lv[q]);
  if (nf == 0.0) nf = 1.0;
  fcg_restart(E, N);
  double err = l2(E, l, N.r) / nf;
  rep.nrm_res_init[q] = err;
  if (pre == PRE_NET) cudaMemcpyAsync(N.usave, E.u.lv[q], 8 * N.NN, cudaMemcpyDeviceToDevice, E.s());
  std::vector<double> hist{err};
  double best = err;
  int it = 0, since = 0, net_its = 0, breaks = 0;
  int mode = pre;
  int rc = WT_OK;
  while (err > o.ir_tol && it < o.ir_max) {
    if ((rc = fcg_launch(E, N, o, mode))) return rc;
    ++it;
    ++since;
    if (mode == PRE_NET) ++net_its;
    double sc[FCG_N];
    cudaMemcpyAsync(sc, N.fcg, 8 * FCG_N, cudaMemcpyDeviceToHost, E.s());
    cudaError_t ce = cudaStreamSynchronize(E.s());
    if (ce != cudaSuccess) return wt_handle_fail("fcg sync", ce);
    err = sc[FCG_RNORM] / nf;
    hist.push_back(err);
    const bool broke = sc[FCG_BREAK] != 0.0 || !std::isfinite(err);
    const bool stalled = (since >= kWin && err > 0.5 * hist[hist.size() - 1 - kWin]) || err > 10.0 * best;
    best = std::min(best, err);
    if (mode == PRE_NET && (broke || stalled)) {
      mode = PRE_MG64;
      rep.precond_fallback = it;
      since = 0;
      if (!(err <= rep.nrm_res_init[q]))
        cudaMemcpyAsync(E.u.lv[q], N.usave, 8 * N.NN, cudaMemcpyDeviceToDevice, E.s());
      fcg_restart(E, N);
      ++rep.restarts;
      err = l2(E, l, N.r) / nf;
      continue;
    }
    if (broke) {
      if (++breaks > 3) break;
      since = 0;
      fcg_restart(E, N);
      ++rep.restarts;
      err = l2(E, l, N.r) / nf;
      continue;
    }
    if (err <= o.ir_tol) {
      // the recurrence's residual drifts from the true one: check and restart
      fcg_restart(E, N);
      err = l2(E, l, N.r) / nf;
      if (err > o.ir_tol) {
        ++rep.restarts;
        since = 0;
      }
    }
  }
  DevLevel& D = E.h->at(l);
  k_lp_fill_ghost<<<nb(D.NN), TPB, 0, E.s()>>>(D.NN, D.nsrc, E.u.lv[q]);
  rep.iterations[q] = it;
  rep.outer_iterations = pre == PRE_NET ? net_its : it;
  rep.nrm_res_final[q] = err;
  return err <= o.ir_tol ? WT_OK : WT_ERR_NOT_CONVERGED;
}

}  // namespace

void lp_release(void* p) {
  if (!p) return;
  auto* N = static_cast<LPNet*>(p);
  for (auto& ex : N->it_exec)
    if (ex) cudaGraphExecDestroy(ex);
  lp_free_pairs(N);
  for (void* q : N->allocs) cudaFree(q);
  delete N;
}

// ---------------------------------------------------------------- C-ABI ----
extern "C" {

static int lp_get(wt_handle* h, Ell** E, LPNet** N) {
  if (!h || !h->ell) return WT_ERR_STATE;
  *E = static_cast<Ell*>(h->ell);
  if (!(*E)->lp) return WT_ERR_STATE;
  *N = static_cast<LPNet*>((*E)->lp);
  return WT_OK;
}

int wt_learned_setup(wt_handle* h, unsigned long long seed) {
  if (!h || !h->ell) return WT_ERR_STATE;
  return lp_build(*static_cast<Ell*>(h->ell), seed);
}

int wt_learned_num_params(void) { return kLpParams; }

int wt_learned_params(wt_handle* h, float* get, const float* set) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  CKE(cudaStreamSynchronize(E->s()));
  if (set) {
    CKE(cudaMemcpy(N->w, set, 4 * kLpParams, cudaMemcpyHostToDevice));
    lp_round_pack(*N, E->s());
    CKE(cudaStreamSynchronize(E->s()));
  }
  if (get) CKE(cudaMemcpy(get, N->w, 4 * kLpParams, cudaMemcpyDeviceToHost));
  return WT_OK;
}

int wt_learned_layout(wt_handle* h, int* ns, int* slot, int* tap) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  if (ns) *ns = N->ns;
  if (slot) CKE(cudaMemcpy(slot, N->slot, 4 * (size_t)N->ns, cudaMemcpyDeviceToHost));
  if (tap) CKE(cudaMemcpy(tap, N->tap, 4 * (size_t)kTaps * N->ns, cudaMemcpyDeviceToHost));
  return WT_OK;
}

int wt_learned_infer(wt_handle* h, const double* r, double* z) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  if (!r || !z) return WT_ERR_ARG;
  cudaStream_t st = E->s();
  CKE(cudaMemcpyAsync(N->rc, r, 8 * (size_t)N->ns, cudaMemcpyHostToDevice, st));
  lp_precondition(*E, *N, nullptr, N->rc, nullptr, N->ec);
  CKE(cudaMemcpyAsync(z, N->ec, 8 * (size_t)N->ns, cudaMemcpyDeviceToHost, st));
  CKE(cudaStreamSynchronize(st));
  return WT_OK;
}

int wt_learned_grad(wt_handle* h, const double* r, const double* e, double* loss, float* grad) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  if (!r || !e) return WT_ERR_ARG;
  cudaStream_t st = E->s();
  CKE(cudaMemcpyAsync(N->rc, r, 8 * (size_t)N->ns, cudaMemcpyHostToDevice, st));
  CKE(cudaMemcpyAsync(N->ec, e, 8 * (size_t)N->ns, cudaMemcpyHostToDevice, st));
  lp_rms(*N, st, nullptr, N->rc, N->rs);
  lp_forward(*E, *N, nullptr, N->rc, N->rs);
  lp_backward(*E, *N, N->ec, N->rs, N->losses);
  if (loss) CKE(cudaMemcpyAsync(loss, N->losses, 8, cudaMemcpyDeviceToHost, st));
  if (grad) CKE(cudaMemcpyAsync(grad, N->g, 4 * kLpParams, cudaMemcpyDeviceToHost, st));
  CKE(cudaStreamSynchronize(st));
  CKE(cudaGetLastError());
  return WT_OK;
}

int wt_learned_train(wt_handle* h, const wt_learn_opts* o, wt_learn_report* rep) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  if (!o || !rep || o->n_rhs < 1 || o->cycles < 1 || o->epochs < 1 || !(o->lr > 0) || o->batch_rhs < 0)
    return WT_ERR_ARG;
  std::memset(rep, 0, sizeof(*rep));
  wt_solver_opts mg{};
  mg.method = WT_SOLVER_MG64;
  mg.down_iter = o->down_iter > 0 ? o->down_iter : 2;
  mg.up_iter = o->up_iter > 0 ? o->up_iter : 2;
  mg.coarse_iter = o->coarse_iter > 0 ? o->coarse_iter : 20;
  mg.ir_max = 60;
  const int batch = o->batch_rhs > 0 ? std::min(o->batch_rhs, o->n_rhs) : o->n_rhs;
  const int total = o->epochs * o->n_rhs * o->cycles;
  double* losses = nullptr;
  std::vector<void*> tmp;
  if (int rc = lpalloc(tmp, &losses, total)) return rc;
  std::mt19937_64 g(o->seed ^ 0x5bd1e995ull);
  CKE(cudaStreamSynchronize(E->s()));
  double ms_gen = 0.0, ms_train = 0.0;
  int rc = WT_OK, step = 0, first_np = 0, last_np = 0;
  for (int k0 = 0; k0 < o->n_rhs && rc == WT_OK; k0 += batch) {
    const int k1 = std::min(o->n_rhs, k0 + batch), np = (k1 - k0) * o->cycles;
    auto t0 = std::chrono::steady_clock::now();
    rc = lp_generate(*E, *N, *o, mg, k0, k1);
    auto t1 = std::chrono::steady_clock::now();
    if (rc == WT_OK) {
      lp_train_batch(*E, *N, *o, np, g, step, total, losses);
      cudaError_t e = cudaStreamSynchronize(E->s());
      if (e != cudaSuccess) rc = wt_handle_fail("learned train", e);
    }
    auto t2 = std::chrono::steady_clock::now();
    ms_gen += std::chrono::duration<double, std::milli>(t1 - t0).count();
    ms_train += std::chrono::duration<double, std::milli>(t2 - t1).count();
    if (k0 == 0) first_np = np;
    last_np = np;
  }
  std::vector<double> hl(total, 0.0);
  if (rc == WT_OK) {
    cudaError_t e = cudaMemcpy(hl.data(), losses, 8 * (size_t)total, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = wt_handle_fail("learned losses", e);
  }
  for (void* p : tmp) cudaFree(p);
  lp_free_pairs(N);
  rep->ms_generate = ms_gen;
  rep->ms_train = ms_train;
  if (rc != WT_OK) return rc;
  // mean loss over the first pass of the first batch and the last pass of the last one
  double a = 0, b = 0;
  for (int k = 0; k < first_np; ++k) a += hl[k];
  for (int k = 0; k < last_np; ++k) b += hl[total - last_np + k];
  rep->pairs = o->n_rhs * o->cycles;
  rep->steps = total;
  rep->loss_first_epoch = a / std::max(1, first_np);
  rep->loss_last_epoch = b / std::max(1, last_np);
  for (int k = 0; k < total; ++k)
    if (!std::isfinite(hl[k])) return WT_ERR_NONFINITE;
  CKE(cudaGetLastError());
  return WT_OK;
}

// Per-layer device time of the network's forward pass on a seeded residual
// (mean over reps launches of each layer, CUDA events on the solver's
// stream): ms[0] layer 1 with the input, ms[1] layer 2 (tensor cores or CUDA
// cores as set), ms[2] layer 3.
int wt_learned_layer_times(wt_handle* h, int reps, float* ms) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  if (reps < 1 || !ms) return WT_ERR_ARG;
  cudaStream_t st = E->s();
  const int ns = N->ns;
  std::vector<double> r(ns);
  Normal rn(12345);
  for (double& v : r) v = rn();
  CKE(cudaMemcpyAsync(N->rc, r.data(), 8 * (size_t)ns, cudaMemcpyHostToDevice, st));
  lp_rms(*N, st, nullptr, N->rc, N->rs);
  k_lp_input<<<lpg(ns), LP_TPB, 0, st>>>(ns, nullptr, N->slot, N->rc, N->rs, E->h->at(N->l).topo, N->x);
  cudaEvent_t ev[2];
  CKE(cudaEventCreate(&ev[0]));
  CKE(cudaEventCreate(&ev[1]));
  auto l1 = [&] {
    k_lp_l1<<<lpg(ns), LP_TPB, 0, st>>>(ns, N->tap, N->x, nullptr, nullptr, nullptr, nullptr, N->wr + kW1, N->slope,
                                        N->h1);
  };
  auto l2 = [&] { lp_l2(*E, *N, st); };
  auto l3 = [&] {
    k_lp_l3<<<lpg(ns), LP_TPB, 0, st>>>(ns, N->tap, N->h2, N->wr + kW3, N->y, nullptr, nullptr, nullptr, nullptr);
  };
  int q = 0;
  const std::function<void()> layers[3] = {l1, l2, l3};
  for (const auto& f : layers) {
    f();  // warm-up
    CKE(cudaEventRecord(ev[0], st));
    for (int k = 0; k < reps; ++k) f();
    CKE(cudaEventRecord(ev[1], st));
    CKE(cudaEventSynchronize(ev[1]));
    float t = 0.f;
    CKE(cudaEventElapsedTime(&t, ev[0], ev[1]));
    ms[q++] = t / reps;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  CKE(cudaGetLastError());
  return WT_OK;
}

// Hidden activation slope (1: identity); takes effect at the next use.
int wt_learned_activation(wt_handle* h, float slope) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  if (!(slope > 0.0f) || slope > 1.0f) return WT_ERR_ARG;
  CKE(cudaStreamSynchronize(E->s()));
  N->slope = slope;
  for (int k = 0; k < 4; ++k) N->it_key[k] = -1;  // the FCG graphs hold the slope
  return WT_OK;
}

// Layer 2 on the tensor cores (1, default) or the CUDA cores (0).
int wt_learned_tensor_cores(wt_handle* h, int on) {
  Ell* E;
  LPNet* N;
  if (int rc = lp_get(h, &E, &N)) return rc;
  if (on != 0 && on != 1) return WT_ERR_ARG;
  CKE(cudaStreamSynchronize(E->s()));
  N->tensor_cores = on;
  for (int k = 0; k < 4; ++k) N->it_key[k] = -1;
  return WT_OK;
}

}  // extern "C"
