// Barotropic elliptic operator, scalar wavelet restriction/prolongation and
// the vector kernels of the multigrid solvers, on the padded lozenge layout.
//
// Ghost cells are read through per-level remap tables instead of being copied:
// nsrc[node] is the node whose value the reference's update_bdry would have
// copied there (itself for owned nodes and for ghosts with no copy entry, such
// as the pole copies), and esrc[edge] is the signed source edge of a ghost edge
// (src/comm.f90:785-808 cp_bdry_inside).  A kernel therefore never needs a
// separate ghost-copy launch, and a ghost always reads its owner's current
// value, which is what the reference's copy produces at the time it is read.
//
// Arithmetic follows the reference expression by expression; the file is built
// with --fmad=false (no contraction) so the FP64 results match the CPU
// restatement bit for bit, reductions excepted (tree order).
#pragma once
#include <cstdint>

namespace wte {

enum { RT = 0, DG = 1, UP = 2 };

struct EllLev {
  int n, P, nd;          // nd = side of a DOMAIN_LEVEL sub-domain at this level
  int64_t NN;
  const double* __restrict__ len;   // 3*NN
  const double* __restrict__ ped;   // 3*NN
  const double* __restrict__ hinv;  // NN
  const double* __restrict__ oa;    // 4*NN overlap areas a(1..4)
  const double* __restrict__ Ie;    // 3*NN interp(csq(a), csq(b)) of each edge's own stencil
  const double* __restrict__ diag;  // NN elliptic_lo_diag
  const int* __restrict__ nsrc;     // NN node read remap
  const int* __restrict__ esrc;     // 3*NN signed edge remap: src*2 + (negate ? 1 : 0)
  const float* __restrict__ Kf;     // 3*NN FP32 coefficient cf*Ie*ped/len (mixed-precision path)
  const float* __restrict__ hinvf;  // NN
  const float* __restrict__ diagf;  // NN
};

__device__ __forceinline__ double interp(double a, double b) { return 0.5 * (a + b); }

__device__ __forceinline__ void decode(const EllLev& L, int t, int& d, int& i, int& j, int m) {
  d = t / (m * m);
  int r = t - d * m * m;
  j = r / m;
  i = r - j * m;
}

__device__ __forceinline__ int64_t nidx(const EllLev& L, int d, int i, int j) {
  return ((int64_t)d * L.P + (j + 2)) * L.P + (i + 2);
}

// Flux of the edge slot through its remap (step1 itype 2, src/ops.f90:202-216):
// interp(csq0, csq1) * (q1/phi1 - q0/phi0) / len * pedlen with phi = 1.
__device__ __forceinline__ double ell_flux(const EllLev& L, const double* __restrict__ q, int64_t slot) {
  const int code = L.esrc[slot];
  const int64_t src = code >> 1;
  const int e = (int)(src / L.NN);
  const int64_t node = src - (int64_t)e * L.NN;
  const double q0 = q[L.nsrc[node]];
  double f;
  if (e == RT) {
    const double q1 = q[L.nsrc[node + 1]];
    f = L.Ie[src] * (q1 / 1.0 - q0 / 1.0) / L.len[src] * L.ped[src];
  } else if (e == DG) {
    const double q2 = q[L.nsrc[node + L.P + 1]];
    f = L.Ie[src] * (q0 / 1.0 - q2 / 1.0) / L.len[src] * L.ped[src];
  } else {
    const double q3 = q[L.nsrc[node + L.P]];
    f = L.Ie[src] * (q3 / 1.0 - q0 / 1.0) / L.len[src] * L.ped[src];
  }
  return (code & 1) ? -f : f;
}

enum { OP_APPLY = 0, OP_JACOBI = 1, OP_RESID = 2 };

// elliptic_lo (src/barotropic_2d.f90:187-250) on [0, n]^2 of one level, fused
// with its consumer: OP_APPLY out = L(q); OP_RESID out = f - L(q) (cal_res,
// src/lin_solve.f90:574); OP_JACOBI out = q + w (f - L(q)) / diag (cal_jacobi,
// src/lin_solve.f90:343).  Ghosts that are copies of another node are not
// computed (every read of them goes to their source).
template <int OP>
__global__ void k_ell_op(EllLev L, double cf, const double* __restrict__ q, const double* __restrict__ f,
                         double* __restrict__ out, double w) {
  const int m = L.n + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  int d, i, j;
  decode(L, t, d, i, j, m);
  const int64_t id = nidx(L, d, i, j);
  if (L.nsrc[id] != id) return;
  const int64_t NN = L.NN, P = L.P;
  const double div = (ell_flux(L, q, RT * NN + id) - ell_flux(L, q, RT * NN + id - 1) + ell_flux(L, q, DG * NN + id - P - 1) -
                      ell_flux(L, q, DG * NN + id) + ell_flux(L, q, UP * NN + id) - ell_flux(L, q, UP * NN + id - P)) *
                     L.hinv[id];
  const double lq = cf * div - q[id];
  if (OP == OP_APPLY) out[id] = lq;
  if (OP == OP_RESID) out[id] = f[id] - lq;
  if (OP == OP_JACOBI) out[id] = q[id] + w * (f[id] - lq) / L.diag[id];
}

// cal_lc (src/lin_solve.f90:529): s = a1 s1 + a2 s2 on [0, n]^2.  The
// coefficients come from device memory when ap1/ap2 are given (solver loops
// that never return to the host), else from a1/a2.
__global__ void k_ell_lc(EllLev L, double* __restrict__ s, double a1, const double* __restrict__ ap1,
                         const double* __restrict__ s1, double a2, const double* __restrict__ ap2, double sgn2,
                         const double* __restrict__ s2) {
  const int m = L.n + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  int d, i, j;
  decode(L, t, d, i, j, m);
  const int64_t id = nidx(L, d, i, j);
  if (L.nsrc[id] != id) return;
  const double c1 = ap1 ? *ap1 : a1;
  const double c2 = ap2 ? sgn2 * *ap2 : a2;
  s[id] = c1 * s1[id] + c2 * s2[id];
}

// Weighted sums of l2 / dp (src/lin_solve.f90:433-502): every (i, j) in
// [0, n]^2 of every lozenge, counted once per DOMAIN_LEVEL sub-domain whose
// (0,1) range contains it.  Block partial sums; k_final_sum adds them in a
// fixed order.
template <int BS>
__global__ void k_ell_dot(EllLev L, const double* __restrict__ a, const double* __restrict__ b,
                          double* __restrict__ partial) {
  __shared__ double sh[BS / 32];
  const int m = L.n + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (t < 10 * m * m) {
    int d, i, j;
    decode(L, t, d, i, j, m);
    const int64_t id = nidx(L, d, i, j);
    const int64_t s = L.nsrc[id];
    const double x = a[s] * b[s];
    const int wi = (i > 0 && i < L.n && i % L.nd == 0) ? 2 : 1;
    const int wj = (j > 0 && j < L.n && j % L.nd == 0) ? 2 : 1;
    v = x;
    if (wi * wj >= 2) v = v + x;
    if (wi * wj == 4) v = v + x + x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < BS / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

// Sum of nb partials by one block in a fixed order; optional sqrt and scaling.
// mode 0: out = sum; 1: out = sqrt(sum); 2: out = sqrt(sum) / *den (res_err).
__global__ void k_final_sum(const double* __restrict__ partial, int nb, double* __restrict__ out, int mode,
                            const double* __restrict__ den) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) v += partial[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (int)(blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) {
      if (mode == 1) v = sqrt(v);
      if (mode == 2) v = sqrt(v) / *den;
      *out = v;
    }
  }
}

// ------------------------------------------------------------- wavelets ----
__device__ __forceinline__ double rdw(const EllLev& L, const double* __restrict__ f, int d, int i, int j) {
  if (i < -2 || j < -2 || i > L.n + 1 || j > L.n + 1) return 0.0;
  return f[L.nsrc[nidx(L, d, i, j)]];
}
__device__ __forceinline__ double oaw(const EllLev& L, int d, int i, int j, int k) {
  if (i < -2 || j < -2 || i > L.n + 1 || j > L.n + 1) return 0.0;
  return L.oa[(int64_t)(k - 1) * L.NN + nidx(L, d, i, j)];
}
// Interp_node (src/wavelet.f90:1487)
__device__ __forceinline__ double interp_node(const EllLev& F, const double* s, int d, int i, int j, int i1, int j1, int i2,
                                              int j2, int i3, int j3, int i4, int j4) {
  return (oaw(F, d, i, j, 1) * rdw(F, s, d, i1, j1) + oaw(F, d, i, j, 2) * rdw(F, s, d, i2, j2) +
          oaw(F, d, i, j, 3) * rdw(F, s, d, i3, j3) + oaw(F, d, i, j, 4) * rdw(F, s, d, i4, j4)) *
         F.hinv[nidx(F, d, i, j)];
}

// Compute_scalar_wavelets (src/wavelet.f90:642) for parents [0, n_c)^2.
__global__ void k_wc_compute(EllLev C, EllLev F, const double* __restrict__ s, double* __restrict__ wc) {
  const int m = C.n;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  int d, ip, jp;
  decode(C, t, d, ip, jp, m);
  const int i = 2 * ip, j = 2 * jp;
  wc[nidx(F, d, i + 1, j)] = rdw(F, s, d, i + 1, j) - interp_node(F, s, d, i + 1, j, i, j, i + 2, j, i + 2, j + 2, i, j - 2);
  wc[nidx(F, d, i + 1, j + 1)] =
      rdw(F, s, d, i + 1, j + 1) - interp_node(F, s, d, i + 1, j + 1, i + 2, j + 2, i, j, i + 2, j, i, j + 2);
  wc[nidx(F, d, i, j + 1)] = rdw(F, s, d, i, j + 1) - interp_node(F, s, d, i, j + 1, i, j, i, j + 2, i - 2, j, i + 2, j + 2);
}

// Restrict_scalar (src/wavelet.f90:520) for parents [0, n_c]^2 (the +1 row
// includes the pole copies); ghost parents that are copies are skipped.
__global__ void k_restrict(EllLev C, EllLev F, const double* __restrict__ sf, const double* __restrict__ wc,
                           double* __restrict__ sc) {
  const int m = C.n + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  int d, ip, jp;
  decode(C, t, d, ip, jp, m);
  const int64_t kp = nidx(C, d, ip, jp);
  if (C.nsrc[kp] != kp) return;
  const int i = 2 * ip, j = 2 * jp;
#define W(a, b, k) (rdw(F, wc, d, i + (a), j + (b)) * oaw(F, d, i + (a), j + (b), k))
  const double sum = W(1, 0, 1) + W(1, 1, 2) + W(2, 1, 3) + W(1, 2, 4) + W(0, 1, 1) + W(-1, 0, 2) + W(-1, 1, 3) +
                     W(-2, -1, 4) + W(-1, -1, 1) + W(0, -1, 2) + W(-1, -2, 3) + W(1, -1, 4);
  sc[kp] = sf[nidx(F, d, i, j)] + sum * C.hinv[kp];
}

// Prolong_scalar (src/wavelet.f90:571; eleven terms, as in the reference) for
// the children (2i, 2j) of parents [0, n_c]^2 that are not copies.
__global__ void k_prolong_even(EllLev C, EllLev F, const double* __restrict__ sc, const double* __restrict__ wc,
                               double* __restrict__ sf) {
  const int m = C.n + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  int d, ip, jp;
  decode(C, t, d, ip, jp, m);
  const int i = 2 * ip, j = 2 * jp;
  const int64_t kc = nidx(F, d, i, j);
  if (F.nsrc[kc] != kc) return;
  const int64_t kp = nidx(C, d, ip, jp);
  const double sum = W(1, 0, 1) + W(1, 1, 2) + W(2, 1, 3) + W(0, 1, 1) + W(-1, 0, 2) + W(-1, 1, 3) + W(-2, -1, 4) +
                     W(-1, -1, 1) + W(0, -1, 2) + W(-1, -2, 3) + W(1, -1, 4);
#undef W
  sf[kc] = sc[C.nsrc[kp]] - sum * C.hinv[kp];
}

// Reconstruct_scalar (src/wavelet.f90:614) for parents [0, n_c)^2.
__global__ void k_prolong_odd(EllLev C, EllLev F, double* __restrict__ s, const double* __restrict__ wc) {
  const int m = C.n;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  int d, ip, jp;
  decode(C, t, d, ip, jp, m);
  const int i = 2 * ip, j = 2 * jp;
  double a = interp_node(F, s, d, i + 1, j, i, j, i + 2, j, i + 2, j + 2, i, j - 2) + rdw(F, wc, d, i + 1, j);
  double b = interp_node(F, s, d, i + 1, j + 1, i + 2, j + 2, i, j, i + 2, j, i, j + 2) + rdw(F, wc, d, i + 1, j + 1);
  double c = interp_node(F, s, d, i, j + 1, i, j, i, j + 2, i - 2, j, i + 2, j + 2) + rdw(F, wc, d, i, j + 1);
  s[nidx(F, d, i + 1, j)] = a;
  s[nidx(F, d, i + 1, j + 1)] = b;
  s[nidx(F, d, i, j + 1)] = c;
}

// ------------------------------------------------ FP32 (mixed precision) ----
// Same operator with per-edge coefficients K = cf*interp(csq)*pedlen/len in
// FP32: L(q) = hinv * sum(+-K (q_b - q_a)) - q.  Used only inside the FP32
// V-cycles of the mixed-precision solver; the outer residual stays FP64.
__device__ __forceinline__ float flux32(const EllLev& L, const float* __restrict__ q, int64_t slot) {
  const int code = L.esrc[slot];
  const int64_t src = code >> 1;
  const int e = (int)(src / L.NN);
  const int64_t node = src - (int64_t)e * L.NN;
  const float q0 = q[L.nsrc[node]];
  float f;
  if (e == RT) f = L.Kf[src] * (q[L.nsrc[node + 1]] - q0);
  else if (e == DG) f = L.Kf[src] * (q0 - q[L.nsrc[node + L.P + 1]]);
  else f = L.Kf[src] * (q[L.nsrc[node + L.P]] - q0);
  return (code & 1) ? -f : f;
}

template <int OP>
__global__ void k_ell_op32(EllLev L, const float* __restrict__ q, const float* __restrict__ f, float* __restrict__ out,
                           float w) {
  const int m = L.n + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 10 * m * m) return;
  int d, i, j;
  decode(L, t, d, i, j, m);
  const int64_t id = nidx(L, d, i, j);
  if (L.nsrc[id] != id) return;
  const int64_t NN = L.NN, P = L.P;
  const float div = (flux32(L, q, RT * NN + id) - flux32(L, q, RT * NN + id - 1) + flux32(L, q, DG * NN + id - P - 1) -
                     flux32(L, q, DG * NN + id) + flux32(L, q, UP * NN + id) - flux32(L, q, UP * NN + id - P)) *
                    L.hinvf[id];
  const float lq = div - q[id];
  if (OP == OP_APPLY) out[id] = lq;
  if (OP == OP_RESID) out[id] = f[id] - lq;
  if (OP == OP_JACOBI) out[id] = q[id] + w * (f[id] - lq) / L.diagf[id];
}

// Operator coefficients of elliptic_lo and elliptic_lo_diag from the old free
// surface eta_old (eta_update keeps it in Laplacian_scalar(S_TEMP),
// src/barotropic_2d.f90:118-129): per edge interp(csq(a), csq(b)) with
// csq = g (|H| phi + eta_old) (src/ops.f90:202-216, phi = 1), the diagonal
// theta1 theta2 (-g 2 sqrt(3) (|H| + eta_old / phi) dt^2 / area) - 1 (the
// exact = .false. branch, :283-296), and their FP32 copies.  eta_old is read
// through the node remap (its ghosts hold their owners' values); with eta_old
// = 0 the results equal those built at setup bit for bit.
__global__ void k_ell_coeffs(int n, int P, int64_t NN, const double* __restrict__ topo, const double* __restrict__ eta,
                             const int* __restrict__ nsrc, const double* __restrict__ len,
                             const double* __restrict__ ped, const double* __restrict__ hinv, double g, double dt,
                             double th1, double th2, double cf, double* __restrict__ Ie, double* __restrict__ diag,
                             float* __restrict__ Kf, float* __restrict__ diagf) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NN) return;
  const int64_t r = k % ((int64_t)P * P);
  const int i = (int)(r % P) - 2, j = (int)(r / P) - 2;
  auto csq = [&](int64_t x) { return g * (fabs(topo[x]) * 1.0 + eta[nsrc[x]]); };
  const double c0 = csq(k);
  if (i + 1 <= n + 1) Ie[RT * NN + k] = 0.5 * (c0 + csq(k + 1));
  if (i + 1 <= n + 1 && j + 1 <= n + 1) Ie[DG * NN + k] = 0.5 * (c0 + csq(k + P + 1));
  if (j + 1 <= n + 1) Ie[UP * NN + k] = 0.5 * (c0 + csq(k + P));
  const double depth = fabs(topo[k]) + eta[nsrc[k]] / 1.0;
  const double wgt = 2.0 * sqrt(3.0) * depth;
  const double lap = -(g * wgt * (dt * dt) * hinv[k]);
  const double dg = th1 * th2 * lap - 1.0;
  diag[k] = dg;
  diagf[k] = (float)dg;
  for (int e = 0; e < 3; ++e) {
    const int64_t q = e * NN + k;
    if (len[q] > 0) Kf[q] = (float)(cf * Ie[q] * ped[q] / len[q]);
  }
}

// compress_scalar (src/adapt.f90:158-172) of one wavelet field: 0 where the
// node mask is below ADJZONE (8).
__global__ void k_compress_wc(int64_t NN, const int* __restrict__ mask_n, double* __restrict__ wc) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < NN && mask_n[k] < 8) wc[k] = 0.0;
}

}  // namespace wte
