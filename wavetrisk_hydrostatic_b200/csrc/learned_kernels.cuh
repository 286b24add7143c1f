// Learned preconditioner of the free-surface solve: a hexagonal-stencil
// convolution network over the nodes of one level, 2 -> 8 -> 8 -> 1 channels.
// Each layer sums over seven taps (the node and its six neighbours in lozenge
// directions (+1,0), (+1,+1), (0,+1), (-1,0), (-1,-1), (0,-1), read through the
// ghost remap) and its input channels:
//   out[co](s) = sum_t sum_ci W[t][ci][co] * in[ci](tap_t(s)).
// The network is linear in the residual (inputs r/rs and (r/rs) * depth
// feature, no biases, identity activations): a fixed, depth-aware linear
// operator of three hops' reach, which generalises from the training
// residuals to any residual.  It corrects what a multigrid V-cycle leaves: the
// preconditioner is z = c + net(r - L c) with c the V-cycle's correction, and
// the network's output is masked to 0 at the pole slots (slots of [0, n]^2
// outside [0, n)^2, whose lozenge-frame taps are degenerate).  The weights
// are FP32 master copies rounded to BF16 for every use (BF16 weights, FP32
// activations and accumulation).  Nodes are numbered compactly: the slots of
// [0, n]^2 of every lozenge that are their own ghost source; a tap that
// leaves that set reads 0.  Activations are channel-major, in[c * ns + s].
//
// Parameter layout (kLpParams floats): W1[7][2][8], W2[7][8][8], W3[7][8][1].
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace wtl {

constexpr int kTaps = 7, kC = 8, kIn = 2;
constexpr int kW1 = 0, kW2 = kW1 + kTaps * kIn * kC, kW3 = kW2 + kTaps * kC * kC, kLpParams = kW3 + kTaps * kC;
constexpr int kDepthRef = 2750;  // depth feature |H| / 2750 m - 1

__device__ __forceinline__ float bf16r(float w) { return __bfloat162float(__float2bfloat16_rn(w)); }

// BF16-rounded copy of the parameters (the weights every kernel below reads).
__global__ void k_lp_round(const float* __restrict__ w, float* __restrict__ wr, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wr[i] = bf16r(w[i]);
}

template <int NT>
__device__ __forceinline__ void block_partial(double v, double* __restrict__ partial) {
  __shared__ double sh[NT / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int q = 0; q < NT / 32; ++q) a += sh[q];
    partial[blockIdx.x] = a;
  }
}

// Block partials of sum_s a(s) b(s) w(s) over the nodes; a, b, w level arrays
// read at slot[s] (slot == nullptr: compact arrays), w == nullptr: weight 1,
// otherwise weight 1 / w (w = hex_inv: the area-weighted inner product in which
// the free-surface operator is symmetric up to its discretisation).
template <int NT>
__global__ void __launch_bounds__(NT) k_lp_dot(int ns, const int* __restrict__ slot, const double* __restrict__ a,
                                               const double* __restrict__ b, const double* __restrict__ w,
                                               double* __restrict__ partial) {
  const int s = blockIdx.x * NT + threadIdx.x;
  double v = 0.0;
  if (s < ns) {
    const int id = slot ? slot[s] : s;
    v = a[id] * b[id];
    if (w) v /= w[id];
  }
  block_partial<NT>(v, partial);
}

// out = scale * (sum of nb partials, fixed order); mode 1: the square root of
// that, replaced by 1 where it is 0 or not finite (the residual scale).
__global__ void k_lp_sum(const double* __restrict__ partial, int nb, double* __restrict__ out, int mode,
                         double scale) {
  __shared__ double sh[256];
  double v = 0.0;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) v += partial[q];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double r = sh[0] * scale;
    if (mode == 1) {
      r = sqrt(r);
      if (!(r > 0.0) || !isfinite(r)) r = 1.0;
    }
    out[0] = r;
  }
}

// Network input of every node: the residual scaled by 1 / rscale, and the same
// times the depth feature |H| / 2750 m - 1.  r read at slot[s] (nullptr:
// compact), topo at tslot[s].
__global__ void k_lp_input(int ns, const int* __restrict__ slot, const int* __restrict__ tslot,
                           const double* __restrict__ r, const double* __restrict__ rscale,
                           const double* __restrict__ topo, float* __restrict__ x) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const double inv = 1.0 / *rscale;
  const float v = (float)(r[slot ? slot[s] : s] * inv);
  x[s] = v;
  x[ns + s] = v * (float)(fabs(topo[tslot[s]]) / (double)kDepthRef - 1.0);
}

// One convolution layer, one thread per node computing all COUT outputs from
// the 7 x CIN tap inputs; BF16-valued weights staged in shared memory.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_lp_conv(int ns, const int* __restrict__ tap, const float* __restrict__ in,
                                                 const float* __restrict__ W, float* __restrict__ out) {
  __shared__ float sw[kTaps * CIN * COUT];
  for (int q = threadIdx.x; q < kTaps * CIN * COUT; q += blockDim.x) sw[q] = W[q];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = 0.0f;
  for (int t = 0; t < kTaps; ++t) {
    const int u = tap[t * ns + s];
    if (u < 0) continue;
    for (int ci = 0; ci < CIN; ++ci) {
      const float v = in[ci * ns + u];
      const float* w = sw + (t * CIN + ci) * COUT;
#pragma unroll
      for (int co = 0; co < COUT; ++co) acc[co] = fmaf(w[co], v, acc[co]);
    }
  }
#pragma unroll
  for (int co = 0; co < COUT; ++co) out[co * ns + s] = acc[co];
}

// The first layer with the input built on the fly, for the solver: the input
// of tap node u is v = (r - lc)(slot[u]) (FP64 difference, then FP32) and
// v * depth feature; the values k_lp_input gives for r - lc at rscale 1.
__global__ void __launch_bounds__(128) k_lp_conv_in(int ns, const int* __restrict__ tap, const int* __restrict__ slot,
                                                    const double* __restrict__ r, const double* __restrict__ lc,
                                                    const double* __restrict__ topo, const float* __restrict__ W,
                                                    float* __restrict__ out) {
  __shared__ float sw[kTaps * kIn * kC];
  for (int q = threadIdx.x; q < kTaps * kIn * kC; q += blockDim.x) sw[q] = W[q];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  float acc[kC];
#pragma unroll
  for (int co = 0; co < kC; ++co) acc[co] = 0.0f;
  for (int t = 0; t < kTaps; ++t) {
    const int u = tap[t * ns + s];
    if (u < 0) continue;
    const int id = slot[u];
    const float v = (float)(r[id] - lc[id]);
    const float x[kIn] = {v, v * (float)(fabs(topo[id]) / (double)kDepthRef - 1.0)};
#pragma unroll
    for (int ci = 0; ci < kIn; ++ci) {
      const float* w = sw + (t * kIn + ci) * kC;
#pragma unroll
      for (int co = 0; co < kC; ++co) acc[co] = fmaf(w[co], x[ci], acc[co]);
    }
  }
#pragma unroll
  for (int co = 0; co < kC; ++co) out[co * ns + s] = acc[co];
}

// The last layer fused with the solver's output: z(slot[s]) = base(slot[s]) +
// own * y(s), y the 1-channel convolution of in.
__global__ void __launch_bounds__(128) k_lp_conv_out(int ns, const int* __restrict__ tap, const int* __restrict__ slot,
                                                     const float* __restrict__ in, const float* __restrict__ W,
                                                     const float* __restrict__ own, const double* __restrict__ base,
                                                     double* __restrict__ z) {
  __shared__ float sw[kTaps * kC];
  for (int q = threadIdx.x; q < kTaps * kC; q += blockDim.x) sw[q] = W[q];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  float acc = 0.0f;
  for (int t = 0; t < kTaps; ++t) {
    const int u = tap[t * ns + s];
    if (u < 0) continue;
#pragma unroll
    for (int ci = 0; ci < kC; ++ci) acc = fmaf(sw[t * kC + ci], in[ci * ns + u], acc);
  }
  const int id = slot[s];
  z[id] = base[id] + (double)(own[s] * acc);
}

// z = base + own * rscale * y into slot[s] of a level array (nullptr:
// compact; base == nullptr: 0), own = 1 on the owned nodes, 0 at the poles.
__global__ void k_lp_output(int ns, const int* __restrict__ slot, const float* __restrict__ y,
                            const double* __restrict__ rscale, const float* __restrict__ own,
                            const double* __restrict__ base, double* __restrict__ z) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const int id = slot ? slot[s] : s;
  z[id] = (base ? base[id] : 0.0) + (double)(own[s] * y[s]) * *rscale;
}


// Training loss: the error of the network in the energy norm of the solve,
//   loss = <d, -L d>_W / |W|,  d = own y - e / rscale,  W = 1 / hex_inv (cell area),
// the norm flexible CG minimises (-L is positive definite in <,>_W).
// k_lp_err writes d on the node slots of a level array; after Ld = L d,
// k_lp_aloss forms the loss partials and dy = 2 W (-Ld) / |W|.
__global__ void k_lp_err(int ns, const int* __restrict__ slot, const float* __restrict__ y,
                         const float* __restrict__ own, const double* __restrict__ e,
                         const double* __restrict__ rscale, double* __restrict__ d) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) d[slot[s]] = (double)(own[s] * y[s]) - e[s] / *rscale;
}
template <int NT>
__global__ void __launch_bounds__(NT) k_lp_aloss(int ns, const int* __restrict__ slot, const double* __restrict__ d,
                                                 const double* __restrict__ Ld, const double* __restrict__ hinv,
                                                 const float* __restrict__ own, double inv_area,
                                                 float* __restrict__ dy, double* __restrict__ partial) {
  const int s = blockIdx.x * NT + threadIdx.x;
  double v = 0.0;
  if (s < ns) {
    const int id = slot[s];
    const double a = -Ld[id] / hinv[id];
    dy[s] = own[s] * (float)(2.0 * a * inv_area);
    v = d[id] * a;
  }
  block_partial<NT>(v, partial);
}

// Weight gradient of one layer: dW[t][ci][co] = sum_s dz[co](s) *
// in[ci](tap_t(s)).  A block stages a chunk of kChunk nodes (their tap inputs
// A[s][t*CIN+ci] and dz) in shared memory; each thread owns fixed entries of
// the gradient and sums them over the block's chunks, then adds them once to
// the global gradient.
constexpr int kChunk = 32;
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_lp_wgrad(int ns, const int* __restrict__ tap, const float* __restrict__ in,
                                                  const float* __restrict__ dz, float* __restrict__ dW) {
  constexpr int K = kTaps * CIN;             // rows of A
  constexpr int NE = K * COUT;               // gradient entries
  constexpr int PER = (NE + 255) / 256;      // entries per thread
  __shared__ float A[kChunk][K];
  __shared__ float G[kChunk][COUT];
  float acc[PER];
#pragma unroll
  for (int r = 0; r < PER; ++r) acc[r] = 0.0f;
  const int nchunk = (ns + kChunk - 1) / kChunk;
  for (int c = blockIdx.x; c < nchunk; c += gridDim.x) {
    const int s0 = c * kChunk;
    __syncthreads();
    for (int q = threadIdx.x; q < kChunk * K; q += 256) {
      const int nl = q / K, k = q % K, s = s0 + nl;
      float v = 0.0f;
      if (s < ns) {
        const int t = k / CIN, ci = k % CIN, u = tap[t * ns + s];
        v = u >= 0 ? in[ci * ns + u] : 0.0f;
      }
      A[nl][k] = v;
    }
    for (int q = threadIdx.x; q < kChunk * COUT; q += 256) {
      const int co = q / kChunk, nl = q % kChunk, s = s0 + nl;
      G[nl][co] = s < ns ? dz[co * ns + s] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < PER; ++r) {
      const int e = threadIdx.x + 256 * r;
      if (e < NE) {
        const int k = e / COUT, co = e % COUT;
        float a = acc[r];
#pragma unroll 8
        for (int nl = 0; nl < kChunk; ++nl) a = fmaf(A[nl][k], G[nl][co], a);
        acc[r] = a;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int e = threadIdx.x + 256 * r;
    if (e < NE) {
      atomicAdd(&dW[e], acc[r]);
    }
  }
}

// Input gradient of one layer: din[ci](tap_t(s)) += sum_co W[t][ci][co] *
// dz[co](s), scattered to the tap's node.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_lp_igrad(int ns, const int* __restrict__ tap, const float* __restrict__ W,
                                                  const float* __restrict__ dz, float* __restrict__ din) {
  __shared__ float sw[kTaps * CIN * COUT];
  for (int q = threadIdx.x; q < kTaps * CIN * COUT; q += blockDim.x) sw[q] = W[q];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  float g[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) g[co] = dz[co * ns + s];
  for (int t = 0; t < kTaps; ++t) {
    const int u = tap[t * ns + s];
    if (u < 0) continue;
    for (int ci = 0; ci < CIN; ++ci) {
      const float* w = sw + (t * CIN + ci) * COUT;
      float a = 0.0f;
#pragma unroll
      for (int co = 0; co < COUT; ++co) a = fmaf(w[co], g[co], a);
      atomicAdd(&din[ci * ns + u], a);
    }
  }
}

// Adam step on the FP32 master parameters (bias-corrected; step t >= 1).
__global__ void k_lp_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, float lr, float b1, float b2, float eps, int t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.0f - powf(b1, (float)t)), vh = vi / (1.0f - powf(b2, (float)t));
  w[i] -= lr * mh / (sqrtf(vh) + eps);
}

// Compact <-> level copies: dst[s] = src[slot[s]] and dst[slot[s]] = src[s].
__global__ void k_lp_gather(int ns, const int* __restrict__ slot, const double* __restrict__ src,
                            double* __restrict__ dst) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) dst[s] = src[slot[s]];
}
__global__ void k_lp_scatter(int ns, const int* __restrict__ slot, const double* __restrict__ src,
                             double* __restrict__ dst) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) dst[slot[s]] = src[s];
}
// e = a - b on the nodes (compact output).
__global__ void k_lp_diff(int ns, const int* __restrict__ slot, const double* __restrict__ a,
                          const double* __restrict__ b, double* __restrict__ e) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) e[s] = a[slot[s]] - b[slot[s]];
}

// ---------------------------------------------------------- flexible CG ----
// Device scalars of the flexible CG recurrences (fcg[]):
enum { FCG_ZLP = 0, FCG_DELTA_PREV = 1, FCG_PR = 2, FCG_DELTA = 3, FCG_RNORM = 4, FCG_BREAK = 5, FCG_N = 8 };

// z = -r on the nodes (no preconditioner: plain CG on -L).
__global__ void k_fcg_neg(int ns, const int* __restrict__ slot, const double* __restrict__ r, double* __restrict__ z) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) z[slot[s]] = -r[slot[s]];
}

// New direction, truncated to one previous direction: beta = <z, Lp'> / <p', Lp'>,
// p = z - beta p', Lp = Lz - beta Lp' (on a restart, FCG_DELTA_PREV == 0: p = z,
// Lp = Lz); fused with the two inner products the step needs, block partials of
// <p, r>_W and <p, Lp>_W (W = 1 / hinv) into pa and pb.
template <int NT>
__global__ void __launch_bounds__(NT) k_fcg_dir_dots(int ns, const int* __restrict__ slot,
                                                     const double* __restrict__ fcg, const double* __restrict__ z,
                                                     const double* __restrict__ lz, const double* __restrict__ r,
                                                     const double* __restrict__ hinv, double* __restrict__ p,
                                                     double* __restrict__ lp, double* __restrict__ pa,
                                                     double* __restrict__ pb) {
  __shared__ double sa[NT / 32], sb[NT / 32];
  const int s = blockIdx.x * NT + threadIdx.x;
  double va = 0.0, vb = 0.0;
  if (s < ns) {
    const double dprev = fcg[FCG_DELTA_PREV];
    const int id = slot[s];
    double pn, lpn;
    if (dprev == 0.0) {
      pn = z[id];
      lpn = lz[id];
    } else {
      const double beta = fcg[FCG_ZLP] / dprev;
      pn = z[id] - beta * p[id];
      lpn = lz[id] - beta * lp[id];
    }
    p[id] = pn;
    lp[id] = lpn;
    va = pn * r[id] / hinv[id];
    vb = pn * lpn / hinv[id];
  }
  for (int o = 16; o > 0; o >>= 1) {
    va += __shfl_down_sync(0xffffffffu, va, o);
    vb += __shfl_down_sync(0xffffffffu, vb, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = va;
    sb[threadIdx.x >> 5] = vb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int q = 0; q < NT / 32; ++q) {
      a += sa[q];
      b += sb[q];
    }
    pa[blockIdx.x] = a;
    pb[blockIdx.x] = b;
  }
}

// out[0] = sum of pa, out[1] = sum of pb (nb partials each, fixed order).
__global__ void k_lp_sum2(const double* __restrict__ pa, const double* __restrict__ pb, int nb,
                          double* __restrict__ out0, double* __restrict__ out1) {
  __shared__ double sa[256], sb[256];
  double a = 0.0, b = 0.0;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) {
    a += pa[q];
    b += pb[q];
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sa[threadIdx.x] += sa[threadIdx.x + o];
      sb[threadIdx.x] += sb[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *out0 = sa[0];
    *out1 = sb[0];
  }
}

// Step: alpha = <p, r> / <p, Lp>; u += alpha p; r -= alpha Lp.  <p, Lp> must be
// negative and finite (L is negative definite); otherwise nothing is updated
// and FCG_BREAK is set.  Thread 0 of block 0 keeps <p, Lp> for the next beta.
__global__ void k_fcg_step(int ns, const int* __restrict__ slot, double* __restrict__ fcg,
                           const double* __restrict__ p, const double* __restrict__ lp, double* __restrict__ u,
                           double* __restrict__ r) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const double delta = fcg[FCG_DELTA], pr = fcg[FCG_PR];
  const bool ok = delta < 0.0 && isfinite(delta) && isfinite(pr);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (ok) fcg[FCG_DELTA_PREV] = delta;
    else fcg[FCG_BREAK] = 1.0;
  }
  if (!ok || s >= ns) return;
  const double alpha = pr / delta;
  const int id = slot[s];
  u[id] += alpha * p[id];
  r[id] -= alpha * lp[id];
}

// Ghost slots of a level field from their sources: q[k] = q[nsrc[k]].
__global__ void k_lp_fill_ghost(int64_t NN, const int* __restrict__ nsrc, double* __restrict__ q) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < NN && nsrc[k] != k) q[k] = q[nsrc[k]];
}

}  // namespace wtl
