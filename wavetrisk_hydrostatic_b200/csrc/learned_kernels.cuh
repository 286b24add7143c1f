// Learned preconditioner of the free-surface solve: a hexagonal-stencil
// convolution network over the nodes of one level, 2 -> 32 -> 32 -> 1
// channels.  Each layer sums over seven taps (the node and its six neighbours
// in lozenge directions (+1,0), (+1,+1), (0,+1), (-1,0), (-1,-1), (0,-1), read
// through the ghost remap) and its input channels:
//   out[co](s) = sum_t sum_ci W[t][ci][co] * in[ci](tap_t(s)),
// the two hidden layers followed by the activation act(p) = p (p > 0),
// slope * p (p <= 0) (slope 1: the identity) and stored in BF16.  No biases:
// the network is positively homogeneous, net(a r) = a net(r) for a > 0, so the
// solver runs it on the unscaled residual.  It corrects what a multigrid
// V-cycle leaves: the preconditioner is z = c + net(r - L c) with c the
// V-cycle's correction, and the network's output is masked to 0 at the pole
// slots (slots of [0, n]^2 outside [0, n)^2, whose lozenge-frame taps are
// degenerate).  The weights are FP32 master copies rounded to BF16 for every
// use; activations are BF16, accumulation FP32.  The middle layer, a
// 224 x 32 contraction per node, runs on the tensor cores (tcgen05, BF16
// operands, FP32 accumulator in tensor memory).  Nodes are numbered compactly:
// the slots of [0, n]^2 of every lozenge that are their own ghost source; a
// tap that leaves that set reads 0.  Activations are node-major, h[s][c].
//
// Parameter layout (kLpParams floats): W1[7][2][32], W2[7][32][32], W3[7][32][1].
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "umma.cuh"

namespace wtl {

constexpr int kTaps = 7, kC = 32, kIn = 2;
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

// Network input of every node, node-major x[2 s + c]: the residual scaled by
// 1 / rscale, and the same times the depth feature |H| / 2750 m - 1.  r read
// at slot[s] (nullptr: compact), topo at tslot[s].
__global__ void k_lp_input(int ns, const int* __restrict__ slot, const int* __restrict__ tslot,
                           const double* __restrict__ r, const double* __restrict__ rscale,
                           const double* __restrict__ topo, float* __restrict__ x) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const double inv = 1.0 / *rscale;
  const float v = (float)(r[slot ? slot[s] : s] * inv);
  x[2 * s] = v;
  x[2 * s + 1] = v * (float)(fabs(topo[tslot[s]]) / (double)kDepthRef - 1.0);
}

__device__ __forceinline__ float lp_act(float p, float slope) { return p > 0.0f ? p : slope * p; }
// Derivative of the activation from its stored (BF16) output: the sign of the
// output is the sign of its argument.
__device__ __forceinline__ float lp_dact(float h, float slope) { return h > 0.0f ? 1.0f : slope; }

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);  // a in the low half
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ void unpack_bf16x8(const uint4& q, float (&f)[8]) {
  const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f[2 * k] = __uint_as_float(w[k] << 16);
    f[2 * k + 1] = __uint_as_float(w[k] & 0xFFFF0000u);
  }
}

// Layer 1 (2 -> 32) with the activation, BF16 output h1[s][32] (64 bytes a
// node).  The input of tap node u is x[u] (x != nullptr, training and
// inference on compact residuals) or, for the solver, built on the fly from
// the level arrays at slot[u]: v = (r - lc) (FP64 difference, then FP32) and
// v * depth feature, the values k_lp_input gives for r - lc at rscale 1.
__global__ void __launch_bounds__(128) k_lp_l1(int ns, const int* __restrict__ tap, const float* __restrict__ x,
                                               const int* __restrict__ slot, const double* __restrict__ r,
                                               const double* __restrict__ lc, const double* __restrict__ topo,
                                               const float* __restrict__ W, float slope, uint4* __restrict__ h1) {
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
    float x0, x1;
    if (x) {
      const float2 v = reinterpret_cast<const float2*>(x)[u];
      x0 = v.x;
      x1 = v.y;
    } else {
      const int id = slot[u];
      x0 = (float)(r[id] - lc[id]);
      x1 = x0 * (float)(fabs(topo[id]) / (double)kDepthRef - 1.0);
    }
    const float* w0 = sw + (t * kIn) * kC;
#pragma unroll
    for (int co = 0; co < kC; ++co) acc[co] = fmaf(w0[co], x0, acc[co]);
#pragma unroll
    for (int co = 0; co < kC; ++co) acc[co] = fmaf(w0[kC + co], x1, acc[co]);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint4 o;
    o.x = pack_bf16x2(lp_act(acc[8 * q + 0], slope), lp_act(acc[8 * q + 1], slope));
    o.y = pack_bf16x2(lp_act(acc[8 * q + 2], slope), lp_act(acc[8 * q + 3], slope));
    o.z = pack_bf16x2(lp_act(acc[8 * q + 4], slope), lp_act(acc[8 * q + 5], slope));
    o.w = pack_bf16x2(lp_act(acc[8 * q + 6], slope), lp_act(acc[8 * q + 7], slope));
    h1[4 * (int64_t)s + q] = o;
  }
}

// ------------------------------------------------ layer 2 on tensor cores ----
// h2 = act(conv(h1)) as one GEMM per tile of 128 nodes: A[m][k] =
// h1[tap_t(s0+m)][ci] (k = 32 t + ci, K = 224, gathered into shared memory),
// B[n][k] = W2[t][ci][n] (BF16, packed once per weight update), D = A B^T
// (128 x 32, FP32) in tensor memory: 14 tcgen05.mma of K 16, one commit to an
// mbarrier, then each warp reads 16 columns of its 32 lanes.  Persistent CTAs
// (grid <= tiles) keep B and the 32 tensor-memory columns over their tiles.
// The gather is a set of 16-byte cp.async copies of whole 8-channel chunks
// (zero-filled for taps outside the node set), issued before the previous
// tile's epilogue so its latency overlaps it.
constexpr int kL2M = 128;
constexpr int kL2Ksteps = kTaps * kC / 16;         // 14
constexpr int kL2StepA = 2 * (kL2M / 8) * 128;     // bytes of A per K step: 2 core columns x 16 row groups
constexpr int kL2StepB = 2 * (kC / 8) * 128;       // bytes of B per K step: 2 core columns x 4 row groups
constexpr int kL2ABytes = kL2Ksteps * kL2StepA;    // 57344
constexpr int kL2BBytes = kL2Ksteps * kL2StepB;    // 14336 (= 2 * kTaps * kC * kC)
constexpr int kL2Smem = kL2ABytes + kL2BBytes + 16;
constexpr int kL2Threads = 256;
constexpr unsigned long long kL2WaitNs = 1000000000ull;  // a CTA gives up on its MMAs after 1 s

// Element (n, k) of the packed B at byte 2 * index: K step k / 16, core
// column (k % 16) / 8, row group n / 8, row n % 8, element k % 8.
__global__ void k_lp_pack_w2(const float* __restrict__ wr, __nv_bfloat16* __restrict__ wpk) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kTaps * kC * kC) return;
  const int ks = idx / 512, rem = idx % 512, kc = rem / 256, g = (rem % 256) / 64, row = (rem % 64) / 8, e = rem % 8;
  const int n = 8 * g + row, k = 16 * ks + 8 * kc + e, t = k / kC, ci = k % kC;
  wpk[idx] = __float2bfloat16_rn(wr[kW2 + (t * kC + ci) * kC + n]);
}

__device__ __forceinline__ void lp_mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool lp_mbar_wait(uint32_t bar, unsigned parity, unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  for (int it = 0;; ++it) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (it == 0) t0 = t;
    else if (t - t0 > limit_ns) return false;
  }
}

// 16-byte global -> shared copy (cp.async, L2 only); src_bytes 0 fills zeros.
__device__ __forceinline__ void cp16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Gather item j of this thread: the 16-byte chunk q (channels 8q..8q+7) of
// tap t of tile row m, item = tid + kL2Threads j.
constexpr int kL2Items = kTaps * kL2M * 4 / kL2Threads;  // 14
__device__ __forceinline__ void l2_item(int tid, int j, int& t, int& m, int& q) {
  const int item = tid + kL2Threads * j;
  q = item & 3;
  m = (item >> 2) & (kL2M - 1);
  t = item >> 9;
}
__device__ __forceinline__ void l2_taps(const int* __restrict__ tap, int ns, int tile, int ntiles, int tid,
                                        int (&tp)[kL2Items]) {
#pragma unroll
  for (int j = 0; j < kL2Items; ++j) {
    int t, m, q;
    l2_item(tid, j, t, m, q);
    const int s = tile * kL2M + m;
    tp[j] = (tile < ntiles && s < ns) ? __ldg(tap + (int64_t)t * ns + s) : -1;
  }
}
__device__ __forceinline__ void l2_gather(uint32_t aaddr, const uint4* __restrict__ h1, int tid,
                                          const int (&tp)[kL2Items]) {
#pragma unroll
  for (int j = 0; j < kL2Items; ++j) {
    int t, m, q;
    l2_item(tid, j, t, m, q);
    const int off = (2 * t + (q >> 1)) * kL2StepA + (q & 1) * (kL2StepA / 2) + (m >> 3) * 128 + (m & 7) * 16;
    const int u = tp[j];
    cp16(aaddr + off, u >= 0 ? (const void*)(h1 + 4 * (int64_t)u + q) : (const void*)h1, u >= 0 ? 16u : 0u);
  }
}

// Persistent CTAs over the tiles, the gather of tile i+1 (cp.async straight
// into the operand layout) in flight while tile i's accumulator is read back
// and stored; the tap indices are fetched a tile further ahead.
__global__ void __launch_bounds__(kL2Threads) k_lp_l2_umma(int ns, const int* __restrict__ tap,
                                                           const uint4* __restrict__ h1,
                                                           const uint4* __restrict__ wpk, float slope,
                                                           uint4* __restrict__ h2, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* sA = sm;
  unsigned char* sB = sm + kL2ABytes;
  uint64_t* bar_p = reinterpret_cast<uint64_t*>(sm + kL2ABytes + kL2BBytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kL2ABytes + kL2BBytes + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t aaddr = umma::smem_u32(sA), baddr = umma::smem_u32(sB), bar = umma::smem_u32(bar_p);
  const int ntiles = (ns + kL2M - 1) / kL2M;
  const int stride = gridDim.x;
  int tile = blockIdx.x;

  int tp[kL2Items];
  l2_taps(tap, ns, tile, ntiles, tid, tp);
  for (int q = tid; q < kL2BBytes / 16; q += kL2Threads) cp16(baddr + 16 * q, wpk + q, 16u);
  l2_gather(aaddr, h1, tid, tp);
  cp_commit();
  l2_taps(tap, ns, tile + stride, ntiles, tid, tp);
  if (tid == 0) lp_mbar_init(bar);
  if (warp == 0) umma::tmem_alloc(tslot, 32);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  constexpr uint32_t kIdesc = umma::idesc_bf16_f32(kL2M, kC);

  unsigned parity = 0;
  for (; tile < ntiles; tile += stride) {
    cp_wait_all();
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < kL2Ksteps; ++ks) {
        const uint64_t ad = umma::desc_kmajor(aaddr + ks * kL2StepA, kL2StepA / 2, 128);
        const uint64_t bd = umma::desc_kmajor(baddr + ks * kL2StepB, kL2StepB / 2, 128);
        umma::mma_bf16(tmem, ad, bd, kIdesc, ks > 0);
      }
      umma::commit_arrive(bar);
    }
    const bool ok = lp_mbar_wait(bar, parity, kL2WaitNs);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicCAS(err, 0, 1);
      if (!ok) lp_mbar_wait(bar, parity, kL2WaitNs);  // the MMAs still read shared memory
      break;
    }
    parity ^= 1u;
    // the operand buffer is free: start the next tile's gather, then its successor's taps
    const int next = tile + stride;
    if (next < ntiles) {
      l2_gather(aaddr, h1, tid, tp);
      cp_commit();
      l2_taps(tap, ns, next + stride, ntiles, tid, tp);
    }
    umma::fence_after_sync();
    float d[16];
    const int quarter = warp & 3, half = warp >> 2;
    umma::tmem_ld16(tmem + ((uint32_t)(32 * quarter) << 16) + 16 * half, d);
    const int s = tile * kL2M + 32 * quarter + lane;
    if (s < ns) {
      uint4 o0, o1;
      o0.x = pack_bf16x2(lp_act(d[0], slope), lp_act(d[1], slope));
      o0.y = pack_bf16x2(lp_act(d[2], slope), lp_act(d[3], slope));
      o0.z = pack_bf16x2(lp_act(d[4], slope), lp_act(d[5], slope));
      o0.w = pack_bf16x2(lp_act(d[6], slope), lp_act(d[7], slope));
      o1.x = pack_bf16x2(lp_act(d[8], slope), lp_act(d[9], slope));
      o1.y = pack_bf16x2(lp_act(d[10], slope), lp_act(d[11], slope));
      o1.z = pack_bf16x2(lp_act(d[12], slope), lp_act(d[13], slope));
      o1.w = pack_bf16x2(lp_act(d[14], slope), lp_act(d[15], slope));
      h2[4 * (int64_t)s + 2 * half] = o0;
      h2[4 * (int64_t)s + 2 * half + 1] = o1;
    }
  }
  cp_wait_all();  // a CTA leaving early (timeout) still has its copies land before it exits
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_free(tmem, 32);
  }
}

// Layer 2 on the CUDA cores (the same sums in FP32, one thread a node): the
// variant for comparison with the tensor-core kernel.
__global__ void __launch_bounds__(128) k_lp_l2_simt(int ns, const int* __restrict__ tap, const uint4* __restrict__ h1,
                                                    const float* __restrict__ W, float slope,
                                                    uint4* __restrict__ h2) {
  __shared__ __align__(16) float sw[kTaps * kC * kC];
  for (int q = threadIdx.x; q < kTaps * kC * kC; q += blockDim.x) sw[q] = W[q];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  float acc[kC];
#pragma unroll
  for (int co = 0; co < kC; ++co) acc[co] = 0.0f;
  for (int t = 0; t < kTaps; ++t) {
    const int u = tap[t * ns + s];
    if (u < 0) continue;
    for (int q = 0; q < 4; ++q) {
      float f[8];
      unpack_bf16x8(h1[4 * (int64_t)u + q], f);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const float4* w = reinterpret_cast<const float4*>(sw + (t * kC + 8 * q + e) * kC);
#pragma unroll
        for (int c4 = 0; c4 < kC / 4; ++c4) {
          const float4 ww = w[c4];
          acc[4 * c4] = fmaf(ww.x, f[e], acc[4 * c4]);
          acc[4 * c4 + 1] = fmaf(ww.y, f[e], acc[4 * c4 + 1]);
          acc[4 * c4 + 2] = fmaf(ww.z, f[e], acc[4 * c4 + 2]);
          acc[4 * c4 + 3] = fmaf(ww.w, f[e], acc[4 * c4 + 3]);
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint4 o;
    o.x = pack_bf16x2(lp_act(acc[8 * q + 0], slope), lp_act(acc[8 * q + 1], slope));
    o.y = pack_bf16x2(lp_act(acc[8 * q + 2], slope), lp_act(acc[8 * q + 3], slope));
    o.z = pack_bf16x2(lp_act(acc[8 * q + 4], slope), lp_act(acc[8 * q + 5], slope));
    o.w = pack_bf16x2(lp_act(acc[8 * q + 6], slope), lp_act(acc[8 * q + 7], slope));
    h2[4 * (int64_t)s + q] = o;
  }
}

// Layer 3 (32 -> 1, no activation): y[s] (z == nullptr), or fused with the
// solver's output, z(slot[s]) = base(slot[s]) + own * y(s).
__global__ void __launch_bounds__(128) k_lp_l3(int ns, const int* __restrict__ tap, const uint4* __restrict__ h2,
                                               const float* __restrict__ W, float* __restrict__ y,
                                               const int* __restrict__ slot, const float* __restrict__ own,
                                               const double* __restrict__ base, double* __restrict__ z) {
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
    for (int q = 0; q < 4; ++q) {
      float f[8];
      unpack_bf16x8(h2[4 * (int64_t)u + q], f);
#pragma unroll
      for (int e = 0; e < 8; ++e) acc = fmaf(sw[t * kC + 8 * q + e], f[e], acc);
    }
  }
  if (z) {
    const int id = slot[s];
    z[id] = base[id] + (double)(own[s] * acc);
  } else {
    y[s] = acc;
  }
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

// Input value ci of node u for the weight gradient: FP32 (the network input)
// or BF16 (the stored activations), node-major.
__device__ __forceinline__ float lp_in(const float* a, int64_t i) { return a[i]; }
__device__ __forceinline__ float lp_in(const __nv_bfloat16* a, int64_t i) { return __bfloat162float(a[i]); }

// Weight gradient of one layer: dW[t][ci][co] = sum_s dz(s)[co] *
// in(tap_t(s))[ci], in and dz node-major.  A block stages a chunk of kChunk
// nodes (their tap inputs A[s][t*CIN+ci] and dz) in shared memory; each
// thread owns fixed entries of the gradient and sums them over the block's
// chunks, then adds them once to the global gradient.
constexpr int kChunk = 32;
template <int CIN, int COUT, class TIn>
__global__ void __launch_bounds__(256) k_lp_wgrad(int ns, const int* __restrict__ tap, const TIn* __restrict__ in,
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
        v = u >= 0 ? lp_in(in, (int64_t)u * CIN + ci) : 0.0f;
      }
      A[nl][k] = v;
    }
    for (int q = threadIdx.x; q < kChunk * COUT; q += 256) {
      const int nl = q / COUT, co = q % COUT, s = s0 + nl;
      G[nl][co] = s < ns ? dz[(int64_t)s * COUT + co] : 0.0f;
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
    if (e < NE) atomicAdd(&dW[e], acc[r]);
  }
}

// Gradient at the input of one layer, gathered: for node u,
//   dh(u)[ci] = sum over (s, t) with tap_t(s) = u of sum_co W[t][ci][co] dz(s)[co],
// the pairs listed in the inverse tap table (inv[inv_ptr[u] .. inv_ptr[u+1]),
// entry 8 s + t), then through the activation whose stored output is h(u):
// dzin(u)[ci] = dh(u)[ci] * act'(h(u)[ci]).  Node-major FP32 output.
template <int COUT>
__global__ void __launch_bounds__(128) k_lp_igrad(int ns, const int* __restrict__ inv_ptr,
                                                  const int* __restrict__ inv, const float* __restrict__ W,
                                                  const float* __restrict__ dz, const __nv_bfloat16* __restrict__ h,
                                                  float slope, float* __restrict__ dzin) {
  __shared__ __align__(16) float sw[kTaps * kC * COUT];
  for (int q = threadIdx.x; q < kTaps * kC * COUT; q += blockDim.x) sw[q] = W[q];
  __syncthreads();
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ns) return;
  float acc[kC];
#pragma unroll
  for (int ci = 0; ci < kC; ++ci) acc[ci] = 0.0f;
  const int e1 = inv_ptr[u + 1];
  for (int e = inv_ptr[u]; e < e1; ++e) {
    const int ent = inv[e], s = ent >> 3, t = ent & 7;
    if (COUT == 1) {
      const float g = dz[s];
#pragma unroll
      for (int ci = 0; ci < kC; ++ci) acc[ci] = fmaf(sw[t * kC + ci], g, acc[ci]);
    } else {
      float g[COUT];
#pragma unroll
      for (int c4 = 0; c4 < COUT / 4; ++c4) {
        const float4 v = reinterpret_cast<const float4*>(dz + (int64_t)s * COUT)[c4];
        g[4 * c4] = v.x;
        g[4 * c4 + 1] = v.y;
        g[4 * c4 + 2] = v.z;
        g[4 * c4 + 3] = v.w;
      }
#pragma unroll
      for (int ci = 0; ci < kC; ++ci) {
        const float4* w = reinterpret_cast<const float4*>(sw + (t * kC + ci) * COUT);
        float a = acc[ci];
#pragma unroll
        for (int c4 = 0; c4 < COUT / 4; ++c4) {
          const float4 ww = w[c4];
          a = fmaf(ww.x, g[4 * c4], a);
          a = fmaf(ww.y, g[4 * c4 + 1], a);
          a = fmaf(ww.z, g[4 * c4 + 2], a);
          a = fmaf(ww.w, g[4 * c4 + 3], a);
        }
        acc[ci] = a;
      }
    }
  }
#pragma unroll
  for (int ci = 0; ci < kC; ++ci)
    dzin[(int64_t)u * kC + ci] = acc[ci] * lp_dact(__bfloat162float(h[(int64_t)u * kC + ci]), slope);
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
