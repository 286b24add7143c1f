// Allocation-free entry point: the solver's weighted l2 norm of one level with
// its block partial sums in a fixed, file-scope device array instead of
// handle-owned scratch.
//
// Some hosts cannot call cudaMalloc: a Fortran or C time loop that runs inside
// a captured or externally managed memory pool, a code that must not grow its
// device footprint after start-up, or a caller in a context where the CUDA
// allocator is not available to it.  Such a caller passes device pointers it
// already owns for the input field (and, optionally, the ghost remap) and for
// the result, and this entry point allocates nothing: no cudaMalloc, no
// cudaFree, no allocating library routine.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>

#include "../../include/wavetrisk_gpu.h"

int wt_handle_fail(const char* where, cudaError_t e);

namespace {

constexpr int NOALLOC_TPB = 256;
constexpr int NOALLOC_MAX_BLOCKS = 4096;   // 32 KiB of partial sums: levels up to 8 (10*257^2 nodes)

// Scratch shared by every call on a device (held until the process exits).
// Each call writes partials [0, nblocks) before the final sum reads them, so
// nothing needs clearing; two calls in flight at the same time on one device
// (different streams) overwrite each other's partials and race.
static __device__ __align__(256) double g_noalloc_partial[NOALLOC_MAX_BLOCKS];

// Device address of g_noalloc_partial per device, looked up on the first call
// made with that device current.  Two host threads making their first call on
// one device at once may both look it up; each stores the same address, and
// the atomics make that a benign race instead of a data race.
constexpr int MAX_DEVICES = 64;
std::atomic<double*> g_partial_addr[MAX_DEVICES] = {};

__global__ void k_noalloc_sq(int n, int P, int nd, const int* __restrict__ nsrc, const double* __restrict__ s,
                             double* __restrict__ partial) {
  __shared__ double sh[NOALLOC_TPB / 32];
  const int m = n + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (t < 10 * m * m) {
    int d = t / (m * m), r = t - d * m * m, j = r / m, i = r - j * m;
    long long id = ((long long)d * P + (j + 2)) * P + (i + 2);
    long long src = nsrc ? (long long)nsrc[id] : id;
    const double x = s[src] * s[src];
    // multiplicity of the node in the (0,1) ranges of the DOMAIN_LEVEL sub-domains
    const int wi = (i > 0 && i < n && i % nd == 0) ? 2 : 1;
    const int wj = (j > 0 && j < n && j % nd == 0) ? 2 : 1;
    v = x;
    if (wi * wj >= 2) v = v + x;
    if (wi * wj == 4) v = v + x + x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < NOALLOC_TPB / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

__global__ void k_noalloc_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
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
    if (threadIdx.x == 0) *out = sqrt(v);
  }
}

}  // namespace

extern "C" int wt_elliptic_l2_noalloc(int level, int domain_level, const int* nsrc, const double* field, double* result,
                                      void* stream) {
  if (level < 0 || domain_level < 0 || !field || !result) return WT_ERR_ARG;
  const int n = 1 << level, P = n + 4;
  const long long threads = 10LL * (n + 1) * (n + 1);
  const long long nblocks = (threads + NOALLOC_TPB - 1) / NOALLOC_TPB;
  if (nblocks > NOALLOC_MAX_BLOCKS) {
    std::fprintf(stderr,
                 "wt_elliptic_l2_noalloc: level %d needs %lld partial sums; the fixed scratch holds %d "
                 "(levels up to 8)\n",
                 level, nblocks, NOALLOC_MAX_BLOCKS);
    return WT_ERR_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return wt_handle_fail("wt_elliptic_l2_noalloc: cudaGetDevice", e);
  if (dev < 0 || dev >= MAX_DEVICES) return WT_ERR_ARG;
  double* partial = g_partial_addr[dev].load(std::memory_order_acquire);
  if (!partial) {
    // The array's name in host code is only a host-side stand-in; the device
    // address is looked up once per device, with that device current.
    e = cudaGetSymbolAddress((void**)&partial, g_noalloc_partial);
    if (e != cudaSuccess) return wt_handle_fail("wt_elliptic_l2_noalloc: cudaGetSymbolAddress", e);
    g_partial_addr[dev].store(partial, std::memory_order_release);
  }
  const int nd = (n >> domain_level) > 0 ? (n >> domain_level) : 1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_noalloc_sq<<<(unsigned)nblocks, NOALLOC_TPB, 0, s>>>(n, P, nd, nsrc, field, partial);
  k_noalloc_final<<<1, 256, 0, s>>>(partial, (int)nblocks, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) return wt_handle_fail("wt_elliptic_l2_noalloc: launch", e);
  return WT_OK;
}
