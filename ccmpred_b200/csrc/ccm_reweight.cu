// Identity-threshold sequence reweighting, bit-exact with the serial reference
// (src/reweighting.c:9-58).
//
// ids(i,j) = #{k : X_ik == X_jk} is counted four columns at a time on packed
// rows (__vcmpeq4 + __popc, padding bytes subtracted), 64 x 64 row pairs per
// block over the upper triangle of row blocks.  count_i gets +1 for every
// j != i with ids > idthres and +2 for j == i (the reference's i <= j loop
// visits the diagonal once and increments w[i] twice).  Counts are integers,
// so the order of the atomic additions does not matter.
#include <cstdio>

#include <cuda_runtime.h>

#include "ccm_internal.cuh"

namespace ccm {

constexpr int kRwTile = 64;
constexpr int kRwChunk = 32;  // packed words per shared-memory chunk

__global__ void rw_pack_kernel(const uint8_t *__restrict__ msa, uint32_t *__restrict__ packed,
                               int L, int N, int words) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)N * words) return;
  const int n = (int)(idx / words), wd = (int)(idx % words);
  uint32_t v = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = wd * 4 + e;
    const uint32_t byte = k < L ? msa[(long long)n * L + k] : 0u;
    v |= byte << (8 * e);
  }
  packed[idx] = v;
}

__global__ void __launch_bounds__(256) rw_count_kernel(const uint32_t *__restrict__ packed,
                                                       int N, int words, int npad, int idthres,
                                                       int *__restrict__ counts) {
  const int IB = blockIdx.y, JB = blockIdx.x;
  if (JB < IB) return;
  __shared__ uint32_t As[kRwTile][kRwChunk + 1];
  __shared__ uint32_t Bs[kRwTile][kRwChunk + 1];
  __shared__ int ci[kRwTile], cj[kRwTile];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int i0 = IB * kRwTile, j0 = JB * kRwTile;
  if (threadIdx.x < kRwTile) { ci[threadIdx.x] = 0; cj[threadIdx.x] = 0; }
  int ids[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) ids[u][v] = 0;

  for (int w0 = 0; w0 < words; w0 += kRwChunk) {
    __syncthreads();
    for (int e = threadIdx.x; e < kRwTile * kRwChunk; e += blockDim.x) {
      const int r = e / kRwChunk, wd = e % kRwChunk;
      const int ia = i0 + r, jb = j0 + r, ww = w0 + wd;
      As[r][wd] = (ia < N && ww < words) ? packed[(long long)ia * words + ww] : 0u;
      Bs[r][wd] = (jb < N && ww < words) ? packed[(long long)jb * words + ww] : 0u;
    }
    __syncthreads();
    const int wmax = (words - w0) < kRwChunk ? (words - w0) : kRwChunk;
    for (int wd = 0; wd < wmax; ++wd) {
      uint32_t a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = As[ty * 4 + u][wd];
#pragma unroll
      for (int v = 0; v < 4; ++v) b[v] = Bs[tx * 4 + v][wd];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) ids[u][v] += __popc(__vcmpeq4(a[u], b[v]));
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 4; ++u) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int il = ty * 4 + u, jl = tx * 4 + v;
      const int i = i0 + il, j = j0 + jl;
      if (i >= N || j >= N) continue;
      const int same = ids[u][v] / 8 - npad;
      if (same <= idthres) continue;
      if (IB == JB) {
        if (i < j) { atomicAdd(&ci[il], 1); atomicAdd(&ci[jl], 1); }
        else if (i == j) atomicAdd(&ci[il], 2);
      } else {
        atomicAdd(&ci[il], 1);
        atomicAdd(&cj[jl], 1);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < kRwTile) {
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.x;
    if (i < N && ci[threadIdx.x]) atomicAdd(&counts[i], ci[threadIdx.x]);
    if (IB != JB && j < N && cj[threadIdx.x]) atomicAdd(&counts[j], cj[threadIdx.x]);
  }
}

// w_i = (float)(1. / ((float)count_i - 1)) as in src/reweighting.c:43-45
__global__ void rw_weights_kernel(const int *__restrict__ counts, float *__restrict__ w, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float cf = (float)counts[i];
  w[i] = (float)(1.0 / (double)(cf - 1.0f));
}

cudaError_t reweight_counts(const uint8_t *d_msa, int L, int N, int idthres, int *d_counts,
                            cudaStream_t stream) {
  const int words = (L + 3) / 4;
  const int npad = words * 4 - L;
  uint32_t *packed = nullptr;
  cudaError_t e = cudaMallocAsync(&packed, sizeof(uint32_t) * (size_t)N * words, stream);
  if (e != cudaSuccess) return e;
  const long long total = (long long)N * words;
  rw_pack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(d_msa, packed, L, N, words);
  cudaMemsetAsync(d_counts, 0, sizeof(int) * N, stream);
  const int nb = (N + kRwTile - 1) / kRwTile;
  rw_count_kernel<<<dim3(nb, nb), 256, 0, stream>>>(packed, N, words, npad, idthres, d_counts);
  cudaFreeAsync(packed, stream);
  return cudaGetLastError();
}

cudaError_t reweight_weights(const int *d_counts, float *d_w, int N, cudaStream_t stream) {
  rw_weights_kernel<<<(N + 255) / 256, 256, 0, stream>>>(d_counts, d_w, N);
  return cudaGetLastError();
}

}  // namespace ccm

// ----------------------------------------------------------------------------
// Allocation-free variant of the sequence reweighting (ccm_calculate_weights_noalloc).
//
// Its only scratch, one identity count per sequence, lives in the file-scope
// device array below instead of memory obtained from cudaMalloc/cudaMallocAsync,
// and the count kernel packs the alignment bytes into words in shared memory
// instead of in a packed copy in global memory.  The array is part of the
// library image: every GPU that loads the library holds it until the process
// exits.  All calls share it and it keeps the counts of the last call, so each
// call clears the part it uses first; calls that overlap on the GPU (different
// streams, or different host threads on one device) race on it.
namespace ccm {

constexpr int kNoAllocMaxRows = 262144;  // 1 MiB of int counts
static __device__ __align__(256) int g_noalloc_counts[kNoAllocMaxRows];

__global__ void __launch_bounds__(256) rw_count_bytes_kernel(const uint8_t *__restrict__ msa,
                                                             int L, int N, int words, int npad,
                                                             int idthres, int *__restrict__ counts) {
  const int IB = blockIdx.y, JB = blockIdx.x;
  if (JB < IB) return;
  __shared__ uint32_t As[kRwTile][kRwChunk + 1];
  __shared__ uint32_t Bs[kRwTile][kRwChunk + 1];
  __shared__ int ci[kRwTile], cj[kRwTile];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int i0 = IB * kRwTile, j0 = JB * kRwTile;
  if (threadIdx.x < kRwTile) { ci[threadIdx.x] = 0; cj[threadIdx.x] = 0; }
  int ids[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) ids[u][v] = 0;

  for (int w0 = 0; w0 < words; w0 += kRwChunk) {
    __syncthreads();
    // bytes straight into the word rows (byte b of word wd = column 4 wd + b):
    // consecutive threads read consecutive bytes of one row, so each warp load
    // covers one 32-byte sector of the alignment
    constexpr int kRowBytes = 4 * kRwChunk;
    for (int e = threadIdx.x; e < kRwTile * kRowBytes; e += blockDim.x) {
      const int r = e / kRowBytes, bt = e % kRowBytes;
      const int k = w0 * 4 + bt;
      const int ia = i0 + r, jb = j0 + r;
      const bool in = k < L;
      reinterpret_cast<uint8_t *>(&As[r][0])[bt] =
          (in && ia < N) ? msa[(long long)ia * L + k] : (uint8_t)0;
      reinterpret_cast<uint8_t *>(&Bs[r][0])[bt] =
          (in && jb < N) ? msa[(long long)jb * L + k] : (uint8_t)0;
    }
    __syncthreads();
    const int wmax = (words - w0) < kRwChunk ? (words - w0) : kRwChunk;
    for (int wd = 0; wd < wmax; ++wd) {
      uint32_t a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = As[ty * 4 + u][wd];
#pragma unroll
      for (int v = 0; v < 4; ++v) b[v] = Bs[tx * 4 + v][wd];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) ids[u][v] += __popc(__vcmpeq4(a[u], b[v]));
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 4; ++u) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int il = ty * 4 + u, jl = tx * 4 + v;
      const int i = i0 + il, j = j0 + jl;
      if (i >= N || j >= N) continue;
      const int same = ids[u][v] / 8 - npad;
      if (same <= idthres) continue;
      if (IB == JB) {
        if (i < j) { atomicAdd(&ci[il], 1); atomicAdd(&ci[jl], 1); }
        else if (i == j) atomicAdd(&ci[il], 2);
      } else {
        atomicAdd(&ci[il], 1);
        atomicAdd(&cj[jl], 1);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < kRwTile) {
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.x;
    if (i < N && ci[threadIdx.x]) atomicAdd(&counts[i], ci[threadIdx.x]);
    if (IB != JB && j < N && cj[threadIdx.x]) atomicAdd(&counts[j], cj[threadIdx.x]);
  }
}

}  // namespace ccm

// See include/ccmpred_b200.h.  Every call looks up the device address of the
// count array with cudaGetSymbolAddress in the context that is current on the
// calling thread -- host code must not use the array's name as a device
// pointer, and an address found in one context (the device's primary context,
// say) is not valid in another context of the same device.  The lookup
// allocates nothing once the library's module is loaded in that context (the
// first call in a context loads it); then a call enqueues a memset and two
// kernels.
extern "C" CCM_API int ccm_calculate_weights_noalloc(const unsigned char *d_msa, int ncol,
                                                     int nrow, float threshold, float *d_w,
                                                     void *stream) {
  using namespace ccm;
  if (!d_msa || !d_w || ncol <= 0 || nrow <= 0) {
    return set_last_error(CCM_ERR_INVALID, "ccm_calculate_weights_noalloc: invalid arguments");
  }
  if (nrow > kNoAllocMaxRows) {
    return set_last_error(CCM_ERR_INVALID,
                          "ccm_calculate_weights_noalloc: nrow=%d exceeds the fixed scratch of %d "
                          "sequences",
                          nrow, kNoAllocMaxRows);
  }
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_counts);
  if (e != cudaSuccess || !p) {
    return set_last_error(CCM_ERR_CUDA,
                          "ccm_calculate_weights_noalloc: cudaGetSymbolAddress failed in the "
                          "current context (%s)",
                          cudaGetErrorString(e));
  }
  int *counts = static_cast<int *>(p);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float prod = threshold * (float)(uint64_t)ncol;  // src/reweighting.c:10
  const int idthres = (int)ceil((double)prod);
  const int words = (ncol + 3) / 4;
  const int npad = words * 4 - ncol;
  e = cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nrow, s);
  if (e == cudaSuccess) {
    const int nb = (nrow + kRwTile - 1) / kRwTile;
    rw_count_bytes_kernel<<<dim3(nb, nb), 256, 0, s>>>(d_msa, ncol, nrow, words, npad, idthres,
                                                        counts);
    rw_weights_kernel<<<(nrow + 255) / 256, 256, 0, s>>>(counts, d_w, nrow);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    return set_last_error(CCM_ERR_CUDA, "ccm_calculate_weights_noalloc: %s", cudaGetErrorString(e));
  }
  return CCM_OK;
}
