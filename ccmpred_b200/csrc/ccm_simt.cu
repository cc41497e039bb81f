// Plain CUDA-core evaluation (no tensor cores), FP32 or FP64.
//
// The FP32 instance is the "plain FP32 path" that the split-bf16 tensor-core
// path is measured against; the FP64 instance serves the FP64 gradient checks.
// Same mathematics as src/evaluate_cpu.c:16-166, organised for the GPU:
//   simt_rows    one block per sequence: logits by gathering the L rows
//                W(X_nk, k, :, :), lse/softmax per column, per-row loss,
//                R(n, a, j) = w_n (P - [X_nj == a]) stored as N x 21L.
//   simt_pairs   G2[(b,k), (a,j)] = sum_n [X_nk == b] R(n,a,j); a block owns
//                4 columns k and 256 (a,j) columns and accumulates the 21 x 4
//                candidate rows in shared memory.
//   simt_single  g1 data term = column sums of R.
//   simt_sym     g2 = G2 + G2^T with zeroed self blocks, + 2 lambda2 x, and the
//                sum of x2^2 partials; then the shared finalize.
#include <cuda_runtime.h>

#include "ccm_internal.cuh"
#include "ccm_layout.cuh"

namespace ccm {

template <typename T> __device__ __forceinline__ T dev_exp(T v);
template <> __device__ __forceinline__ float dev_exp<float>(float v) { return expf(v); }
template <> __device__ __forceinline__ double dev_exp<double>(double v) { return exp(v); }
template <typename T> __device__ __forceinline__ T dev_log(T v);
template <> __device__ __forceinline__ float dev_log<float>(float v) { return logf(v); }
template <> __device__ __forceinline__ double dev_log<double>(double v) { return log(v); }

template <typename T>
__global__ void __launch_bounds__(256) simt_rows_kernel(const uint8_t *__restrict__ msa,
                                                        const float *__restrict__ w,
                                                        const T *__restrict__ x1,
                                                        const T *__restrict__ x2, T *__restrict__ R,
                                                        double *__restrict__ part_f, int L, int N) {
  extern __shared__ uint8_t xs[];
  __shared__ double red[8];
  const long long QL = (long long)kQ * L;
  for (int n = blockIdx.x; n < N; n += gridDim.x) {
    __syncthreads();
    for (int k = threadIdx.x; k < L; k += blockDim.x) xs[k] = msa[(long long)n * L + k];
    __syncthreads();
    const T wn = (T)w[n];
    double fsum = 0.0;
    for (int j = threadIdx.x; j < L; j += blockDim.x) {
      T acc[kQ];
#pragma unroll
      for (int a = 0; a < kQ - 1; ++a) acc[a] = x1[a * L + j];
      acc[kQ - 1] = (T)0;
      for (int k = 0; k < L; ++k) {
        const T *row = x2 + x2_index(xs[k], k, 0, j, L);
#pragma unroll
        for (int a = 0; a < kQ; ++a) acc[a] += row[(long long)a * L];
      }
      T mx = acc[0];
#pragma unroll
      for (int a = 1; a < kQ; ++a) mx = acc[a] > mx ? acc[a] : mx;
      T s = (T)0;
#pragma unroll
      for (int a = 0; a < kQ; ++a) s += dev_exp<T>(acc[a] - mx);
      const T lse = mx + dev_log<T>(s);
      const int xj = xs[j];
      T tgt = (T)0;
#pragma unroll
      for (int a = 0; a < kQ; ++a) tgt = (a == xj) ? acc[a] : tgt;
      fsum += (double)(wn * (lse - tgt));
      T *rrow = R + (long long)n * QL + j;
#pragma unroll
      for (int a = 0; a < kQ; ++a)
        rrow[(long long)a * L] = wn * (dev_exp<T>(acc[a] - lse) - (a == xj ? (T)1 : (T)0));
    }
    for (int o = 16; o > 0; o >>= 1) fsum += __shfl_xor_sync(0xffffffffu, fsum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = fsum;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
      part_f[n] = t;
    }
  }
}

constexpr int kPairK = 4;     // columns k per block
constexpr int kPairCols = 256;

template <typename T>
__global__ void __launch_bounds__(kPairCols) simt_pairs_kernel(const uint8_t *__restrict__ msa,
                                                              const T *__restrict__ R,
                                                              T *__restrict__ G2, int L, int N) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  T *acc = reinterpret_cast<T *>(smem_raw);  // [kPairK][kQ][kPairCols]
  const long long QL = (long long)kQ * L;
  const long long col = (long long)blockIdx.x * kPairCols + threadIdx.x;
  const int k0 = blockIdx.y * kPairK;
  for (int i = threadIdx.x; i < kPairK * kQ * kPairCols; i += blockDim.x) acc[i] = (T)0;
  __syncthreads();
  if (col < QL) {
    for (int n = 0; n < N; ++n) {
      const T r = R[(long long)n * QL + col];
      const uint8_t *xr = msa + (long long)n * L + k0;
#pragma unroll
      for (int kk = 0; kk < kPairK; ++kk) {
        if (k0 + kk < L) acc[(kk * kQ + xr[kk]) * kPairCols + threadIdx.x] += r;
      }
    }
  }
  __syncthreads();
  if (col < QL) {
    for (int kk = 0; kk < kPairK && k0 + kk < L; ++kk)
      for (int b = 0; b < kQ; ++b)
        G2[((long long)b * L + k0 + kk) * QL + col] = acc[(kk * kQ + b) * kPairCols + threadIdx.x];
  }
}

template <typename T>
__global__ void simt_single_kernel(const T *__restrict__ R, T *__restrict__ g1d, int L, int N) {
  const long long QL = (long long)kQ * L;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;  // a*L + j, a < 20
  if (v >= (kQ - 1) * L) return;
  T s = (T)0;
  for (int n = 0; n < N; ++n) s += R[(long long)n * QL + v];
  g1d[v] = s;
}

// tied (reference): g2 = G2 + G2^T, self blocks 0, + 2 lambda2 x;
// partial: g2 = G2 (self blocks kept) + lambda2 x -- the true partial derivatives.
template <typename T>
__global__ void __launch_bounds__(256) simt_sym_kernel(const T *__restrict__ G2,
                                                       const T *__restrict__ x2,
                                                       T *__restrict__ g2,
                                                       double *__restrict__ part_reg, int L,
                                                       T lambda_pair, int partial) {
  const int row = blockIdx.x;  // b*L + k
  const int b = row / L, k = row % L;
  const long long QL = (long long)kQ * L;
  const T two_l2 = (partial ? (T)1 : (T)2) * lambda_pair;
  double acc = 0.0;
  for (int a = 0; a < kQPad; ++a) {
    for (int j = threadIdx.x; j < L; j += blockDim.x) {
      const long long id = x2_index(b, k, a, j, L);
      const T xv = x2[id];
      acc += (double)xv * (double)xv;
      T gv = (T)0;
      if (a < kQ && partial)
        gv = G2[(long long)row * QL + (long long)a * L + j];
      else if (a < kQ && k != j)
        gv = G2[(long long)row * QL + (long long)a * L + j] +
             G2[((long long)a * L + j) * QL + row];
      g2[id] = gv + two_l2 * xv;
    }
  }
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    part_reg[row] = s;
  }
}

template <typename T>
__global__ void __launch_bounds__(1024) simt_finalize_kernel(const double *part_f, int n_part_f,
                                                             const double *part_reg,
                                                             int n_part_reg, const T *x1,
                                                             const T *g1d, T *g1, long long nsp,
                                                             int L, T lambda_single,
                                                             T lambda_pair, ccm_result *out) {
  __shared__ double red[32];
  double af = 0.0, ar2 = 0.0, ar1 = 0.0;
  for (int i = threadIdx.x; i < n_part_f; i += blockDim.x) af += part_f[i];
  for (int i = threadIdx.x; i < n_part_reg; i += blockDim.x) ar2 += part_reg[i];
  const long long ns = nsingle_of(L);
  const T two_l1 = (T)2 * lambda_single;
  for (long long v = threadIdx.x; v < nsp; v += blockDim.x) {
    if (v < ns) {
      const T xv = x1[v];
      ar1 += (double)xv * (double)xv;
      g1[v] = g1d[v] + two_l1 * xv;
    } else {
      g1[v] = (T)0;
    }
  }
  auto block_sum = [&](double x) -> double {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    return s;
  };
  const double F = block_sum(af), R2 = block_sum(ar2), R1 = block_sum(ar1);
  if (threadIdx.x == 0) {
    const double fx = F + (double)lambda_single * R1 + 0.5 * (double)lambda_pair * R2;
    out->fx = fx;
    out->f_data = F;
    out->reg = fx - F;
  }
}

template <typename T>
static cudaError_t simt_run(ccm_context *c, const T *d_x, T *d_g) {
  const int L = c->L, N = c->N;
  const long long QL = (long long)kQ * L;
  const T *x1 = d_x;
  const T *x2 = d_x + c->nsp;
  T *g1 = d_g;
  T *g2 = d_g + c->nsp;
  T *R = static_cast<T *>(c->d_simt_pc);
  T *G2 = static_cast<T *>(c->d_simt_g2);
  T *g1d = static_cast<T *>(c->d_simt_g1);
  double *part_f = static_cast<double *>(c->d_simt_part);
  double *part_reg = part_f + N;

  int threads = ((L + 31) / 32) * 32;
  if (threads > 256) threads = 256;
  const int grid_rows = N < 65535 ? N : 65535;
  prof_mark(c);
  simt_rows_kernel<T><<<grid_rows, threads, L, c->stream>>>(c->d_msa, c->d_w, x1, x2, R, part_f, L, N);

  const size_t pair_smem = sizeof(T) * kPairK * kQ * kPairCols;
  dim3 pgrid((unsigned)((QL + kPairCols - 1) / kPairCols), (unsigned)((L + kPairK - 1) / kPairK));
  prof_mark(c);
  simt_pairs_kernel<T><<<pgrid, kPairCols, pair_smem, c->stream>>>(c->d_msa, R, G2, L, N);
  prof_mark(c);

  const int nsingle = (kQ - 1) * L;
  simt_single_kernel<T><<<(nsingle + 127) / 128, 128, 0, c->stream>>>(R, g1d, L, N);
  prof_mark(c);

  simt_sym_kernel<T><<<kQ * L, 256, 0, c->stream>>>(G2, x2, g2, part_reg, L, (T)c->lambda_pair,
                                                     c->gradient == CCM_GRADIENT_PARTIAL);
  prof_mark(c);

  simt_finalize_kernel<T><<<1, 1024, 0, c->stream>>>(part_f, N, part_reg, kQ * L, x1, g1d, g1,
                                                     c->nsp, L, (T)c->lambda_single,
                                                     (T)c->lambda_pair, c->d_out);
  prof_mark(c);
  count_launch(c, 5);
  return cudaGetLastError();
}

cudaError_t simt_configure_kernels() {
  cudaError_t e = cudaFuncSetAttribute(simt_pairs_kernel<float>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(float) * kPairK * kQ * kPairCols));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(simt_pairs_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(double) * kPairK * kQ * kPairCols));
}

cudaError_t simt_evaluate(ccm_context *c, const float *d_x, float *d_g) {
  return simt_run<float>(c, d_x, d_g);
}

cudaError_t simt_evaluate_f64(ccm_context *c, const double *d_x, double *d_g) {
  return simt_run<double>(c, d_x, d_g);
}

size_t simt_scratch_bytes(int L, int N, size_t elem) {
  const size_t QL = (size_t)kQ * L;
  return elem * ((size_t)N * QL + QL * QL + (size_t)(kQ - 1) * L);
}

}  // namespace ccm
