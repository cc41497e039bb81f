// Contact scores on the device: the Frobenius norm of the mean-centred 20x20
// coupling block of every column pair, as the reference's sum_submatrices
// (src/util.c:16-64) computes it on the host.  One thread per (k, j); each
// thread sums in the reference's order (a outer, b inner) with explicitly
// rounded float operations (no contraction to FMA), so the result equals the
// host function bit for bit.  Adjacent threads take adjacent j, so every W load
// of a warp is one contiguous run of the padded coupling layout.
#include <cuda_runtime.h>

#include "ccm_internal.cuh"
#include "ccm_layout.cuh"

namespace ccm {

__global__ void contact_scores_kernel(const float *__restrict__ x2, float *__restrict__ out, int L) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)L * L) return;
  const int k = (int)(idx / L), j = (int)(idx % L);
  // W(b,k,a,j) = x2[((b*L + k)*32 + a)*L + j]
  const long long bstride = (long long)kQPad * L * L;
  const float *base = x2 + (long long)k * kQPad * L + j;
  float mean = 0.0f;
  for (int a = 0; a < kQ; ++a)
    for (int b = 0; b < kQ; ++b) mean = __fadd_rn(mean, base[b * bstride + (long long)a * L]);
  mean = __fdiv_rn(mean, (float)(kQ * kQ));
  float acc = 0.0f;
  for (int a = 0; a < kQ - 1; ++a)
    for (int b = 0; b < kQ - 1; ++b) {
      const float w = __fsub_rn(base[b * bstride + (long long)a * L], mean);
      acc = __fadd_rn(acc, __fmul_rn(w, w));
    }
  out[idx] = k == j ? 0.0f : __fsqrt_rn(acc);
}

cudaError_t launch_contact_scores(const float *d_x, float *d_out, int L, cudaStream_t stream) {
  const long long n = (long long)L * L;
  contact_scores_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      d_x + nsingle_padded_of(L), d_out, L);
  return cudaGetLastError();
}

}  // namespace ccm

extern "C" CCM_API int ccm_sum_submatrices_gpu(const float *d_x, float *d_out, int ncol,
                                               void *stream) {
  if (!d_x || !d_out || ncol <= 0)
    return ccm::set_last_error(CCM_ERR_INVALID, "ccm_sum_submatrices_gpu: invalid arguments");
  const cudaError_t e =
      ccm::launch_contact_scores(d_x, d_out, ncol, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return ccm::set_last_error(CCM_ERR_CUDA, "ccm_sum_submatrices_gpu: %s", cudaGetErrorString(e));
  return CCM_OK;
}
