// Device-side nonlinear conjugate gradient over the evaluation of a context:
// the replacement of libconjugrad's conjugrad_gpu (called at src/ccmpred.c:644
// with the parameters of src/ccmpred.c:526-534; the library itself is absent
// from the reference checkout, so the rules below are this project's own,
// written from the parameter names and the standard method, Nocedal & Wright,
// "Numerical Optimization", 2nd ed., ch. 3 and 5.2):
//
//   s0 = -g0, alpha0 = 1 / ||g0||
//   per iteration k:
//     line search, at most max_linesearch trials x_t = x + alpha s; accept on
//       sufficient decrease f_t <= f + ftol * alpha * (g.s); otherwise the
//       next trial is the minimiser of the quadratic through f, g.s and f_t,
//       safeguarded to [0.1, alpha_mul] times alpha (N&W sec. 3.5);
//       if all trials fail and s is not -g, restart along s = -g with
//       alpha = 1/||g|| and search once more
//     beta = max(0, g_t.(g_t - g) / g.g)                        (Polak-Ribiere+)
//     s = -g_t + beta s; if s is not a descent direction, s = -g_t
//     next alpha = 2 (f_old - f_new) / -(g_t.s_new)             (N&W eq. 3.60)
//     stop when k >= K and (f_{k-K} - f_k) / |f_k| < epsilon    ("-e/-k", src/ccmpred.c:192-196)
//   The reference's "wolfe" parameter (src/ccmpred.c:533) has no role in these
//   rules; it is kept in ccm_cg_params for the reference's parameter list.
//
// Vectors stay in float on the device; every dot product and the line-search
// tests are FP64.  One trial step (x_t = x + alpha s, the four evaluation
// kernels, the dots, the copy of the scalars to pinned host memory) is
// captured once in a CUDA graph per buffer parity and replayed; the host only
// reads back 40 bytes per trial.  On the tensor-core paths the step is fused
// into tc_prep, which reads x and s once and writes x_t while it splits the
// couplings into their bf16 terms.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "ccm_internal.cuh"

namespace ccm {

int set_last_error(int code, const char *fmt, ...);
int enqueue_evaluation(ccm_context *c, const float *d_x, float *d_g);
int enqueue_evaluation_step(ccm_context *c, const float *d_x, const float *d_s,
                            const double *d_alpha, float *d_xt, float *d_g);

constexpr int kDotBlocks = 592;  // 4 x 148 SMs

// x_t = x + alpha * s  (alpha read from device memory)
__global__ void cg_step_kernel(const float *__restrict__ x, const float *__restrict__ s,
                               const double *__restrict__ alpha, float *__restrict__ xt,
                               long long n) {
  const float a = (float)alpha[0];
  const long long n4 = n / 4;
  const float4 *x4 = reinterpret_cast<const float4 *>(x);
  const float4 *s4 = reinterpret_cast<const float4 *>(s);
  float4 *t4 = reinterpret_cast<float4 *>(xt);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4;
       i += (long long)gridDim.x * blockDim.x) {
    const float4 xv = x4[i], sv = s4[i];
    t4[i] = make_float4(fmaf(a, sv.x, xv.x), fmaf(a, sv.y, xv.y), fmaf(a, sv.z, xv.z),
                        fmaf(a, sv.w, xv.w));
  }
  for (long long i = n4 * 4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    xt[i] = fmaf(a, s[i], x[i]);
}

// Per-block FP64 partials of  a.b, a.a, a.c  (c may be null).  Fixed grid and
// fixed summation order: the result does not depend on scheduling.
__global__ void __launch_bounds__(256) cg_dots_kernel(const float *__restrict__ a,
                                                      const float *__restrict__ b,
                                                      const float *__restrict__ c,
                                                      long long n, double *__restrict__ part) {
  double ab = 0.0, aa = 0.0, ac = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double av = a[i];
    ab += av * (double)b[i];
    aa += av * av;
    if (c) ac += av * (double)c[i];
  }
  __shared__ double red[3][8];
  for (int o = 16; o > 0; o >>= 1) {
    ab += __shfl_xor_sync(0xffffffffu, ab, o);
    aa += __shfl_xor_sync(0xffffffffu, aa, o);
    ac += __shfl_xor_sync(0xffffffffu, ac, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = ab;
    red[1][threadIdx.x >> 5] = aa;
    red[2][threadIdx.x >> 5] = ac;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[threadIdx.x][w];
    part[blockIdx.x * 3 + threadIdx.x] = t;
  }
}

// Final FP64 reduction of the dot partials into out[0..2].
__global__ void cg_dots_final_kernel(const double *__restrict__ part, int nblocks,
                                     double *__restrict__ out) {
  __shared__ double red[3][32];
  double v[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x)
    for (int k = 0; k < 3; ++k) v[k] += part[i * 3 + k];
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
    out[threadIdx.x] = t;
  }
}

// s = -g + beta * s  (beta == 0 gives steepest descent).  beta is a launch
// argument: it is fixed when the kernel is enqueued, with no host buffer that
// the host could overwrite before the copy runs.
__global__ void cg_direction_kernel(const float *__restrict__ g, double beta,
                                    float *__restrict__ s, long long n) {
  const float b = (float)beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    s[i] = fmaf(b, s[i], -g[i]);
}

}  // namespace ccm

using namespace ccm;

namespace {

// Scalars exchanged with the host per trial (pinned).
struct TrialOut {
  double f;      // f(x_t)
  double gs;     // g_t . s
  double gg;     // g_t . g_t
  double ggold;  // g_t . g  (for Polak-Ribiere)
  double xx;     // x_t . x_t
  int status;
  int pad;
};

struct CgState {
  ccm_context *c = nullptr;
  long long n = 0;
  float *xb[2] = {nullptr, nullptr};  // x ping-pong (xb[0] may be the caller's x)
  float *gb[2] = {nullptr, nullptr};
  float *s = nullptr;
  double *d_alpha = nullptr, *d_part = nullptr, *d_dots = nullptr;
  double *h_alpha = nullptr;  // pinned
  TrialOut *h_out = nullptr;  // pinned
  cudaGraphExec_t trial[2] = {nullptr, nullptr};
  bool own_x0 = false;
  bool want_xx = true;   // compute x_t . x_t in every trial (needed by a progress callback)
  int eval_kernels = 0;  // kernels of the step and the evaluation inside the trial graph
};

int free_state(CgState &st) {
  for (int i = 0; i < 2; ++i) {
    if (st.trial[i]) cudaGraphExecDestroy(st.trial[i]);
    if ((i == 1 || st.own_x0) && st.xb[i]) cudaFreeAsync(st.xb[i], st.c->stream);
    if (st.gb[i]) cudaFreeAsync(st.gb[i], st.c->stream);
  }
  // stream-ordered frees and pooled pinned slots: nothing here waits for the
  // other streams of the device
  for (void *p : {(void *)st.s, (void *)st.d_alpha, (void *)st.d_part, (void *)st.d_dots})
    if (p) cudaFreeAsync(p, st.c->stream);
  pinned_small_free(st.h_alpha);
  pinned_small_free(st.h_out);
  return CCM_OK;
}

int grid_for(long long n) {
  const long long b = (n / 4 + 255) / 256;
  return (int)(b < 4 * 148 * 4 ? (b > 0 ? b : 1) : 4 * 148 * 4);
}

// Enqueue the dots of (a = gt) with (b = s), (a.a), (c = gold) and the copy of
// f, the dots and x_t.x_t into the pinned TrialOut.
cudaError_t enqueue_trial_tail(CgState &st, const float *xt, const float *gt, const float *gold) {
  cudaStream_t s = st.c->stream;
  cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(gt, st.s, gold, st.n, st.d_part);
  cg_dots_final_kernel<<<1, 1024, 0, s>>>(st.d_part, kDotBlocks, st.d_dots);
  if (st.want_xx) {  // ||x_t|| is reported to the progress callback only
    cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(xt, xt, nullptr, st.n, st.d_part);
    cg_dots_final_kernel<<<1, 1024, 0, s>>>(st.d_part, kDotBlocks, st.d_dots + 3);
  }
  cudaError_t e = cudaMemcpyAsync(&st.h_out->f, &st.c->d_out->fx, sizeof(double),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&st.h_out->gs, st.d_dots, 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && st.want_xx)
    e = cudaMemcpyAsync(&st.h_out->xx, st.d_dots + 4, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&st.h_out->status, &st.c->d_out->status, sizeof(int),
                        cudaMemcpyDeviceToHost, s);
  return e;
}

// Capture: alpha (pinned) -> device; x_t = x + alpha s; evaluate(x_t) -> g_t;
// dots; scalars -> pinned.  Parity p: x = xb[p], trial into xb[1-p].
int capture_trial(CgState &st, int p) {
  cudaStream_t s = st.c->stream;
  float *x = st.xb[p], *xt = st.xb[1 - p];
  float *g = st.gb[p], *gt = st.gb[1 - p];
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg capture: %s", cudaGetErrorString(e));
  cudaMemcpyAsync(st.d_alpha, st.h_alpha, sizeof(double), cudaMemcpyHostToDevice, s);
  // tensor-core paths take the step inside tc_prep (one pass over x and s that
  // also splits the couplings into the bf16 terms); the CUDA-core paths step first
  const bool fused = st.c->path == CCM_PATH_TC_BF16X2 || st.c->path == CCM_PATH_TC_BF16X3 ||
                     st.c->path == CCM_PATH_TC_I8X3 || st.c->path == CCM_PATH_TC_I8SP;
  if (!fused) cg_step_kernel<<<grid_for(st.n), 256, 0, s>>>(x, st.s, st.d_alpha, xt, st.n);
  const long long before = st.c->launches;
  int rc = fused ? enqueue_evaluation_step(st.c, x, st.s, st.d_alpha, xt, gt)
                 : enqueue_evaluation(st.c, xt, gt);
  st.eval_kernels = (int)(st.c->launches - before) + (fused ? 0 : 1);
  st.c->launches = before;  // counted per replay instead
  e = enqueue_trial_tail(st, xt, gt, g);
  cudaError_t e2 = cudaStreamEndCapture(s, &graph);
  if (rc != CCM_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&st.trial[p], graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg capture: %s", cudaGetErrorString(e));
  return CCM_OK;
}

}  // namespace

extern "C" {

void ccm_cg_params_default(ccm_cg_params *p) {
  if (!p) return;
  // src/ccmpred.c:222-229, 526-534
  p->max_iterations = 250;
  p->epsilon = 0.01;
  p->k = 5;
  p->max_linesearch = 5;
  p->alpha_mul = 0.5;
  p->ftol = 1e-4;
  p->wolfe = 0.2;
}

int ccm_conjugrad_gpu(ccm_context *c, float *d_x, long long n, const ccm_cg_params *params,
                      ccm_progress_t progress, void *instance, ccm_cg_result *result) {
  if (!c || !d_x || !params) return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_gpu: null argument");
  if (n != c->nvarp)
    return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_gpu: n %lld != nvar_padded %lld", n, c->nvarp);
  if (c->path == CCM_PATH_SIMT_F64)
    return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_gpu: needs a float evaluation path");
  if (params->max_iterations < 0 || params->k < 1 || params->max_linesearch < 1 ||
      !(params->alpha_mul > 0.0 && params->alpha_mul < 1.0))
    return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_gpu: invalid parameters");
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  CgState st;
  st.c = c;
  st.n = n;
  st.xb[0] = d_x;
  st.want_xx = progress != nullptr;
  const size_t bytes = sizeof(float) * (size_t)n;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&st.xb[1]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&st.gb[0]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&st.gb[1]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&st.s), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&st.d_alpha), sizeof(double)));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&st.d_part), sizeof(double) * 3 * kDotBlocks));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&st.d_dots), sizeof(double) * 6));
  static_assert(sizeof(TrialOut) <= 256, "TrialOut must fit a pinned slot");
  st.h_alpha = static_cast<double *>(pinned_small_alloc(sizeof(double)));
  st.h_out = static_cast<TrialOut *>(pinned_small_alloc(sizeof(TrialOut)));
  if (!st.h_alpha || !st.h_out) chk(cudaErrorMemoryAllocation);
  if (e != cudaSuccess) {
    free_state(st);
    (void)cudaGetLastError();  // a failed allocation must not surface in a later launch check
    return set_last_error(e == cudaErrorMemoryAllocation ? CCM_ERR_NOMEM : CCM_ERR_CUDA,
                          "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
  }
  ccm_cg_result res;
  std::memset(&res, 0, sizeof(res));
  int p = 0;  // x = xb[p], g = gb[p]

  // initial evaluation: f0, g0 and the dots with s := 0 (g.s unused)
  cudaMemsetAsync(st.s, 0, bytes, s);
  int rc = enqueue_evaluation(c, st.xb[0], st.gb[0]);
  if (rc == CCM_OK) {
    e = enqueue_trial_tail(st, st.xb[0], st.gb[0], st.gb[0]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = set_last_error(CCM_ERR_CUDA, "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
  }
  if (rc == CCM_OK && st.h_out->status != 0)
    rc = set_last_error(CCM_ERR_DEVICE, "ccm_conjugrad_gpu: device wait timed out in evaluation");
  if (rc != CCM_OK) { free_state(st); return rc; }
  double f = st.h_out->f, gg = st.h_out->gg;
  res.evaluations = 1;
  std::vector<double> fhist;
  fhist.push_back(f);
  if (!(gg > 0.0) || !std::isfinite(f)) {
    res.status = std::isfinite(f) ? CCM_CG_ALREADY_MINIMIZED : CCM_CG_ERR_NONFINITE;
    res.fx = f;
    free_state(st);
    if (result) *result = res;
    return CCM_OK;
  }
  // s0 = -g0
  cg_direction_kernel<<<grid_for(n), 256, 0, s>>>(st.gb[0], 0.0, st.s, n);
  double gs = -gg;  // g.s with s = -g
  double alpha = 1.0 / std::sqrt(gg);
  bool steepest = true;  // s == -g
  int status = CCM_CG_ERR_MAXITER;
  for (int k = 1; k <= params->max_iterations; ++k) {
    bool accepted = false;
    int ls = 0, trials = 0;
    for (int attempt = 0; attempt < 2 && !accepted; ++attempt) {
      for (ls = 1; ls <= params->max_linesearch; ++ls) {
        if (!st.trial[p]) {
          rc = capture_trial(st, p);
          if (rc != CCM_OK) { free_state(st); return rc; }
        }
        *st.h_alpha = alpha;
        e = cudaGraphLaunch(st.trial[p], s);
        // (step +) evaluation + (1 or 2) x (dots + final)
        c->launches += st.eval_kernels + (st.want_xx ? 4 : 2);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
          free_state(st);
          return set_last_error(CCM_ERR_CUDA, "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
        }
        res.evaluations++;
        trials++;
        if (st.h_out->status != 0) {
          free_state(st);
          return set_last_error(CCM_ERR_DEVICE, "ccm_conjugrad_gpu: device wait timed out in evaluation");
        }
        const double ft = st.h_out->f;
        if (std::isfinite(ft) && ft <= f + params->ftol * alpha * gs) {
          accepted = true;
          break;
        }
        const double den = 2.0 * (ft - f - gs * alpha);
        double aq = (std::isfinite(ft) && den > 0.0) ? -gs * alpha * alpha / den
                                                    : params->alpha_mul * alpha;
        aq = std::fmin(aq, params->alpha_mul * alpha);
        alpha = std::fmax(aq, 0.1 * alpha);
      }
      if (!accepted && !steepest) {
        // restart along the steepest-descent direction
        cg_direction_kernel<<<grid_for(n), 256, 0, s>>>(st.gb[p], 0.0, st.s, n);
        c->launches += 1;
        gs = -gg;
        alpha = 1.0 / std::sqrt(gg);
        steepest = true;
      } else if (!accepted) {
        break;
      }
    }
    if (!accepted) { status = CCM_CG_ERR_LINESEARCH; break; }
    ls = trials;
    // accept: x, g <- trial buffers
    const double fnew = st.h_out->f, ggnew = st.h_out->gg, gtg = st.h_out->ggold;
    const double xx = st.h_out->xx;
    p = 1 - p;
    const double step = alpha;
    // Polak-Ribiere+ direction
    double beta = (ggnew - gtg) / gg;
    if (!(beta > 0.0)) beta = 0.0;
    steepest = beta == 0.0;
    cg_direction_kernel<<<grid_for(n), 256, 0, s>>>(st.gb[p], beta, st.s, n);
    c->launches += 1;
    // g.s for the new direction: -||g||^2 + beta * (g_t.s_old)
    double gs_new = -ggnew + beta * st.h_out->gs;
    if (!(gs_new < 0.0)) {
      // not a descent direction: restart with steepest descent
      cg_direction_kernel<<<grid_for(n), 256, 0, s>>>(st.gb[p], 0.0, st.s, n);
      gs_new = -ggnew;
      steepest = true;
    }
    alpha = 2.0 * (f - fnew) / -gs_new;
    gs = gs_new;
    f = fnew;
    gg = ggnew;
    fhist.push_back(f);
    res.iterations = k;
    if (progress) {
      e = cudaStreamSynchronize(s);
      const int stop = progress(instance, st.xb[p], st.gb[p], (float)f, (float)std::sqrt(xx),
                                (float)std::sqrt(gg), (float)step, (int)n, k, ls);
      if (stop) { status = CCM_CG_STOPPED; break; }
    }
    if (k >= params->k) {
      const double fk = fhist[fhist.size() - 1 - params->k];
      if ((fk - f) / std::fabs(f) < params->epsilon) { status = CCM_CG_SUCCESS; break; }
    }
  }
  // leave the final x in the caller's buffer
  if (p == 1) cudaMemcpyAsync(d_x, st.xb[1], bytes, cudaMemcpyDeviceToDevice, s);
  e = cudaStreamSynchronize(s);
  res.fx = f;
  res.gnorm = std::sqrt(gg);
  res.status = status;
  free_state(st);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
  if (result) *result = res;
  return CCM_OK;
}

}  // extern "C"

extern "C" int ccm_conjugrad_host(ccm_context *c, float *x, long long n, const ccm_cg_params *params,
                                  ccm_progress_t progress, void *instance, ccm_cg_result *result) {
  if (!c || !x) return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_host: null argument");
  if (n != c->nvarp)
    return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_host: n %lld != nvar_padded %lld", n, c->nvarp);
  cudaSetDevice(c->device);
  float *d_x = nullptr;
  const size_t bytes = sizeof(float) * (size_t)n;
  cudaError_t e = dev_alloc_raw(c, reinterpret_cast<void **>(&d_x), bytes);
  if (e != cudaSuccess)
    return set_last_error(CCM_ERR_NOMEM, "ccm_conjugrad_host: %s", cudaGetErrorString(e));
  e = cudaMemcpyAsync(d_x, x, bytes, cudaMemcpyHostToDevice, c->stream);
  int rc = CCM_OK;
  if (e == cudaSuccess) rc = ccm_conjugrad_gpu(c, d_x, n, params, progress, instance, result);
  if (e == cudaSuccess && rc == CCM_OK) e = cudaMemcpyAsync(x, d_x, bytes, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFreeAsync(d_x, c->stream);
  if (rc != CCM_OK) return rc;
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "ccm_conjugrad_host: %s", cudaGetErrorString(e));
  return CCM_OK;
}

extern "C" int ccm_device_info(int device, char *name, int name_len, size_t *mem_free,
                               size_t *mem_total) {
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "ccm_device_info: %s", cudaGetErrorString(e));
  if (name && name_len > 0) {
    std::strncpy(name, prop.name, (size_t)name_len - 1);
    name[name_len - 1] = 0;
  }
  if (mem_free || mem_total) {
    size_t fr = 0, to = 0;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMemGetInfo(&fr, &to);
    if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "ccm_device_info: %s", cudaGetErrorString(e));
    if (mem_free) *mem_free = fr;
    if (mem_total) *mem_total = to;
  }
  return CCM_OK;
}

extern "C" int ccm_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}
