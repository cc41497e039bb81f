// Device-side nonlinear conjugate gradient: the replacement of libconjugrad's
// conjugrad_gpu (called at src/ccmpred.c:632 with the parameters of
// src/ccmpred.c:526-534; the library is absent from the reference checkout).
// The rules -- line search, Polak-Ribiere+ direction, stopping test -- are in
// ccm_cg_rules.cuh; here they run on the device.
//
// Per line-search trial, on the context's stream:
//   cg_dir_kernel      s <- -g or -g + beta s when the last decision asks for it
//   step + evaluation  x_t = x + alpha s (alpha read from the control record;
//                      fused into the first pass over x on the tensor-core
//                      paths), f(x_t), g_t
//   cg_dots_kernel     FP64 partials of g_t.s, g_t.g_t, g_t.g (and x_t.x_t)
//   cg_control_kernel  one block: the partials summed in a fixed order, then
//                      one thread applies the rules to the control record and
//                      sets the conditional nodes' values
// The trials form the body of a CUDA-graph WHILE node (the line search), and
// the iterations -- two of them per round, one for each buffer parity, the x
// and g of one iteration being the trial buffers of the previous one -- the
// body of an outer WHILE node: without a progress callback the whole solve is
// one graph launch and the host waits once.  With a progress callback (which
// the reference calls after every iteration, src/ccmpred.c:50-61) the host
// launches one line-search graph per iteration and reads the control record
// back after each.  Vectors stay in float; every dot product and every
// line-search quantity is FP64.
//
// conjugrad_gpu with another evaluate callback than this library's own
// (conjugrad_callback_gpu below) runs the same kernels around one call of
// the callback per trial, from the host.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "ccm_cg_rules.cuh"
#include "ccm_internal.cuh"
#include "ccm_layout.cuh"

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

// The elements a vector pass of the CG visits.  cols == 0: all n.  Else the
// single-field block [0, nsp) and, of each of the `rows` coupling rows (stride
// `row`), its first `cols` elements: the 21 states, the padding states skipped
// (a solve whose x0 has zero padding states keeps them zero in x, g and s).
// Fixed grid, fixed assignment of elements to threads.
struct VecSpan {
  long long n, nsp, row;
  int rows, cols;
};

template <class F>
__device__ __forceinline__ void for_span(const VecSpan &v, F f) {
  const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (v.cols == 0) {
    for (long long i = t0; i < v.n; i += stride) f(i);
    return;
  }
  for (long long i = t0; i < v.nsp; i += stride) f(i);
  for (int r = blockIdx.x; r < v.rows; r += gridDim.x) {
    const long long base = v.nsp + (long long)r * v.row;
    for (int c = threadIdx.x; c < v.cols; c += blockDim.x) f(base + c);
  }
}

// Per-block FP64 partials of  a.b, a.a, a.c  (b and c may be null).  Fixed grid
// and fixed summation order: the result does not depend on scheduling.
__global__ void __launch_bounds__(256) cg_dots_kernel(const float *__restrict__ a,
                                                      const float *__restrict__ b,
                                                      const float *__restrict__ c, VecSpan v,
                                                      double *__restrict__ part) {
  double ab = 0.0, aa = 0.0, ac = 0.0;
  for_span(v, [&](long long i) {
    const double av = a[i];
    if (b) ab += av * (double)b[i];
    aa += av * av;
    if (c) ac += av * (double)c[i];
  });
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

// s <- -g (dir_mode 1) or fmaf(beta, s, -g) (dir_mode 2); dir_mode 0 keeps s.
__global__ void cg_dir_kernel(const float *__restrict__ g, float *__restrict__ s,
                              const CgCtl *__restrict__ ctl, VecSpan v) {
  const int mode = ctl->dir_mode;
  if (mode == 0) return;
  const float b = (float)ctl->beta;
  for_span(v, [&](long long i) { s[i] = mode == 1 ? -g[i] : fmaf(b, s[i], -g[i]); });
}

// Sum of the partials part[i * 3 + k], i < nblocks, in a fixed order, for a block
// of 256 threads; the result in thread 0.
__device__ double reduce_part(const double *part, int nblocks, int k, double *red) {
  double v = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) v += part[i * 3 + k];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// Conditional-node values a control kernel sets: the value of the WHILE node
// whose body holds it (its line search) when mode >= 1.  Mode 0: none
// (host-driven).  Every conditional value in these graphs is set in one of two
// ways only: by a kernel in the body of a WHILE node, for that node (the
// control and the guard), or by a kernel upstream of an IF or WHILE node in the
// same graph (the selectors and arms).
struct CgHandles {
  cudaGraphConditionalHandle ls_self;
  int mode, parity;
};

// Opens a WHILE node in the same graph for its next execution while the solve runs.
__global__ void cg_arm_kernel(const CgCtl *ctl, cudaGraphConditionalHandle h) {
  cudaGraphSetConditional(h, ctl->status == kCgRunning ? 1u : 0u);
}

// Selects the IF node of parity p in the same graph: the solve runs and its x
// is buffer p.
__global__ void cg_select_kernel(const CgCtl *ctl, cudaGraphConditionalHandle h, int p) {
  cudaGraphSetConditional(h, ctl->status == kCgRunning && ctl->parity == p ? 1u : 0u);
}

// Last node of every round of the whole-solve graph's outer loop (in its body):
// counts the round and keeps the loop open while the solve runs.  It bounds the
// loop on its own: past max_rounds (a round holds at least one trial, so a solve
// within its trial budget never gets there) it ends the solve (reported as
// CCM_ERR_DEVICE).
__global__ void cg_guard_kernel(CgCtl *ctl, cudaGraphConditionalHandle h_out, int max_rounds) {
  const int round = ++ctl->rounds;
  if (ctl->status == kCgRunning && round > max_rounds) {
    ctl->status = kCgLoopBound;
    ctl->ls_active = 0;
  }
  cudaGraphSetConditional(h_out, ctl->status == kCgRunning ? 1u : 0u);
}

// After the initial evaluation: f0 (from the evaluation record, or from f_slot
// when a callback evaluated), g0.g0 from the partials.  In a graph (set_out) it
// also sets the value of the solve's outer WHILE node: no iteration when x0 is
// already a minimum or f0 is not finite.
__global__ void __launch_bounds__(256) cg_start_kernel(CgCtl *ctl, const double *part,
                                                       int nblocks, const ccm_result *res,
                                                       const double *f_slot,
                                                       cudaGraphConditionalHandle h_out,
                                                       int set_out) {
  __shared__ double red[8];
  const double gg = reduce_part(part, nblocks, 1, red);
  if (threadIdx.x == 0) {
    cg_rules_start(*ctl, f_slot ? *f_slot : res->fx, gg);
    if (res && res->status != 0) {
      ctl->status = CCM_ERR_DEVICE;
      ctl->ls_active = 0;
    }
    if (set_out) cudaGraphSetConditional(h_out, ctl->status == kCgRunning ? 1u : 0u);
  }
}

// The solve's x ends in the trial buffer when the last accepted step had parity
// 0: copy it to the caller's buffer (a no-op otherwise).
__global__ void cg_final_x_kernel(const CgCtl *__restrict__ ctl, const float *__restrict__ x1,
                                  float *__restrict__ x0, long long n) {
  if (ctl->parity != 1) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x0[i] = x1[i];
}

__global__ void __launch_bounds__(256) cg_control_kernel(CgCtl *ctl, CgRuleParams p,
                                                         const double *part, int nblocks,
                                                         int with_xx, const ccm_result *res,
                                                         const double *f_slot, CgHandles h) {
  __shared__ double red[8];
  CgTrial t;
  t.gts = reduce_part(part, nblocks, 0, red);
  t.gtgt = reduce_part(part, nblocks, 1, red);
  t.gtg = reduce_part(part, nblocks, 2, red);
  t.xtxt = with_xx ? reduce_part(part + 3 * nblocks, nblocks, 1, red) : 0.0;
  if (threadIdx.x != 0) return;
  if (ctl->status != kCgRunning) {  // a finished solve takes no more trials
    if (h.mode >= 1) cudaGraphSetConditional(h.ls_self, 0u);
    return;
  }
  t.f = f_slot ? *f_slot : res->fx;
  t.status = res ? res->status : 0;
  t.pad = 0;
  const bool accepted = cg_rules_trial(*ctl, t, p);
  // a bound on the loop whatever the rules do: two full line searches per iteration
  if (ctl->status == kCgRunning &&
      ctl->evals > (p.max_iterations + 1) * 2 * (p.max_linesearch + 1) + 1) {
    ctl->status = CCM_CG_ERR_LINESEARCH;
    ctl->ls_active = 0;
  }
  (void)accepted;
  if (h.mode >= 1) cudaGraphSetConditional(h.ls_self, ctl->ls_active ? 1u : 0u);
}

}  // namespace ccm

using namespace ccm;

namespace {

int grid_for(long long n) {
  const long long b = (n / 4 + 255) / 256;
  return (int)(b < 4 * 148 * 4 ? (b > 0 ? b : 1) : 4 * 148 * 4);
}

CgRuleParams rule_params(const ccm_cg_params &p) {
  CgRuleParams r;
  r.max_iterations = p.max_iterations;
  r.k = p.k;
  r.max_linesearch = p.max_linesearch;
  r.pad = 0;
  r.epsilon = p.epsilon;
  r.alpha_mul = p.alpha_mul;
  r.ftol = p.ftol;
  r.wolfe = p.wolfe;
  r.min_gnorm = p.min_gnorm;
  return r;
}

int check_params(const ccm_cg_params *p, const char *who) {
  if (p->max_iterations < 0 || p->k < 1 || p->k >= kCgHist || p->max_linesearch < 1 ||
      !(p->alpha_mul > 0.0 && p->alpha_mul < 1.0) || !(p->wolfe < 1.0))
    return set_last_error(CCM_ERR_INVALID, "%s: invalid parameters", who);
  return CCM_OK;
}

// Buffers of one solve on a context: x and g of both parities (xb[0] is the
// caller's x), the direction, the control record and the dot partials.
struct CgRun {
  ccm_context *c = nullptr;
  long long n = 0;
  float *xb[2] = {nullptr, nullptr};
  float *gb[2] = {nullptr, nullptr};
  float *s = nullptr;
  CgCtl *d_ctl = nullptr;
  double *d_part = nullptr;
  CgCtl *h_ctl = nullptr;  // pinned, the kCgCtlHead bytes before fhist
  cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};  // whole solve | parity 0 | parity 1
  bool want_xx = false;
  bool fused = false;
  bool padfree = false;  // x0's padding states are zero: every pass skips them
  VecSpan span{};        // the elements the vector passes visit
  size_t mem_mark = 0;  // the context's mem_used before this solve's buffers
  int trial_kernels = 0;  // kernels of one trial (launch accounting)
};

// OR of the bit patterns of the padding states a in [21, 32) of every coupling
// row of x into *flag.
__global__ void cg_pad_bits_kernel(const float *__restrict__ x, long long nsp, int L,
                                   int *__restrict__ flag) {
  const int rows = kQ * L, pad = (kQPad - kQ) * L;
  unsigned acc = 0;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const unsigned *p =
        reinterpret_cast<const unsigned *>(x + nsp + (long long)r * kQPad * L + kQ * L);
    for (int i = threadIdx.x; i < pad; i += blockDim.x) acc |= p[i];
  }
  if (__any_sync(0xffffffffu, acc != 0) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// The elements the solve's vector passes visit.  On the integer paths, when x0's
// padding states are zero (checked here, or known: the batch solver starts its
// couplings at zero), they stay zero in x, g and s (g = 2 lambda2 x there,
// s = -g + beta s), so every pass skips them: the evaluation's column-maximum and
// prep passes and the CG's direction and dot passes.  The work buffers' padding
// states are zeroed once; nothing writes them afterwards.
int choose_span(CgRun &r, bool known_zero) {
  ccm_context *c = r.c;
  const int L = c->L;
  r.span = VecSpan{r.n, 0, 0, 0, 0};
  r.padfree = false;
  const bool i8 = c->path == CCM_PATH_TC_I8X3 || c->path == CCM_PATH_TC_I8SP;
  if (!i8 || !c->cg_skip_padding) return CCM_OK;
  cudaStream_t s = c->stream;
  cudaError_t e = cudaSuccess;
  if (!known_zero) {
    int *d_flag = reinterpret_cast<int *>(r.d_part);
    e = cudaMemsetAsync(d_flag, 0, sizeof(int), s);
    if (e == cudaSuccess) {
      cg_pad_bits_kernel<<<kDotBlocks, 256, 0, s>>>(r.xb[0], c->nsp, L, d_flag);
      e = cudaMemcpyAsync(r.h_ctl, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
      return set_last_error(CCM_ERR_CUDA, "cg padding check: %s", cudaGetErrorString(e));
    if (*reinterpret_cast<const int *>(r.h_ctl) != 0) return CCM_OK;
  }
  const size_t bytes = sizeof(float) * (size_t)r.n;
  for (float *b : {r.xb[1], r.gb[0], r.gb[1], r.s})
    if (e == cudaSuccess) e = cudaMemsetAsync(b, 0, bytes, s);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg buffers: %s", cudaGetErrorString(e));
  r.padfree = true;
  r.span = VecSpan{r.n, c->nsp, (long long)kQPad * L, kQ * L, kQ * L};
  c->skip_padding = true;
  return CCM_OK;
}

void free_run(CgRun &r) {
  r.c->skip_padding = false;
  for (auto &g : r.exec)
    if (g) cudaGraphExecDestroy(g);
  cudaStream_t s = r.c->stream;
  // stream-ordered frees and a pooled pinned slot: nothing here waits for the
  // other streams of the device
  for (void *p : {(void *)r.xb[1], (void *)r.gb[0], (void *)r.gb[1], (void *)r.s,
                  (void *)r.d_ctl, (void *)r.d_part})
    if (p) cudaFreeAsync(p, s);
  pinned_small_free(r.h_ctl);
  r.c->mem_used = r.mem_mark;
}

// One trial on the stream (in capture): direction, step + evaluation, dots,
// control.  Parity p: x = xb[p], trial into xb[1 - p].
int enqueue_trial(CgRun &r, int p, const CgRuleParams &rp, CgHandles h) {
  ccm_context *c = r.c;
  cudaStream_t s = c->stream;
  float *x = r.xb[p], *xt = r.xb[1 - p], *g = r.gb[p], *gt = r.gb[1 - p];
  const long long before = c->launches;
  cg_dir_kernel<<<grid_for(r.n), 256, 0, s>>>(g, r.s, r.d_ctl, r.span);
  int rc;
  if (r.fused) {
    rc = enqueue_evaluation_step(c, x, r.s, &r.d_ctl->alpha, xt, gt);
  } else {
    cg_step_kernel<<<grid_for(r.n), 256, 0, s>>>(x, r.s, &r.d_ctl->alpha, xt, r.n);
    rc = enqueue_evaluation(c, xt, gt);
  }
  if (rc != CCM_OK) return rc;
  cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(gt, r.s, g, r.span, r.d_part);
  if (r.want_xx) cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(xt, nullptr, nullptr, r.span,
                                                           r.d_part + 3 * kDotBlocks);
  cg_control_kernel<<<1, 256, 0, s>>>(r.d_ctl, rp, r.d_part, kDotBlocks, r.want_xx ? 1 : 0,
                                      c->d_out, nullptr, h);
  r.trial_kernels = (int)(c->launches - before) + (r.fused ? 0 : 1) + (r.want_xx ? 4 : 3);
  c->launches = before;  // counted from the evaluations of each run instead
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg trial: %s", cudaGetErrorString(e));
  return CCM_OK;
}

// Add a conditional node of `type` to `graph` after `deps`; its handle is
// created on `graph` with `deflt`; the node's body graph is returned.
cudaError_t add_conditional(cudaGraph_t graph, cudaGraphConditionalNodeType type, unsigned deflt,
                            const cudaGraphNode_t *deps, size_t ndeps,
                            cudaGraphConditionalHandle *handle, cudaGraphNode_t *node,
                            cudaGraph_t *body, bool have_handle = false) {
  cudaError_t e = have_handle ? cudaSuccess
                              : cudaGraphConditionalHandleCreate(handle, graph, deflt,
                                                                 cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = *handle;
  np.conditional.type = type;
  np.conditional.size = 1;
  e = cudaGraphAddNode(node, graph, deps, ndeps, &np);
  if (e != cudaSuccess) return e;
  *body = np.conditional.phGraph_out[0];
  return cudaSuccess;
}

// Capture one trial into `body` (the body graph of a WHILE node).
int capture_trial_into(CgRun &r, cudaGraph_t body, int p, const CgRuleParams &rp, CgHandles h) {
  cudaStream_t s = r.c->stream;
  cudaError_t e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg capture: %s", cudaGetErrorString(e));
  const int rc = enqueue_trial(r, p, rp, h);
  cudaGraph_t out = nullptr;
  e = cudaStreamEndCapture(s, &out);
  if (rc != CCM_OK) return rc;
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg capture: %s", cudaGetErrorString(e));
  return CCM_OK;
}

// The copy of the control record's scalars to pinned memory, appended to
// `graph` after `dep`.
int capture_readback(CgRun &r, cudaGraph_t graph, cudaGraphNode_t dep) {
  cudaStream_t s = r.c->stream;
  cudaError_t e = cudaStreamBeginCaptureToGraph(s, graph, &dep, nullptr, 1,
                                                cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(r.h_ctl, r.d_ctl, kCgCtlHead, cudaMemcpyDeviceToHost, s);
  cudaGraph_t out = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(s, &out);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg capture: %s", cudaGetErrorString(e));
  return CCM_OK;
}

// One small kernel captured into `graph` after `deps` (through the context's
// stream); its node in *node.  kind 0: arm h; 1: select parity p on h; 2: guard.
int capture_small(CgRun &r, cudaGraph_t graph, const cudaGraphNode_t *deps, size_t ndeps,
                  int kind, cudaGraphConditionalHandle h, int arg, cudaGraphNode_t *node) {
  cudaStream_t s = r.c->stream;
  cudaError_t e = cudaStreamBeginCaptureToGraph(s, graph, deps, nullptr, ndeps,
                                                cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    if (kind == 0) cg_arm_kernel<<<1, 1, 0, s>>>(r.d_ctl, h);
    else if (kind == 1) cg_select_kernel<<<1, 1, 0, s>>>(r.d_ctl, h, arg);
    else cg_guard_kernel<<<1, 1, 0, s>>>(r.d_ctl, h, arg);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *fr = nullptr;
    size_t nd = 0;
    e = cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &fr, &nd);
    if (e == cudaSuccess && nd == 1) *node = fr[0];
    else if (e == cudaSuccess) e = cudaErrorUnknown;
    cudaGraph_t tmp = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s, &tmp);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg capture: %s", cudaGetErrorString(e));
  return CCM_OK;
}

// The trial of parity p inside the outer loop's body `b_out`, after `dep`:
//   select(p) -> IF(sel_p) { trial parity p }
// Its IF node in *node.
int add_parity_trial(CgRun &r, const CgRuleParams &rp, cudaGraph_t b_out, cudaGraphNode_t dep,
                     int p, cudaGraphNode_t *node) {
  cudaGraphConditionalHandle h_sel;
  cudaGraphNode_t n_sel, n_if;
  cudaGraph_t b_if;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h_sel, b_out, 0, cudaGraphCondAssignDefault);
  int rc = e == cudaSuccess ? CCM_OK
                            : set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  if (rc == CCM_OK) rc = capture_small(r, b_out, &dep, 1, 1, h_sel, p, &n_sel);
  if (rc == CCM_OK) {
    e = add_conditional(b_out, cudaGraphCondTypeIf, 0, &n_sel, 1, &h_sel, &n_if, &b_if, true);
    if (e != cudaSuccess) rc = set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  }
  if (rc == CCM_OK) rc = capture_trial_into(r, b_if, p, rp, CgHandles{0, 0, p});
  *node = n_if;
  return rc;
}

// The iteration loop of a whole solve, added to `g` after `deps`, one level of
// conditional nodes deep:
//   WHILE(outer) { select(0) -> IF { trial parity 0 } -> select(1) -> IF { trial
//                  parity 1 } -> guard }
// A round takes the next trial from the buffer parity that holds x (one trial,
// or two when the first one is accepted); the control kernels only update the
// state record, the selectors read it, and the guard keeps the loop open while
// the solve runs and bounds the rounds by itself.  (Line searches as WHILE
// nodes nested inside this loop stopped iterating after a few rounds on B200
// with driver 580; one level of IF nodes inside one WHILE does not need it.)
int add_solve_loop(CgRun &r, const CgRuleParams &rp, cudaGraph_t g,
                   cudaGraphConditionalHandle h_out, const cudaGraphNode_t *deps, size_t ndeps,
                   cudaGraphNode_t *n_out) {
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h_out;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaError_t e = cudaGraphAddNode(n_out, g, deps, ndeps, &np);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  cudaGraph_t b_out = np.conditional.phGraph_out[0];
  cudaGraphNode_t n_start = nullptr, n_t0 = nullptr, n_t1 = nullptr, n_guard = nullptr;
  e = cudaGraphAddEmptyNode(&n_start, b_out, nullptr, 0);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  // every round takes at least one trial while the solve runs; the control
  // kernels end a solve after (max_iterations + 1) 2 (max_linesearch + 1) trials
  const int max_rounds = (rp.max_iterations + 1) * 2 * (rp.max_linesearch + 1) + 4;
  int rc = add_parity_trial(r, rp, b_out, n_start, 0, &n_t0);
  if (rc == CCM_OK) rc = add_parity_trial(r, rp, b_out, n_t0, 1, &n_t1);
  if (rc == CCM_OK) rc = capture_small(r, b_out, &n_t1, 1, 2, h_out, max_rounds, &n_guard);
  return rc;
}

// Whole solve after the initial evaluation (on the host's stream): the loop,
// then the read-back.
int build_solve_graph(CgRun &r, const CgRuleParams &rp) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg graph: %s", cudaGetErrorString(e));
  cudaGraphConditionalHandle h_out;
  cudaGraphNode_t n_out = nullptr;
  e = cudaGraphConditionalHandleCreate(&h_out, g, 1, cudaGraphCondAssignDefault);
  int rc = e == cudaSuccess ? CCM_OK
                            : set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  if (rc == CCM_OK) rc = add_solve_loop(r, rp, g, h_out, nullptr, 0, &n_out);
  if (rc == CCM_OK) rc = capture_readback(r, g, n_out);
  if (rc == CCM_OK) {
    e = cudaGraphInstantiate(&r.exec[0], g, 0);
    if (e != cudaSuccess) rc = set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  }
  cudaGraphDestroy(g);
  return rc;
}

// One iteration of parity p: WHILE(ls) { trial }, then the read-back.
int build_iteration_graph(CgRun &r, int p, const CgRuleParams &rp) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "cg graph: %s", cudaGetErrorString(e));
  cudaGraphConditionalHandle h_ls;
  cudaGraphNode_t n_ls;
  cudaGraph_t b_ls;
  e = add_conditional(g, cudaGraphCondTypeWhile, 1, nullptr, 0, &h_ls, &n_ls, &b_ls);
  int rc = e == cudaSuccess ? CCM_OK
                            : set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  if (rc == CCM_OK) rc = capture_trial_into(r, b_ls, p, rp, CgHandles{h_ls, 1, p});
  if (rc == CCM_OK) rc = capture_readback(r, g, n_ls);
  if (rc == CCM_OK) {
    e = cudaGraphInstantiate(&r.exec[1 + p], g, 0);
    if (e != cudaSuccess) rc = set_last_error(CCM_ERR_UNSUPPORTED, "cg graph: %s", cudaGetErrorString(e));
  }
  cudaGraphDestroy(g);
  return rc;
}

// CCM_ERR_DEVICE for a solve that ended on a device-side bound, with its state.
int device_error(const char *who, const CgCtl &h) {
  return set_last_error(CCM_ERR_DEVICE,
                        "%s: %s (round %d, iteration %d, evaluation %d, parity %d, trial %d)", who,
                        h.status == kCgLoopBound ? "the solve graph's round bound was reached"
                                                 : "device wait timed out in an evaluation",
                        h.rounds, h.iter, h.evals, h.parity, h.ls);
}

int finish(CgRun &r, float *d_x, ccm_cg_result *result, int stopped) {
  ccm_context *c = r.c;
  const CgCtl &h = *r.h_ctl;
  cudaError_t e = cudaSuccess;
  // leave the final x in the caller's buffer
  if (h.parity == 1)
    e = cudaMemcpyAsync(d_x, r.xb[1], sizeof(float) * (size_t)r.n, cudaMemcpyDeviceToDevice,
                        c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  ccm_cg_result res;
  std::memset(&res, 0, sizeof(res));
  res.status = stopped ? CCM_CG_STOPPED : h.status;
  res.iterations = h.iter;
  res.evaluations = h.evals;
  res.fx = h.f;
  res.gnorm = std::sqrt(h.gg);
  const CgCtl hc = h;
  free_run(r);
  if (e != cudaSuccess) return set_last_error(CCM_ERR_CUDA, "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
  if (hc.status == CCM_ERR_DEVICE || hc.status == kCgLoopBound) return device_error("ccm_conjugrad_gpu", hc);
  if (result) *result = res;
  return CCM_OK;
}

}  // namespace

// ---------------------------------------------------------------- solves in a shared graph
// The batch solver puts the solves of many alignments into one graph: each one
// a chain initial evaluation -> start -> outer WHILE -> final x -> read-back,
// with no edge between alignments, so the graph's independent branches run
// concurrently.  All captures go through the context's stream.
struct ccm::CgGraphSolve {
  CgRun r;
};

int ccm::cg_graph_solve_add(ccm_context *c, float *d_x, const ccm_cg_params *params,
                            cudaGraph_t graph, CgGraphSolve **out, cudaGraphNode_t *last) {
  *out = nullptr;
  int rc = check_params(params, "ccm_solve_batch");
  if (rc != CCM_OK) return rc;
  if (c->path == CCM_PATH_SIMT_F64)
    return set_last_error(CCM_ERR_INVALID, "ccm_solve_batch: needs a float evaluation path");
  const CgRuleParams rp = rule_params(*params);
  CgGraphSolve *gs = new CgGraphSolve();
  CgRun &r = gs->r;
  r.c = c;
  r.mem_mark = c->mem_used;
  r.n = c->nvarp;
  r.xb[0] = d_x;
  r.fused = c->path == CCM_PATH_TC_BF16X2 || c->path == CCM_PATH_TC_BF16X3 ||
            c->path == CCM_PATH_TC_I8X3 || c->path == CCM_PATH_TC_I8SP;
  const size_t bytes = sizeof(float) * (size_t)r.n;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.xb[1]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.gb[0]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.gb[1]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.s), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.d_ctl), sizeof(CgCtl)));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.d_part), sizeof(double) * 6 * kDotBlocks));
  r.h_ctl = static_cast<CgCtl *>(pinned_small_alloc(kCgCtlHead));
  if (!r.h_ctl) chk(cudaErrorMemoryAllocation);
  if (e != cudaSuccess) {
    free_run(r);
    delete gs;
    (void)cudaGetLastError();
    return set_last_error(e == cudaErrorMemoryAllocation ? CCM_ERR_NOMEM : CCM_ERR_CUDA,
                          "ccm_solve_batch: %s", cudaGetErrorString(e));
  }
  // the batch solver starts every alignment's couplings at zero
  if ((rc = choose_span(r, true)) != CCM_OK) {
    free_run(r);
    delete gs;
    return rc;
  }
  const bool prof = c->prof_on;
  c->prof_on = false;
  cudaStream_t s = c->stream;
  cudaGraphConditionalHandle h_out;
  e = cudaGraphConditionalHandleCreate(&h_out, graph, 1, cudaGraphCondAssignDefault);
  std::vector<cudaGraphNode_t> front;
  // initial evaluation, g0.g0, start (which sets the outer loop's value)
  if (e == cudaSuccess)
    e = cudaStreamBeginCaptureToGraph(s, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = enqueue_evaluation(c, r.xb[0], r.gb[0]);
    cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(r.gb[0], nullptr, nullptr, r.span, r.d_part);
    cg_start_kernel<<<1, 256, 0, s>>>(r.d_ctl, r.d_part, kDotBlocks, c->d_out, nullptr, h_out, 1);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    if (cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &nd) == cudaSuccess)
      front.assign(deps, deps + nd);
    cudaGraph_t tmp = nullptr;
    e = cudaStreamEndCapture(s, &tmp);
  }
  cudaGraphNode_t n_out = nullptr;
  if (e != cudaSuccess && rc == CCM_OK)
    rc = set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: %s", cudaGetErrorString(e));
  if (rc == CCM_OK && front.empty()) rc = set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: capture");
  if (rc == CCM_OK) rc = add_solve_loop(r, rp, graph, h_out, front.data(), front.size(), &n_out);
  // the final x into the caller's buffer, the state record to the host
  if (rc == CCM_OK) {
    e = cudaStreamBeginCaptureToGraph(s, graph, &n_out, nullptr, 1, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cg_final_x_kernel<<<grid_for(r.n), 256, 0, s>>>(r.d_ctl, r.xb[1], r.xb[0], r.n);
      cudaMemcpyAsync(r.h_ctl, r.d_ctl, kCgCtlHead, cudaMemcpyDeviceToHost, s);
      cudaStreamCaptureStatus cs;
      const cudaGraphNode_t *deps = nullptr;
      size_t nd = 0;
      if (cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &nd) == cudaSuccess && nd == 1)
        *last = deps[0];
      else
        e = cudaErrorUnknown;
      cudaGraph_t tmp = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(s, &tmp);
      if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) rc = set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: %s", cudaGetErrorString(e));
  }
  c->prof_on = prof;
  if (rc != CCM_OK) {
    free_run(r);
    delete gs;
    return rc;
  }
  *out = gs;
  return CCM_OK;
}

int ccm::cg_graph_solve_result(const CgGraphSolve *gs, ccm_cg_result *res) {
  const CgCtl &h = *gs->r.h_ctl;
  std::memset(res, 0, sizeof(*res));
  res->status = h.status;
  res->iterations = h.iter;
  res->evaluations = h.evals;
  res->fx = h.f;
  res->gnorm = std::sqrt(h.gg);
  if (h.status == CCM_ERR_DEVICE || h.status == kCgLoopBound) return device_error("ccm_solve_batch", h);
  return CCM_OK;
}

void ccm::cg_graph_solve_free(CgGraphSolve *gs) {
  if (!gs) return;
  free_run(gs->r);
  delete gs;
}

extern "C" {

void ccm_cg_params_default(ccm_cg_params *p) {
  if (!p) return;
  // src/ccmpred.c:222-229, 526-534, as the reference holds them (float)
  p->max_iterations = 250;
  p->epsilon = (double)0.01f;
  p->k = 5;
  p->max_linesearch = 5;
  p->alpha_mul = 0.5;
  p->ftol = (double)1e-4f;
  p->wolfe = (double)0.2f;
  p->min_gnorm = 0.0;
}

int ccm_conjugrad_gpu(ccm_context *c, float *d_x, long long n, const ccm_cg_params *params,
                      ccm_progress_t progress, void *instance, ccm_cg_result *result) {
  if (!c || !d_x || !params) return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_gpu: null argument");
  if (n != c->nvarp)
    return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_gpu: n %lld != nvar_padded %lld", n, c->nvarp);
  if (c->path == CCM_PATH_SIMT_F64)
    return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_gpu: needs a float evaluation path");
  int rc = check_params(params, "ccm_conjugrad_gpu");
  if (rc != CCM_OK) return rc;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  const CgRuleParams rp = rule_params(*params);
  CgRun r;
  r.c = c;
  r.mem_mark = c->mem_used;
  r.n = n;
  r.xb[0] = d_x;
  r.want_xx = progress != nullptr;
  // tensor-core paths take the step inside the first pass over x
  r.fused = c->path == CCM_PATH_TC_BF16X2 || c->path == CCM_PATH_TC_BF16X3 ||
            c->path == CCM_PATH_TC_I8X3 || c->path == CCM_PATH_TC_I8SP;
  const size_t bytes = sizeof(float) * (size_t)n;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.xb[1]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.gb[0]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.gb[1]), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.s), bytes));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.d_ctl), sizeof(CgCtl)));
  chk(dev_alloc_raw(c, reinterpret_cast<void **>(&r.d_part), sizeof(double) * 6 * kDotBlocks));
  static_assert(kCgCtlHead <= 256, "the control record's scalars must fit a pinned slot");
  r.h_ctl = static_cast<CgCtl *>(pinned_small_alloc(kCgCtlHead));
  if (!r.h_ctl) chk(cudaErrorMemoryAllocation);
  if (e != cudaSuccess) {
    free_run(r);
    (void)cudaGetLastError();  // a failed allocation must not surface in a later launch check
    return set_last_error(e == cudaErrorMemoryAllocation ? CCM_ERR_NOMEM : CCM_ERR_CUDA,
                          "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
  }
  if ((rc = choose_span(r, false)) != CCM_OK) {
    free_run(r);
    return rc;
  }
  // profiling marks are not captured into the solve's graphs
  const bool prof = c->prof_on;
  c->prof_on = false;

  // initial evaluation at x0: f0, g0, g0.g0
  rc = enqueue_evaluation(c, r.xb[0], r.gb[0]);
  if (rc == CCM_OK) {
    cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(r.gb[0], nullptr, nullptr, r.span, r.d_part);
    cg_start_kernel<<<1, 256, 0, s>>>(r.d_ctl, r.d_part, kDotBlocks, c->d_out, nullptr, 0, 0);
    count_launch(c, 2);
    e = cudaMemcpyAsync(r.h_ctl, r.d_ctl, kCgCtlHead, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = set_last_error(CCM_ERR_CUDA, "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
  }
  // the graphs: the whole solve without a progress callback, else one per parity
  bool whole = progress == nullptr;
  if (rc == CCM_OK && r.h_ctl->status == kCgRunning) {
    if (!progress) {
      rc = build_solve_graph(r, rp);
      if (rc == CCM_ERR_UNSUPPORTED) {
        // nested conditional nodes refused by this driver: one graph per iteration
        (void)cudaGetLastError();
        whole = false;
        rc = CCM_OK;
      }
    }
    if (rc == CCM_OK && !whole) {
      rc = build_iteration_graph(r, 0, rp);
      if (rc == CCM_OK) rc = build_iteration_graph(r, 1, rp);
    }
  }
  c->prof_on = prof;
  if (rc != CCM_OK) { free_run(r); return rc; }

  int stopped = 0;
  if (r.h_ctl->status == kCgRunning) {
    if (whole) {
      e = cudaGraphLaunch(r.exec[0], s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    } else {
      while (e == cudaSuccess && r.h_ctl->status == kCgRunning) {
        const int iter0 = r.h_ctl->iter;
        e = cudaGraphLaunch(r.exec[1 + r.h_ctl->parity], s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
        const CgCtl &h = *r.h_ctl;
        if (h.iter > iter0 && progress &&
            progress(instance, r.xb[h.parity], r.gb[h.parity], (float)h.f, (float)std::sqrt(h.xx),
                     (float)std::sqrt(h.gg), (float)h.step, (int)n, h.iter, h.ls_last)) {
          stopped = 1;
          break;
        }
      }
    }
    if (e != cudaSuccess) {
      free_run(r);
      return set_last_error(CCM_ERR_CUDA, "ccm_conjugrad_gpu: %s", cudaGetErrorString(e));
    }
  }
  c->launches += (long long)(r.h_ctl->evals - 1) * r.trial_kernels;
  return finish(r, d_x, result, stopped);
}

}  // extern "C"

// ---------------------------------------------------------------- callback CG
// conjugrad_gpu with an evaluate callback that is not this library's own: the
// same kernels and rules, one host call of the callback per trial, on the legacy
// default stream (the stream of the reference's evaluate_cuda).
int ccm::conjugrad_callback_gpu(float *d_x, long long n, ccm_eval_callback eval,
                                ccm_progress_t progress, void *instance,
                                const ccm_cg_params *params, ccm_cg_result *result) {
  int rc = check_params(params, "conjugrad_gpu");
  if (rc != CCM_OK) return rc;
  const CgRuleParams rp = rule_params(*params);
  cudaStream_t s = 0;  // legacy default stream
  const size_t bytes = sizeof(float) * (size_t)n;
  const VecSpan flat{n, 0, 0, 0, 0};  // a foreign evaluation: every element
  float *xb[2] = {d_x, nullptr}, *gb[2] = {nullptr, nullptr}, *dir = nullptr;
  CgCtl *d_ctl = nullptr;
  double *d_part = nullptr, *d_f = nullptr;
  cudaError_t e = cudaMallocAsync(&xb[1], bytes, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&gb[0], bytes, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&gb[1], bytes, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&dir, bytes, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_ctl, sizeof(CgCtl), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_part, sizeof(double) * 6 * kDotBlocks, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_f, sizeof(double), s);
  CgCtl *h = static_cast<CgCtl *>(pinned_small_alloc(kCgCtlHead));
  double *h_f = static_cast<double *>(pinned_small_alloc(sizeof(double)));
  if (e == cudaSuccess && (!h || !h_f)) e = cudaErrorMemoryAllocation;
  const CgHandles none{0, 0, 0};
  int stopped = 0;
  // one evaluation by the callback at xb[q] into gb[q]; its f goes to the device
  auto evaluate = [&](int q) -> cudaError_t {
    cudaError_t r = cudaStreamSynchronize(s);  // x complete before the callback reads it
    if (r != cudaSuccess) return r;
    *h_f = (double)eval(instance, xb[q], gb[q], (int)n);
    return cudaMemcpyAsync(d_f, h_f, sizeof(double), cudaMemcpyHostToDevice, s);
  };
  if (e == cudaSuccess) e = evaluate(0);
  if (e == cudaSuccess) {
    cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(gb[0], nullptr, nullptr, flat, d_part);
    cg_start_kernel<<<1, 256, 0, s>>>(d_ctl, d_part, kDotBlocks, nullptr, d_f, 0, 0);
    e = cudaMemcpyAsync(h, d_ctl, kCgCtlHead, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  while (e == cudaSuccess && h->status == kCgRunning) {
    const int p = h->parity, iter0 = h->iter;
    cg_dir_kernel<<<grid_for(n), 256, 0, s>>>(gb[p], dir, d_ctl, flat);
    cg_step_kernel<<<grid_for(n), 256, 0, s>>>(xb[p], dir, &d_ctl->alpha, xb[1 - p], n);
    e = evaluate(1 - p);
    if (e != cudaSuccess) break;
    cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(gb[1 - p], dir, gb[p], flat, d_part);
    if (progress) cg_dots_kernel<<<kDotBlocks, 256, 0, s>>>(xb[1 - p], nullptr, nullptr, flat,
                                                           d_part + 3 * kDotBlocks);
    cg_control_kernel<<<1, 256, 0, s>>>(d_ctl, rp, d_part, kDotBlocks, progress ? 1 : 0, nullptr,
                                        d_f, none);
    e = cudaMemcpyAsync(h, d_ctl, kCgCtlHead, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && progress && h->iter > iter0 &&
        progress(instance, xb[h->parity], gb[h->parity], (float)h->f, (float)std::sqrt(h->xx),
                 (float)std::sqrt(h->gg), (float)h->step, (int)n, h->iter, h->ls_last)) {
      stopped = 1;
      break;
    }
  }
  ccm_cg_result res;
  std::memset(&res, 0, sizeof(res));
  if (e == cudaSuccess && h->parity == 1)
    e = cudaMemcpyAsync(d_x, xb[1], bytes, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    res.status = stopped ? CCM_CG_STOPPED : h->status;
    res.iterations = h->iter;
    res.evaluations = h->evals;
    res.fx = h->f;
    res.gnorm = std::sqrt(h->gg);
  }
  for (void *p : {(void *)xb[1], (void *)gb[0], (void *)gb[1], (void *)dir, (void *)d_ctl,
                  (void *)d_part, (void *)d_f})
    if (p) cudaFreeAsync(p, s);
  pinned_small_free(h);
  pinned_small_free(h_f);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return set_last_error(e == cudaErrorMemoryAllocation ? CCM_ERR_NOMEM : CCM_ERR_CUDA,
                          "conjugrad_gpu: %s", cudaGetErrorString(e));
  }
  if (result) *result = res;
  return CCM_OK;
}

// ---------------------------------------------------------------- host-vector CG
// conjugrad: host x, a callback with host pointers.  The same rules
// (ccm_cg_rules.cuh) on the host; dot products accumulate in FP64 in a fixed
// order, the vector updates are the device kernels' float operations.
int ccm::conjugrad_host_vectors(float *x, long long n, ccm_eval_callback eval,
                                ccm_progress_t progress, void *instance,
                                const ccm_cg_params *params, ccm_cg_result *result) {
  int rc = check_params(params, "conjugrad");
  if (rc != CCM_OK) return rc;
  const CgRuleParams rp = rule_params(*params);
  std::vector<float> xo((size_t)n), g0((size_t)n), g1((size_t)n), dir((size_t)n);
  float *xb[2] = {x, xo.data()}, *gb[2] = {g0.data(), g1.data()};
  std::vector<double> fhist;
  CgCtl c;
  std::memset(&c, 0, sizeof(c));
  auto dots = [&](const float *a, const float *b, const float *d, double out[3]) {
    double ab = 0.0, aa = 0.0, ad = 0.0;
    for (long long i = 0; i < n; ++i) {
      const double av = a[i];
      if (b) ab += av * (double)b[i];
      aa += av * av;
      if (d) ad += av * (double)d[i];
    }
    out[0] = ab;
    out[1] = aa;
    out[2] = ad;
  };
  double d3[3];
  const double f0 = (double)eval(instance, xb[0], gb[0], (int)n);
  dots(gb[0], nullptr, nullptr, d3);
  cg_rules_start(c, f0, d3[1]);
  int stopped = 0;
  while (c.status == kCgRunning) {
    const int p = c.parity, iter0 = c.iter;
    float *xp = xb[p], *xt = xb[1 - p], *gp = gb[p], *gt = gb[1 - p];
    if (c.dir_mode != 0) {
      const float b = (float)c.beta;
      for (long long i = 0; i < n; ++i)
        dir[(size_t)i] = c.dir_mode == 1 ? -gp[i] : fmaf(b, dir[(size_t)i], -gp[i]);
    }
    const float a = (float)c.alpha;
    for (long long i = 0; i < n; ++i) xt[i] = fmaf(a, dir[(size_t)i], xp[i]);
    CgTrial t;
    std::memset(&t, 0, sizeof(t));
    t.f = (double)eval(instance, xt, gt, (int)n);
    dots(gt, dir.data(), gp, d3);
    t.gts = d3[0];
    t.gtgt = d3[1];
    t.gtg = d3[2];
    if (progress) {
      dots(xt, nullptr, nullptr, d3);
      t.xtxt = d3[1];
    }
    cg_rules_trial(c, t, rp);
    if (progress && c.iter > iter0 &&
        progress(instance, xb[c.parity], gb[c.parity], (float)c.f, (float)std::sqrt(c.xx),
                 (float)std::sqrt(c.gg), (float)c.step, (int)n, c.iter, c.ls_last)) {
      stopped = 1;
      break;
    }
  }
  if (c.parity == 1) std::memcpy(x, xb[1], sizeof(float) * (size_t)n);
  if (result) {
    std::memset(result, 0, sizeof(*result));
    result->status = stopped ? CCM_CG_STOPPED : c.status;
    result->iterations = c.iter;
    result->evaluations = c.evals;
    result->fx = c.f;
    result->gnorm = std::sqrt(c.gg);
  }
  return CCM_OK;
}

extern "C" int ccm_conjugrad_host(ccm_context *c, float *x, long long n, const ccm_cg_params *params,
                                  ccm_progress_t progress, void *instance, ccm_cg_result *result) {
  if (!c || !x) return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_host: null argument");
  if (n != c->nvarp)
    return set_last_error(CCM_ERR_INVALID, "ccm_conjugrad_host: n %lld != nvar_padded %lld", n, c->nvarp);
  cudaSetDevice(c->device);
  float *d_x = nullptr;
  const size_t bytes = sizeof(float) * (size_t)n;
  cudaError_t e = dev_alloc_raw(c, reinterpret_cast<void **>(&d_x), bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return set_last_error(CCM_ERR_NOMEM, "ccm_conjugrad_host: %s", cudaGetErrorString(e));
  }
  e = cudaMemcpyAsync(d_x, x, bytes, cudaMemcpyHostToDevice, c->stream);
  int rc = CCM_OK;
  if (e == cudaSuccess) rc = ccm_conjugrad_gpu(c, d_x, n, params, progress, instance, result);
  if (e == cudaSuccess && rc == CCM_OK) e = cudaMemcpyAsync(x, d_x, bytes, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFreeAsync(d_x, c->stream);
  c->mem_used -= bytes;
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
