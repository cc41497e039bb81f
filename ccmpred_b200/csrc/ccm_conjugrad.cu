// The optimizer entry points under libconjugrad's names (include/conjugrad.h),
// which the reference's driver calls: conjugrad_init and the parameter fields at
// src/ccmpred.c:526-534, conjugrad_gpu at src/ccmpred.c:632 (device x, the
// evaluate_cuda callback), conjugrad at src/ccmpred.c:644,647 (host x),
// conjugrad_malloc / conjugrad_free at src/ccmpred.c:493,514,671,766-768.
//
// conjugrad_gpu recognises this library's own evaluate_cuda with an instance
// set up by init_cuda and then runs the device CG of ccm_conjugrad_gpu on the
// instance's context (line search and iteration on the device, the trial step
// fused into the evaluation); any other callback is driven per trial by
// conjugrad_callback_gpu.  conjugrad recognises evaluate_b200 (the host-pointer
// backend) the same way and otherwise applies the rules on host vectors.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/conjugrad.h"
#include "ccm_internal.cuh"

using namespace ccm;

namespace {

ccm_cg_params to_params(const conjugrad_parameter_t *p) {
  ccm_cg_params c;
  std::memset(&c, 0, sizeof(c));
  c.max_iterations = p->max_iterations;
  c.k = p->k;
  c.max_linesearch = p->max_linesearch;
  c.epsilon = (double)p->epsilon;
  c.alpha_mul = (double)p->alpha_mul;
  c.ftol = (double)p->ftol;
  c.wolfe = (double)p->wolfe;
  c.min_gnorm = (double)p->min_gnorm;
  return c;
}

// CCM_CG_* -> the return values the reference prints (src/ccmpred.c:650-660)
int to_conjugrad_status(int s) {
  switch (s) {
    case CCM_CG_SUCCESS: return CONJUGRAD_SUCCESS;
    case CCM_CG_ALREADY_MINIMIZED: return CONJUGRAD_ALREADY_MINIMIZED;
    case CCM_CG_STOPPED: return CONJUGRAD_SUCCESS;
    case CCM_CG_ERR_MAXITER: return CONJUGRADERR_MAXIMUMITERATION;
    case CCM_CG_ERR_LINESEARCH: return CONJUGRADERR_MAXIMUMLINESEARCH;
    default: return CONJUGRADERR_UNKNOWN;
  }
}

ccm_context *own_context(conjugrad_evaluate_t ev, conjugrad_evaluate_t ours, void *instance) {
  if (ev != ours || !instance) return nullptr;
  void *extra = static_cast<ccm_userdata *>(instance)->extra;
  return is_context(extra) ? static_cast<ccm_context *>(extra) : nullptr;
}

int finish(const char *who, int rc, const ccm_cg_result &res, conjugrad_float_t *fx) {
  if (rc != CCM_OK) {
    fprintf(stderr, "%s: %s\n", who, ccm_last_error());
    return CONJUGRADERR_UNKNOWN;
  }
  if (fx) *fx = (conjugrad_float_t)res.fx;
  return to_conjugrad_status(res.status);
}

}  // namespace

extern "C" {

conjugrad_parameter_t *conjugrad_init(void) {
  conjugrad_parameter_t *p =
      static_cast<conjugrad_parameter_t *>(std::malloc(sizeof(conjugrad_parameter_t)));
  if (!p) return nullptr;
  ccm_cg_params d;
  ccm_cg_params_default(&d);
  p->max_linesearch = d.max_linesearch;
  p->max_iterations = d.max_iterations;
  p->k = d.k;
  p->epsilon = (conjugrad_float_t)d.epsilon;
  p->ftol = (conjugrad_float_t)d.ftol;
  p->wolfe = (conjugrad_float_t)d.wolfe;
  p->alpha_mul = (conjugrad_float_t)d.alpha_mul;
  p->min_gnorm = (conjugrad_float_t)d.min_gnorm;
  return p;
}

conjugrad_float_t *conjugrad_malloc(int n) {
  if (n <= 0) return nullptr;
  void *p = nullptr;
  if (posix_memalign(&p, 64, sizeof(conjugrad_float_t) * (size_t)n) != 0) return nullptr;
  return static_cast<conjugrad_float_t *>(p);
}

void conjugrad_free(conjugrad_float_t *x) { std::free(x); }

int conjugrad_gpu(int n, conjugrad_float_t *d_x, conjugrad_float_t *fx,
                  conjugrad_evaluate_t proc_evaluate, conjugrad_progress_t proc_progress,
                  void *instance, conjugrad_parameter_t *param) {
  if (n <= 0 || !d_x || !proc_evaluate || !param) {
    fprintf(stderr, "conjugrad_gpu: invalid arguments\n");
    return CONJUGRADERR_UNKNOWN;
  }
  const ccm_cg_params cp = to_params(param);
  ccm_cg_result res;
  std::memset(&res, 0, sizeof(res));
  const ccm_progress_t progress = reinterpret_cast<ccm_progress_t>(proc_progress);
  int rc;
  ccm_context *c = own_context(proc_evaluate, evaluate_cuda, instance);
  if (c && c->nvarp == (long long)n)
    rc = ccm_conjugrad_gpu(c, d_x, n, &cp, progress, instance, &res);
  else
    rc = conjugrad_callback_gpu(d_x, n, proc_evaluate, progress, instance, &cp, &res);
  return finish("conjugrad_gpu", rc, res, fx);
}

int conjugrad(int n, conjugrad_float_t *x, conjugrad_float_t *fx,
              conjugrad_evaluate_t proc_evaluate, conjugrad_progress_t proc_progress,
              void *instance, conjugrad_parameter_t *param) {
  if (n <= 0 || !x || !proc_evaluate || !param) {
    fprintf(stderr, "conjugrad: invalid arguments\n");
    return CONJUGRADERR_UNKNOWN;
  }
  const ccm_cg_params cp = to_params(param);
  ccm_cg_result res;
  std::memset(&res, 0, sizeof(res));
  const ccm_progress_t progress = reinterpret_cast<ccm_progress_t>(proc_progress);
  int rc;
  // evaluate_b200 without a progress callback: the device CG on the context (a
  // progress callback of conjugrad expects host pointers, which it would not get)
  ccm_context *c = progress ? nullptr : own_context(proc_evaluate, evaluate_b200, instance);
  if (c && c->nvarp == (long long)n)
    rc = ccm_conjugrad_host(c, x, n, &cp, progress, instance, &res);
  else
    rc = conjugrad_host_vectors(x, n, proc_evaluate, progress, instance, &cp, &res);
  return finish("conjugrad", rc, res, fx);
}

}  // extern "C"
