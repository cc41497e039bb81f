// The rules of the nonlinear conjugate-gradient optimizer, as one set of
// __host__ __device__ functions over a small state record: the device CG
// (ccm_cg.cu) applies them in a one-thread control kernel after every
// line-search trial, the host-vector CG (conjugrad) applies the same code on the
// host.  libconjugrad, the reference's optimizer (called at
// src/ccmpred.c:632,644 with the parameters of src/ccmpred.c:526-534), is absent
// from the reference checkout, so these rules are this project's own, written
// from the parameter names and Nocedal & Wright, "Numerical Optimization", 2nd
// ed., ch. 3 and 5.2:
//
//   s0 = -g0, alpha0 = 1 / ||g0||
//   per iteration, at most max_linesearch trials x_t = x + alpha s:
//     sufficient decrease (A):  f_t <= f + ftol alpha g.s
//     curvature (C):            g_t.s >= wolfe g.s        (g.s < 0)
//     A and C                  -> accept
//     A, not C (slope still steep: the step is short), two trials left
//                              -> remember alpha, try the secant step
//                                 alpha g.s / (g.s - g_t.s), the zero of the
//                                 line through the two slopes, kept in
//                                 [1.5, 16] alpha (alpha / alpha_mul when
//                                 g_t.s <= g.s, no zero ahead)
//     A, not C, fewer trials   -> accept
//     not A after an expansion -> retreat: the remembered step once more
//                                 (it met A; the trial repeats it exactly, and
//                                 is accepted)
//     not A otherwise          -> the minimiser of the quadratic through f,
//                                 g.s and f_t, kept in [0.1, alpha_mul] alpha
//   trials exhausted without a step: if s is not -g, restart along s = -g with
//     alpha = 1 / ||g|| and a fresh trial budget, else fail (line search)
//   after a step: beta = max(0, g_t.(g_t - g) / g.g)      (Polak-Ribiere+)
//     s = -g_t + beta s; if that is not a descent direction, s = -g_t
//     next alpha = 2 (f - f_t) / -(g_t.s)                  (N&W eq. 3.60)
//   stop after an iteration i when i >= k and (f_{i-k} - f_i) / |f_i| < epsilon
//     (src/ccmpred.c:192-196, "-e/-k"), when ||g|| <= min_gnorm (if set),
//     or at max_iterations.
#pragma once

#include <cmath>
#include <cstddef>

#include "../../include/ccmpred_b200.h"

namespace ccm {

constexpr int kCgHist = 257;  // ring of accepted f: k <= 256
constexpr int kCgRunning = 0x7fff;
constexpr int kCgLoopBound = -1019;  // the whole-solve graph's round bound was reached

struct CgRuleParams {
  int max_iterations, k, max_linesearch;
  int pad;
  double epsilon, alpha_mul, ftol, wolfe, min_gnorm;
};

// What a trial produces: f(x_t) and the dot products of its gradient g_t with
// the direction s, with itself and with the gradient g at x; x_t.x_t when asked.
struct CgTrial {
  double f, gts, gtgt, gtg, xtxt;
  int status;  // device error bits of the evaluation, 0 when clean
  int pad;
};

// State of the optimizer between trials (device memory in the device CG).  The
// scalars come first: the host reads back only the part before fhist.
struct CgCtl {
  double f, gg, gs;     // at the current x: f, g.g, g.s (s the current direction)
  double alpha;         // step of the next trial
  double alpha_good;    // a step of this line search that met A (0: none)
  double beta;          // of the direction update that dir_mode 2 applies
  double step, xx;      // last accepted step and x.x there (progress reports)
  int iter;             // accepted iterations
  int ls;               // trials of the current line search
  int ls_last;          // trials the last accepted iteration took
  int evals;            // evaluations, the initial one included
  int steepest;         // s == -g
  int retreat;          // the next trial repeats alpha_good
  int dir_mode;         // before the next trial: 0 keep s, 1 s = -g, 2 s = -g + beta s
  int parity;           // x is buffer `parity` (the trial writes the other one)
  int status;           // kCgRunning, or the CCM_CG_* outcome (CCM_ERR_DEVICE: a kernel timed out)
  int ls_active;        // 1 while the current line search continues
  int rounds;           // rounds of the whole-solve graph's outer loop (its bound)
  int pad;
  double fhist[kCgHist];  // f after iteration i at i % kCgHist
};
constexpr int kCgCtlHead = 8 * 8 + 12 * 4;  // bytes before fhist
static_assert(offsetof(CgCtl, fhist) == kCgCtlHead, "CgCtl: scalars before fhist");

__host__ __device__ inline bool cg_finite(double v) { return v - v == 0.0; }

// Growth of a step that met sufficient decrease with the slope gts at x_t still
// steeper than wolfe gs (gs < 0): the secant estimate of where the slope along s
// reaches zero, gs / (gs - gts) of the step, limited to [kCgGrowMin, kCgGrowMax];
// 1 / alpha_mul when gts <= gs (the slope has not risen: no zero ahead).
constexpr double kCgGrowMin = 1.5, kCgGrowMax = 16.0;
__host__ __device__ inline double cg_expansion(double gs, double gts, double alpha_mul) {
  if (!(gts > gs)) return 1.0 / alpha_mul;
  return fmin(fmax(gs / (gs - gts), kCgGrowMin), kCgGrowMax);
}

// After the initial evaluation at x0 (f0, g0.g0).
__host__ __device__ inline void cg_rules_start(CgCtl &c, double f0, double gg0) {
  c.f = f0;
  c.gg = gg0;
  c.iter = 0;
  c.ls = 0;
  c.ls_last = 0;
  c.evals = 1;
  c.fhist[0] = f0;
  c.alpha_good = 0.0;
  c.retreat = 0;
  c.beta = 0.0;
  c.step = 0.0;
  c.parity = 0;
  c.rounds = 0;
  if (!cg_finite(f0)) {
    c.status = CCM_CG_ERR_NONFINITE;
  } else if (!(gg0 > 0.0)) {
    c.status = CCM_CG_ALREADY_MINIMIZED;
  } else {
    c.status = kCgRunning;
  }
  c.ls_active = c.status == kCgRunning;
  c.dir_mode = 1;  // s0 = -g0
  c.steepest = 1;
  c.gs = -gg0;
  c.alpha = gg0 > 0.0 ? 1.0 / sqrt(gg0) : 0.0;
}

// Stop test after iteration c.iter.
__host__ __device__ inline void cg_rules_stop(CgCtl &c, const CgRuleParams &p) {
  const int i = c.iter;
  if (p.min_gnorm > 0.0 && sqrt(c.gg) <= p.min_gnorm) {
    c.status = CCM_CG_SUCCESS;
  } else if (i >= p.k && (c.fhist[(i - p.k) % kCgHist] - c.f) / fabs(c.f) < p.epsilon) {
    c.status = CCM_CG_SUCCESS;
  } else if (i >= p.max_iterations) {
    c.status = CCM_CG_ERR_MAXITER;
  }
}

// Apply one trial's result.  Returns true when the trial was accepted (the
// caller's x is then the trial point: c.parity has flipped).
__host__ __device__ inline bool cg_rules_trial(CgCtl &c, const CgTrial &t, const CgRuleParams &p) {
  c.ls++;
  c.evals++;
  c.dir_mode = 0;
  if (t.status != 0) {
    c.status = CCM_ERR_DEVICE;
    c.ls_active = 0;
    return false;
  }
  const bool suff = cg_finite(t.f) && t.f <= c.f + p.ftol * c.alpha * c.gs;
  const bool curv = p.wolfe <= 0.0 || t.gts >= p.wolfe * c.gs;  // wolfe <= 0: no curvature test
  bool accept = false;
  if (c.retreat) {
    accept = suff;  // the same step as an earlier trial that met A
  } else if (suff && (curv || c.ls + 2 > p.max_linesearch)) {
    accept = true;
  } else if (suff) {
    c.alpha_good = c.alpha;  // expand: the slope at x_t is still steep
    c.alpha = c.alpha * cg_expansion(c.gs, t.gts, p.alpha_mul);
  } else if (c.alpha_good > 0.0) {
    c.alpha = c.alpha_good;  // the expansion overshot: back to the good step
    c.retreat = 1;
  } else {
    const double den = 2.0 * (t.f - c.f - c.gs * c.alpha);
    double aq = (cg_finite(t.f) && den > 0.0) ? -c.gs * c.alpha * c.alpha / den
                                              : p.alpha_mul * c.alpha;
    aq = fmin(aq, p.alpha_mul * c.alpha);
    c.alpha = fmax(aq, 0.1 * c.alpha);
  }
  if (accept) {
    const double fnew = t.f, ggnew = t.gtgt;
    double beta = (ggnew - t.gtg) / c.gg;  // Polak-Ribiere+
    if (!(beta > 0.0)) beta = 0.0;
    double gs_new = -ggnew + beta * t.gts;
    if (!(gs_new < 0.0)) {  // not a descent direction: steepest descent
      beta = 0.0;
      gs_new = -ggnew;
    }
    c.step = c.alpha;
    c.xx = t.xtxt;
    double anext = 2.0 * (c.f - fnew) / -gs_new;
    if (!(anext > 0.0) || !cg_finite(anext)) anext = ggnew > 0.0 ? 1.0 / sqrt(ggnew) : 0.0;
    c.alpha = anext;
    c.beta = beta;
    c.dir_mode = beta == 0.0 ? 1 : 2;
    c.steepest = beta == 0.0;
    c.f = fnew;
    c.gg = ggnew;
    c.gs = gs_new;
    c.iter++;
    c.fhist[c.iter % kCgHist] = fnew;
    c.parity ^= 1;
    c.ls_last = c.ls;
    c.ls = 0;
    c.alpha_good = 0.0;
    c.retreat = 0;
    c.ls_active = 0;
    if (!(ggnew > 0.0)) c.status = CCM_CG_SUCCESS;  // a stationary point
    else cg_rules_stop(c, p);
    return true;
  }
  // (an expansion is taken only with two trials left, so a retreat always fits)
  if (c.ls >= p.max_linesearch) {
    if (!c.steepest) {  // restart along -g with a fresh budget
      c.dir_mode = 1;
      c.steepest = 1;
      c.gs = -c.gg;
      c.alpha = 1.0 / sqrt(c.gg);
      c.alpha_good = 0.0;
      c.retreat = 0;
      c.ls = 0;
    } else {
      c.status = CCM_CG_ERR_LINESEARCH;
      c.ls_active = 0;
    }
  }
  return false;
}

}  // namespace ccm
