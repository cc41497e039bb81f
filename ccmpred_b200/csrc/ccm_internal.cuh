// Internal state of a ccm_context and the argument blocks of its kernels.
#pragma once

#include <cstdint>
#include <utility>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/ccmpred_b200.h"

namespace ccm {

// Launch `k` on `s` with programmatic stream serialisation: it may be scheduled
// before the previous kernel of the stream completes and waits for it on the
// device (griddep_wait in every kernel of the evaluation).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

// device status bits (ccm_result.status)
constexpr int kErrFwdTimeout = 1;
constexpr int kErrBwdTimeout = 2;

struct FwdMaps {
  CUtensorMap a;      // one-hot O [Npad][S], box 32 (slots, K) x 128 (rows), 64B swizzle
  CUtensorMap b[3];   // Wperm_i  [S][S],   box 64 (out slots, N) x 32 (in slots, K)
};

struct BwdMaps {
  CUtensorMap o;      // one-hot O [Npad][S], box 64 (slots, M/N) x 32 (rows, K)
  CUtensorMap r[3];   // R_i       [Npad][S], same box
};

// Integer path (CCM_PATH_TC_I8X3): 8-bit operands, s32 tensor-core accumulation.
struct I8FwdMaps {
  CUtensorMap a1, a128;  // one-hot O x1 / x128 [Npad][S] u8, box 64 (slots, K) x 128 (rows), 64B swizzle
  CUtensorMap b[3];      // digits of W [S][S] s8, box 128 (out slots, N) x 64 (in slots, K), 128B swizzle
};

struct I8BwdMaps {
  CUtensorMap o1, o128;  // one-hot O x1 / x128 [Npad][S] u8, box 128 (slots) x 32 (rows), 128B swizzle
  CUtensorMap r[3];      // digits of R [Npad][S] s8, same box
};

// Sparse integer forward (CCM_PATH_TC_I8SP): compressed one-hot A and its
// metadata, K in the order k' = l * 21 + q.
// All four are tiled stores of shared-memory images (see ccm_tc_i8.cu) viewed
// as rows of 256 bytes, no TMA swizzle; one box is one tile of one stage.
struct I8SpMaps {
  CUtensorMap a1, a128;  // compressed one-hot x1 / x128: 8 KB tiles, box 256 x 32
  CUtensorMap e;         // metadata: 2 KB tiles, box 256 x 8
  CUtensorMap b[3];      // digits of W: 12 KB tiles (128 K rows x 96 slots), box 256 x 48
};

struct I8PrepArgs {
  int8_t *wdig[3];
  const uint32_t *colmax;  // per coupling column (a*L + j): max |W| as float bits
  const float *enc;        // per slot: the digit encoding factor 2^(21 - e), 0 for padding
  double *part_reg;
  int L, S;
  int KB;  // sparse forward: K blocks of 128 rows (tiled digit layout)
  float inv_L;
  float lambda_pair;
  float g2_coef;
  int ncols;  // elements of a row that prep reads and writes: 32 L, or 21 L (padding skipped)
};

struct I8FwdArgs {
  const uint8_t *msa;
  const float *w;
  const float *x1;
  const uint32_t *colmax;
  int8_t *r[3];
  double *part_f;
  int *status;
  int L, N, S, T, Npad, m_tiles;
  int KP;  // sparse forward: logical K (a multiple of 256)
  // digits of R: R * r_enc with r_enc = 2^(21 - eR), eR = ceil(log2 max |w|) (0 for
  // uniform weights), so that |R| <= max |w| fills, and stays within, 21 bits
  float r_enc;
  // > 0: instead of waiting for a finished accumulator, the epilogue waits this
  // many clock cycles on a barrier that nothing arrives on, so that the wait runs
  // out and the kernel takes its timeout path (a test of that path; 0 normally)
  long long acc_wait_cycles;
};

struct PrepArgs {
  __nv_bfloat16 *wperm[3];
  // Fused CG step (tc_prep<.., true>): the parameters evaluated are
  // xt = x + alpha * s, computed here, written to xt and used at once.
  const float *step_x, *step_s;  // full vectors (nvar_padded)
  const double *alpha;           // device scalar
  float *xt;                     // full vector out
  long long nsp;                 // nsingle_padded
  double *part_reg;
  int L, S;
  float lambda_pair;
  float g2_coef;  // g2 starts at g2_coef * lambda_pair * x
};

struct FwdArgs {
  const uint8_t *msa;
  const float *w;
  const float *x1;
  __nv_bfloat16 *r[3];
  double *part_f;
  int *status;
  int L, N, S, T, Npad, m_tiles;
};

struct BwdArgs {
  const float *x2;
  float *g2;
  float *g1d;
  const int2 *tiles;
  int *status;
  int n_tiles, L, S, Npad;
  float lambda_pair;
  float r_dec;  // integer path: 2^(eR - 21), the inverse of I8FwdArgs::r_enc
};

struct FinalizeArgs {
  const double *part_f;
  long long n_part_f;
  const double *part_reg;
  long long n_part_reg;
  const float *x1;
  const float *g1d;
  float *g1;
  long long nsp;
  int L;
  float lambda_single, lambda_pair;
  ccm_result *out;
  double *block_part;  // kFinBlocks x 3 sums
  unsigned *done;      // blocks finished (0 between evaluations)
};
constexpr int kFinBlocks = 16, kFinThreads = 512;

// Per-kernel CUDA-event timing of evaluations (ccm_profile_begin/end): one
// event before the first kernel of an evaluation and one after each kernel.
constexpr int kMaxProfMarks = 8;
void prof_mark(ccm_context *c);
// Stream-ordered device allocation on the context's stream, from its pool.
cudaError_t dev_alloc_raw(ccm_context *c, void **p, size_t bytes);
// ccm_create with the pool that the context's device memory comes from.
int create_context(ccm_context **out, const unsigned char *msa, int ncol, int nrow,
                   const float *weights, const ccm_options *opt, cudaMemPool_t pool);
// init_bias restricted to the single fields x[0 .. 20L) (host).
void init_single_fields(const unsigned char *msa, int ncol, int nrow, float *x);
// sum_submatrices of a device x into a device L x L map.
cudaError_t launch_contact_scores(const float *d_x, float *d_out, int L, cudaStream_t stream);
// Pinned host slots of at most 256 bytes, never returned to CUDA (no device sync).
void *pinned_small_alloc(size_t bytes);
void pinned_small_free(void *p);
void count_launch(ccm_context *c, int n = 1);
// Zero `words` 32-bit words on stream s with a kernel (capturable into the
// bodies of conditional graph nodes).
cudaError_t zero_words(void *p, long long words, cudaStream_t s);

cudaError_t tc_configure_kernels();
// CTA pairs of tc_forward that can be resident at once on the current device.
cudaError_t tc_forward_max_pairs(int nsplit, int *pairs);
cudaError_t tc_backward_max_pairs(int nsplit, int *pairs);
cudaError_t tc_evaluate(ccm_context *c, const float *d_x, float *d_g);
// The integer path: evaluation at d_x, or (d_s != null) at d_xt = d_x + alpha d_s.
cudaError_t i8_evaluate(ccm_context *c, const float *d_x, float *d_g, const float *d_s,
                        const double *d_alpha, float *d_xt);
cudaError_t i8_configure_kernels();
cudaError_t i8_forward_max_pairs(int *pairs);
cudaError_t i8_backward_max_pairs(int *pairs);
cudaError_t i8_build_onehot(ccm_context *c);
cudaError_t i8sp_forward_max_pairs(int *pairs);
// tc_finalize over the loss partials of n_fwd_tiles 128-row forward tiles.
cudaError_t launch_tc_finalize(ccm_context *c, const float *x1, float *d_g, long long n_fwd_tiles);
// One CG trial on a tensor-core context: xt = x + alpha s (alpha on the device),
// then the evaluation at xt, with the step fused into tc_prep.
cudaError_t tc_evaluate_step(ccm_context *c, const float *d_x, const float *d_s,
                             const double *d_alpha, float *d_xt, float *d_g);
int tc_fwd_smem_bytes(int nsplit);
int tc_bwd_smem_bytes(int nsplit);

cudaError_t simt_evaluate(ccm_context *c, const float *d_x, float *d_g);
cudaError_t simt_evaluate_f64(ccm_context *c, const double *d_x, double *d_g);

// Record a message for ccm_last_error() and return `code`.
int set_last_error(int code, const char *fmt, ...);

// Enqueue one evaluation of the context's path on its stream (no host sync).
int enqueue_evaluation(ccm_context *c, const float *d_x, float *d_g);
// Tensor-core paths: d_xt = d_x + alpha d_s (alpha on the device) fused into the
// evaluation at d_xt.
int enqueue_evaluation_step(ccm_context *c, const float *d_x, const float *d_s,
                            const double *d_alpha, float *d_xt, float *d_g);

cudaError_t reweight_counts(const uint8_t *d_msa, int L, int N, int idthres, int *d_counts,
                            cudaStream_t stream);

// An evaluate callback of the reference's shape (include/evaluate_cuda.h:8-13).
typedef float (*ccm_eval_callback)(void *instance, const float *x, float *g, const int n);
// The device CG around a foreign callback (device x; one callback call per trial).
int conjugrad_callback_gpu(float *d_x, long long n, ccm_eval_callback eval,
                           ccm_progress_t progress, void *instance, const ccm_cg_params *params,
                           ccm_cg_result *result);
// The same rules over host vectors (host x; the callback gets host pointers).
int conjugrad_host_vectors(float *x, long long n, ccm_eval_callback eval,
                           ccm_progress_t progress, void *instance, const ccm_cg_params *params,
                           ccm_cg_result *result);
// True when p points at a live context of this library.
bool is_context(const void *p);

// A whole device-side solve added to a graph that holds many (the batch
// solver's waves): initial evaluation, the iteration loop, the final x in d_x,
// the state record copied to pinned memory.  `last` receives the solve's last
// node.  After the graph ran, cg_graph_solve_result reads the outcome.
struct CgGraphSolve;
int cg_graph_solve_add(ccm_context *c, float *d_x, const ccm_cg_params *params, cudaGraph_t graph,
                       CgGraphSolve **out, cudaGraphNode_t *last);
int cg_graph_solve_result(const CgGraphSolve *gs, ccm_cg_result *res);
void cg_graph_solve_free(CgGraphSolve *gs);
// Upper bound of the device memory of a context of `path` (bytes), without the
// optimizer's vectors.
size_t context_bytes_estimate(int L, int N, int path);

constexpr uint32_t kContextMagic = 0xCC3B2000u;

}  // namespace ccm

struct ccm_context {
  uint32_t magic = ccm::kContextMagic;  // cleared when the context is destroyed
  int device = 0;
  int num_sms = 148;
  int fwd_pairs = 74;             // resident CTA pairs of tc_forward
  int bwd_pairs = 74;             // resident CTA pairs of tc_backward
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;   // device memory pool, or null for the device's default pool
  size_t mem_limit = 0;           // ccm_options.mem_limit (0: none)
  size_t mem_used = 0;            // device bytes held through dev_alloc_raw
  bool own_stream = false;
  int path = CCM_PATH_TC_BF16X2;
  int nsplit = 2;
  int gradient = CCM_GRADIENT_TIED;

  int L = 0, N = 0;
  long long nsingle = 0, nsp = 0, nvarp = 0;
  int r_exp = 0;                   // eR of the integer path's R digits: 2^eR >= max |w|
  long long acc_wait_cycles = 0;   // ccm_debug_set_wait_limit (0: default budget)
  float lambda_single = 0.01f, lambda_pair = 0.0f;

  uint8_t *d_msa = nullptr;       // N x L
  float *d_w = nullptr;           // N
  float *h_w = nullptr;           // N (host copy)
  ccm_result *d_out = nullptr;    // result of the last evaluation
  ccm_result *h_out = nullptr;    // pinned host mirror
  int *d_status = nullptr;        // == &d_out->status

  // tensor-core path
  int T = 0, S = 0, Npad = 0;
  __nv_bfloat16 *d_onehot = nullptr;     // Npad x S
  __nv_bfloat16 *d_wperm[3] = {nullptr, nullptr, nullptr};  // S x S
  __nv_bfloat16 *d_r[3] = {nullptr, nullptr, nullptr};      // Npad x S
  double *d_part_f = nullptr;
  double *d_part_reg = nullptr;
  double *d_fin_part = nullptr;     // tc_finalize: per-block sums
  unsigned *d_fin_done = nullptr;   // tc_finalize: its ticket counter
  float *d_g1d = nullptr;                // 20 L single-field data gradient
  int2 *d_bwd_tiles = nullptr;
  int n_bwd_tiles = 0;
  ccm::FwdMaps fwd_maps;
  ccm::BwdMaps bwd_maps;

  // integer tensor-core path
  uint8_t *d_o1 = nullptr, *d_o128 = nullptr;          // Npad x S one-hot, values 1 / 128
  int8_t *d_wdig[3] = {nullptr, nullptr, nullptr};     // S x S digits of W
  int8_t *d_rdig[3] = {nullptr, nullptr, nullptr};     // Npad x S digits of R
  uint32_t *d_colmax = nullptr;  // 21 L column maxima of |W|, then S per-slot encoding factors
  // the column-maximum and prep passes skip the padding states a >= 21 (set by a
  // device-side solve whose x0 has zero padding states, while it captures and
  // runs; ccm_debug_set_cg_skip_padding clears cg_skip_padding to forbid it)
  bool skip_padding = false;
  bool cg_skip_padding = true;
  ccm::I8FwdMaps i8fwd_maps;
  ccm::I8BwdMaps i8bwd_maps;
  // sparse integer forward: W digits are KP x SW (K rows l * 21 + q, 192-slot
  // groups as columns); compressed one-hot Npad x KP/2 and metadata Npad x KP/8
  int KP = 0, SW = 0;
  uint8_t *d_ac1 = nullptr, *d_ac128 = nullptr, *d_meta = nullptr;
  ccm::I8SpMaps i8sp_maps;

  // SIMT paths
  void *d_simt_pc = nullptr;      // N x 21 x L probabilities (float or double)
  void *d_simt_g2 = nullptr;      // (21L) x (21L) unsymmetrised coupling gradient
  void *d_simt_part = nullptr;    // partial sums
  void *d_simt_g1 = nullptr;

  // host-pointer evaluation scratch
  float *d_xh = nullptr, *d_gh = nullptr;
  bool xh_pad_dirty = false;           // d_xh holds nonzero padding states
  long long host_h2d = 0, host_d2h = 0;  // bytes the last ccm_evaluate_host copied

  // instrumentation
  long long launches = 0;              // kernels launched by this context
  bool prof_on = false;
  int prof_max = 0, prof_eval = 0, prof_idx = 0, prof_marks_used = 0;
  cudaEvent_t *prof_events = nullptr;  // prof_max * kMaxProfMarks
};
