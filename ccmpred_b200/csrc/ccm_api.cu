// C ABI of libccmpred_b200.so: context lifecycle, evaluation dispatch and the
// reference-compatible backend triples.  See include/ccmpred_b200.h.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "ccm_internal.cuh"
#include "ccm_layout.cuh"
#include "ccm_ptx.cuh"

namespace ccm {

void prof_mark(ccm_context *c) {
  if (!c->prof_on || c->prof_eval >= c->prof_max || c->prof_idx >= kMaxProfMarks) return;
  cudaEventRecord(c->prof_events[c->prof_eval * kMaxProfMarks + c->prof_idx], c->stream);
  c->prof_idx++;
}

void count_launch(ccm_context *c, int n) { c->launches += n; }

// Zero `words` 32-bit words.  A kernel rather than cudaMemsetAsync: the
// evaluation is also captured into the bodies of conditional graph nodes (the
// device-side CG), which hold kernel nodes.
__global__ void zero_words_kernel(uint32_t *__restrict__ p, long long words) {
  griddep_wait();
  griddep_launch();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < words;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = 0u;
}

cudaError_t zero_words(void *p, long long words, cudaStream_t s) {
  const long long blocks = (words + 255) / 256;
  return launch_pdl(zero_words_kernel, dim3((unsigned)(blocks < 1184 ? (blocks > 0 ? blocks : 1) : 1184)),
                    dim3(256), 0, s, static_cast<uint32_t *>(p), words);
}

bool is_context(const void *p) {
  return p && static_cast<const ccm_context *>(p)->magic == kContextMagic;
}

cudaError_t dev_alloc_raw(ccm_context *c, void **p, size_t bytes) {
  // the cap of ccm_options.mem_limit: the bytes this context holds
  if (c->mem_limit > 0 && c->mem_used + bytes > c->mem_limit) return cudaErrorMemoryAllocation;
  const cudaError_t e = c->pool ? cudaMallocFromPoolAsync(p, bytes, c->pool, c->stream)
                                : cudaMallocAsync(p, bytes, c->stream);
  if (e == cudaSuccess) c->mem_used += bytes;
  return e;
}

// Small pinned host records (a context's result, the CG's step scalars) come
// from one process-wide slab of 256-byte slots that is never returned to CUDA:
// cudaFreeHost waits for the whole device, which would stall the streams of
// every other context at each context tear-down.
static constexpr size_t kPinnedSlot = 256;
static constexpr size_t kPinnedChunk = 256 * kPinnedSlot;
static std::mutex pinned_mutex;
static std::vector<void *> pinned_free;

void *pinned_small_alloc(size_t bytes) {
  if (bytes > kPinnedSlot) return nullptr;
  std::lock_guard<std::mutex> lock(pinned_mutex);
  if (pinned_free.empty()) {
    void *chunk = nullptr;
    if (cudaHostAlloc(&chunk, kPinnedChunk, cudaHostAllocPortable) != cudaSuccess) return nullptr;
    for (size_t i = kPinnedChunk / kPinnedSlot; i-- > 0;)
      pinned_free.push_back(static_cast<char *>(chunk) + i * kPinnedSlot);
  }
  void *p = pinned_free.back();
  pinned_free.pop_back();
  std::memset(p, 0, kPinnedSlot);
  return p;
}

void pinned_small_free(void *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(pinned_mutex);
  pinned_free.push_back(p);
}

int set_last_error(int code, const char *fmt, ...);

cudaError_t simt_configure_kernels();
size_t simt_scratch_bytes(int L, int N, size_t elem);
cudaError_t reweight_weights(const int *d_counts, float *d_w, int N, cudaStream_t stream);
}  // namespace ccm

using namespace ccm;

namespace {

thread_local char g_last_error[512] = "";
int g_default_path = CCM_PATH_TC_I8SP;

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

}  // namespace

int ccm::set_last_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

namespace {

#define CCM_CUDA_TRY(expr)                                                                  \
  do {                                                                                      \
    cudaError_t _e = (expr);                                                                \
    if (_e != cudaSuccess)                                                                  \
      return set_error(_e == cudaErrorMemoryAllocation ? CCM_ERR_NOMEM : CCM_ERR_CUDA,      \
                       "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__,    \
                       __LINE__);                                                           \
  } while (0)

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn lookup_encode_fn() {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
          cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    return reinterpret_cast<EncodeTiledFn>(p);
  return nullptr;
}

EncodeTiledFn get_encode_fn() {
  static const EncodeTiledFn fn = lookup_encode_fn();  // thread-safe one-time init
  return fn;
}

// 2-D bf16 row-major [rows][cols] tensor, swizzled boxes of box_cols x box_rows
// (128-byte swizzle for 64-column boxes, 64-byte swizzle for 32-column boxes).
int make_map_bf16(CUtensorMap *map, void *base, long long rows, long long cols, int box_cols,
                  int box_rows) {
  const CUtensorMapSwizzle swz =
      box_cols * 2 == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
  EncodeTiledFn enc = get_encode_fn();
  if (!enc) return set_error(CCM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(CCM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CCM_OK;
}

// 2-D 8-bit row-major [rows][cols] tensor, boxes of box_cols x box_rows bytes
// (128-byte swizzle for 128-column boxes, 64-byte swizzle for 64-column boxes).
// 8-bit row-major [rows][cols] map; the swizzle spans the box's 128 or 64 bytes
// unless given.
int make_map_u8(CUtensorMap *map, void *base, long long rows, long long cols, int box_cols,
                int box_rows, int swizzle = -1) {
  const CUtensorMapSwizzle swz =
      swizzle >= 0 ? (CUtensorMapSwizzle)swizzle
                   : (box_cols == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B);
  EncodeTiledFn enc = get_encode_fn();
  if (!enc) return set_error(CCM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(CCM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CCM_OK;
}

// One-hot matrix O[n][s] (bf16): 1 where the state of column l(s) in row n is
// q(s); 1 in the ones slot for every real row; 0 elsewhere (padding rows,
// padding slots).
__global__ void build_onehot_kernel(const uint8_t *__restrict__ msa, __nv_bfloat16 *__restrict__ O,
                                    int L, int N, int S, int Npad) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Npad * S) return;
  const int n = (int)(idx / S), s = (int)(idx % S);
  const int t = s / kGroupSlots, r = s % kGroupSlots;
  float v = 0.0f;
  if (n < N) {
    if (s == kOnesSlot) {
      v = 1.0f;
    } else if (r < kGroupUsed) {
      const int q = r / kGroupCols, l = t * kGroupCols + r % kGroupCols;
      if (l < L && msa[(long long)n * L + l] == q) v = 1.0f;
    }
  }
  O[idx] = __float2bfloat16_rn(v);
}

// Device memory of a context is allocated and freed stream-ordered on the
// context's stream.  Plain cudaFree waits for the whole device, which in the
// batch solver would stall every other worker's stream at each alignment.
template <class T>
cudaError_t dev_alloc(ccm_context *c, T **p, size_t bytes) {
  return dev_alloc_raw(c, reinterpret_cast<void **>(p), bytes);
}

bool configured[64] = {false};
std::mutex configure_mutex;

int ensure_configured(int device) {
  if (device < 0 || device >= 64) return set_error(CCM_ERR_INVALID, "bad device %d", device);
  std::lock_guard<std::mutex> lock(configure_mutex);
  if (configured[device]) return CCM_OK;
  CCM_CUDA_TRY(tc_configure_kernels());
  CCM_CUDA_TRY(i8_configure_kernels());
  CCM_CUDA_TRY(simt_configure_kernels());
  configured[device] = true;
  return CCM_OK;
}

int alloc_tc(ccm_context *c) {
  const bool sp = c->path == CCM_PATH_TC_I8SP;
  if (sp) {
    // sparse integer path: forward tiles are 192-slot groups (9 columns); the
    // slot space is padded to the backward's 256-slot pair tiles; K of the
    // forward is 21 L in the order l * 21 + q, padded to 256
    c->T = Groups192::groups(c->L);
    c->SW = c->T * Groups192::kSlots;
    c->S = ((c->SW + 255) / 256) * 256;
    c->KP = ((kQ * c->L + 255) / 256) * 256;
  } else {
    c->T = n_groups(c->L);
    c->S = c->T * kGroupSlots;
  }
  // rows padded to the forward's 256-row CTA-pair tiles
  c->Npad = ((c->N + 255) / 256) * 256;
  const size_t S = c->S, Np = c->Npad;
  const bool i8 = c->path == CCM_PATH_TC_I8X3 || sp;
  if (i8) {
    // integer path: one-hot x1 / x128 bytes, three digit matrices of W and of R
    const size_t wbytes = sp ? (size_t)c->KP * c->SW : S * S;
    CCM_CUDA_TRY(dev_alloc(c, &c->d_o1, Np * S));
    CCM_CUDA_TRY(dev_alloc(c, &c->d_o128, Np * S));
    for (int i = 0; i < 3; ++i) {
      CCM_CUDA_TRY(dev_alloc(c, &c->d_wdig[i], wbytes));
      CCM_CUDA_TRY(cudaMemsetAsync(c->d_wdig[i], 0, wbytes, c->stream));
      CCM_CUDA_TRY(dev_alloc(c, &c->d_rdig[i], Np * S));
      CCM_CUDA_TRY(cudaMemsetAsync(c->d_rdig[i], 0, Np * S, c->stream));
    }
    if (sp) {
      CCM_CUDA_TRY(dev_alloc(c, &c->d_ac1, Np * c->KP / 2));
      CCM_CUDA_TRY(dev_alloc(c, &c->d_ac128, Np * c->KP / 2));
      CCM_CUDA_TRY(dev_alloc(c, &c->d_meta, Np * c->KP / 8));
    }
    CCM_CUDA_TRY(dev_alloc(c, &c->d_colmax, sizeof(uint32_t) * (((kQ * c->L + 3) & ~3) + S)));
  } else {
    CCM_CUDA_TRY(dev_alloc(c, &c->d_onehot, sizeof(__nv_bfloat16) * Np * S));
    for (int i = 0; i < c->nsplit; ++i) {
      CCM_CUDA_TRY(dev_alloc(c, &c->d_wperm[i], sizeof(__nv_bfloat16) * S * S));
      CCM_CUDA_TRY(cudaMemsetAsync(c->d_wperm[i], 0, sizeof(__nv_bfloat16) * S * S, c->stream));
      CCM_CUDA_TRY(dev_alloc(c, &c->d_r[i], sizeof(__nv_bfloat16) * Np * S));
      CCM_CUDA_TRY(cudaMemsetAsync(c->d_r[i], 0, sizeof(__nv_bfloat16) * Np * S, c->stream));
    }
  }
  const long long fwd_tiles = (long long)(c->Npad / 128) * c->T;
  CCM_CUDA_TRY(dev_alloc(c, &c->d_part_f, sizeof(double) * fwd_tiles * 8));
  CCM_CUDA_TRY(dev_alloc(c, &c->d_part_reg, sizeof(double) * kQ * c->L));
  CCM_CUDA_TRY(dev_alloc(c, &c->d_fin_part, sizeof(double) * 3 * kFinBlocks));
  CCM_CUDA_TRY(dev_alloc(c, &c->d_fin_done, sizeof(unsigned)));
  CCM_CUDA_TRY(cudaMemsetAsync(c->d_fin_done, 0, sizeof(unsigned), c->stream));
  CCM_CUDA_TRY(dev_alloc(c, &c->d_g1d, sizeof(float) * (kQ - 1) * c->L));

  std::vector<int2> tiles;
  // P and Q in 256-slot blocks (rows, columns of C); the symmetric gradient
  // needs only the tiles that hold some s1 <= s2
  const int blocks = c->S / 256;
  for (int Q = 0; Q < blocks; ++Q)
    for (int P = 0; P < blocks; ++P)
      if (c->gradient == CCM_GRADIENT_PARTIAL || P <= Q) tiles.push_back(make_int2(P, Q));
  c->n_bwd_tiles = (int)tiles.size();
  CCM_CUDA_TRY(dev_alloc(c, &c->d_bwd_tiles, sizeof(int2) * tiles.size()));
  CCM_CUDA_TRY(cudaMemcpyAsync(c->d_bwd_tiles, tiles.data(), sizeof(int2) * tiles.size(),
                               cudaMemcpyHostToDevice, c->stream));

  int rc;
  if (i8) {
    CCM_CUDA_TRY(i8_build_onehot(c));
    std::memset(&c->i8fwd_maps, 0, sizeof(c->i8fwd_maps));
    std::memset(&c->i8bwd_maps, 0, sizeof(c->i8bwd_maps));
    if ((rc = make_map_u8(&c->i8fwd_maps.a1, c->d_o1, Np, S, 64, 128)) != CCM_OK) return rc;
    if ((rc = make_map_u8(&c->i8fwd_maps.a128, c->d_o128, Np, S, 64, 128)) != CCM_OK) return rc;
    // backward operands: the dense path reads 128-slot x 32-row boxes of the
    // row-major matrices (128-byte swizzle); the sparse path stores them tiled
    // (4 KB shared-memory images, swizzle applied) and reads 16 rows of 256 bytes
    const long long trows = (long long)Np * S / 256;
    const int none = CU_TENSOR_MAP_SWIZZLE_NONE;
    auto bwd_map = [&](CUtensorMap *m, void *p) {
      return sp ? make_map_u8(m, p, trows, 256, 256, 16, none) : make_map_u8(m, p, Np, S, 128, 32);
    };
    if ((rc = bwd_map(&c->i8bwd_maps.o1, c->d_o1)) != CCM_OK) return rc;
    if ((rc = bwd_map(&c->i8bwd_maps.o128, c->d_o128)) != CCM_OK) return rc;
    for (int i = 0; i < 3; ++i) {
      if (!sp && (rc = make_map_u8(&c->i8fwd_maps.b[i], c->d_wdig[i], S, S, 128, 64)) != CCM_OK)
        return rc;
      if ((rc = bwd_map(&c->i8bwd_maps.r[i], c->d_rdig[i])) != CCM_OK) return rc;
    }
    if (sp) {
      std::memset(&c->i8sp_maps, 0, sizeof(c->i8sp_maps));
      // tiled operand storage viewed as rows of 256 bytes; one box = one stage tile
      const long long KP = c->KP;
      if ((rc = make_map_u8(&c->i8sp_maps.a1, c->d_ac1, Np * KP / 512, 256, 256, 32, none)) !=
              CCM_OK ||
          (rc = make_map_u8(&c->i8sp_maps.a128, c->d_ac128, Np * KP / 512, 256, 256, 32, none)) !=
              CCM_OK ||
          (rc = make_map_u8(&c->i8sp_maps.e, c->d_meta, Np * KP / 2048, 256, 256, 8, none)) !=
              CCM_OK)
        return rc;
      for (int i = 0; i < 3; ++i)
        if ((rc = make_map_u8(&c->i8sp_maps.b[i], c->d_wdig[i], KP * c->SW / 256, 256, 256, 48,
                              none)) != CCM_OK)
          return rc;
    }
    return CCM_OK;
  }
  const long long total = (long long)Np * S;
  build_onehot_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(
      c->d_msa, c->d_onehot, c->L, c->N, c->S, c->Npad);
  CCM_CUDA_TRY(cudaGetLastError());

  std::memset(&c->fwd_maps, 0, sizeof(c->fwd_maps));
  std::memset(&c->bwd_maps, 0, sizeof(c->bwd_maps));
  if ((rc = make_map_bf16(&c->fwd_maps.a, c->d_onehot, Np, S, 32, 128)) != CCM_OK) return rc;
  if ((rc = make_map_bf16(&c->bwd_maps.o, c->d_onehot, Np, S, 64, 32)) != CCM_OK) return rc;
  for (int i = 0; i < c->nsplit; ++i) {
    if ((rc = make_map_bf16(&c->fwd_maps.b[i], c->d_wperm[i], S, S, 64, 32)) != CCM_OK) return rc;
    if ((rc = make_map_bf16(&c->bwd_maps.r[i], c->d_r[i], Np, S, 64, 32)) != CCM_OK) return rc;
  }
  return CCM_OK;
}

int alloc_simt(ccm_context *c, size_t elem) {
  const size_t QL = (size_t)kQ * c->L;
  CCM_CUDA_TRY(dev_alloc(c, &c->d_simt_pc, elem * (size_t)c->N * QL));
  CCM_CUDA_TRY(dev_alloc(c, &c->d_simt_g2, elem * QL * QL));
  CCM_CUDA_TRY(dev_alloc(c, &c->d_simt_g1, elem * (size_t)(kQ - 1) * c->L));
  CCM_CUDA_TRY(dev_alloc(c, &c->d_simt_part, sizeof(double) * ((size_t)c->N + QL)));
  return CCM_OK;
}

void free_all(ccm_context *c) {
  // stream-ordered frees: cudaFree would wait for every stream of the device
  auto f = [c](void *p) { if (p) cudaFreeAsync(p, c->stream); };
  f(c->d_msa); f(c->d_w); f(c->d_out); f(c->d_onehot);
  for (int i = 0; i < 3; ++i) { f(c->d_wperm[i]); f(c->d_r[i]); f(c->d_wdig[i]); f(c->d_rdig[i]); }
  f(c->d_o1); f(c->d_o128); f(c->d_colmax); f(c->d_ac1); f(c->d_ac128); f(c->d_meta);
  f(c->d_part_f); f(c->d_part_reg); f(c->d_fin_part); f(c->d_fin_done); f(c->d_g1d); f(c->d_bwd_tiles);
  f(c->d_simt_pc); f(c->d_simt_g2); f(c->d_simt_part); f(c->d_simt_g1);
  f(c->d_xh); f(c->d_gh);
  if (c->h_out) pinned_small_free(c->h_out);
  std::free(c->h_w);
  if (c->prof_events) {
    for (int i = 0; i < c->prof_max * kMaxProfMarks; ++i) cudaEventDestroy(c->prof_events[i]);
    std::free(c->prof_events);
  }
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
}

int check_status(ccm_context *c) {
  if (c->h_out->status != 0)
    return set_error(CCM_ERR_DEVICE, "device wait timed out in %s (status 0x%x)",
                     (c->h_out->status & kErrFwdTimeout) ? "tc_forward" : "tc_backward",
                     c->h_out->status);
  return CCM_OK;
}

int enqueue_eval(ccm_context *c, const float *d_x, float *d_g) {
  CCM_CUDA_TRY(zero_words(c->d_out, sizeof(ccm_result) / 4, c->stream));
  count_launch(c);
  c->prof_idx = 0;
  cudaError_t e;
  switch (c->path) {
    case CCM_PATH_TC_BF16X2:
    case CCM_PATH_TC_BF16X3: e = tc_evaluate(c, d_x, d_g); break;
    case CCM_PATH_TC_I8X3:
    case CCM_PATH_TC_I8SP: e = i8_evaluate(c, d_x, d_g, nullptr, nullptr, nullptr); break;
    case CCM_PATH_SIMT_F32: e = simt_evaluate(c, d_x, d_g); break;
    case CCM_PATH_SIMT_F64:
      return set_error(CCM_ERR_INVALID, "CCM_PATH_SIMT_F64 takes double buffers: use ccm_evaluate_f64");
    default: return set_error(CCM_ERR_INVALID, "unknown path %d", c->path);
  }
  if (e != cudaSuccess)
    return set_error(CCM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  if (c->prof_on && c->prof_eval < c->prof_max) {
    c->prof_marks_used = c->prof_idx;
    c->prof_eval++;
  }
  return CCM_OK;
}

void free_prof(ccm_context *c) {
  if (c->prof_events) {
    for (int i = 0; i < c->prof_max * kMaxProfMarks; ++i) cudaEventDestroy(c->prof_events[i]);
    std::free(c->prof_events);
  }
  c->prof_events = nullptr;
  c->prof_on = false;
  c->prof_max = c->prof_eval = 0;
}

}  // namespace

int ccm::enqueue_evaluation_step(ccm_context *c, const float *d_x, const float *d_s,
                                  const double *d_alpha, float *d_xt, float *d_g) {
  const bool i8 = c->path == CCM_PATH_TC_I8X3 || c->path == CCM_PATH_TC_I8SP;
  if (c->path != CCM_PATH_TC_BF16X2 && c->path != CCM_PATH_TC_BF16X3 && !i8)
    return set_error(CCM_ERR_INVALID, "fused step: tensor-core paths only");
  CCM_CUDA_TRY(zero_words(c->d_out, sizeof(ccm_result) / 4, c->stream));
  count_launch(c);
  c->prof_idx = 0;
  const cudaError_t e = i8
                            ? i8_evaluate(c, d_x, d_g, d_s, d_alpha, d_xt)
                            : tc_evaluate_step(c, d_x, d_s, d_alpha, d_xt, d_g);
  if (e != cudaSuccess)
    return set_error(CCM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  if (c->prof_on && c->prof_eval < c->prof_max) {
    c->prof_marks_used = c->prof_idx;
    c->prof_eval++;
  }
  return CCM_OK;
}

int ccm::enqueue_evaluation(ccm_context *c, const float *d_x, float *d_g) {
  return enqueue_eval(c, d_x, d_g);
}

namespace {

ccm_userdata *as_ud(void *instance) { return static_cast<ccm_userdata *>(instance); }

[[noreturn]] void die_ref(const char *what) {
  // reference error behaviour: print and exit (include/evaluate_cuda_kernels.h:9)
  printf("CUDA error in %s: %s\n", what, ccm_last_error());
  exit(EXIT_FAILURE);
}

int init_backend(ccm_userdata *ud) {
  if (!ud || !ud->msa || ud->ncol <= 0 || ud->nrow <= 0)
    return set_error(CCM_ERR_INVALID, "init: invalid userdata");
  const int L = ud->ncol, N = ud->nrow;
  // the device the caller made current (the reference selects it with
  // cudaSetDevice before init, src/ccmpred.c:421-426)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  std::vector<float> w(N, 1.0f);
  if (ud->reweighting_threshold < 1.0f) {
    int rc = ccm_calculate_weights(ud->msa, L, N, ud->reweighting_threshold, w.data(), dev);
    if (rc != CCM_OK) return rc;
    float wsum = 0.0f, wmin = w[0], wmax = w[0];
    for (int i = 0; i < N; ++i) {
      wsum += w[i];
      if (w[i] > wmax) wmax = w[i];
      if (w[i] < wmin) wmin = w[i];
    }
    printf("Reweighted %d sequences with threshold %.1f to Beff=%g weight mean=%g, min=%g, max=%g\n",
           N, ud->reweighting_threshold, wsum, wsum / N, wmin, wmax);
  } else {
    printf("Using uniform weights\n");
  }
  if (ud->weights) std::memcpy(ud->weights, w.data(), sizeof(float) * N);
  ccm_options opt;
  ccm_options_default(&opt, L);
  opt.lambda_single = ud->lambda_single;
  opt.lambda_pair = ud->lambda_pair;
  opt.path = g_default_path;
  opt.device = dev;
  ccm_context *ctx = nullptr;
  int rc = ccm_create(&ctx, ud->msa, L, N, w.data(), &opt);
  if (rc != CCM_OK) return rc;
  ud->extra = ctx;
  return CCM_OK;
}

}  // namespace

int ccm::create_context(ccm_context **out, const unsigned char *msa, int ncol, int nrow,
                        const float *weights, const ccm_options *opt, cudaMemPool_t pool) {
  if (!out || !msa || ncol <= 0 || nrow <= 0)
    return set_error(CCM_ERR_INVALID, "ccm_create: invalid arguments");
  *out = nullptr;
  ccm_options o;
  if (opt) o = *opt; else ccm_options_default(&o, ncol);
  if (o.path < CCM_PATH_TC_BF16X2 || o.path > CCM_PATH_TC_I8SP)
    return set_error(CCM_ERR_INVALID, "ccm_create: unknown path %d", o.path);
  if (o.gradient != CCM_GRADIENT_TIED && o.gradient != CCM_GRADIENT_PARTIAL)
    return set_error(CCM_ERR_INVALID, "ccm_create: unknown gradient mode %d", o.gradient);
  for (long long i = 0; i < (long long)ncol * nrow; ++i)
    if (msa[i] > 20) return set_error(CCM_ERR_INVALID, "ccm_create: MSA state %d > 20 at %lld", msa[i], i);
  // the integer paths encode R = w (P - onehot), |R| <= max |w|, with 21
  // fractional bits below the smallest power of two 2^eR >= max |w| (below 1 too:
  // an alignment whose rows all carry small weights keeps its residuals' bits)
  float wmax = weights ? 0.0f : 1.0f;
  if (weights)
    for (int i = 0; i < nrow; ++i) {
      if (!std::isfinite(weights[i]))
        return set_error(CCM_ERR_INVALID, "ccm_create: weight %d is not finite", i);
      wmax = std::max(wmax, std::fabs(weights[i]));
    }
  int r_exp = 0;
  if (wmax > 0.0f) {
    (void)std::frexp(wmax, &r_exp);                   // wmax = m 2^r_exp, m in [0.5, 1)
    if (std::ldexp(1.0f, r_exp - 1) == wmax) --r_exp;  // an exact power of two
    if (r_exp > 100) return set_error(CCM_ERR_INVALID, "ccm_create: weight %g too large", wmax);
    r_exp = std::max(r_exp, -100);
  }
  // the coupling block has 21*32*L^2 entries; keep every index in 32-bit range of int callers
  if (nvar_padded_of(ncol) > 0x7fffffffLL)
    return set_error(CCM_ERR_INVALID, "ccm_create: L=%d exceeds the int nvar of the reference ABI", ncol);

  CCM_CUDA_TRY(cudaSetDevice(o.device));
  cudaDeviceProp prop;
  CCM_CUDA_TRY(cudaGetDeviceProperties(&prop, o.device));
  const bool tc_path = o.path == CCM_PATH_TC_BF16X2 || o.path == CCM_PATH_TC_BF16X3 ||
                       o.path == CCM_PATH_TC_I8X3 || o.path == CCM_PATH_TC_I8SP;
  if (tc_path && prop.major != 10)
    return set_error(CCM_ERR_UNSUPPORTED, "tensor-core path needs an sm_100 device (found sm_%d%d)",
                     prop.major, prop.minor);
  int rc = ensure_configured(o.device);
  if (rc != CCM_OK) return rc;

  ccm_context *c = new ccm_context();
  c->pool = pool;
  c->mem_limit = o.mem_limit;
  c->r_exp = r_exp;
  c->device = o.device;
  c->num_sms = prop.multiProcessorCount;
  if (tc_path) {
    const int ns = o.path == CCM_PATH_TC_BF16X3 ? 3 : 2;
    const bool i8 = o.path == CCM_PATH_TC_I8X3 || o.path == CCM_PATH_TC_I8SP;
    cudaError_t e = o.path == CCM_PATH_TC_I8SP ? i8sp_forward_max_pairs(&c->fwd_pairs)
                    : i8                       ? i8_forward_max_pairs(&c->fwd_pairs)
                                               : tc_forward_max_pairs(ns, &c->fwd_pairs);
    if (e == cudaSuccess)
      e = i8 ? i8_backward_max_pairs(&c->bwd_pairs) : tc_backward_max_pairs(ns, &c->bwd_pairs);
    if (e != cudaSuccess || c->fwd_pairs < 1 || c->bwd_pairs < 1) {
      delete c;
      return set_error(CCM_ERR_CUDA, "tc_forward cluster occupancy: %s", cudaGetErrorString(e));
    }
    if (o.max_sms > 0) {
      const int pairs = std::max(1, o.max_sms / 2);
      c->fwd_pairs = std::min(c->fwd_pairs, pairs);
      c->bwd_pairs = std::min(c->bwd_pairs, pairs);
    }
  }
  c->path = o.path;
  c->nsplit = (o.path == CCM_PATH_TC_BF16X3) ? 3 : 2;
  c->gradient = o.gradient;
  c->L = ncol;
  c->N = nrow;
  c->nsingle = nsingle_of(ncol);
  c->nsp = nsingle_padded_of(ncol);
  c->nvarp = nvar_padded_of(ncol);
  c->lambda_single = o.lambda_single;
  c->lambda_pair = o.lambda_pair;
  if (o.stream) {
    c->stream = static_cast<cudaStream_t>(o.stream);
  } else {
    // a blocking stream: ordered with the legacy default stream, on which callers
    // (and torch by default) produce x and consume g
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault);
    if (e != cudaSuccess) {
      delete c;
      return set_error(CCM_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
    }
    c->own_stream = true;
  }
  auto fail = [&](int code) {
    free_all(c);
    delete c;
    (void)cudaGetLastError();  // a failed allocation must not surface in a later launch check
    return code;
  };
#define CCM_CTX_TRY(expr)                                                                    \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess)                                                                   \
      return fail(set_error(_e == cudaErrorMemoryAllocation ? CCM_ERR_NOMEM : CCM_ERR_CUDA,  \
                            "%s failed: %s", #expr, cudaGetErrorString(_e)));                \
  } while (0)
  c->h_w = static_cast<float *>(std::malloc(sizeof(float) * nrow));
  if (!c->h_w) return fail(set_error(CCM_ERR_NOMEM, "host weights"));
  for (int i = 0; i < nrow; ++i) c->h_w[i] = weights ? weights[i] : 1.0f;
  CCM_CTX_TRY(dev_alloc(c, &c->d_msa, (size_t)ncol * nrow));
  CCM_CTX_TRY(cudaMemcpyAsync(c->d_msa, msa, (size_t)ncol * nrow, cudaMemcpyHostToDevice, c->stream));
  CCM_CTX_TRY(dev_alloc(c, &c->d_w, sizeof(float) * nrow));
  CCM_CTX_TRY(cudaMemcpyAsync(c->d_w, c->h_w, sizeof(float) * nrow, cudaMemcpyHostToDevice, c->stream));
  CCM_CTX_TRY(dev_alloc(c, &c->d_out, sizeof(ccm_result)));
  CCM_CTX_TRY(cudaMemsetAsync(c->d_out, 0, sizeof(ccm_result), c->stream));
  c->h_out = static_cast<ccm_result *>(pinned_small_alloc(sizeof(ccm_result)));
  if (!c->h_out) return fail(set_error(CCM_ERR_NOMEM, "pinned result record"));
  c->d_status = &c->d_out->status;

  if (tc_path) {
    if ((rc = alloc_tc(c)) != CCM_OK) return fail(rc);
  } else {
    if ((rc = alloc_simt(c, c->path == CCM_PATH_SIMT_F64 ? sizeof(double) : sizeof(float))) != CCM_OK)
      return fail(rc);
  }
  CCM_CTX_TRY(cudaStreamSynchronize(c->stream));
#undef CCM_CTX_TRY
  *out = c;
  return CCM_OK;
}

extern "C" {

const char *ccm_last_error(void) { return g_last_error; }

void ccm_set_default_path(int path) { g_default_path = path; }

long long ccm_nsingle_padded(int ncol) { return nsingle_padded_of(ncol); }
long long ccm_nvar_padded(int ncol) { return nvar_padded_of(ncol); }

void ccm_options_default(ccm_options *opt, int ncol) {
  if (!opt) return;
  opt->lambda_single = 0.01f;
  opt->lambda_pair = 0.2f * (float)(ncol - 1);
  opt->path = CCM_PATH_TC_I8SP;
  opt->device = 0;
  opt->stream = nullptr;
  opt->gradient = CCM_GRADIENT_TIED;
  opt->max_sms = 0;
  opt->mem_limit = 0;
}

int ccm_create(ccm_context **out, const unsigned char *msa, int ncol, int nrow,
               const float *weights, const ccm_options *opt) {
  return ccm::create_context(out, msa, ncol, nrow, weights, opt, nullptr);
}

int ccm_destroy(ccm_context *ctx) {
  if (!ctx) return CCM_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  ctx->magic = 0;
  delete ctx;
  return CCM_OK;
}

int ccm_evaluate_async(ccm_context *c, const float *d_x, float *d_g, long long nvar) {
  if (!c || !d_x || !d_g) return set_error(CCM_ERR_INVALID, "ccm_evaluate: null argument");
  if (nvar != c->nvarp)
    return set_error(CCM_ERR_INVALID, "ccm_evaluate: nvar %lld != nvar_padded %lld", nvar, c->nvarp);
  return enqueue_eval(c, d_x, d_g);
}

int ccm_evaluate(ccm_context *c, const float *d_x, float *d_g, long long nvar, double *fx) {
  int rc = ccm_evaluate_async(c, d_x, d_g, nvar);
  if (rc != CCM_OK) return rc;
  CCM_CUDA_TRY(cudaMemcpyAsync(c->h_out, c->d_out, sizeof(ccm_result), cudaMemcpyDeviceToHost, c->stream));
  CCM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if ((rc = check_status(c)) != CCM_OK) return rc;
  if (fx) *fx = c->h_out->fx;
  return CCM_OK;
}

namespace {

// A few host threads that stay alive for the process, for the host-side passes
// of ccm_evaluate_host.  parallel_for(n, f) runs f(i) for every i < n on the
// workers and the calling thread; one job at a time.
class HostWorkers {
 public:
  static HostWorkers &get() {
    static HostWorkers w;
    return w;
  }
  void parallel_for(long long n, const std::function<void(long long)> &f) {
    std::lock_guard<std::mutex> job_lock(job_mutex_);
    {
      std::lock_guard<std::mutex> lk(m_);
      fn_ = &f;
      n_ = n;
      next_.store(0);
      busy_ = (int)threads_.size();
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(m_);
    done_cv_.wait(lk, [&] { return busy_ == 0; });
    fn_ = nullptr;
  }

 private:
  HostWorkers() {
    const unsigned hw = std::thread::hardware_concurrency();
    const int n = (int)std::min(7u, hw > 1 ? hw / 2 : 1u);
    for (int i = 0; i < n; ++i) threads_.emplace_back([this] { loop(); });
  }
  ~HostWorkers() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : threads_) t.join();
  }
  void work() {
    for (long long i; (i = next_.fetch_add(1)) < n_;) (*fn_)(i);
  }
  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
      std::lock_guard<std::mutex> lk(m_);
      if (--busy_ == 0) done_cv_.notify_all();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex job_mutex_, m_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(long long)> *fn_ = nullptr;
  long long n_ = 0;
  std::atomic<long long> next_{0};
  int busy_ = 0;
  unsigned long long gen_ = 0;
  bool stop_ = false;
};

}  // namespace

// Host x and g.  The padding states a in [21, 32) of the coupling block are 34 %
// of x and are zero on every path that starts from init_bias or a .raw file
// (src/ccmpred.c:101, src/io.c:81-95); where they are zero (checked on the host,
// bit patterns, while the DMA copies the rest) neither they nor the gradient's
// padding states (2 lambda2 x = 0) cross PCIe: x and g move as 21 L rows of 21 L
// floats with a pitch of 32 L, and the host writes g's padding states as zeros
// during the device-to-host copy.  Any nonzero bit there: the padding is copied
// both ways as well.
int ccm_evaluate_host(ccm_context *c, const float *x, float *g, long long nvar, double *fx) {
  if (!c || !x || !g) return set_error(CCM_ERR_INVALID, "ccm_evaluate_host: null argument");
  if (nvar != c->nvarp)
    return set_error(CCM_ERR_INVALID, "ccm_evaluate_host: nvar %lld != nvar_padded %lld", nvar, c->nvarp);
  const size_t bytes = sizeof(float) * (size_t)nvar;
  if (!c->d_xh) {
    CCM_CUDA_TRY(dev_alloc(c, &c->d_xh, bytes));
    CCM_CUDA_TRY(dev_alloc(c, &c->d_gh, bytes));
    CCM_CUDA_TRY(cudaMemsetAsync(c->d_xh, 0, bytes, c->stream));
    c->xh_pad_dirty = false;
  }
  const int L = c->L;
  const long long nsp = c->nsp, rows = (long long)kQ * L;
  const size_t pitch = sizeof(float) * kQPad * (size_t)L;
  const size_t real = sizeof(float) * kQ * (size_t)L, pad = pitch - real;
  // single fields, then the 21 states of every row
  CCM_CUDA_TRY(cudaMemcpyAsync(c->d_xh, x, sizeof(float) * nsp, cudaMemcpyHostToDevice, c->stream));
  CCM_CUDA_TRY(cudaMemcpy2DAsync(c->d_xh + nsp, pitch, x + nsp, pitch, real, rows,
                                 cudaMemcpyHostToDevice, c->stream));
  long long h2d = sizeof(float) * nsp + (long long)real * rows;
  std::atomic<int> nonzero{0};
  const long long kRowsPerJob = 64;
  HostWorkers::get().parallel_for((rows + kRowsPerJob - 1) / kRowsPerJob, [&](long long job) {
    uint32_t acc = 0;
    for (long long r = job * kRowsPerJob; r < std::min(rows, (job + 1) * kRowsPerJob); ++r) {
      const uint32_t *p = reinterpret_cast<const uint32_t *>(x + nsp + r * kQPad * L + kQ * L);
      for (size_t i = 0; i < pad / 4; ++i) acc |= p[i];
    }
    if (acc) nonzero.store(1, std::memory_order_relaxed);
  });
  const bool pad_nonzero = nonzero.load() != 0;
  if (pad_nonzero) {
    CCM_CUDA_TRY(cudaMemcpy2DAsync(c->d_xh + nsp + kQ * L, pitch, x + nsp + kQ * L, pitch, pad, rows,
                                   cudaMemcpyHostToDevice, c->stream));
    h2d += (long long)pad * rows;
  } else if (c->xh_pad_dirty) {
    CCM_CUDA_TRY(cudaMemset2DAsync(c->d_xh + nsp + kQ * L, pitch, 0, pad, rows, c->stream));
  }
  c->xh_pad_dirty = pad_nonzero;
  int rc = enqueue_eval(c, c->d_xh, c->d_gh);
  if (rc != CCM_OK) return rc;
  CCM_CUDA_TRY(cudaMemcpyAsync(g, c->d_gh, sizeof(float) * nsp, cudaMemcpyDeviceToHost, c->stream));
  CCM_CUDA_TRY(cudaMemcpy2DAsync(g + nsp, pitch, c->d_gh + nsp, pitch, pad_nonzero ? pitch : real,
                                 rows, cudaMemcpyDeviceToHost, c->stream));
  long long d2h = sizeof(float) * nsp + (long long)(pad_nonzero ? pitch : real) * rows;
  CCM_CUDA_TRY(cudaMemcpyAsync(c->h_out, c->d_out, sizeof(ccm_result), cudaMemcpyDeviceToHost, c->stream));
  d2h += sizeof(ccm_result);
  if (!pad_nonzero)  // g's padding states, disjoint from what the copy writes
    HostWorkers::get().parallel_for((rows + kRowsPerJob - 1) / kRowsPerJob, [&](long long job) {
      for (long long r = job * kRowsPerJob; r < std::min(rows, (job + 1) * kRowsPerJob); ++r)
        std::memset(g + nsp + r * kQPad * L + kQ * L, 0, pad);
    });
  CCM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->host_h2d = h2d;
  c->host_d2h = d2h;
  if ((rc = check_status(c)) != CCM_OK) return rc;
  if (fx) *fx = c->h_out->fx;
  return CCM_OK;
}

int ccm_host_copy_bytes(const ccm_context *c, long long *h2d, long long *d2h) {
  if (!c || !h2d || !d2h) return set_error(CCM_ERR_INVALID, "ccm_host_copy_bytes: null argument");
  *h2d = c->host_h2d;
  *d2h = c->host_d2h;
  return CCM_OK;
}

int ccm_evaluate_f64(ccm_context *c, const double *d_x, double *d_g, long long nvar, double *fx) {
  if (!c || !d_x || !d_g) return set_error(CCM_ERR_INVALID, "ccm_evaluate_f64: null argument");
  if (c->path != CCM_PATH_SIMT_F64)
    return set_error(CCM_ERR_INVALID, "ccm_evaluate_f64 needs a CCM_PATH_SIMT_F64 context");
  if (nvar != c->nvarp)
    return set_error(CCM_ERR_INVALID, "ccm_evaluate_f64: nvar %lld != nvar_padded %lld", nvar, c->nvarp);
  CCM_CUDA_TRY(cudaMemsetAsync(c->d_out, 0, sizeof(ccm_result), c->stream));
  CCM_CUDA_TRY(simt_evaluate_f64(c, d_x, d_g));
  CCM_CUDA_TRY(cudaMemcpyAsync(c->h_out, c->d_out, sizeof(ccm_result), cudaMemcpyDeviceToHost, c->stream));
  CCM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (fx) *fx = c->h_out->fx;
  return CCM_OK;
}

long long ccm_debug_copy(ccm_context *c, int which, void *dst, long long bytes) {
  if (!c) return set_error(CCM_ERR_INVALID, "ccm_debug_copy: null context");
  const void *src = nullptr;
  long long size = 0;
  const long long slots = (long long)c->S;
  if (c->path == CCM_PATH_TC_I8X3 || c->path == CCM_PATH_TC_I8SP) {
    // integer paths: 0 one-hot (x1 bytes), 1-3 digits of W, 4-6 digits of R,
    // 7 single-field data gradient, 8 column maxima of |W| (float bits); sparse
    // path: W digits are KP x SW, 9 compressed one-hot x1 (Npad x KP/2),
    // 10 its metadata (Npad x KP/8)
    const bool sp = c->path == CCM_PATH_TC_I8SP;
    if (which == 0) { src = c->d_o1; size = (long long)c->Npad * slots; }
    else if (which >= 1 && which <= 3) {
      src = c->d_wdig[which - 1];
      size = sp ? (long long)c->KP * c->SW : slots * slots;
    }
    else if (which == 9 && sp) { src = c->d_ac1; size = (long long)c->Npad * c->KP / 2; }
    else if (which == 10 && sp) { src = c->d_meta; size = (long long)c->Npad * c->KP / 8; }
    else if (which >= 4 && which <= 6) { src = c->d_rdig[which - 4]; size = (long long)c->Npad * slots; }
    else if (which == 7) { src = c->d_g1d; size = 4LL * (kQ - 1) * c->L; }
    else if (which == 8) { src = c->d_colmax; size = 4LL * kQ * c->L; }
  } else if (which == 0) { src = c->d_onehot; size = 2LL * c->Npad * slots; }
  else if (which >= 1 && which <= 3) { src = c->d_wperm[which - 1]; size = 2LL * slots * slots; }
  else if (which >= 4 && which <= 6) { src = c->d_r[which - 4]; size = 2LL * c->Npad * slots; }
  else if (which == 7) { src = c->d_g1d; size = 4LL * (kQ - 1) * c->L; }
  if (!src) return set_error(CCM_ERR_INVALID, "ccm_debug_copy: buffer %d not allocated", which);
  if (!dst) return size;
  if (bytes < size) return set_error(CCM_ERR_INVALID, "ccm_debug_copy: need %lld bytes", size);
  CCM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  CCM_CUDA_TRY(cudaMemcpy(dst, src, (size_t)size, cudaMemcpyDeviceToHost));
  return CCM_OK;
}

int ccm_profile_begin(ccm_context *c, int max_evals) {
  if (!c || max_evals <= 0) return set_error(CCM_ERR_INVALID, "ccm_profile_begin: invalid arguments");
  free_prof(c);
  c->prof_events = static_cast<cudaEvent_t *>(std::calloc((size_t)max_evals * kMaxProfMarks, sizeof(cudaEvent_t)));
  if (!c->prof_events) return set_error(CCM_ERR_NOMEM, "ccm_profile_begin: host allocation");
  c->prof_max = max_evals;
  for (int i = 0; i < max_evals * kMaxProfMarks; ++i) CCM_CUDA_TRY(cudaEventCreate(&c->prof_events[i]));
  c->prof_eval = 0;
  c->prof_on = true;
  return CCM_OK;
}

int ccm_profile_end(ccm_context *c, double *kernel_ms, int max_kernels, int *n_kernels, int *n_evals) {
  if (!c || !c->prof_on) return set_error(CCM_ERR_INVALID, "ccm_profile_end: profiling not active");
  CCM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const int nk = c->prof_marks_used > 0 ? c->prof_marks_used - 1 : 0;
  for (int k = 0; k < max_kernels; ++k) kernel_ms[k] = 0.0;
  for (int e = 0; e < c->prof_eval; ++e)
    for (int k = 0; k < nk && k < max_kernels; ++k) {
      float ms = 0.0f;
      CCM_CUDA_TRY(cudaEventElapsedTime(&ms, c->prof_events[e * kMaxProfMarks + k],
                                        c->prof_events[e * kMaxProfMarks + k + 1]));
      kernel_ms[k] += ms;
    }
  if (n_kernels) *n_kernels = nk;
  if (n_evals) *n_evals = c->prof_eval;
  free_prof(c);
  return CCM_OK;
}

long long ccm_launch_count(const ccm_context *c) { return c ? c->launches : -1; }

int ccm_debug_set_wait_limit(ccm_context *c, long long cycles) {
  if (!c || cycles < 0) return set_error(CCM_ERR_INVALID, "ccm_debug_set_wait_limit: invalid arguments");
  c->acc_wait_cycles = cycles;
  return CCM_OK;
}

int ccm_debug_set_cg_skip_padding(ccm_context *c, int allow) {
  if (!c) return set_error(CCM_ERR_INVALID, "ccm_debug_set_cg_skip_padding: null context");
  c->cg_skip_padding = allow != 0;
  return CCM_OK;
}

const ccm_result *ccm_result_device(const ccm_context *c) { return c ? c->d_out : nullptr; }

int ccm_get_result(ccm_context *c, ccm_result *out) {
  if (!c || !out) return set_error(CCM_ERR_INVALID, "ccm_get_result: null argument");
  CCM_CUDA_TRY(cudaMemcpyAsync(c->h_out, c->d_out, sizeof(ccm_result), cudaMemcpyDeviceToHost, c->stream));
  CCM_CUDA_TRY(cudaStreamSynchronize(c->stream));
  *out = *c->h_out;
  return CCM_OK;
}

int ccm_get_weights(const ccm_context *c, float *w) {
  if (!c || !w) return set_error(CCM_ERR_INVALID, "ccm_get_weights: null argument");
  std::memcpy(w, c->h_w, sizeof(float) * c->N);
  return CCM_OK;
}

void *ccm_stream(const ccm_context *c) { return c ? static_cast<void *>(c->stream) : nullptr; }

int ccm_calculate_weights(const unsigned char *msa, int ncol, int nrow, float threshold, float *w,
                          int device) {
  if (!msa || !w || ncol <= 0 || nrow <= 0)
    return set_error(CCM_ERR_INVALID, "ccm_calculate_weights: invalid arguments");
  CCM_CUDA_TRY(cudaSetDevice(device));
  // src/reweighting.c:10 -- threshold * ncol in float (ncol converted from uint64_t)
  const float prod = threshold * (float)(uint64_t)ncol;
  const int idthres = (int)ceil((double)prod);
  cudaStream_t s;
  CCM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  uint8_t *d_msa = nullptr;
  int *d_cnt = nullptr;
  float *d_w = nullptr;
  cudaError_t e = cudaMallocAsync(&d_msa, (size_t)ncol * nrow, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_cnt, sizeof(int) * nrow, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_w, sizeof(float) * nrow, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_msa, msa, (size_t)ncol * nrow, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = reweight_counts(d_msa, ncol, nrow, idthres, d_cnt, s);
  if (e == cudaSuccess) e = reweight_weights(d_cnt, d_w, nrow, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w, d_w, sizeof(float) * nrow, cudaMemcpyDeviceToHost, s);
  if (d_msa) cudaFreeAsync(d_msa, s);
  if (d_cnt) cudaFreeAsync(d_cnt, s);
  if (d_w) cudaFreeAsync(d_w, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess)
    return set_error(CCM_ERR_CUDA, "ccm_calculate_weights: %s", cudaGetErrorString(e));
  return CCM_OK;
}

// ------------------------------------------------------------ reference triple
int init_cuda(void *instance) {
  if (init_backend(as_ud(instance)) != CCM_OK) die_ref("init_cuda");
  return EXIT_SUCCESS;
}

float evaluate_cuda(void *instance, const float *x, float *g, const int nvar) {
  ccm_userdata *ud = as_ud(instance);
  double fx = 0.0;
  if (ccm_evaluate(static_cast<ccm_context *>(ud->extra), x, g, nvar, &fx) != CCM_OK)
    die_ref("evaluate_cuda");
  return (float)fx;
}

int destroy_cuda(void *instance) {
  ccm_userdata *ud = as_ud(instance);
  ccm_destroy(static_cast<ccm_context *>(ud->extra));
  ud->extra = nullptr;
  return EXIT_SUCCESS;
}

int init_b200(void *instance) {
  if (init_backend(as_ud(instance)) != CCM_OK) die_ref("init_b200");
  return 1;
}

float evaluate_b200(void *instance, const float *x, float *g, const int nvar) {
  ccm_userdata *ud = as_ud(instance);
  double fx = 0.0;
  if (ccm_evaluate_host(static_cast<ccm_context *>(ud->extra), x, g, nvar, &fx) != CCM_OK)
    die_ref("evaluate_b200");
  return (float)fx;
}

int destroy_b200(void *instance) { return destroy_cuda(instance) == EXIT_SUCCESS ? EXIT_SUCCESS : 1; }

}  // extern "C"
