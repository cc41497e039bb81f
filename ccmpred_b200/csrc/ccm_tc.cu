// Tensor-core (tcgen05) evaluation of the pseudo-likelihood f and its gradient.
//
// One evaluation = four launches on the context's stream:
//   1. tc_prep     x2 -> Wperm_i (bf16 split terms, permuted slot layout),
//                  2*lambda2*x on the a >= 21 padding of g2, sum of x2^2 partials.
//   2. tc_forward  logits = onehot(X) . Wperm (+ V in the epilogue), softmax over
//                  the 21 states of every (row, column), per-row loss, and
//                  R = w (P - onehot) split into bf16 terms.       [tcgen05 GEMM]
//   3. tc_backward C = [O;R]^T [R;O] on the upper triangle of slot tiles, written
//                  to g2 both as (s1,s2) and (s2,s1) with the self-edge mask and
//                  + 2*lambda2*x; the ones slot row of C is the single-field
//                  data gradient.                                  [tcgen05 GEMM]
//   4. tc_finalize FP64 sums of the loss and regulariser partials, g1.
//
// Semantics follow src/evaluate_cpu.c:16-166 (see oracle/ccm_oracle.c for the
// line-by-line restatement used as the checker).
#include <cuda_bf16.h>

#include "ccm_internal.cuh"
#include "ccm_layout.cuh"
#include "ccm_ptx.cuh"

namespace ccm {

// ------------------------------------------------------------------ tc_prep
// One block per row (b,k) of the reference W matrix.  The row's 21 L real
// entries are staged in shared memory (coalesced float4 loads); every thread
// then emits 8 consecutive slots of row s(b,k) of each Wperm_i as one 16-byte
// store (padding slots written as 0).  The whole g2 row is initialised to the
// regulariser gradient 2*lambda2*x (src/evaluate_cpu.c:158-161); tc_backward
// later adds the data term with one atomic add per element.  One FP64 partial
// of sum x^2 per row (all 32 L slots).
//
// STEP = true fuses the conjugate-gradient trial step into this pass: each
// element is v = fmaf(alpha, s, x) of the current iterate x and direction s
// (the same operation as the stand-alone step kernel), written to xt and used
// for everything above; one extra block (the last) steps the single fields.
template <int NSPLIT, bool STEP>
__global__ void __launch_bounds__(256) tc_prep_kernel(const float *__restrict__ x2,
                                                      float *__restrict__ g2, PrepArgs args) {
  extern __shared__ __align__(16) float xrow[];  // 21 L floats
  const int L = args.L;
  const int row = blockIdx.x;  // b*L + k
  float a = 0.0f;
  const float *s2 = nullptr;
  float *xt2 = nullptr;
  if (STEP) {
    a = (float)args.alpha[0];
    if (row == kQ * L) {
      for (long long i = threadIdx.x; i < args.nsp; i += blockDim.x)
        args.xt[i] = fmaf(a, args.step_s[i], args.step_x[i]);
      return;
    }
    s2 = args.step_s + args.nsp;
    xt2 = args.xt + args.nsp;
  }
  const int b = row / L, k = row % L;
  const long long base = (long long)row * kQPad * L;
  const float two_l2 = args.g2_coef * args.lambda_pair;  // 2 (tied) or 1 (partial)
  const int nreal = kQ * L;
  double acc = 0.0;
  // rows start at a multiple of 32 L floats (16-byte aligned); L % 4 == 0 allows float4
  if ((L & 3) == 0) {
    // the whole 32 L row as float4: four independent 16-byte loads in flight per
    // thread; the real states (first 21 L floats) are also staged in shared memory
    const float4 *src = reinterpret_cast<const float4 *>(x2 + base);
    float4 *dst = reinterpret_cast<float4 *>(g2 + base);
    const int n4 = kQPad * L / 4, nreal4 = nreal / 4;
    constexpr int kU = 4;
    for (int i0 = threadIdx.x; i0 < n4; i0 += kU * blockDim.x) {
      float4 v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int i = i0 + u * blockDim.x;
        v[u] = i < n4 ? __ldcs(src + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        if (STEP && i < n4) {
          const float4 sv = __ldcs(reinterpret_cast<const float4 *>(s2 + base) + i);
          v[u] = make_float4(fmaf(a, sv.x, v[u].x), fmaf(a, sv.y, v[u].y), fmaf(a, sv.z, v[u].z),
                             fmaf(a, sv.w, v[u].w));
          reinterpret_cast<float4 *>(xt2 + base)[i] = v[u];
        }
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int i = i0 + u * blockDim.x;
        if (i < n4) {
          acc += (double)v[u].x * v[u].x + (double)v[u].y * v[u].y + (double)v[u].z * v[u].z +
                 (double)v[u].w * v[u].w;
          if (i < nreal4) reinterpret_cast<float4 *>(xrow)[i] = v[u];
          __stcs(dst + i, make_float4(two_l2 * v[u].x, two_l2 * v[u].y, two_l2 * v[u].z,
                                      two_l2 * v[u].w));
        }
      }
    }
  } else {
    for (int i = threadIdx.x; i < nreal; i += blockDim.x) {
      float v = x2[base + i];
      if (STEP) { v = fmaf(a, s2[base + i], v); xt2[base + i] = v; }
      acc += (double)v * v;
      xrow[i] = v;
      g2[base + i] = two_l2 * v;
    }
    for (int i = nreal + threadIdx.x; i < kQPad * L; i += blockDim.x) {
      float v = x2[base + i];
      if (STEP) { v = fmaf(a, s2[base + i], v); xt2[base + i] = v; }
      acc += (double)v * v;
      g2[base + i] = two_l2 * v;
    }
  }
  __syncthreads();
  const long long srow = (long long)slot_of(b, k) * args.S;
  for (int u = threadIdx.x; u < args.S / 8; u += blockDim.x) {
    uint32_t p0[4], p1[4], p2[4];
#pragma unroll
    for (int e2 = 0; e2 < 4; ++e2) {
      uint32_t h0 = 0, h1 = 0, h2 = 0;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int sl = u * 8 + e2 * 2 + e;
        const int t = sl / kGroupSlots, r = sl % kGroupSlots;
        float v = 0.0f;
        if (r < kGroupUsed) {
          const int a = r / kGroupCols, j = t * kGroupCols + r % kGroupCols;
          if (j < L) v = xrow[a * L + j];
        }
        const __nv_bfloat16 hb = __float2bfloat16_rn(v);
        const float r1 = v - __bfloat162float(hb);
        const __nv_bfloat16 lb = __float2bfloat16_rn(r1);
        h0 |= (uint32_t)__bfloat16_as_ushort(hb) << (16 * e);
        h1 |= (uint32_t)__bfloat16_as_ushort(lb) << (16 * e);
        if (NSPLIT > 2)
          h2 |= (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(r1 - __bfloat162float(lb)))
                << (16 * e);
      }
      p0[e2] = h0; p1[e2] = h1; p2[e2] = h2;
    }
    const long long off = srow + (long long)u * 8;
    *reinterpret_cast<uint4 *>(args.wperm[0] + off) = make_uint4(p0[0], p0[1], p0[2], p0[3]);
    *reinterpret_cast<uint4 *>(args.wperm[1] + off) = make_uint4(p1[0], p1[1], p1[2], p1[3]);
    if (NSPLIT > 2)
      *reinterpret_cast<uint4 *>(args.wperm[2] + off) = make_uint4(p2[0], p2[1], p2[2], p2[3]);
  }
  // block reduction, fixed order
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += red[w];
    args.part_reg[row] = sum;
  }
}

// --------------------------------------------------------------- tc_forward
// The forward runs on CTA pairs (clusters of 2): one pair MMA of M = 256 rows x
// N = 256 slots per K step, each CTA holding 128 of the rows (kFwdBM) and 128 of
// the slot columns of B.  Per CTA and K step that is half the B bytes of a
// single-CTA 128 x 256 tile, which is what keeps the tensor pipe fed.
constexpr int kFwdBM = 128, kFwdBN = 256, kFwdBK = 32;
constexpr int kFwdPairM = 2 * kFwdBM;   // rows per pair tile
constexpr int kFwdHalfN = kFwdBN / 2;   // B columns held by each CTA
// forward: warp 0 TMA, warp 1 MMA (leader CTA), warps 2-9 epilogue (two warps per
// TMEM lane quarter, each owning half of the 256 accumulator columns)
constexpr int kFwdThreads = 320;

template <int NSPLIT>
struct FwdSmem {
  static constexpr int kStages = NSPLIT == 2 ? 8 : 6;
  static constexpr int kABytes = kFwdBM * kFwdBK * 2;            // 8 KB, K-major, 64B swizzle
  static constexpr int kBBytes = kFwdHalfN * kFwdBK * 2;         // 8 KB per term, MN-major
  static constexpr int kStage = kABytes + NSPLIT * kBBytes;
  static constexpr int kBarOff = kStages * kStage;
  static constexpr int kVOff = kBarOff + 256;                     // V of the tile's 12 columns
  static constexpr int kXOff = kVOff + 1024;                       // half-to-half exchange
  static constexpr int kXBytes = 2 * kFwdBM * 12 * 4;              // [half][row][12]
  static constexpr int kTotal = kXOff + kXBytes + 1024;            // + alignment slack
};

__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
  const uint32_t s = smem_u32(p);
  return p + ((1024u - (s & 1023u)) & 1023u);
}

__device__ __forceinline__ void record_error(int *status, int bit, int *abort_flag) {
  atomicOr(status, bit);
  *reinterpret_cast<volatile int *>(abort_flag) = 1;
}

__device__ __forceinline__ bool aborted(const int *abort_flag) {
  return *reinterpret_cast<const volatile int *>(abort_flag) != 0;
}

// Forward epilogue for one warp: TMEM lane quarter q, column half H (chunks
// 4H..4H+3 of the 8 x 32 accumulator columns).  The softmax over the 21
// states of each of the 12 alignment columns of the tile needs both halves:
// the per-column max and sum of exp are exchanged with the partner warp
// (same rows, other half) through shared memory.
template <int NSPLIT, int H>
__device__ __forceinline__ void fwd_epilogue_tile(const FwdArgs &args, uint32_t taddr, const float *Vs,
                                                  float *xbuf, int q, int lane, int n, int t,
                                                  long long part) {
  const int L = args.L;
  const int j0 = t * kGroupCols;
  const bool live = n < args.N;
  const float wn = live ? args.w[n] : 0.0f;
  const int row = q * 32 + lane;
  const int pair_bar = 2 + q;
  int xr[kGroupCols];
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) {
    const int j = j0 + jj;
    xr[jj] = (live && j < L) ? (int)args.msa[(long long)n * L + j] : -1;
  }
  const volatile float *Vv = Vs;
  float *mine = xbuf + (H * kFwdBM + row) * kGroupCols;
  const float *other = xbuf + ((1 - H) * kFwdBM + row) * kGroupCols;

  float mx[kGroupCols], tg[kGroupCols], se[kGroupCols];
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) { mx[jj] = -INFINITY; tg[jj] = 0.0f; se[jj] = 0.0f; }
  // pass A: max over own states, logit of the observed state if it is ours
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint32_t v[32];
    __syncwarp();
    tmem_ld32(taddr + (4 * H + c) * 32, v);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int col = (4 * H + c) * 32 + i;
      if (col < kGroupUsed) {
        const int a = col / kGroupCols, jj = col % kGroupCols;
        const float z = __uint_as_float(v[i]) + (a < kQ - 1 ? Vv[a * kGroupCols + jj] : 0.0f);
        mx[jj] = fmaxf(mx[jj], z);
        if (xr[jj] == a) tg[jj] = z;
      }
    }
  }
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) mine[jj] = mx[jj];
  named_bar_sync(pair_bar, 64);
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) mx[jj] = fmaxf(mx[jj], other[jj]);
  named_bar_sync(pair_bar, 64);  // partner has read `mine`
  // pass B: own part of the sum of exp
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint32_t v[32];
    __syncwarp();
    tmem_ld32(taddr + (4 * H + c) * 32, v);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int col = (4 * H + c) * 32 + i;
      if (col < kGroupUsed) {
        const int a = col / kGroupCols, jj = col % kGroupCols;
        const float z = __uint_as_float(v[i]) + (a < kQ - 1 ? Vv[a * kGroupCols + jj] : 0.0f);
        se[jj] += expf(z - mx[jj]);
      }
    }
  }
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) mine[jj] = se[jj];
  named_bar_sync(pair_bar, 64);
  float lse[kGroupCols];
  double floss = 0.0;
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) {
    // both halves form the same sum: H=0 adds (own + partner), H=1 (partner + own)
    const float tot = H == 0 ? se[jj] + other[jj] : other[jj] + se[jj];
    lse[jj] = mx[jj] + logf(tot);
    // the loss term belongs to the half holding the observed state's column
    if (xr[jj] >= 0 && ((xr[jj] * kGroupCols + jj) >> 7) == H)
      floss += (double)(wn * (lse[jj] - tg[jj]));
  }
  // pass C: R = w (P - onehot) over own 128 slots, split into bf16 terms
  const long long rbase = (long long)n * args.S + (long long)t * kGroupSlots;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int cc = 4 * H + c;
    uint32_t v[32];
    __syncwarp();
    tmem_ld32(taddr + cc * 32, v);
    tmem_wait_ld();
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      // 16 columns = 32 bytes of each bf16 term: one full-sector store per term
      uint32_t ph[8], pl[8], pl2[8];
#pragma unroll
      for (int e2 = 0; e2 < 8; ++e2) {
        uint32_t hh = 0, ll = 0, l2 = 0;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = u * 16 + e2 * 2 + e;
          const int col = cc * 32 + i;
          float r = 0.0f;
          if (col < kGroupUsed) {
            const int a = col / kGroupCols, jj = col % kGroupCols;
            const float z = __uint_as_float(v[i]) + (a < kQ - 1 ? Vv[a * kGroupCols + jj] : 0.0f);
            if (xr[jj] >= 0) r = wn * (expf(z - lse[jj]) - (xr[jj] == a ? 1.0f : 0.0f));
          }
          const __nv_bfloat16 hb = __float2bfloat16_rn(r);
          const float rr = r - __bfloat162float(hb);
          const __nv_bfloat16 lb = __float2bfloat16_rn(rr);
          hh |= (uint32_t)__bfloat16_as_ushort(hb) << (16 * e);
          ll |= (uint32_t)__bfloat16_as_ushort(lb) << (16 * e);
          if (NSPLIT > 2)
            l2 |= (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(rr - __bfloat162float(lb)))
                  << (16 * e);
        }
        ph[e2] = hh; pl[e2] = ll; pl2[e2] = l2;
      }
      const long long off = rbase + cc * 32 + u * 16;
      st_global_v8(args.r[0] + off, ph);
      st_global_v8(args.r[1] + off, pl);
      if (NSPLIT > 2) st_global_v8(args.r[2] + off, pl2);
    }
  }
  // loss partial, one per (tile, epilogue warp), summed in fixed order by tc_finalize
  for (int o = 16; o > 0; o >>= 1) floss += __shfl_xor_sync(0xffffffffu, floss, o);
  if (lane == 0) args.part_f[part * 8 + H * 4 + q] = floss;
}

template <int NSPLIT>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kFwdThreads, 1)
    tc_forward_kernel(const __grid_constant__ FwdMaps maps, FwdArgs args) {
  using SM = FwdSmem<NSPLIT>;
  constexpr int kFwdStages = SM::kStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align1024(smem_raw);
  // barriers: full[] is used in the leader only (it counts the bytes of both
  // CTAs' loads); empty[] and tfull[] in both (the leader's commits reach both);
  // tempty[] in the leader only (all 16 epilogue warps of the pair arrive there)
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + SM::kBarOff);
  uint64_t *empty = full + kFwdStages;
  uint64_t *tfull = empty + kFwdStages;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
  float *Vs = reinterpret_cast<float *>(smem + SM::kVOff);
  float *xbuf = reinterpret_cast<float *>(smem + SM::kXOff);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int n_tiles = args.m_tiles * args.T;  // m_tiles counts 256-row pair tiles
  const int k_blocks = args.S / kFwdBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kFwdStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&tfull[a], 1); mbar_init(&tempty[a], 16); }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&maps.a);
    for (int i = 0; i < NSPLIT; ++i) prefetch_tmap(&maps.b[i]);
  }
  if (warp == 1) { tmem_alloc_pair(tmem_slot, 512); tmem_relinquish_pair(); }
  // both CTAs' barriers initialised and TMEM allocated before any remote use
  tc_fence_before();
  cluster_sync();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer (both CTAs): own A rows, own half of B
      uint32_t it = 0;
      for (int tile = pair; tile < n_tiles && !aborted(abort_flag); tile += npairs) {
        const int m = tile % args.m_tiles, t = tile / args.m_tiles;
        const int row0 = m * kFwdPairM + (int)rank * kFwdBM;
        const int col0 = t * kFwdBN + (int)rank * kFwdHalfN;
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int stage = it % kFwdStages;
          const uint32_t round = it / kFwdStages;
          if (!mbar_wait(&empty[stage], (round & 1) ^ 1)) {
            record_error(args.status, kErrFwdTimeout, abort_flag);
            break;
          }
          uint8_t *sa = smem + stage * SM::kStage;
          const uint32_t fb = mapa_shared(smem_u32(&full[stage]), 0);
          if (rank == 0) mbar_arrive_expect_tx(&full[stage], 2 * SM::kStage);
          tma_load_2d_pair(sa, &maps.a, fb, kb * kFwdBK, row0);
          for (int i = 0; i < NSPLIT; ++i) {
            uint8_t *sb = sa + SM::kABytes + i * SM::kBBytes;
            for (int c = 0; c < kFwdHalfN / 64; ++c)
              tma_load_2d_pair(sb + c * (kFwdBK * 128), &maps.b[i], fb, col0 + c * 64,
                               kb * kFwdBK);
          }
        }
      }
      // drain: every issued load must land before the CTA may exit.  The leader
      // sees both CTAs' bytes on its full barriers; the other CTA sees the MMA's
      // release of each stage (issued after the stage's loads were consumed).
      const uint32_t issued = it;
      for (uint32_t r = (issued > kFwdStages ? issued - kFwdStages : 0); r < issued; ++r) {
        const bool ok = rank == 0 ? mbar_wait(&full[r % kFwdStages], (r / kFwdStages) & 1)
                                  : mbar_wait(&empty[r % kFwdStages], (r / kFwdStages) & 1);
        if (!ok) {
          record_error(args.status, kErrFwdTimeout, abort_flag);
          break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---------------- MMA issuer (leader CTA): 256 x 256 x 16 pair MMAs
      constexpr uint32_t idesc = idesc_bf16_f32(kFwdPairM, kFwdBN, 0, 1);
      uint32_t it = 0;
      int local = 0;
      for (int tile = pair; tile < n_tiles && !aborted(abort_flag); tile += npairs, ++local) {
        const int acc = local & 1;
        const uint32_t use = local >> 1;
        if (!mbar_wait(&tempty[acc], (use & 1) ^ 1)) {
          record_error(args.status, kErrFwdTimeout, abort_flag);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + acc * kFwdBN;
        bool ok = true;
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int stage = it % kFwdStages;
          const uint32_t round = it / kFwdStages;
          if (!mbar_wait(&full[stage], round & 1)) {
            record_error(args.status, kErrFwdTimeout, abort_flag);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + stage * SM::kStage);
          const uint32_t b0 = a0 + SM::kABytes;
#pragma unroll
          for (int k16 = 0; k16 < kFwdBK / 16; ++k16) {
            const uint64_t ad = sdesc_sw64(a0 + k16 * 32, 16, 512);
#pragma unroll
            for (int i = 0; i < NSPLIT; ++i) {
              const uint64_t bd =
                  sdesc_sw128(b0 + i * SM::kBBytes + k16 * 16 * 128, kFwdBK * 128, 1024);
              umma_bf16_pair(d, ad, bd, idesc, (kb | k16 | i) != 0);
            }
          }
          umma_commit_pair(&empty[stage], 0x3);
        }
        if (!ok) break;
        umma_commit_pair(&tfull[acc], 0x3);
      }
      umma_commit_pair(drain, 0x1);
      if (!mbar_wait(drain, 0)) record_error(args.status, kErrFwdTimeout, abort_flag);
    }
  } else {
    // ---------------- epilogue (both CTAs): 8 warps; warp w owns TMEM lanes
    // 32*(w%4) ... and column half (w-2)/4 of this CTA's 128 rows
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int ethr = threadIdx.x - 64;
    const int L = args.L;
    int local = 0;
    for (int tile = pair; tile < n_tiles; tile += npairs, ++local) {
      // all eight epilogue warps agree here: every one finished the previous
      // tile (so Vs may be overwritten) and none has seen an abort
      if (named_bar_or(1, 256, aborted(abort_flag))) break;
      const int acc = local & 1;
      const uint32_t use = local >> 1;
      const int m = tile % args.m_tiles, t = tile / args.m_tiles;
      const int j0 = t * kGroupCols;
      if (ethr < (kQ - 1) * kGroupCols) {
        const int a = ethr / kGroupCols, j = j0 + ethr % kGroupCols;
        Vs[ethr] = (j < L) ? args.x1[a * L + j] : 0.0f;
      }
      named_bar_sync(1, 256);
      const int n = m * kFwdPairM + (int)rank * kFwdBM + q * 32 + lane;
      bool ok = mbar_wait(&tfull[acc], use & 1);
      if (__any_sync(0xffffffffu, !ok)) {
        // leave through the agreement barrier at the top of the loop; the
        // partner warp times out on the same barrier
        if (lane == 0) record_error(args.status, kErrFwdTimeout, abort_flag);
        continue;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + acc * kFwdBN + ((uint32_t)(q * 32) << 16);
      const long long part = (long long)tile * 2 + rank;
      if (half == 0)
        fwd_epilogue_tile<NSPLIT, 0>(args, taddr, Vs, xbuf, q, lane, n, t, part);
      else
        fwd_epilogue_tile<NSPLIT, 1>(args, taddr, Vs, xbuf, q, lane, n, t, part);
      // accumulator may be reused by the leader's MMA warp
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&tempty[acc]), 0));
    }
  }

  // neither CTA leaves while the other may still read its shared memory or
  // signal its barriers
  tc_fence_before();
  cluster_sync();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 512);
  }
}

// -------------------------------------------------------------- tc_backward
// Like the forward, the backward runs on CTA pairs: a pair tile is 256 slots P
// (C rows, 128 per CTA) x kBwdBN slots Q (C columns, half of the B operand per
// CTA).  N = 256 keeps the operand bytes per MMA clock low enough for shared
// memory to feed the tensor pipe (N = 128 tiles measured 25 % slower).
constexpr int kBwdBM = 128, kBwdBN = 256, kBwdBK = 32;
constexpr int kBwdPairM = 2 * kBwdBM;
constexpr int kBwdHalfN = kBwdBN / 2;
constexpr int kBwdBufs = 512 / kBwdBN;  // TMEM accumulators of kBwdBN columns
// The K loop (rows of the alignment) is cut into chunks of kBwdChunkKB k-blocks
// (1280 rows).  Each chunk is accumulated by the tensor cores into one of the two
// TMEM buffers, and the epilogue adds the finished chunk into FP32 registers
// (round-to-nearest).  The tensor-core accumulator then never sums more than
// one chunk, which keeps its rounding error from growing with N.
constexpr int kBwdChunkKB = 40;
// warp 0 TMA, warp 1 MMA (leader CTA), warps 2-9 epilogue (two warps per TMEM
// lane quarter, one per half of the 256 columns)
constexpr int kBwdThreads = 320;

template <int NSPLIT>
struct BwdSmem {
  static constexpr int kStages = NSPLIT == 2 ? 4 : 3;
  static constexpr int kChunk = kBwdBK * 128;                    // 64 slots x BK rows = 4 KB
  static constexpr int kA = 2 * kChunk;                          // this CTA's 128 P slots
  static constexpr int kB = (kBwdHalfN / 64) * kChunk;           // this CTA's Q slots
  // stage: O_P | R_P[i] | O_Q | R_Q[i]
  static constexpr int kOffOP = 0;
  static constexpr int kOffRP = kA;
  static constexpr int kOffOQ = kA + NSPLIT * kA;
  static constexpr int kOffRQ = kOffOQ + kB;
  static constexpr int kStage = kOffRQ + NSPLIT * kB;
  static constexpr int kBarOff = kStages * kStage;
  static constexpr int kTOff = kBarOff + 256;                    // epilogue transpose buffers
  static constexpr int kTBytes = 8 * 32 * 9 * 4;                 // 8 warps x 32 rows x 8(+1) cols
  static constexpr int kTotal = kTOff + kTBytes + 1024;
};

// SYM = true: C = [O;R]^T [R;O] on the upper triangle of tiles, written to
// g2 directly and transposed (the reference's tied gradient).  SYM = false:
// G = O^T R on all tiles, written directly only, self blocks included (the
// true partial derivatives, for gradient checks and autograd).
template <int NSPLIT, bool SYM>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kBwdThreads, 1)
    tc_backward_kernel(const __grid_constant__ BwdMaps maps, BwdArgs args) {
  using SM = BwdSmem<NSPLIT>;
  constexpr int kStages = SM::kStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align1024(smem_raw);
  // full[] and tempty[] are used in the leader only; empty[] and tfull[] in both
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + SM::kBarOff);
  uint64_t *empty = full + kStages;
  uint64_t *tfull = empty + kStages;
  uint64_t *tempty = tfull + kBwdBufs;
  uint64_t *drain = tempty + kBwdBufs;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int n_tiles = args.n_tiles;
  const int k_blocks = args.Npad / kBwdBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int a = 0; a < kBwdBufs; ++a) { mbar_init(&tfull[a], 1); mbar_init(&tempty[a], 16); }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&maps.o);
    for (int i = 0; i < NSPLIT; ++i) prefetch_tmap(&maps.r[i]);
  }
  if (warp == 1) { tmem_alloc_pair(tmem_slot, 512); tmem_relinquish_pair(); }
  tc_fence_before();
  cluster_sync();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      for (int tile = pair; tile < n_tiles && !aborted(abort_flag); tile += npairs) {
        const int2 pq = args.tiles[tile];
        const int xP = pq.x * kBwdPairM + (int)rank * kBwdBM;
        const int xQ = pq.y * kBwdBN + (int)rank * kBwdHalfN;
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int stage = it % kStages;
          const uint32_t round = it / kStages;
          if (!mbar_wait(&empty[stage], (round & 1) ^ 1)) {
            record_error(args.status, kErrBwdTimeout, abort_flag);
            break;
          }
          uint8_t *st = smem + stage * SM::kStage;
          const int y = kb * kBwdBK;
          const uint32_t fb = mapa_shared(smem_u32(&full[stage]), 0);
          if (rank == 0)
            mbar_arrive_expect_tx(&full[stage],
                                  2 * (SYM ? SM::kStage : SM::kA + NSPLIT * SM::kB));
          for (int c = 0; c < 2; ++c)
            tma_load_2d_pair(st + SM::kOffOP + c * SM::kChunk, &maps.o, fb, xP + 64 * c, y);
          if (SYM) {
            for (int i = 0; i < NSPLIT; ++i)
              for (int c = 0; c < 2; ++c)
                tma_load_2d_pair(st + SM::kOffRP + i * SM::kA + c * SM::kChunk, &maps.r[i], fb,
                                 xP + 64 * c, y);
            for (int c = 0; c < kBwdHalfN / 64; ++c)
              tma_load_2d_pair(st + SM::kOffOQ + c * SM::kChunk, &maps.o, fb, xQ + 64 * c, y);
          }
          for (int i = 0; i < NSPLIT; ++i)
            for (int c = 0; c < kBwdHalfN / 64; ++c)
              tma_load_2d_pair(st + SM::kOffRQ + i * SM::kB + c * SM::kChunk, &maps.r[i], fb,
                               xQ + 64 * c, y);
        }
      }
      // drain (as in tc_forward): the leader's full barriers count both CTAs'
      // bytes; the other CTA waits for the MMA's release of its last stages
      const uint32_t issued = it;
      for (uint32_t r = (issued > (uint32_t)kStages ? issued - kStages : 0); r < issued; ++r) {
        const bool ok = rank == 0 ? mbar_wait(&full[r % kStages], (r / kStages) & 1)
                                  : mbar_wait(&empty[r % kStages], (r / kStages) & 1);
        if (!ok) {
          record_error(args.status, kErrBwdTimeout, abort_flag);
          break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      constexpr uint32_t idesc = idesc_bf16_f32(kBwdPairM, kBwdBN, 1, 1);
      uint32_t it = 0;
      uint32_t chunk = 0;  // chunks issued by this pair, across tiles
      bool ok = true;
      for (int tile = pair; tile < n_tiles && ok && !aborted(abort_flag); tile += npairs) {
        for (int kb0 = 0; kb0 < k_blocks && ok; kb0 += kBwdChunkKB, ++chunk) {
          const int buf = chunk % kBwdBufs;
          const uint32_t use = chunk / kBwdBufs;
          if (!mbar_wait(&tempty[buf], (use & 1) ^ 1)) {
            record_error(args.status, kErrBwdTimeout, abort_flag);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem_base + buf * kBwdBN;
          const int kb1 = min(kb0 + kBwdChunkKB, k_blocks);
          for (int kb = kb0; kb < kb1; ++kb, ++it) {
            const int stage = it % kStages;
            const uint32_t round = it / kStages;
            if (!mbar_wait(&full[stage], round & 1)) {
              record_error(args.status, kErrBwdTimeout, abort_flag);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t s0 = smem_u32(smem + stage * SM::kStage);
#pragma unroll
            for (int k16 = 0; k16 < kBwdBK / 16; ++k16) {
              const uint32_t ko = k16 * 16 * 128;
              const uint64_t dOP = sdesc_sw128(s0 + SM::kOffOP + ko, SM::kChunk, 1024);
              const uint64_t dOQ = sdesc_sw128(s0 + SM::kOffOQ + ko, SM::kChunk, 1024);
#pragma unroll
              for (int i = 0; i < NSPLIT; ++i) {
                const uint64_t dRQ =
                    sdesc_sw128(s0 + SM::kOffRQ + i * SM::kB + ko, SM::kChunk, 1024);
                umma_bf16_pair(d, dOP, dRQ, idesc, ((kb - kb0) | k16 | i) != 0);
              }
              if (SYM) {
#pragma unroll
                for (int i = 0; i < NSPLIT; ++i) {
                  const uint64_t dRP =
                      sdesc_sw128(s0 + SM::kOffRP + i * SM::kA + ko, SM::kChunk, 1024);
                  umma_bf16_pair(d, dRP, dOQ, idesc, 1);
                }
              }
            }
            umma_commit_pair(&empty[stage], 0x3);
          }
          if (!ok) break;
          umma_commit_pair(&tfull[buf], 0x3);
        }
      }
      umma_commit_pair(drain, 0x1);
      if (!mbar_wait(drain, 0)) record_error(args.status, kErrBwdTimeout, abort_flag);
    }
  } else {
    // Epilogue.  Each thread owns one row s1 of the tile (TMEM lane) and one
    // half of its 256 columns; it sums the tile's K chunks in FP32 registers,
    // then writes every element (s1, s2), s1 <= s2, of the symmetric C to
    //   direct      g2 row (b,k) = s1, column (a,j) = s2
    //   transposed  g2 row (a,j) = s2, column (b,k) = s1   (s1 != s2)
    // (SYM = false: direct only, all elements).  Transposed writes are issued
    // thread-major (consecutive lanes = consecutive k: contiguous runs); direct
    // writes go through a per-warp shared-memory transpose so that one warp
    // instruction covers 4 rows x 8 columns (runs of consecutive j).  g2 already
    // holds the regulariser term (tc_prep) and every element receives exactly one
    // atomic add, so the result does not depend on the order of the adds.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int L = args.L;
    float *__restrict__ g2 = args.g2;
    float *Tb = reinterpret_cast<float *>(smem + SM::kTOff) + (warp - 2) * 32 * 9;
    uint32_t chunk = 0;
    bool ok = true;
    for (int tile = pair; tile < n_tiles && ok; tile += npairs) {
      float accv[kBwdHalfN];
#pragma unroll
      for (int i = 0; i < kBwdHalfN; ++i) accv[i] = 0.0f;
      for (int kb0 = 0; kb0 < k_blocks; kb0 += kBwdChunkKB, ++chunk) {
        const int buf = chunk % kBwdBufs;
        const uint32_t use = chunk / kBwdBufs;
        const bool w_ok = mbar_wait(&tfull[buf], use & 1);
        if (__any_sync(0xffffffffu, !w_ok)) {
          if (lane == 0) record_error(args.status, kErrBwdTimeout, abort_flag);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr =
            tmem_base + buf * kBwdBN + half * kBwdHalfN + ((uint32_t)(q * 32) << 16);
#pragma unroll
        for (int c = 0; c < kBwdHalfN / 32; ++c) {
          uint32_t v[32];
          __syncwarp();
          tmem_ld32(taddr + c * 32, v);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 32; ++i) accv[c * 32 + i] += __uint_as_float(v[i]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&tempty[buf]), 0));
      }
      if (!ok) break;

      const int2 pq = args.tiles[tile];
      const int rowbase = pq.x * kBwdPairM + (int)rank * kBwdBM + q * 32;
      const int s1 = rowbase + lane;
      const int t1 = s1 / kGroupSlots, r1 = s1 % kGroupSlots;
      const int b = r1 / kGroupCols, k = t1 * kGroupCols + r1 % kGroupCols;
      const bool valid1 = r1 < kGroupUsed && k < L;
      const long long colt = (long long)b * L + k;  // transposed: + ((a*L+j)*32)*L
      // columns: Q block pq.y of kBwdBN slots, inside slot group tQ from slot rQ
      const int tQ = pq.y * kBwdBN / kGroupSlots;
      const int rQ = pq.y * kBwdBN % kGroupSlots + half * kBwdHalfN;
      const int sQ = tQ * kGroupSlots + rQ;
      // 8 rounds of 8 columns through the transpose buffer Tb[row][col]
#pragma unroll
      for (int cb = 0; cb < kBwdHalfN / 8; ++cb) {
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 8; ++e) Tb[lane * 9 + e] = accv[cb * 8 + e];
        __syncwarp();
        // (A) transposed writes and the ones-slot column: thread = row s1
        if (SYM) {
#pragma unroll 1
          for (int col = 0; col < 8; ++col) {
            const int r2 = rQ + cb * 8 + col;
            const int s2 = sQ + cb * 8 + col;
            const int a = r2 / kGroupCols, j = tQ * kGroupCols + r2 % kGroupCols;
            const bool valid2 = r2 < kGroupUsed && j < L;
            if (s1 < s2) {
              const float val = Tb[lane * 9 + col];
              if (valid1 && valid2) {
                if (k != j) atomicAdd(g2 + ((long long)a * L + j) * kQPad * L + colt, val);
              } else if (s2 == kOnesSlot && valid1 && b < kQ - 1) {
                args.g1d[b * L + k] = val;
              }
            }
          }
        }
        // (B) direct writes and the ones-slot row: lanes = 4 rows x 8 columns
        const int col = lane & 7;
        const int r2 = rQ + cb * 8 + col;
        const int s2 = sQ + cb * 8 + col;
        const int a = r2 / kGroupCols, j = tQ * kGroupCols + r2 % kGroupCols;
        const bool valid2 = r2 < kGroupUsed && j < L;
#pragma unroll
        for (int it = 0; it < 8; ++it) {
          const int row = 4 * it + (lane >> 3);
          const int s1r = rowbase + row;
          if (SYM && s1r > s2) continue;
          const float val = Tb[row * 9 + col];
          const int tr = s1r / kGroupSlots, rr = s1r % kGroupSlots;
          const int br = rr / kGroupCols, kr = tr * kGroupCols + rr % kGroupCols;
          if (rr < kGroupUsed && kr < L) {
            if (valid2 && (!SYM || kr != j)) atomicAdd(g2 + x2_index(br, kr, a, j, L), val);
          } else if (s1r == kOnesSlot && valid2 && a < kQ - 1) {
            args.g1d[a * L + j] = val;
          }
        }
      }
    }
  }

  tc_fence_before();
  cluster_sync();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 512);
  }
}

// -------------------------------------------------------------- tc_finalize
// fx = sum(loss partials) + lambda1 sum V^2 + 0.5 lambda2 sum x2^2 (all in FP64,
// fixed summation order); g1 = g1d + 2 lambda1 V, g1 padding = 0
// (src/evaluate_cpu.c:151-163).  kFinBlocks blocks each sum a fixed share of
// the partials; the block that finishes last (a ticket counter, reset by it)
// adds the blocks' sums in block order and writes the result.
__global__ void __launch_bounds__(kFinThreads) tc_finalize_kernel(FinalizeArgs args) {
  __shared__ double red[kFinThreads / 32][3];
  __shared__ bool last;
  griddep_wait();
  griddep_launch();
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  double acc_f = 0.0, acc_r2 = 0.0, acc_r1 = 0.0;
  for (long long i = tid; i < args.n_part_f; i += stride) acc_f += args.part_f[i];
  for (long long i = tid; i < args.n_part_reg; i += stride) acc_r2 += args.part_reg[i];
  const long long ns = nsingle_of(args.L);
  const float two_l1 = 2.0f * args.lambda_single;
  for (long long v = tid; v < args.nsp; v += stride) {
    if (v < ns) {
      const float xv = args.x1[v];
      acc_r1 += (double)xv * (double)xv;
      if (args.g1 != nullptr) args.g1[v] = args.g1d[v] + two_l1 * xv;
    } else if (args.g1 != nullptr) {
      args.g1[v] = 0.0f;
    }
  }
  double acc[3] = {acc_f, acc_r2, acc_r1};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = acc[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[3] = {0.0, 0.0, 0.0};
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
      for (int k = 0; k < 3; ++k) s[k] += red[w][k];
    for (int k = 0; k < 3; ++k) args.block_part[3 * blockIdx.x + k] = s[k];
    __threadfence();
    last = atomicAdd(args.done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double s[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < (int)gridDim.x; ++b)
      for (int k = 0; k < 3; ++k) s[k] += __ldcg(args.block_part + 3 * b + k);
    const double F = s[0], R2 = s[1], R1 = s[2];
    const double fx = F + (double)args.lambda_single * R1 + 0.5 * (double)args.lambda_pair * R2;
    args.out->fx = fx;
    args.out->f_data = F;
    args.out->reg = fx - F;
    *args.done = 0u;  // for the next evaluation (also inside a replayed graph)
  }
}

// ---------------------------------------------------------------- launchers
// Without a step: evaluate at d_x.  With one (step_x, step_s, alpha): evaluate
// at d_x := step_x + alpha * step_s, which tc_prep computes and writes to d_x.
template <int NSPLIT>
static cudaError_t launch_tc(ccm_context *c, const float *d_x, float *d_g,
                             const float *step_x = nullptr, const float *step_s = nullptr,
                             const double *alpha = nullptr) {
  const int L = c->L;
  const float *x1 = d_x;
  const float *x2 = d_x + c->nsp;
  float *g2 = d_g + c->nsp;
  const bool step = step_x != nullptr;

  PrepArgs pa{};
  pa.L = L; pa.S = c->S; pa.lambda_pair = c->lambda_pair; pa.part_reg = c->d_part_reg;
  pa.g2_coef = c->gradient == CCM_GRADIENT_PARTIAL ? 1.0f : 2.0f;
  for (int i = 0; i < 3; ++i) pa.wperm[i] = c->d_wperm[i];
  prof_mark(c);
  if (step) {
    pa.step_x = step_x; pa.step_s = step_s; pa.alpha = alpha;
    pa.xt = const_cast<float *>(d_x); pa.nsp = c->nsp;
    tc_prep_kernel<NSPLIT, true><<<kQ * L + 1, 256, sizeof(float) * kQ * L, c->stream>>>(
        step_x + c->nsp, g2, pa);
  } else {
    tc_prep_kernel<NSPLIT, false><<<kQ * L, 256, sizeof(float) * kQ * L, c->stream>>>(x2, g2, pa);
  }
  prof_mark(c);

  FwdArgs fa{};
  fa.msa = c->d_msa; fa.w = c->d_w; fa.x1 = x1; fa.part_f = c->d_part_f; fa.status = c->d_status;
  for (int i = 0; i < 3; ++i) fa.r[i] = c->d_r[i];
  fa.L = L; fa.N = c->N; fa.S = c->S; fa.T = c->T; fa.Npad = c->Npad;
  fa.m_tiles = c->Npad / kFwdPairM;
  const int pair_tiles = fa.m_tiles * c->T;
  const int fwd_tiles = 2 * pair_tiles;  // 128-row halves, one loss partial set each
  const int pairs = pair_tiles < c->fwd_pairs ? pair_tiles : c->fwd_pairs;
  tc_forward_kernel<NSPLIT><<<2 * pairs, kFwdThreads, FwdSmem<NSPLIT>::kTotal, c->stream>>>(
      c->fwd_maps, fa);
  prof_mark(c);

  BwdArgs ba{};
  ba.x2 = x2; ba.g2 = g2; ba.g1d = c->d_g1d; ba.tiles = c->d_bwd_tiles;
  ba.n_tiles = c->n_bwd_tiles; ba.status = c->d_status; ba.L = L; ba.S = c->S; ba.Npad = c->Npad;
  ba.lambda_pair = c->lambda_pair;
  const int bwd_pairs = c->n_bwd_tiles < c->bwd_pairs ? c->n_bwd_tiles : c->bwd_pairs;
  if (c->gradient == CCM_GRADIENT_PARTIAL)
    tc_backward_kernel<NSPLIT, false>
        <<<2 * bwd_pairs, kBwdThreads, BwdSmem<NSPLIT>::kTotal, c->stream>>>(c->bwd_maps, ba);
  else
    tc_backward_kernel<NSPLIT, true>
        <<<2 * bwd_pairs, kBwdThreads, BwdSmem<NSPLIT>::kTotal, c->stream>>>(c->bwd_maps, ba);
  prof_mark(c);

  launch_tc_finalize(c, x1, d_g, fwd_tiles);
  prof_mark(c);
  count_launch(c, 4);
  return cudaGetLastError();
}

cudaError_t launch_tc_finalize(ccm_context *c, const float *x1, float *d_g, long long n_fwd_tiles) {
  FinalizeArgs za{};
  za.part_f = c->d_part_f; za.n_part_f = n_fwd_tiles * 8;
  za.part_reg = c->d_part_reg; za.n_part_reg = (long long)kQ * c->L;
  za.x1 = x1; za.g1d = c->d_g1d; za.g1 = d_g; za.L = c->L; za.nsp = c->nsp;
  za.lambda_single = c->lambda_single; za.lambda_pair = c->lambda_pair; za.out = c->d_out;
  za.block_part = c->d_fin_part; za.done = c->d_fin_done;
  return launch_pdl(tc_finalize_kernel, dim3(kFinBlocks), dim3(kFinThreads), 0, c->stream, za);
}

cudaError_t tc_backward_max_pairs(int nsplit, int *pairs) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(kBwdThreads, 1, 1);
  cfg.dynamicSmemBytes = nsplit == 3 ? BwdSmem<3>::kTotal : BwdSmem<2>::kTotal;
  int n = 0;
  cudaError_t e = nsplit == 3
                      ? cudaOccupancyMaxActiveClusters(&n, tc_backward_kernel<3, true>, &cfg)
                      : cudaOccupancyMaxActiveClusters(&n, tc_backward_kernel<2, true>, &cfg);
  *pairs = n;
  return e;
}

cudaError_t tc_forward_max_pairs(int nsplit, int *pairs) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(kFwdThreads, 1, 1);
  cfg.dynamicSmemBytes = nsplit == 3 ? FwdSmem<3>::kTotal : FwdSmem<2>::kTotal;
  int n = 0;
  cudaError_t e = nsplit == 3
                      ? cudaOccupancyMaxActiveClusters(&n, tc_forward_kernel<3>, &cfg)
                      : cudaOccupancyMaxActiveClusters(&n, tc_forward_kernel<2>, &cfg);
  *pairs = n;
  return e;
}

cudaError_t tc_configure_kernels() {
  cudaError_t e;
  // the staged W row is 21 L floats: up to L = 2000 (168 KB)
  e = cudaFuncSetAttribute(tc_prep_kernel<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 168000);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_prep_kernel<3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 168000);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_prep_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 168000);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_prep_kernel<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 168000);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_forward_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           FwdSmem<2>::kTotal);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_forward_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           FwdSmem<3>::kTotal);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_backward_kernel<2, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, BwdSmem<2>::kTotal);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_backward_kernel<2, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, BwdSmem<2>::kTotal);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tc_backward_kernel<3, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, BwdSmem<3>::kTotal);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(tc_backward_kernel<3, false>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, BwdSmem<3>::kTotal);
}

cudaError_t tc_evaluate(ccm_context *c, const float *d_x, float *d_g) {
  return c->nsplit == 3 ? launch_tc<3>(c, d_x, d_g) : launch_tc<2>(c, d_x, d_g);
}

cudaError_t tc_evaluate_step(ccm_context *c, const float *d_x, const float *d_s,
                             const double *d_alpha, float *d_xt, float *d_g) {
  return c->nsplit == 3 ? launch_tc<3>(c, d_xt, d_g, d_x, d_s, d_alpha)
                        : launch_tc<2>(c, d_xt, d_g, d_x, d_s, d_alpha);
}

int tc_fwd_smem_bytes(int nsplit) { return nsplit == 3 ? FwdSmem<3>::kTotal : FwdSmem<2>::kTotal; }
int tc_bwd_smem_bytes(int nsplit) { return nsplit == 3 ? BwdSmem<3>::kTotal : BwdSmem<2>::kTotal; }

}  // namespace ccm
