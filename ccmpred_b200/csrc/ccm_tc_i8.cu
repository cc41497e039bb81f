// Integer tensor-core evaluation (CCM_PATH_TC_I8X3): the same two contractions as
// the split-bf16 path (ccm_tc.cu), with 8-bit operands and exact 32-bit integer
// accumulation on tcgen05 (kind::i8, cta_group::2).
//
// Fixed-point digits.  A value v with scale 2^e (|v| <= 2^e) is represented by the
// integer Q = clamp(rint(v * 2^(21 - e)), -2^21, 2^21 - 1) and stored as three
// bytes: d0 = Q >> 14 (signed, -128..127), d1 = (Q >> 7) & 127, d2 = Q & 127, so
// that Q = d0 * 2^14 + d1 * 2^7 + d2.  The one-hot operand is stored twice, as
// unsigned bytes 1 and 128, and the contractions accumulate
//   hi = sum O1 * d0,   lo = sum O128 * d1 + sum O1 * d2 = sum O * (Q & 0x3fff)
// in two s32 TMEM accumulators; sum O * Q = hi * 2^14 + lo exactly.  W takes one
// power-of-two scale per coupling column (a, j) (its column maximum rounded up),
// R = w (P - onehot), |R| < 1, takes the scale 1.  Quantisation error: at most
// 2^-22 of the column scale per element; modelled against FP64 it gives a 3x
// smaller gradient error than the hi+lo bf16 split, and the sums are exact.
// Per K element the tensor cores do three 8-bit products (at twice the bf16
// rate) where the split-bf16 path does two bf16 products: 3/4 of the cycles.
//
// One evaluation = colmax (+ the fused CG step), prep (digits of W, g2 <- 2 l2 x,
// sum x^2), forward, backward, finalize (shared with ccm_tc.cu).
#include <cmath>

#include <cuda_bf16.h>

#include "ccm_internal.cuh"
#include "ccm_layout.cuh"
#include "ccm_ptx.cuh"

namespace ccm {

constexpr int kI8FracBits = 21;

__device__ __forceinline__ uint8_t *i8_align1024(uint8_t *p) {
  const uint32_t s = smem_u32(p);
  return p + ((1024u - (s & 1023u)) & 1023u);
}

__device__ __forceinline__ void i8_record_error(int *status, int bit, int *abort_flag) {
  atomicOr(status, bit);
  *reinterpret_cast<volatile int *>(abort_flag) = 1;
}

__device__ __forceinline__ bool i8_aborted(const int *abort_flag) {
  return *reinterpret_cast<const volatile int *>(abort_flag) != 0;
}

// 2^s as a float, s in [-126, 127].
__device__ __forceinline__ float pow2f(int s) { return __int_as_float((s + 127) << 23); }
inline float pow2_host(int s) { return std::ldexp(1.0f, s); }

// Smallest e with 2^e >= m for the float m with bits `mbits` (m >= 0), limited to
// [-100, 127] so that 2^(21 - e) stays a normal float; 0 for m == 0.
__device__ __forceinline__ int col_exponent(uint32_t mbits) {
  if (mbits == 0) return 0;
  const int E = (int)(mbits >> 23) - 127;
  const int e = (mbits & 0x7FFFFFu) ? E + 1 : E;
  return max(e, -100);
}

// ---------------------------------------------------------------- colmax
// Column maxima of |W| over the 21 L rows (b, k), per coupling column c = a*L + j
// (a < 21), as float bits with atomicMax (|v| >= 0 orders like its bits).  Block
// (bx, by): 256 consecutive columns c of a 32 L row, rows [by*R, by*R + R).
// STEP = true also takes the CG trial step: v = fmaf(alpha, s, x) is written to
// xt for every element of x (the last row of blocks steps the single fields).
// cols = 21 L instead of 32 L leaves out the padding states (a solve that keeps
// them zero in x, s and xt).
template <bool STEP>
__global__ void __launch_bounds__(256) i8_colmax_kernel(const float *__restrict__ x,
                                                        const float *__restrict__ s,
                                                        const double *__restrict__ alpha,
                                                        float *__restrict__ xt,
                                                        uint32_t *__restrict__ colmax, int L,
                                                        long long nsp, int rows_per_block,
                                                        int krow_order, int cols) {
  griddep_wait();
  griddep_launch();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int w32 = kQPad * L;
  float a = 0.0f;
  if (STEP) {
    a = (float)alpha[0];
    if (blockIdx.y == gridDim.y - 1) {
      for (long long i = c; i < nsp; i += (long long)gridDim.x * blockDim.x)
        xt[i] = fmaf(a, s[i], x[i]);
      return;
    }
  }
  if (c >= cols) return;  // cols = 32 L, or 21 L when the padding states are skipped
  const int r0 = blockIdx.y * rows_per_block;
  const int r1 = min(r0 + rows_per_block, kQ * L);
  float m = 0.0f;
  for (int r = r0; r < r1; ++r) {
    // rows in the reverse of the order in which prep reads them (plain row order, or
    // the sparse path's K-row order k * 21 + b), so that prep's first rows are the
    // ones read last here and are still in L2
    const int rr = kQ * L - 1 - r;
    const int row = krow_order ? (rr % kQ) * L + rr / kQ : rr;
    const long long i = nsp + (long long)row * w32 + c;
    float v = x[i];
    if (STEP) {
      v = fmaf(a, s[i], v);
      xt[i] = v;
    }
    m = fmaxf(m, fabsf(v));
  }
  if (c < kQ * L && m > 0.0f) atomicMax(colmax + c, __float_as_uint(m));
}

// Per slot s (of the slot groups G): the encoding factor 2^(21 - e) of the digits
// of its coupling column (e the column's exponent, from the maxima above), 0 for
// padding slots; read by prep.
template <class G>
__global__ void i8_scales_kernel(const uint32_t *__restrict__ colmax, float *__restrict__ enc,
                                 int L, int S) {
  griddep_wait();
  griddep_launch();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int t = s / G::kSlots, r = s % G::kSlots;
  float f = 0.0f;
  if (r < G::kUsed) {
    const int a = r / G::kCols, j = t * G::kCols + r % G::kCols;
    if (j < L) f = pow2f(kI8FracBits - col_exponent(colmax[a * L + j]));
  }
  enc[s] = f;
}

// Operand storage of the sparse forward.  Every operand tile a stage needs is
// stored contiguously in global memory as the exact shared-memory image the
// MMA reads (swizzle included), so that one TMA box of 256-byte rows moves it;
// tiles with 16-, 32- or 64-byte rows cost one TMA request per row and leave the
// kernel bound by the L1/TMA request rate.  KB = KP / 128 K blocks.
//   A (compressed one-hot, 128 rows x 64 bytes, 64-byte swizzle): tile
//     (m128, kb) at ((m128 * KB + kb) * 128 + r) * 64; 16-byte chunk c of row r
//     stored at chunk c ^ ((r >> 1) & 3).
//   E (metadata, 128 rows x 16 bytes, no swizzle): tile (m128, kb) at
//     ((m128 * KB + kb) * 128 + r) * 16.
//   B (digits of W; per forward tile t and CTA half h, 128 K rows x 96 slots as
//     three atoms of 32 slots, 32-byte swizzle): atom i at
//     (((t * 2 + h) * KB + kb) * 3 + i) * 4096 + r * 32; chunk c of row r stored
//     at chunk c ^ ((r >> 2) & 1).
__host__ __device__ constexpr long long i8sp_a_offset(int n, int col, int KB) {
  // col: byte of the compressed row (0 .. KP/2)
  return (((long long)(n >> 7) * KB + (col >> 6)) * 128 + (n & 127)) * 64 +
         ((((col >> 4) & 3) ^ (((n & 127) >> 1) & 3)) << 4) + (col & 15);
}
__host__ __device__ constexpr long long i8sp_e_offset(int n, int byte, int KB) {
  return (((long long)(n >> 7) * KB + (byte >> 4)) * 128 + (n & 127)) * 16 + (byte & 15);
}
__host__ __device__ constexpr long long i8sp_b_offset(int kr, int s, int KB) {
  // kr: K row (l * 21 + q), s: slot of the 192-slot groups
  const int t = s / Groups192::kSlots, c = s % Groups192::kSlots;
  const int h = c / 96, i = (c % 96) >> 5, x = c & 31, r = kr & 127;
  return ((((long long)t * 2 + h) * KB + (kr >> 7)) * 3 + i) * 4096 + r * 32 +
         ((((x >> 4) ^ (r >> 2)) & 1) << 4) + (x & 15);
}

// ---------------------------------------------------------------- prep
// One block per row (b, k) of W, as tc_prep: g2 <- g2_coef * lambda2 * x, the FP64
// partial of sum x^2, and one row of the three digit matrices of W (16 slots per
// thread, one 16-byte store per digit matrix).  Columns are the slots of the
// groups G; the row is s(b, k) (NAT = false: Wperm, both sides permuted) or
// K row k * 21 + b of the sparse forward (NAT = true, alignment column major,
// stored in its tiled layout).  args.S is the row length.  The row is staged in shared memory in slot order,
// so that the digit pass reads 16 consecutive slots per thread (vector loads, no
// index arithmetic) with their per-slot factors.
template <class G, bool NAT>
__global__ void __launch_bounds__(256) i8_prep_kernel(const float *__restrict__ x2,
                                                      float *__restrict__ g2, I8PrepArgs args) {
  griddep_wait();
  griddep_launch();
  extern __shared__ __align__(16) float xrow[];  // S floats: the row in slot order
  const int L = args.L;
  // NAT: blocks in K-row order k * 21 + b, so that blocks running together fill
  // neighbouring rows of the same stored tiles
  const int row = NAT ? (int)(blockIdx.x % kQ) * L + (int)(blockIdx.x / kQ) : (int)blockIdx.x;
  const int b = row / L, k = row % L;
  const long long base = (long long)row * kQPad * L;
  const float two_l2 = args.g2_coef * args.lambda_pair;
  const int nreal = kQ * L;
  double acc = 0.0;
  if ((L & 3) == 0) {
    const float4 *src = reinterpret_cast<const float4 *>(x2 + base);
    float4 *dst = reinterpret_cast<float4 *>(g2 + base);
    const int n4 = args.ncols / 4, nreal4 = nreal / 4;
    constexpr int kU = 4;
    for (int i0 = threadIdx.x; i0 < n4; i0 += kU * blockDim.x) {
      float4 v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int i = i0 + u * blockDim.x;
        v[u] = i < n4 ? __ldcs(src + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int i = i0 + u * blockDim.x;
        if (i < n4) {
          // four squares in float, their sum added in FP64
          acc += (double)fmaf(v[u].w, v[u].w,
                              fmaf(v[u].z, v[u].z, fmaf(v[u].y, v[u].y, v[u].x * v[u].x)));
          if (i < nreal4) {
            // c = 4i = a L + j, j a multiple of 4: the four elements share a, and
            // j .. j+3 stay inside the row's column range
            const int c = 4 * i;
            const int a = (int)(((float)c + 0.5f) * args.inv_L);
            const int j = c - a * L;
            const float vv[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) xrow[G::slot_of(a, j + e)] = vv[e];
          }
          __stcs(dst + i, make_float4(two_l2 * v[u].x, two_l2 * v[u].y, two_l2 * v[u].z,
                                      two_l2 * v[u].w));
        }
      }
    }
  } else {
    for (int i = threadIdx.x; i < args.ncols; i += blockDim.x) {
      const float v = x2[base + i];
      acc += (double)v * v;
      if (i < nreal) xrow[G::slot_of(i / L, i % L)] = v;
      g2[base + i] = two_l2 * v;
    }
  }
  __syncthreads();
  const long long srow = (long long)G::slot_of(b, k) * args.S;  // (NAT: tiled, i8sp_b_offset)
  for (int u = threadIdx.x; u < args.S / 16; u += blockDim.x) {
    uint32_t p0[4], p1[4], p2[4];
#pragma unroll
    for (int e4 = 0; e4 < 4; ++e4) {
      const float4 xv = reinterpret_cast<const float4 *>(xrow)[u * 4 + e4];
      const float4 fv = __ldg(reinterpret_cast<const float4 *>(args.enc) + u * 4 + e4);
      const float xs[4] = {xv.x, xv.y, xv.z, xv.w}, fs[4] = {fv.x, fv.y, fv.z, fv.w};
      int qv[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        // padding slots have factor 0 and are never staged: their digits are 0
        const int q = fs[e] != 0.0f ? __float2int_rn(xs[e] * fs[e]) : 0;  // exact scaling
        qv[e] = min(max(q, -(1 << kI8FracBits)), (1 << kI8FracBits) - 1);
      }
      // byte e of each word = digit of element e (as in the forward's R digits)
      auto pack = [](int b0, int b1, int b2, int b3) {
        return __byte_perm(__byte_perm(b0, b1, 0x0040), __byte_perm(b2, b3, 0x0040), 0x5410);
      };
      p0[e4] = pack(qv[0] >> 14, qv[1] >> 14, qv[2] >> 14, qv[3] >> 14);
      p1[e4] = pack(qv[0] >> 7, qv[1] >> 7, qv[2] >> 7, qv[3] >> 7) & 0x7F7F7F7Fu;
      p2[e4] = pack(qv[0], qv[1], qv[2], qv[3]) & 0x7F7F7F7Fu;
    }
    const long long off = NAT ? i8sp_b_offset(k * kQ + b, u * 16, args.KB) : srow + (long long)u * 16;
    *reinterpret_cast<uint4 *>(args.wdig[0] + off) = make_uint4(p0[0], p0[1], p0[2], p0[3]);
    *reinterpret_cast<uint4 *>(args.wdig[1] + off) = make_uint4(p1[0], p1[1], p1[2], p1[3]);
    *reinterpret_cast<uint4 *>(args.wdig[2] + off) = make_uint4(p2[0], p2[1], p2[2], p2[3]);
  }
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

// Tiled storage of the backward's operands on the sparse path (one-hot x1 /
// x128 and the digits of R, Npad x S bytes each): the 32-row x 128-slot tile
// (kb = n / 32, sb = s / 128) that one pipeline stage of one CTA reads is stored
// contiguously (4 KB) as the shared-memory image the MMA reads -- rows of 128
// slots, 16-byte chunk c of row r at chunk c ^ (r & 7) (128-byte swizzle) --
// tiles in the order sb * KB + kb, KB = Npad / 32.  One TMA box of 16 rows of
// 256 bytes moves a tile (twice the bytes per TMA row request of a 128-slot box
// of the row-major matrix).
__host__ __device__ constexpr long long i8_bwd_tile_offset(int n, int s, int KB) {
  return ((long long)(s >> 7) * KB + (n >> 5)) * 4096 + (n & 31) * 128 +
         (((((s & 127) >> 4) ^ (n & 7)) & 7) << 4) + (s & 15);
}

// One-hot operands of the integer path (slot groups G): O1[n][s] = 1 and
// O128[n][s] = 128 where the state of column l(s) in row n is q(s), and in the
// ones slot of every real row; 0 elsewhere.  TILED: stored as i8_bwd_tile_offset.
template <class G, bool TILED>
__global__ void i8_onehot_kernel(const uint8_t *__restrict__ msa, uint8_t *__restrict__ o1,
                                 uint8_t *__restrict__ o128, int L, int N, int S, int Npad) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Npad * S) return;
  const int n = (int)(idx / S), s = (int)(idx % S);
  const long long at = TILED ? i8_bwd_tile_offset(n, s, Npad >> 5) : idx;
  const int t = s / G::kSlots, r = s % G::kSlots;
  bool one = false;
  if (n < N) {
    if (s == G::kOnes) {
      one = true;
    } else if (r < G::kUsed) {
      const int q = r / G::kCols, l = t * G::kCols + r % G::kCols;
      one = l < L && msa[(long long)n * L + l] == q;
    }
  }
  o1[at] = one ? 1 : 0;
  o128[at] = one ? 128 : 0;
}

}  // namespace ccm

namespace ccm {

// ---------------------------------------------------------------- forward
// Pair tiles of 256 rows x 256 slots as in tc_forward.  Per tile the MMAs run in
// two phases: first the low digits into `lo` (O128 x d1 + O1 x d2), then the high
// digit into `hi` (O1 x d0).  The epilogue merges z = (hi * 2^14 + lo) * scale + V
// into float logits written back over `hi`, releases `lo` (the next tile's low
// phase may start), runs the softmax passes on `hi`, writes the digits of R and
// releases `hi`.  TMEM: hi = columns [0, 256), lo = [256, 512).
constexpr int kI8BM = 128, kI8PairM = 256, kI8BN = 256, kI8HalfN = 128, kI8FwdBK = 64;
constexpr int kI8Threads = 320;

struct I8FwdSmem {
  static constexpr int kStages = 6;
  static constexpr int kTile = kI8BM * kI8FwdBK;  // 8 KB: A 128 rows x 64 B, B 64 rows x 128 B
  static constexpr int kOffA1 = 0;
  static constexpr int kOffA128 = kTile;
  static constexpr int kOffB = 2 * kTile;          // lo phase: d1, d2
  // hi phase: two K blocks per stage: O1 (kb) at 0, O1 (kb+1) at kTile, d0 (kb) at
  // 2 kTile, d0 (kb+1) at 3 kTile, so that a stage feeds four MMAs in both phases
  static constexpr int kStage = 4 * kTile;
  static constexpr int kBarOff = kStages * kStage;
  static constexpr int kTabOff = kBarOff + 256;    // per tile: scale[256], V[256]
  static constexpr int kXOff = kTabOff + 2 * kGroupSlots * 4;
  static constexpr int kXBytes = 2 * kI8BM * 2 * kGroupCols * 4;  // (max, sum) per half
  static constexpr int kTotal = kXOff + kXBytes + 1024;
};

// Epilogue of one tile for one warp (TMEM lane quarter q, column half H: columns
// 128 H .. 128 H + 127 of the tile).  Three passes over TMEM, one exp per element:
//   merge: z = (hi * 2^14 + lo) * scale + V (exact integer sum, one rounding),
//          written over hi; per alignment column jj the maximum m of the own
//          states and the logit of the observed state; then `lo` is released;
//   B:     e = exp(z - m) written over z, s = sum e;
//          (m, s) exchanged with the partner warp (same rows, other half):
//          M = max(m, m'), S = s exp(m - M) + s' exp(m' - M) (same order in both
//          halves), lse = M + log S;
//   C:     P = e * exp(m - M) / S, R = w (P - onehot) as its three digits.
// G: the slot groups of the tile (one group = one tile, G::kSlots columns, half
// of them per warp).  REGS: the merged logits leave both accumulators during the
// merge -- the half's first 32-column chunk into a TMEM stash that no MMA writes
// (t_stash), the other chunks into registers -- and the arrival on `lo_bar` after
// the merge then releases both accumulators, so that the next tile's MMAs run
// during passes B and C.  TILED: the digits of R go to the backward's tiled
// storage (i8_bwd_tile_offset) instead of row-major Npad x S.
// hi * 2^14 + lo, rounded once to float.  A row of the one-hot operand holds L
// ones, so |hi| <= 128 L and 0 <= lo <= 16383 L: with L <= kI8NarrowMaxL the exact
// sum lies in [-2^31, 2^31) and the 32-bit conversion (NARROW) gives the float the
// 64-bit one gives.
constexpr int kI8NarrowMaxL = 1024;
template <bool NARROW>
__device__ __forceinline__ float i8_merge_digits(uint32_t hi, uint32_t lo) {
  if constexpr (NARROW) {
    return __int2float_rn((int)(hi * 16384u + lo));
  } else {
    return __ll2float_rn((long long)(int)hi * 16384 + (long long)(int)lo);
  }
}

template <class G, int H, bool REGS = false, bool TILED = false, bool NARROW = false>
__device__ __forceinline__ void i8_fwd_epilogue_tile(const I8FwdArgs &args, uint32_t t_hi,
                                                     uint32_t t_lo, const float *tab_scale,
                                                     const float *tab_v, float *xbuf, int q,
                                                     int lane, int n, int t, long long part,
                                                     uint32_t lo_bar, uint32_t t_stash = 0) {
  constexpr int kGroupCols = G::kCols, kGroupUsed = G::kUsed;
  constexpr int kChunks = G::kSlots / 64;  // 32-column chunks per half
  uint32_t zr[REGS ? (kChunks - 1) * 32 : 1];  // REGS: chunks 1.. of the half
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
  float mx[kGroupCols], tg[kGroupCols], se[kGroupCols];
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) { mx[jj] = -INFINITY; tg[jj] = 0.0f; se[jj] = 0.0f; }
  // merge + maxima
  if constexpr (REGS) {
    // 16-column steps: steps 0 and 1 fill the stash, the others the registers
    uint32_t st[32];
#pragma unroll
    for (int c = 0; c < 2 * kChunks; ++c) {
      const int cc = 2 * kChunks * H + c;
      uint32_t vh[16], vl[16];
      __syncwarp();
      tmem_ld16(t_hi + cc * 16, vh);
      tmem_ld16(t_lo + cc * 16, vl);
      tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int col = cc * 16 + i;
        const float z = fmaf(i8_merge_digits<NARROW>(vh[i], vl[i]), tab_scale[col], tab_v[col]);
        if (c < 2) st[c * 16 + i] = __float_as_uint(z);
        else zr[(c - 2) * 16 + i] = __float_as_uint(z);
        if (col < kGroupUsed) {
          const int a = col / kGroupCols, jj = col % kGroupCols;
          mx[jj] = fmaxf(mx[jj], z);
          if (xr[jj] == a) tg[jj] = z;
        }
      }
      if (c == 1) tmem_st32(t_stash, st);
    }
  }
#pragma unroll
  for (int c = 0; c < (REGS ? 0 : kChunks); ++c) {
    const int cc = kChunks * H + c;
    uint32_t vh[32], vl[32];
    __syncwarp();
    tmem_ld32(t_hi + cc * 32, vh);
    tmem_ld32(t_lo + cc * 32, vl);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int col = cc * 32 + i;
      const float z = fmaf(i8_merge_digits<NARROW>(vh[i], vl[i]), tab_scale[col], tab_v[col]);
      vh[i] = __float_as_uint(z);
      if (col < kGroupUsed) {
        const int a = col / kGroupCols, jj = col % kGroupCols;
        mx[jj] = fmaxf(mx[jj], z);
        if (xr[jj] == a) tg[jj] = z;
      }
    }
    tmem_st32(t_hi + cc * 32, vh);
  }
  tmem_wait_st();
  tc_fence_before();
  __syncwarp();
  // the next tile's low phase (REGS: its MMAs) may start
  if (lane == 0) mbar_arrive_cluster(lo_bar);
  // B: e = exp(z - m), sum
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int cc = kChunks * H + c;
    if constexpr (REGS) {
      if (c > 0) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int col = cc * 32 + i;
          if (col < kGroupUsed) {
            const int jj = col % kGroupCols;
            const float e = expf(__uint_as_float(zr[(c - 1) * 32 + i]) - mx[jj]);
            se[jj] += e;
            zr[(c - 1) * 32 + i] = __float_as_uint(e);
          }
        }
        continue;
      }
    }
    uint32_t v[32];
    __syncwarp();
    tmem_ld32(REGS ? t_stash : t_hi + cc * 32, v);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int col = cc * 32 + i;
      if (col < kGroupUsed) {
        const int jj = col % kGroupCols;
        const float e = expf(__uint_as_float(v[i]) - mx[jj]);
        se[jj] += e;
        v[i] = __float_as_uint(e);
      }
    }
    tmem_st32(REGS ? t_stash : t_hi + cc * 32, v);
  }
  float *mine = xbuf + (H * kI8BM + row) * (2 * kGroupCols);
  const float *other = xbuf + ((1 - H) * kI8BM + row) * (2 * kGroupCols);
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) {
    mine[jj] = mx[jj];
    mine[kGroupCols + jj] = se[jj];
  }
  named_bar_sync(pair_bar, 64);
  double floss = 0.0;
  // R * 2^21 = e * cw - [observed] * won, with cw = w exp(m - M) / S * 2^21
  float cw[kGroupCols];
  const float won = live ? wn * args.r_enc : 0.0f;
#pragma unroll
  for (int jj = 0; jj < kGroupCols; ++jj) {
    const float mo = other[jj], so = other[kGroupCols + jj];
    const float M = fmaxf(mx[jj], mo);
    const float fa = expf(mx[jj] - M), fo = expf(mo - M);
    const float S = H == 0 ? se[jj] * fa + so * fo : so * fo + se[jj] * fa;
    const float lse = M + logf(S);
    cw[jj] = xr[jj] >= 0 ? (fa / S) * won : 0.0f;
    if (xr[jj] >= 0 && (xr[jj] * kGroupCols + jj) / (G::kSlots / 2) == H)
      floss += (double)(wn * (lse - tg[jj]));
  }
  tmem_wait_st();
  // C: R = w (P - onehot), three digits per element
  const long long rbase = (long long)n * args.S + (long long)t * G::kSlots;
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int cc = kChunks * H + c;
    uint32_t vbuf[32];
    if (!REGS || c == 0) {
      __syncwarp();
      tmem_ld32(REGS ? t_stash : t_hi + cc * 32, vbuf);
      tmem_wait_ld();
    }
    auto v = [&](int i) -> uint32_t {
      if constexpr (REGS) return c == 0 ? vbuf[i] : zr[(c - 1) * 32 + i];
      else return vbuf[i];
    };
    uint32_t w0[8], w1[8], w2[8];
#pragma unroll
    for (int e4 = 0; e4 < 8; ++e4) {
      int qv[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int i = e4 * 4 + e;
        const int col = cc * 32 + i;
        float t = 0.0f;
        if (col < kGroupUsed) {
          const int a = col / kGroupCols, jj = col % kGroupCols;
          t = fmaf(__uint_as_float(v(i)), cw[jj], xr[jj] == a ? -won : 0.0f);
        }
        // |R| 2^-eR <= 1: only the top of the range needs the clamp (P rounding to 1)
        qv[e] = min(__float2int_rn(t), (1 << kI8FracBits) - 1);
      }
      // byte e of each word = digit of element e: d0 = q >> 14, d1 = (q >> 7) & 127,
      // d2 = q & 127 (two byte permutes per pair, one per word)
      auto pack = [](int b0, int b1, int b2, int b3) {
        return __byte_perm(__byte_perm(b0, b1, 0x0040), __byte_perm(b2, b3, 0x0040), 0x5410);
      };
      w0[e4] = pack(qv[0] >> 14, qv[1] >> 14, qv[2] >> 14, qv[3] >> 14);
      w1[e4] = pack(qv[0] >> 7, qv[1] >> 7, qv[2] >> 7, qv[3] >> 7) & 0x7F7F7F7Fu;
      w2[e4] = pack(qv[0], qv[1], qv[2], qv[3]) & 0x7F7F7F7Fu;
    }
    long long off = rbase + cc * 32;
    if constexpr (TILED) {
      // the 32 slots [s0, s0 + 32) of row n are 16-byte chunks c, c + 1 (c even) of
      // the tile row; swizzled to c ^ m and (c ^ m) ^ 1, m = n & 7: one aligned
      // 32-byte pair, its halves exchanged when m is odd
      const int s0 = t * G::kSlots + cc * 32;
      const int m = n & 7, c = (s0 & 127) >> 4;
      off = ((long long)(s0 >> 7) * (args.Npad >> 5) + (n >> 5)) * 4096 + (n & 31) * 128 +
            (((c ^ m) & 6) << 4);
      if (m & 1) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          uint32_t v = w0[i]; w0[i] = w0[i + 4]; w0[i + 4] = v;
          v = w1[i]; w1[i] = w1[i + 4]; w1[i + 4] = v;
          v = w2[i]; w2[i] = w2[i + 4]; w2[i + 4] = v;
        }
      }
    }
    st_global_v8(args.r[0] + off, w0);
    st_global_v8(args.r[1] + off, w1);
    st_global_v8(args.r[2] + off, w2);
  }
  for (int o = 16; o > 0; o >>= 1) floss += __shfl_xor_sync(0xffffffffu, floss, o);
  if (lane == 0) args.part_f[part * 8 + H * 4 + q] = floss;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kI8Threads, 1)
    i8_forward_kernel(const __grid_constant__ I8FwdMaps maps, I8FwdArgs args) {
  using SM = I8FwdSmem;
  constexpr int kStages = SM::kStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = i8_align1024(smem_raw);
  // full[] and the *_empty barriers are used in the leader only; empty[] and
  // acc_full in both CTAs (the leader's commits reach both)
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + SM::kBarOff);
  uint64_t *empty = full + kStages;
  uint64_t *acc_full = empty + kStages;
  uint64_t *lo_empty = acc_full + 1;
  uint64_t *hi_empty = lo_empty + 1;
  uint64_t *drain = hi_empty + 1;
  // a barrier that no thread ever arrives on: the epilogue waits on it instead
  // of on acc_full when a test asks for a wait that runs out (acc_wait_cycles)
  uint64_t *never = drain + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(never + 1);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
  float *tab_scale = reinterpret_cast<float *>(smem + SM::kTabOff);
  float *tab_v = tab_scale + kGroupSlots;
  float *xbuf = reinterpret_cast<float *>(smem + SM::kXOff);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int n_tiles = args.m_tiles * args.T;
  const int k_blocks = args.S / kI8FwdBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(acc_full, 1);
    mbar_init(lo_empty, 16);
    mbar_init(hi_empty, 16);
    mbar_init(drain, 1);
    mbar_init(never, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&maps.a1);
    prefetch_tmap(&maps.a128);
    for (int i = 0; i < 3; ++i) prefetch_tmap(&maps.b[i]);
  }
  if (warp == 1) { tmem_alloc_pair(tmem_slot, 512); tmem_relinquish_pair(); }
  tc_fence_before();
  cluster_sync();
  tc_fence_after();
  // the prologue above overlaps the previous kernel's tail; its outputs from here
  griddep_launch();
  griddep_wait();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t t_hi = tmem_base, t_lo = tmem_base + kI8BN;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer (both CTAs), in the MMA's order
      uint32_t it = 0;
      bool ok = true;
      for (int tile = pair; tile < n_tiles && ok && !i8_aborted(abort_flag); tile += npairs) {
        const int m = tile % args.m_tiles, t = tile / args.m_tiles;
        const int row0 = m * kI8PairM + (int)rank * kI8BM;
        const int col0 = t * kI8BN + (int)rank * kI8HalfN;
        for (int phase = 0; phase < 2 && ok; ++phase) {  // 0: low digits, 1: high digit
          for (int kb = 0; kb < k_blocks; kb += (phase == 0 ? 1 : 2), ++it) {
            const int stage = it % kStages;
            const uint32_t round = it / kStages;
            if (!mbar_wait(&empty[stage], (round & 1) ^ 1)) {
              i8_record_error(args.status, kErrFwdTimeout, abort_flag);
              ok = false;
              break;
            }
            uint8_t *st = smem + stage * SM::kStage;
            const uint32_t fb = mapa_shared(smem_u32(&full[stage]), 0);
            const int kx = kb * kI8FwdBK;
            if (phase == 0) {
              if (rank == 0) mbar_arrive_expect_tx(&full[stage], 2 * 4 * SM::kTile);
              tma_load_2d_pair(st + SM::kOffA1, &maps.a1, fb, kx, row0);
              tma_load_2d_pair(st + SM::kOffA128, &maps.a128, fb, kx, row0);
              tma_load_2d_pair(st + SM::kOffB, &maps.b[1], fb, col0, kx);
              tma_load_2d_pair(st + SM::kOffB + SM::kTile, &maps.b[2], fb, col0, kx);
            } else {
              if (rank == 0) mbar_arrive_expect_tx(&full[stage], 2 * 4 * SM::kTile);
              tma_load_2d_pair(st, &maps.a1, fb, kx, row0);
              tma_load_2d_pair(st + SM::kTile, &maps.a1, fb, kx + kI8FwdBK, row0);
              tma_load_2d_pair(st + 2 * SM::kTile, &maps.b[0], fb, col0, kx);
              tma_load_2d_pair(st + 3 * SM::kTile, &maps.b[0], fb, col0, kx + kI8FwdBK);
            }
          }
        }
      }
      const uint32_t issued = it;
      for (uint32_t r = (issued > kStages ? issued - kStages : 0); r < issued; ++r) {
        const bool w = rank == 0 ? mbar_wait(&full[r % kStages], (r / kStages) & 1)
                                 : mbar_wait(&empty[r % kStages], (r / kStages) & 1);
        if (!w) {
          i8_record_error(args.status, kErrFwdTimeout, abort_flag);
          break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---------------- MMA issuer (leader): 256 x 256 x 32 pair MMAs, u8 x s8 -> s32
      constexpr uint32_t idesc = idesc_i8_s32(kI8PairM, kI8BN, 0, 1, 0, 1);
      uint32_t it = 0;
      int local = 0;
      bool ok = true;
      for (int tile = pair; tile < n_tiles && ok && !i8_aborted(abort_flag);
           tile += npairs, ++local) {
        const uint32_t wpar = (local & 1) ^ 1;
        for (int phase = 0; phase < 2 && ok; ++phase) {
          if (!mbar_wait(phase == 0 ? lo_empty : hi_empty, wpar)) {
            i8_record_error(args.status, kErrFwdTimeout, abort_flag);
            ok = false;
            break;
          }
          tc_fence_after();
          for (int kb = 0; kb < k_blocks; kb += (phase == 0 ? 1 : 2), ++it) {
            const int stage = it % kStages;
            const uint32_t round = it / kStages;
            if (!mbar_wait(&full[stage], round & 1)) {
              i8_record_error(args.status, kErrFwdTimeout, abort_flag);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t s0 = smem_u32(smem + stage * SM::kStage);
#pragma unroll
            for (int k32 = 0; k32 < kI8FwdBK / 32; ++k32) {
              if (phase == 0) {
                const uint64_t a1 = sdesc_sw64(s0 + SM::kOffA1 + k32 * 32, 16, 512);
                const uint64_t a128 = sdesc_sw64(s0 + SM::kOffA128 + k32 * 32, 16, 512);
                const uint64_t bA = sdesc_sw128(s0 + SM::kOffB + k32 * 32 * 128, SM::kTile, 1024);
                const uint64_t bB =
                    sdesc_sw128(s0 + SM::kOffB + SM::kTile + k32 * 32 * 128, SM::kTile, 1024);
                umma_i8_pair(t_lo, a128, bA, idesc, (kb | k32) != 0);
                umma_i8_pair(t_lo, a1, bB, idesc, 1);
              } else {
#pragma unroll
                for (int sub = 0; sub < 2; ++sub) {
                  const uint64_t a1 = sdesc_sw64(s0 + sub * SM::kTile + k32 * 32, 16, 512);
                  const uint64_t b0 = sdesc_sw128(s0 + (2 + sub) * SM::kTile + k32 * 32 * 128,
                                                  SM::kTile, 1024);
                  umma_i8_pair(t_hi, a1, b0, idesc, (kb | sub | k32) != 0);
                }
              }
            }
            umma_commit_pair(&empty[stage], 0x3);
          }
        }
        if (ok) umma_commit_pair(acc_full, 0x3);
      }
      umma_commit_pair(drain, 0x1);
      if (!mbar_wait(drain, 0)) i8_record_error(args.status, kErrFwdTimeout, abort_flag);
    }
  } else {
    // ---------------- epilogue (both CTAs): 8 warps, lane quarter q, column half
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int ethr = threadIdx.x - 64;
    const int L = args.L;
    const uint32_t lo_bar = mapa_shared(smem_u32(lo_empty), 0);
    const uint32_t hi_bar = mapa_shared(smem_u32(hi_empty), 0);

    int local = 0;
    for (int tile = pair; tile < n_tiles; tile += npairs, ++local) {
      // all eight warps finished the previous tile (tables free) and saw no abort
      if (named_bar_or(1, 256, i8_aborted(abort_flag))) break;
      const int m = tile % args.m_tiles, t = tile / args.m_tiles;
      {
        // slot tables of this tile: merge scale 2^(e - 21) and the single field V
        const int r = ethr;
        float sc = 0.0f, vv = 0.0f;
        if (r < kGroupUsed) {
          const int a = r / kGroupCols, j = t * kGroupCols + r % kGroupCols;
          if (j < L) {
            sc = pow2f(col_exponent(args.colmax[a * L + j]) - kI8FracBits);
            if (a < kQ - 1) vv = args.x1[a * L + j];
          }
        }
        tab_scale[r] = sc;
        tab_v[r] = vv;
      }
      named_bar_sync(1, 256);
      const int n = m * kI8PairM + (int)rank * kI8BM + q * 32 + lane;
      // (with acc_wait_cycles set, a wait that runs out by design: see `never`)
      const bool ok = args.acc_wait_cycles > 0 ? mbar_wait(never, 0, args.acc_wait_cycles)
                                               : mbar_wait(acc_full, local & 1);
      if (__any_sync(0xffffffffu, !ok)) {
        if (lane == 0) i8_record_error(args.status, kErrFwdTimeout, abort_flag);
        continue;
      }
      tc_fence_after();
      const uint32_t lq = (uint32_t)(q * 32) << 16;
      const long long part = (long long)tile * 2 + rank;
      const bool narrow = L <= kI8NarrowMaxL;
      if (half == 0 && narrow)
        i8_fwd_epilogue_tile<Groups256, 0, false, false, true>(args, t_hi + lq, t_lo + lq, tab_scale,
                                                           tab_v, xbuf, q, lane, n, t, part, lo_bar);
      else if (half == 0)
        i8_fwd_epilogue_tile<Groups256, 0>(args, t_hi + lq, t_lo + lq, tab_scale, tab_v, xbuf, q, lane, n, t,
                                part, lo_bar);
      else if (narrow)
        i8_fwd_epilogue_tile<Groups256, 1, false, false, true>(args, t_hi + lq, t_lo + lq, tab_scale,
                                                           tab_v, xbuf, q, lane, n, t, part, lo_bar);
      else
        i8_fwd_epilogue_tile<Groups256, 1>(args, t_hi + lq, t_lo + lq, tab_scale, tab_v, xbuf, q, lane, n, t,
                                part, lo_bar);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(hi_bar);
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

// ---------------------------------------------------------------- sparse forward
// CCM_PATH_TC_I8SP.  The one-hot operand with its K order changed to
// k' = l * 21 + q (alignment column major): any four consecutive k' span at most
// two alignment columns, and a row has exactly one 1 per column, so every group
// of four holds at most two ones -- the 2:4 structured sparsity that
// tcgen05.mma.sp runs at twice the dense rate.  A is stored compressed (the two
// kept values of each group) with 4 bits of metadata per group: the kept
// positions i0 < i1 in bits 0-1 and 2-3, group c of a row in nibble c of the
// row's metadata bytes (low nibble first).  A group with a single 1 keeps it
// with a zero partner, an empty group keeps (0, 1) with two zeros.
// One thread per metadata byte (two groups, eight logical K).
__global__ void i8sp_onehot_kernel(const uint8_t *__restrict__ msa, uint32_t *__restrict__ ac1,
                                   uint32_t *__restrict__ ac128, uint8_t *__restrict__ meta,
                                   int L, int N, int KP, int Npad) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = KP / 8;
  if (idx >= (long long)Npad * nb) return;
  const int n = (int)(idx / nb), byte = (int)(idx % nb);
  uint32_t vals = 0, m = 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int c = 2 * byte + h;
    int pos[2] = {0, 0}, cnt = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int k = 4 * c + p;
      if (n < N && k < kQ * L && msa[(long long)n * L + k / kQ] == k % kQ) {
        if (cnt < 2) pos[cnt] = p;
        ++cnt;
      }
    }
    int i0 = 0, i1 = 1, v0 = 0, v1 = 0;
    if (cnt >= 2) {
      i0 = pos[0]; i1 = pos[1]; v0 = 1; v1 = 1;
    } else if (cnt == 1) {
      if (pos[0] < 3) { i0 = pos[0]; i1 = 3; v0 = 1; }
      else { i0 = 2; i1 = 3; v1 = 1; }
    }
    m |= (uint32_t)(i0 | (i1 << 2)) << (4 * h);
    vals |= (uint32_t)(v0 | (v1 << 8)) << (16 * h);
  }
  // compressed row n: KP / 2 bytes, four per metadata byte (one aligned word)
  const int KB = KP / 128;
  meta[i8sp_e_offset(n, byte, KB)] = (uint8_t)m;
  const long long ao = i8sp_a_offset(n, 4 * byte, KB) >> 2;
  ac1[ao] = vals;
  ac128[ao] = vals * 128;  // the same with values 128
}

// As i8_forward_kernel on 256 x 192 tiles (Groups192, nine alignment columns per
// tile), with sparse MMAs (K = 64 logical per instruction).  Per 128 logical K
// the CTA holds A compressed as 128 rows x 64 bytes (64-byte swizzle), the
// metadata as 128 rows x 16 bytes (no swizzle), copied into TMEM by tcgen05.cp
// ahead of the MMAs that read it (the copy and the MMAs issue from one thread and
// execute in order; two metadata slots alternate), and B -- the digits of W with
// rows in the K order k' -- MN-major, 96 columns per CTA as three 32-byte
// swizzled atoms of 128 K rows.  Each of these is one TMA box of the tiled
// storage above (no TMA swizzle: the images are stored swizzled).
// One pass per tile: a stage holds everything one block of 128 logical K needs
// for the three digit products (A x1, A x128, B d0..d2, E; 54 KB), so the one-hot
// operand and its metadata cross L2 once per tile, not once per digit phase; the
// kernel is bound by this L2 -> shared-memory operand stream.  The epilogue takes
// the merged logits out of both accumulators during its merge pass (into TMEM
// columns [192, 256) and registers) and releases them at once, so the next tile's
// MMAs overlap the softmax and the R digits.
// TMEM: hi = [0, 192), epilogue stash = [192, 256), lo = [256, 448), metadata
// slots at 448 and 452.
constexpr int kSpBN = Groups192::kSlots, kSpBK = 128;

struct I8SpSmem {
  static constexpr int kStages = 3;
  static constexpr int kA = kI8BM * kSpBK / 2;  // 8 KB
  static constexpr int kAtom = kSpBK * 32;      // 4 KB: 128 K rows x 32 columns
  static constexpr int kB = 3 * kAtom;          // 12 KB: 96 columns
  static constexpr int kE = kI8BM * kSpBK / 8;  // 2 KB
  // one K block of 128 logical K for all three digit products:
  // A x1 | A x128 | B d0 | B d1 | B d2 | E
  static constexpr int kOffA1 = 0, kOffA128 = kA, kOffB = 2 * kA, kOffE = 2 * kA + 3 * kB;
  static constexpr int kStage = kOffE + kE;
  static constexpr int kBarOff = kStages * kStage;
  static constexpr int kTabOff = kBarOff + 256;  // per tile: scale[192], V[192]
  static constexpr int kXOff = kTabOff + 2 * kSpBN * 4;
  static constexpr int kXBytes = 2 * kI8BM * 2 * Groups192::kCols * 4;
  static constexpr int kTotal = kXOff + kXBytes + 1024;
};

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kI8Threads, 1)
    i8sp_forward_kernel(const __grid_constant__ I8SpMaps maps, I8FwdArgs args) {
  using SM = I8SpSmem;
  constexpr int kStages = SM::kStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = i8_align1024(smem_raw);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + SM::kBarOff);
  uint64_t *empty = full + kStages;
  uint64_t *acc_full = empty + kStages;
  uint64_t *acc_empty = acc_full + 1;
  uint64_t *drain = acc_empty + 1;
  // a barrier that no thread ever arrives on: the epilogue waits on it instead
  // of on acc_full when a test asks for a wait that runs out (acc_wait_cycles)
  uint64_t *never = drain + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(never + 1);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
  float *tab_scale = reinterpret_cast<float *>(smem + SM::kTabOff);
  float *tab_v = tab_scale + kSpBN;
  float *xbuf = reinterpret_cast<float *>(smem + SM::kXOff);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int n_tiles = args.m_tiles * args.T;
  const int k_blocks = args.KP / kSpBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 16);
    mbar_init(drain, 1);
    mbar_init(never, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&maps.a1);
    prefetch_tmap(&maps.a128);
    prefetch_tmap(&maps.e);
    for (int i = 0; i < 3; ++i) prefetch_tmap(&maps.b[i]);
  }
  if (warp == 1) { tmem_alloc_pair(tmem_slot, 512); tmem_relinquish_pair(); }
  tc_fence_before();
  cluster_sync();
  tc_fence_after();
  // the prologue above overlaps the previous kernel's tail; its outputs from here
  griddep_launch();
  griddep_wait();
  const uint32_t tmem_base = *tmem_slot;
  // TMEM: hi [0, 192), the epilogue's stash [192, 256), lo [256, 448), metadata 448 / 452
  const uint32_t t_hi = tmem_base, t_lo = tmem_base + 256, t_e = tmem_base + 448;
  const uint32_t t_stash = tmem_base + kSpBN;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer (both CTAs), in the MMA's order
      uint32_t it = 0;
      bool ok = true;
      for (int tile = pair; tile < n_tiles && ok && !i8_aborted(abort_flag); tile += npairs) {
        const int m = tile % args.m_tiles, t = tile / args.m_tiles;
        // tile rows of the tiled operands (256-byte rows): A 32, E 8, B 48 per K block
        const int m128 = 2 * m + (int)rank, tb = 2 * t + (int)rank;
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int stage = it % kStages;
          const uint32_t round = it / kStages;
          if (!mbar_wait(&empty[stage], (round & 1) ^ 1)) {
            i8_record_error(args.status, kErrFwdTimeout, abort_flag);
            ok = false;
            break;
          }
          uint8_t *st = smem + stage * SM::kStage;
          const uint32_t fb = mapa_shared(smem_u32(&full[stage]), 0);
          const int ya = (m128 * k_blocks + kb) * 32, yb = (tb * k_blocks + kb) * 48;
          if (rank == 0) mbar_arrive_expect_tx(&full[stage], 2 * SM::kStage);
          tma_load_2d_pair(st + SM::kOffA1, &maps.a1, fb, 0, ya);
          tma_load_2d_pair(st + SM::kOffA128, &maps.a128, fb, 0, ya);
          for (int i = 0; i < 3; ++i)
            tma_load_2d_pair(st + SM::kOffB + i * SM::kB, &maps.b[i], fb, 0, yb);
          tma_load_2d_pair(st + SM::kOffE, &maps.e, fb, 0, (m128 * k_blocks + kb) * 8);
        }
      }
      const uint32_t issued = it;
      for (uint32_t r = (issued > kStages ? issued - kStages : 0); r < issued; ++r) {
        const bool w = rank == 0 ? mbar_wait(&full[r % kStages], (r / kStages) & 1)
                                 : mbar_wait(&empty[r % kStages], (r / kStages) & 1);
        if (!w) {
          i8_record_error(args.status, kErrFwdTimeout, abort_flag);
          break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---------------- MMA issuer (leader): 256 x 192 x 64 (logical) sparse pair MMAs
      constexpr uint32_t idesc = idesc_i8_s32(kI8PairM, kSpBN, 0, 1, 0, 1) | kIdescSparse;
      uint32_t it = 0, ecopies = 0;
      int local = 0;
      bool ok = true;
      for (int tile = pair; tile < n_tiles && ok && !i8_aborted(abort_flag);
           tile += npairs, ++local) {
        // both accumulators free: the previous tile's epilogue finished its merge
        if (!mbar_wait(acc_empty, (local & 1) ^ 1)) {
          i8_record_error(args.status, kErrFwdTimeout, abort_flag);
          break;
        }
        tc_fence_after();
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int stage = it % kStages;
          const uint32_t round = it / kStages;
          if (!mbar_wait(&full[stage], round & 1)) {
            i8_record_error(args.status, kErrFwdTimeout, abort_flag);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t s0 = smem_u32(smem + stage * SM::kStage);
          const uint32_t te = t_e + 4 * (ecopies++ & 1);
          tmem_cp_pair_128x128b(te, sdesc_noswz(s0 + SM::kOffE, 2048, 128));
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const uint64_t a1 = sdesc_sw64(s0 + SM::kOffA1 + k * 32, 16, 512);
            const uint64_t a128 = sdesc_sw64(s0 + SM::kOffA128 + k * 32, 16, 512);
            const uint64_t b0 = sdesc_sw32(s0 + SM::kOffB + k * 2048, SM::kAtom, 256);
            const uint64_t b1 = sdesc_sw32(s0 + SM::kOffB + SM::kB + k * 2048, SM::kAtom, 256);
            const uint64_t b2 = sdesc_sw32(s0 + SM::kOffB + 2 * SM::kB + k * 2048, SM::kAtom, 256);
            const uint32_t first = (kb | k) != 0;
            umma_i8sp_pair(t_hi, a1, b0, idesc, te + 2 * k, first);    // O1 x d0
            umma_i8sp_pair(t_lo, a128, b1, idesc, te + 2 * k, first);  // O128 x d1
            umma_i8sp_pair(t_lo, a1, b2, idesc, te + 2 * k, 1);        // O1 x d2
          }
          umma_commit_pair(&empty[stage], 0x3);
        }
        if (ok) umma_commit_pair(acc_full, 0x3);
      }
      umma_commit_pair(drain, 0x1);
      if (!mbar_wait(drain, 0)) i8_record_error(args.status, kErrFwdTimeout, abort_flag);
    }
  } else {
    // ---------------- epilogue (both CTAs): 8 warps, lane quarter q, column half
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int ethr = threadIdx.x - 64;
    const int L = args.L;
    const uint32_t empty_bar = mapa_shared(smem_u32(acc_empty), 0);

    int local = 0;
    for (int tile = pair; tile < n_tiles; tile += npairs, ++local) {
      if (named_bar_or(1, 256, i8_aborted(abort_flag))) break;
      const int m = tile % args.m_tiles, t = tile / args.m_tiles;
      if (ethr < kSpBN) {
        const int r = ethr;
        float sc = 0.0f, vv = 0.0f;
        if (r < Groups192::kUsed) {
          const int a = r / Groups192::kCols, j = t * Groups192::kCols + r % Groups192::kCols;
          if (j < L) {
            sc = pow2f(col_exponent(args.colmax[a * L + j]) - kI8FracBits);
            if (a < kQ - 1) vv = args.x1[a * L + j];
          }
        }
        tab_scale[r] = sc;
        tab_v[r] = vv;
      }
      named_bar_sync(1, 256);
      const int n = m * kI8PairM + (int)rank * kI8BM + q * 32 + lane;
      // (with acc_wait_cycles set, a wait that runs out by design: see `never`)
      const bool ok = args.acc_wait_cycles > 0 ? mbar_wait(never, 0, args.acc_wait_cycles)
                                               : mbar_wait(acc_full, local & 1);
      if (__any_sync(0xffffffffu, !ok)) {
        if (lane == 0) i8_record_error(args.status, kErrFwdTimeout, abort_flag);
        continue;
      }
      tc_fence_after();
      const uint32_t lq = (uint32_t)(q * 32) << 16;
      const long long part = (long long)tile * 2 + rank;
      // both accumulators are released inside, right after the merge
      const bool narrow = L <= kI8NarrowMaxL;
      if (half == 0 && narrow)
        i8_fwd_epilogue_tile<Groups192, 0, true, true, true>(args, t_hi + lq, t_lo + lq, tab_scale,
                                                       tab_v, xbuf, q, lane, n, t, part, empty_bar,
                                                       t_stash + lq);
      else if (half == 0)
        i8_fwd_epilogue_tile<Groups192, 0, true, true>(args, t_hi + lq, t_lo + lq, tab_scale, tab_v,
                                                 xbuf, q, lane, n, t, part, empty_bar,
                                                 t_stash + lq);
      else if (narrow)
        i8_fwd_epilogue_tile<Groups192, 1, true, true, true>(args, t_hi + lq, t_lo + lq, tab_scale,
                                                       tab_v, xbuf, q, lane, n, t, part, empty_bar,
                                                       t_stash + 32 + lq);
      else
        i8_fwd_epilogue_tile<Groups192, 1, true, true>(args, t_hi + lq, t_lo + lq, tab_scale, tab_v,
                                                 xbuf, q, lane, n, t, part, empty_bar,
                                                 t_stash + 32 + lq);
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

}  // namespace ccm

namespace ccm {

// ---------------------------------------------------------------- backward
// Pair tiles of 256 x 256 slots (P <= Q for the symmetric gradient) as in
// tc_backward.  Per K step of 32 rows, with the digits r0..r2 of R and the two
// one-hot operands O1, O128 (both sides MN-major, 8-bit):
//   hi += O1_P^T r0_Q + r0_P^T O1_Q
//   lo += O128_P^T r1_Q + O1_P^T r2_Q + r1_P^T O128_Q + r2_P^T O1_Q
// (SYM = false: the O^T R products only).  The sums are exact in s32 for up to
// 32768 rows; longer alignments are cut into K chunks of that length, each merged
// as (hi * 2^14 + lo) * 2^-21 (exact, one rounding) into FP32 registers.  The
// output phase is tc_backward's: one atomic add per g2 element.
constexpr int kI8BwdBK = 32;
constexpr int kI8BwdChunkKB = 1024;  // 32768 rows: |lo| <= 32768 * 2 * 16383 < 2^31

struct I8BwdSmem {
  static constexpr int kStages = 5;
  static constexpr int kTile = 128 * kI8BwdBK;  // 4 KB: 128 slots x 32 rows, 8-bit
  // P side: O1, O128, r0, r1, r2 (this CTA's 128 P slots); Q side: the same (its 128 Q slots)
  static constexpr int kStage = 10 * kTile;
  static constexpr int kBarOff = kStages * kStage;
  static constexpr int kTOff = kBarOff + 256;
  static constexpr int kTBytes = 8 * 32 * 9 * 4;
  static constexpr int kTotal = kTOff + kTBytes + 1024;
};

// TILED: the operands are in the tiled storage of i8_bwd_tile_offset (the sparse
// path); else row-major Npad x S.  The shared-memory images are the same.
template <bool SYM, class G, bool TILED>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kI8Threads, 1)
    i8_backward_kernel(const __grid_constant__ I8BwdMaps maps, BwdArgs args) {
  using SM = I8BwdSmem;
  constexpr int kStages = SM::kStages;
  constexpr int kBN = 256, kHalfN = 128, kPairM = 256, kBM = 128;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = i8_align1024(smem_raw);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + SM::kBarOff);
  uint64_t *empty = full + kStages;
  uint64_t *acc_full = empty + kStages;
  uint64_t *acc_empty = acc_full + 1;
  uint64_t *drain = acc_empty + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int n_tiles = args.n_tiles;
  const int k_blocks = args.Npad / kI8BwdBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 16);
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&maps.o1);
    prefetch_tmap(&maps.o128);
    for (int i = 0; i < 3; ++i) prefetch_tmap(&maps.r[i]);
  }
  if (warp == 1) { tmem_alloc_pair(tmem_slot, 512); tmem_relinquish_pair(); }
  tc_fence_before();
  cluster_sync();
  tc_fence_after();
  // the prologue above overlaps the previous kernel's tail; its outputs from here
  griddep_launch();
  griddep_wait();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t t_hi = tmem_base, t_lo = tmem_base + kBN;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      bool ok = true;
      for (int tile = pair; tile < n_tiles && ok && !i8_aborted(abort_flag); tile += npairs) {
        const int2 pq = args.tiles[tile];
        const int xP = pq.x * kPairM + (int)rank * kBM;
        const int xQ = pq.y * kBN + (int)rank * kHalfN;
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int stage = it % kStages;
          const uint32_t round = it / kStages;
          if (!mbar_wait(&empty[stage], (round & 1) ^ 1)) {
            i8_record_error(args.status, kErrBwdTimeout, abort_flag);
            ok = false;
            break;
          }
          uint8_t *st = smem + stage * SM::kStage;
          // row-major: box (slot x, row y); tiled: the 4 KB tile of (slot block,
          // K block) is 16 rows of 256 bytes at row 16 * (sb * KB + kb)
          const int y = kb * kI8BwdBK;
          const int xp = TILED ? 0 : xP, xq = TILED ? 0 : xQ;
          const int yp = TILED ? ((xP >> 7) * k_blocks + kb) * 16 : y;
          const int yq = TILED ? ((xQ >> 7) * k_blocks + kb) * 16 : y;
          const uint32_t fb = mapa_shared(smem_u32(&full[stage]), 0);
          if (rank == 0) mbar_arrive_expect_tx(&full[stage], 2 * (SYM ? 10 : 5) * SM::kTile);
          tma_load_2d_pair(st + 0 * SM::kTile, &maps.o1, fb, xp, yp);
          tma_load_2d_pair(st + 1 * SM::kTile, &maps.o128, fb, xp, yp);
          if (SYM)
            for (int i = 0; i < 3; ++i)
              tma_load_2d_pair(st + (2 + i) * SM::kTile, &maps.r[i], fb, xp, yp);
          if (SYM) {
            tma_load_2d_pair(st + 5 * SM::kTile, &maps.o1, fb, xq, yq);
            tma_load_2d_pair(st + 6 * SM::kTile, &maps.o128, fb, xq, yq);
          }
          for (int i = 0; i < 3; ++i)
            tma_load_2d_pair(st + (7 + i) * SM::kTile, &maps.r[i], fb, xq, yq);
        }
      }
      const uint32_t issued = it;
      for (uint32_t r = (issued > (uint32_t)kStages ? issued - kStages : 0); r < issued; ++r) {
        const bool w = rank == 0 ? mbar_wait(&full[r % kStages], (r / kStages) & 1)
                                 : mbar_wait(&empty[r % kStages], (r / kStages) & 1);
        if (!w) {
          i8_record_error(args.status, kErrBwdTimeout, abort_flag);
          break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      constexpr uint32_t id_us = idesc_i8_s32(kPairM, kBN, 0, 1, 1, 1);  // A = one-hot, B = R
      constexpr uint32_t id_su = idesc_i8_s32(kPairM, kBN, 1, 0, 1, 1);  // A = R, B = one-hot
      uint32_t it = 0, chunk = 0;
      bool ok = true;
      for (int tile = pair; tile < n_tiles && ok && !i8_aborted(abort_flag); tile += npairs) {
        for (int kb0 = 0; kb0 < k_blocks && ok; kb0 += kI8BwdChunkKB, ++chunk) {
          if (!mbar_wait(acc_empty, (chunk & 1) ^ 1)) {
            i8_record_error(args.status, kErrBwdTimeout, abort_flag);
            ok = false;
            break;
          }
          tc_fence_after();
          const int kb1 = min(kb0 + kI8BwdChunkKB, k_blocks);
          for (int kb = kb0; kb < kb1; ++kb, ++it) {
            const int stage = it % kStages;
            const uint32_t round = it / kStages;
            if (!mbar_wait(&full[stage], round & 1)) {
              i8_record_error(args.status, kErrBwdTimeout, abort_flag);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t s0 = smem_u32(smem + stage * SM::kStage);
            auto d = [&](int i) { return sdesc_sw128(s0 + i * SM::kTile, SM::kTile, 1024); };
            const uint32_t first = kb == kb0 ? 0u : 1u;
            umma_i8_pair(t_hi, d(0), d(7), id_us, first);  // O1_P^T r0_Q
            umma_i8_pair(t_lo, d(1), d(8), id_us, first);  // O128_P^T r1_Q
            umma_i8_pair(t_lo, d(0), d(9), id_us, 1);      // O1_P^T r2_Q
            if (SYM) {
              umma_i8_pair(t_hi, d(2), d(5), id_su, 1);    // r0_P^T O1_Q
              umma_i8_pair(t_lo, d(3), d(6), id_su, 1);    // r1_P^T O128_Q
              umma_i8_pair(t_lo, d(4), d(5), id_su, 1);    // r2_P^T O1_Q
            }
            umma_commit_pair(&empty[stage], 0x3);
          }
          if (!ok) break;
          umma_commit_pair(acc_full, 0x3);
        }
      }
      umma_commit_pair(drain, 0x1);
      if (!mbar_wait(drain, 0)) i8_record_error(args.status, kErrBwdTimeout, abort_flag);
    }
  } else {
    // Epilogue: as tc_backward, with each K chunk merged from the two integer
    // accumulators (16 columns per TMEM load) into FP32 registers.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int L = args.L;
    float *__restrict__ g2 = args.g2;
    float *Tb = reinterpret_cast<float *>(smem + SM::kTOff) + (warp - 2) * 32 * 9;
    const float r_dec = args.r_dec;
    const uint32_t empty_bar = mapa_shared(smem_u32(acc_empty), 0);
    uint32_t chunk = 0;
    bool ok = true;
    for (int tile = pair; tile < n_tiles && ok; tile += npairs) {
      float accv[kHalfN];
#pragma unroll
      for (int i = 0; i < kHalfN; ++i) accv[i] = 0.0f;
      for (int kb0 = 0; kb0 < k_blocks; kb0 += kI8BwdChunkKB, ++chunk) {
        const bool w_ok = mbar_wait(acc_full, chunk & 1);
        if (__any_sync(0xffffffffu, !w_ok)) {
          if (lane == 0) i8_record_error(args.status, kErrBwdTimeout, abort_flag);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t col0 = half * kHalfN + ((uint32_t)(q * 32) << 16);
#pragma unroll
        for (int c = 0; c < kHalfN / 16; ++c) {
          uint32_t vh[16], vl[16];
          __syncwarp();
          tmem_ld16(t_hi + col0 + c * 16, vh);
          tmem_ld16(t_lo + col0 + c * 16, vl);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const long long qs = (long long)(int)vh[i] * 16384 + (long long)(int)vl[i];
            // exact 64-bit sum, one rounding to float, exact scaling by 2^(eR - 21)
            accv[c * 16 + i] += __ll2float_rn(qs) * r_dec;
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(empty_bar);
      }
      if (!ok) break;

      const int2 pq = args.tiles[tile];
      const int rowbase = pq.x * kPairM + (int)rank * kBM + q * 32;
      const int s1 = rowbase + lane;
      const int t1 = s1 / G::kSlots, r1 = s1 % G::kSlots;
      const int b = r1 / G::kCols, k = t1 * G::kCols + r1 % G::kCols;
      const bool valid1 = r1 < G::kUsed && k < L;
      const long long colt = (long long)b * L + k;
      // the Q slots of this warp: sQ + i, i < 128 (with 192-slot groups a 256-slot
      // tile half may cross a group boundary: decode each slot on its own)
      const int sQ = pq.y * kBN + half * kHalfN;
#pragma unroll
      for (int cb = 0; cb < kHalfN / 8; ++cb) {
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 8; ++e) Tb[lane * 9 + e] = accv[cb * 8 + e];
        __syncwarp();
        if (SYM) {
#pragma unroll 1
          for (int col = 0; col < 8; ++col) {
            const int s2 = sQ + cb * 8 + col;
            const int t2 = s2 / G::kSlots, r2 = s2 % G::kSlots;
            const int a = r2 / G::kCols, j = t2 * G::kCols + r2 % G::kCols;
            const bool valid2 = r2 < G::kUsed && j < L;
            if (s1 < s2) {
              const float val = Tb[lane * 9 + col];
              if (valid1 && valid2) {
                if (k != j) atomicAdd(g2 + ((long long)a * L + j) * kQPad * L + colt, val);
              } else if (s2 == G::kOnes && valid1 && b < kQ - 1) {
                args.g1d[b * L + k] = val;
              }
            }
          }
        }
        const int col = lane & 7;
        const int s2 = sQ + cb * 8 + col;
        const int t2 = s2 / G::kSlots, r2 = s2 % G::kSlots;
        const int a = r2 / G::kCols, j = t2 * G::kCols + r2 % G::kCols;
        const bool valid2 = r2 < G::kUsed && j < L;
#pragma unroll
        for (int it = 0; it < 8; ++it) {
          const int row = 4 * it + (lane >> 3);
          const int s1r = rowbase + row;
          if (SYM && s1r > s2) continue;
          const float val = Tb[row * 9 + col];
          const int tr = s1r / G::kSlots, rr = s1r % G::kSlots;
          const int br = rr / G::kCols, kr = tr * G::kCols + rr % G::kCols;
          if (rr < G::kUsed && kr < L) {
            if (valid2 && (!SYM || kr != j)) atomicAdd(g2 + x2_index(br, kr, a, j, L), val);
          } else if (s1r == G::kOnes && valid2 && a < kQ - 1) {
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

}  // namespace ccm

namespace ccm {

// ---------------------------------------------------------------- launchers
// Evaluation at d_x, or, with d_s, at d_xt = d_x + alpha d_s (the step is taken
// by the column-max pass, which writes d_xt).  Profile marks: [colmax + prep |
// forward | backward | finalize].
cudaError_t i8_evaluate(ccm_context *c, const float *d_x, float *d_g, const float *d_s,
                        const double *d_alpha, float *d_xt) {
  const int L = c->L;
  const bool step = d_s != nullptr;
  const bool sp = c->path == CCM_PATH_TC_I8SP;
  const float *xe = step ? d_xt : d_x;
  const float *x1 = xe;
  const float *x2 = xe + c->nsp;
  float *g2 = d_g + c->nsp;
  cudaError_t e;

  prof_mark(c);
  if ((e = zero_words(c->d_colmax, (long long)kQ * L, c->stream)) != cudaSuccess) return e;
  constexpr int kRows = 32;
  const int cols = (c->skip_padding ? kQ : kQPad) * L;
  const dim3 cgrid((cols + 255) / 256, (kQ * L + kRows - 1) / kRows + (step ? 1 : 0));
  if (step)
    e = launch_pdl(i8_colmax_kernel<true>, cgrid, dim3(256), 0, c->stream, d_x, d_s, d_alpha, d_xt,
                   c->d_colmax, L, c->nsp, kRows, sp ? 1 : 0, cols);
  else
    e = launch_pdl(i8_colmax_kernel<false>, cgrid, dim3(256), 0, c->stream, d_x,
                   (const float *)nullptr, (const double *)nullptr, (float *)nullptr, c->d_colmax,
                   L, c->nsp, kRows, sp ? 1 : 0, cols);
  if (e != cudaSuccess) return e;
  // per-slot factors after the column maxima, 16-byte aligned for the float4 loads
  float *enc = reinterpret_cast<float *>(c->d_colmax + ((kQ * L + 3) & ~3));
  // W digit rows: S slots (dense forward) or SW slots of 192-slot groups (sparse)
  const int wcols = sp ? c->SW : c->S;
  if (sp)
    e = launch_pdl(i8_scales_kernel<Groups192>, dim3((wcols + 255) / 256), dim3(256), 0, c->stream,
                   (const uint32_t *)c->d_colmax, enc, L, wcols);
  else
    e = launch_pdl(i8_scales_kernel<Groups256>, dim3((wcols + 255) / 256), dim3(256), 0, c->stream,
                   (const uint32_t *)c->d_colmax, enc, L, wcols);
  if (e != cudaSuccess) return e;
  I8PrepArgs pa{};
  for (int i = 0; i < 3; ++i) pa.wdig[i] = c->d_wdig[i];
  pa.colmax = c->d_colmax;
  pa.enc = enc;
  pa.part_reg = c->d_part_reg;
  pa.L = L; pa.S = wcols; pa.KB = c->KP / 128; pa.lambda_pair = c->lambda_pair;
  pa.g2_coef = c->gradient == CCM_GRADIENT_PARTIAL ? 1.0f : 2.0f;
  pa.inv_L = 1.0f / (float)L;
  pa.ncols = cols;
  if (sp)
    e = launch_pdl(i8_prep_kernel<Groups192, true>, dim3(kQ * L), dim3(256), sizeof(float) * wcols,
                   c->stream, x2, g2, pa);
  else
    e = launch_pdl(i8_prep_kernel<Groups256, false>, dim3(kQ * L), dim3(256), sizeof(float) * wcols,
                   c->stream, x2, g2, pa);
  if (e != cudaSuccess) return e;
  prof_mark(c);

  I8FwdArgs fa{};
  fa.msa = c->d_msa; fa.w = c->d_w; fa.x1 = x1; fa.colmax = c->d_colmax;
  for (int i = 0; i < 3; ++i) fa.r[i] = c->d_rdig[i];
  fa.part_f = c->d_part_f; fa.status = c->d_status;
  fa.L = L; fa.N = c->N; fa.S = c->S; fa.T = c->T; fa.Npad = c->Npad;
  fa.m_tiles = c->Npad / kI8PairM;
  fa.KP = c->KP;
  fa.r_enc = pow2_host(kI8FracBits - c->r_exp);
  fa.acc_wait_cycles = c->acc_wait_cycles;
  const int pair_tiles = fa.m_tiles * c->T;
  const int fpairs = pair_tiles < c->fwd_pairs ? pair_tiles : c->fwd_pairs;
  if (sp)
    e = launch_pdl(i8sp_forward_kernel, dim3(2 * fpairs), dim3(kI8Threads), I8SpSmem::kTotal,
                   c->stream, c->i8sp_maps, fa);
  else
    e = launch_pdl(i8_forward_kernel, dim3(2 * fpairs), dim3(kI8Threads), I8FwdSmem::kTotal,
                   c->stream, c->i8fwd_maps, fa);
  if (e != cudaSuccess) return e;
  prof_mark(c);

  BwdArgs ba{};
  ba.x2 = x2; ba.g2 = g2; ba.g1d = c->d_g1d; ba.tiles = c->d_bwd_tiles;
  ba.n_tiles = c->n_bwd_tiles; ba.status = c->d_status; ba.L = L; ba.S = c->S; ba.Npad = c->Npad;
  ba.lambda_pair = c->lambda_pair;
  ba.r_dec = pow2_host(c->r_exp - kI8FracBits);
  const int bpairs = c->n_bwd_tiles < c->bwd_pairs ? c->n_bwd_tiles : c->bwd_pairs;
  const bool sym = c->gradient != CCM_GRADIENT_PARTIAL;
  const dim3 bgrid(2 * bpairs);
  auto bwd = sp && sym ? i8_backward_kernel<true, Groups192, true>
             : sp        ? i8_backward_kernel<false, Groups192, true>
             : sym       ? i8_backward_kernel<true, Groups256, false>
                         : i8_backward_kernel<false, Groups256, false>;
  e = launch_pdl(bwd, bgrid, dim3(kI8Threads), I8BwdSmem::kTotal, c->stream, c->i8bwd_maps, ba);
  if (e != cudaSuccess) return e;
  prof_mark(c);

  if ((e = launch_tc_finalize(c, x1, d_g, 2LL * pair_tiles)) != cudaSuccess) return e;
  prof_mark(c);
  count_launch(c, 7);
  return cudaGetLastError();
}

cudaError_t i8_configure_kernels() {
  cudaError_t e;
  const int kMax = cudaFuncAttributeMaxDynamicSharedMemorySize;
  // the staged row is S floats: up to L = 2688 (the 227 KB per block, less the
  // kernel's static reduction buffer)
  if ((e = cudaFuncSetAttribute(i8_prep_kernel<Groups256, false>, (cudaFuncAttribute)kMax,
                                230000)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(i8_prep_kernel<Groups192, true>, (cudaFuncAttribute)kMax,
                                230000)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(i8_forward_kernel, (cudaFuncAttribute)kMax, I8FwdSmem::kTotal)) !=
          cudaSuccess ||
      (e = cudaFuncSetAttribute(i8sp_forward_kernel, (cudaFuncAttribute)kMax, I8SpSmem::kTotal)) !=
          cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(i8_backward_kernel<true, Groups256, false>, (cudaFuncAttribute)kMax,
                                I8BwdSmem::kTotal)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(i8_backward_kernel<false, Groups256, false>, (cudaFuncAttribute)kMax,
                                I8BwdSmem::kTotal)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(i8_backward_kernel<true, Groups192, true>, (cudaFuncAttribute)kMax,
                                I8BwdSmem::kTotal)) != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(i8_backward_kernel<false, Groups192, true>, (cudaFuncAttribute)kMax,
                              I8BwdSmem::kTotal);
}

cudaError_t i8_forward_max_pairs(int *pairs) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(kI8Threads, 1, 1);
  cfg.dynamicSmemBytes = I8FwdSmem::kTotal;
  *pairs = 0;
  return cudaOccupancyMaxActiveClusters(pairs, i8_forward_kernel, &cfg);
}

cudaError_t i8sp_forward_max_pairs(int *pairs) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(kI8Threads, 1, 1);
  cfg.dynamicSmemBytes = I8SpSmem::kTotal;
  *pairs = 0;
  return cudaOccupancyMaxActiveClusters(pairs, i8sp_forward_kernel, &cfg);
}

cudaError_t i8_backward_max_pairs(int *pairs) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(kI8Threads, 1, 1);
  cfg.dynamicSmemBytes = I8BwdSmem::kTotal;
  *pairs = 0;
  return cudaOccupancyMaxActiveClusters(pairs, i8_backward_kernel<true, Groups256, false>, &cfg);
}

// One-hot operands for a context of the integer paths (Npad x S bytes each), and
// for the sparse path the compressed forward operand with its metadata.
cudaError_t i8_build_onehot(ccm_context *c) {
  const long long total = (long long)c->Npad * c->S;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (c->path != CCM_PATH_TC_I8SP) {
    i8_onehot_kernel<Groups256, false><<<grid, 256, 0, c->stream>>>(c->d_msa, c->d_o1, c->d_o128, c->L,
                                                             c->N, c->S, c->Npad);
    return cudaGetLastError();
  }
  // the sparse path's backward reads its operands from tiled storage
  i8_onehot_kernel<Groups192, true><<<grid, 256, 0, c->stream>>>(c->d_msa, c->d_o1, c->d_o128, c->L,
                                                           c->N, c->S, c->Npad);
  const long long bytes = (long long)c->Npad * (c->KP / 8);
  i8sp_onehot_kernel<<<(unsigned)((bytes + 255) / 256), 256, 0, c->stream>>>(
      c->d_msa, reinterpret_cast<uint32_t *>(c->d_ac1), reinterpret_cast<uint32_t *>(c->d_ac128),
      c->d_meta, c->L, c->N, c->KP, c->Npad);
  return cudaGetLastError();
}

}  // namespace ccm
