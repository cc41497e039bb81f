// Index maps shared by the host and the kernels.
//
// Reference layout (include/ccmpred.h:1-17, PADDING on):
//   x = [ V(j,a) at a*L + j (a < 20) | pad to nsingle_padded |
//         W(b,k,a,j) at ((b*L + k)*32 + a)*L + j ]
// so W is a (21L) x (32L) row-major matrix with rows (b,k) and columns (a,j).
//
// Tensor-core layout.  The 21*L (state, column) pairs are permuted into
// "groups" of 12 alignment columns, 256 slots per group:
//   s(q, l) = (l / 12) * 256 + q * 12 + (l % 12)          q < 21, l < L
// Slots 252..255 of every group and slots of columns l >= L are padding.
// One group is exactly one 256-wide MMA tile, so the 21 states of a column
// sit inside one accumulator tile and the softmax over states is done in the
// GEMM epilogue.  Slot 252 of group 0 is the "ones" slot: the one-hot matrix
// holds 1 there for every real row, which makes the symmetric backward GEMM
// also produce the column sums of R, i.e. the single-field gradient.
#pragma once

#include <cstdint>

namespace ccm {

constexpr int kQ = 21;           // states: 20 amino acids + gap (src/sequence.c:10-27)
constexpr int kQPad = 32;        // N_ALPHA_PAD (include/ccmpred.h:5-9)
constexpr int kGroupCols = 12;   // alignment columns per 256-slot group
constexpr int kGroupSlots = 256;
constexpr int kGroupUsed = kQ * kGroupCols;  // 252
constexpr int kOnesSlot = 252;

__host__ __device__ constexpr long long nsingle_of(int L) { return (long long)L * (kQ - 1); }

// src/ccmpred.c:389: nsingle + 32 - nsingle % 32 (a full extra 32 when divisible)
__host__ __device__ constexpr long long nsingle_padded_of(int L) {
  return nsingle_of(L) + kQPad - nsingle_of(L) % kQPad;
}

__host__ __device__ constexpr long long nvar_padded_of(int L) {
  return nsingle_padded_of(L) + (long long)L * L * kQ * kQPad;
}

__host__ __device__ constexpr int n_groups(int L) { return (L + kGroupCols - 1) / kGroupCols; }

__host__ __device__ constexpr int slot_of(int q, int l) {
  return (l / kGroupCols) * kGroupSlots + q * kGroupCols + (l % kGroupCols);
}

// The same permutation with a general group width, as a traits type: COLS
// alignment columns per group of SLOTS slots, s(q, l) = (l / COLS) * SLOTS +
// q * COLS + l % COLS, ones slot q = 21 of group 0 (slot 21 * COLS).
//   Groups256: 12 columns per 256 slots (the layout above).
//   Groups192: 9 columns per 192 slots, for the sparse integer forward, whose
//              two 192-column s32 accumulators leave TMEM columns free for the
//              sparsity metadata (two 256-column ones fill all 512).
template <int COLS, int SLOTS>
struct SlotGroups {
  static constexpr int kCols = COLS;
  static constexpr int kSlots = SLOTS;
  static constexpr int kUsed = kQ * COLS;
  static constexpr int kOnes = kQ * COLS;
  __host__ __device__ static constexpr int groups(int L) { return (L + COLS - 1) / COLS; }
  __host__ __device__ static constexpr int slot_of(int q, int l) {
    return (l / COLS) * SLOTS + q * COLS + (l % COLS);
  }
};
using Groups256 = SlotGroups<kGroupCols, kGroupSlots>;
using Groups192 = SlotGroups<9, 192>;

__host__ __device__ constexpr long long x2_index(int b, int k, int a, int j, int L) {
  return (((long long)b * L + k) * kQPad + a) * L + j;
}

}  // namespace ccm
