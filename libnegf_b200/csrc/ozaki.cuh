// Complex128 block products on the integer tensor cores (sm_100a tcgen05,
// kind::i8) by an exact-splitting (Ozaki) scheme.
//
// Every real part and imaginary part of a row of A (a column of B) is scaled
// by the same power of two 2^-e so that it lies in (-1, 1), then cut into S
// digits rounded to nearest: x = sum_t d_t 2^(-6-7t) + r, |d_t| <= 64,
// |r| <= 2^(-7S).  The digit matrices are int8; their products accumulate
// exactly in int32 (|sum| <= 8 * 2K * 64^2 < 2^31 for K <= 1024).  The digit
// pairs (t, u), 0-based, with t + u < min(S + 1, 8) are kept, one TMEM
// accumulator per level t + u, and the epilogue rebuilds
// C = 2^(eA_r + eB_c) sum_levels 2^(-12-7 level) acc in FP64.  The result
// carries about 7S bits relative to the row / column scales (S = 7: a few
// units of the rounding of an FP64 product).
//
// Complex: C_re = [Ar | -Ai] [Br ; Bi] and C_im = [Ai | Ar] [Br ; Bi], two
// real products over the concatenated K (the digits of Ar, Ai and -Ai are
// all stored, so the B tiles are shared).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace negf {

constexpr int kOzTileM = 128;       // UMMA M (one CTA)
constexpr int kOzTileN = 128;       // UMMA N (the full-rate width); 4 levels x 128 columns of TMEM
constexpr int kOzKChunk = 32;       // bytes of K per pipeline stage (one 32-byte swizzle row, one MMA K step)
constexpr int kOzStages = 3;
constexpr int kOzMinSlices = 4, kOzMaxSlices = 8;

// Workspace of one batched product (bytes), laid out by ozaki_layout():
// digit planes of A and B, exponents, non-finite flags, an FP64 m x n
// buffer per item for the real part.
struct OzakiLayout {
  int m, n, k, kp, slices, batch;
  size_t qa_off, qb_off, ea_off, eb_off, flag_off, t0_off, total;
};
OzakiLayout ozaki_layout(int batch, int m, int n, int k, int slices);

// C_p = alpha * A_p * B_p + beta * C_p for the problems p = item_map[b],
// b < batch (item_map null: p = b); complex128, column major, element
// strides sA/sB/sC in complex elements.  beta == 0: C is not read.  C may
// alias A or B (the operands are split into the workspace first).  maxabs
// (optional, one double per problem, non-negative, updated with atomicMax on
// its bit pattern): max |C_p| over the stored elements, NaN when one of them
// is NaN or Inf.  status (optional,
// one int per problem): 3 on a non-finite operand (C is NaN), 7 when a
// pipeline wait ran out (C is not written).
cudaError_t launch_ozaki_zgemm(int batch, int m, int n, int k, double2 alpha, const double2* A, int64_t sA,
                               const double2* B, int64_t sB, double2 beta, double2* C, int64_t sC, int slices,
                               void* work, double* maxabs, int* status, cudaStream_t s,
                               const int* item_map = nullptr);

}  // namespace negf
