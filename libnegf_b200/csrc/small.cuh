// Small-order block operations (n <= 32) for the lock-step FP64 form: one
// CTA per product, one warp per inversion, every problem of a batch in one
// launch.  At these orders
// a product or an inversion is a few microseconds of dependent steps, so a
// CTA working through one point's chain of them (the persistent engine)
// leaves the FP64 pipe idle; a batch of warps, each holding one problem's
// rows in registers, keeps it fed.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace negf {

constexpr int kSmallMax = 32;      // largest order of the one-warp kernels

// C_p = alpha A_p B_p + beta C_p (complex128, column major, n x n) for the
// problems p = map[b] (map null: p = b), b < *count (count null: batch).
// A, B, C: problem p at p * Q complex elements.  beta == 0: C is not read.
// maxabs (optional): max |C_p| (modulus) of the written elements, folded
// into maxabs[p] by atomicMax on the bit pattern (non-negative doubles); a
// NaN or Inf element makes it NaN.  C must not alias A or B.
cudaError_t launch_small_zgemm(int batch, int n, double2 alpha, const double2* A, const double2* B, double2 beta,
                               double2* C, int64_t Q, const int* map, const int* count, double* maxabs,
                               cudaStream_t s);

// X_p = A_p^-1 by Gauss-Jordan elimination with partial pivoting (pivot =
// max |Re|+|Im| over the rows not yet used, the lowest row on a tie: the
// izamax rule of zgetrf) for the same problem selection; info[p] = 0 or the
// 1-based column of the first zero pivot, and status[p] (optional) gets
// singular_code there unless it holds a code already.  X may alias A.
cudaError_t launch_small_zinv(int batch, int n, const double2* A, double2* X, int64_t Q, const int* map,
                              const int* count, int* info, int* status, int singular_code, cudaStream_t s);

// One decimation iteration (src/contselfenergy.F90:271-340) for the points
// of list[], b < *count, in one launch, one CTA per point (Go, Co, Bo
// staged in shared memory once): X = Go Co, C1 = Co X, the CPU convergence
// rule on max|C1| (ok[], ncyc_c[], iteration `it`; the points that go on are
// appended to next[] / *next_count, in no fixed order), and for those
// Self = Bo X, Ao -= Self, Aos -= Self, Y = Go Bo, B1 = Bo Y, Ao -= Co Y; a
// point whose max|C1| is Inf / NaN leaves the list with redo[p] = 1.  P
// bounds the list length.
cudaError_t launch_small_dec(int P, int n, const int* list, const int* count, const double2* Go, const double2* Co,
                             const double2* Bo, double2* C1, double2* B1, double2* Ao, double2* Aos, int64_t Q, int* ok,
                             int* ncyc_c, double tol, int it, int* next, int* next_count, int* redo, cudaStream_t s);

// The residual probe of each inverse X_p of A_p (same problem selection) and
// up to two Newton steps X <- X + X (I - A X) where it shows a loss of
// accuracy (kInvProbeTol); X_p is left untouched where it does not.
// sens (optional): sens[p] = 1 where the probe's condition estimate of A
// exceeds kSensitiveCond (a nearly singular matrix).
cudaError_t launch_small_refine(int batch, int n, const double2* A, double2* X, int64_t Q, const int* map,
                                const int* count, cudaStream_t s, int* sens = nullptr);

}  // namespace negf
