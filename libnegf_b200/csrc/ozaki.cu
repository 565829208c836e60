// Complex128 block products on the integer tensor cores of sm_100a: an exact
// int8 splitting of the operands (see ozaki.cuh), tcgen05.mma kind::i8 with
// the int32 accumulators in tensor memory, operand tiles staged by TMA.
//
// One product is three launches on the caller's stream:
//   k_split_rows  A -> int8 digit planes of Ar, Ai, -Ai (K contiguous) and a
//                 power-of-two exponent per row;
//   k_split_cols  B -> digit planes of Br, Bi and an exponent per column;
//   k_ozaki       persistent CTAs over 128 x 128 tiles of C.  Per tile four
//                 mainloops over the concatenated K: (real, imaginary part) x
//                 (digit levels 0-3, levels 4-7), each with one accumulator of
//                 128 columns per level in tensor memory (4 x 128 = all 512
//                 columns), then an FP64 epilogue: the four levels of a group
//                 combine exactly (Horner, 2^7 apart, below 2^48); the first
//                 group's sum stays in registers until the second group's is
//                 added, scaled by 2^(eA_r + eB_c); the real part goes
//                 through an FP64 buffer, C = alpha (re + i im) + beta C at
//                 the end of the imaginary part.
// Roles: warp 8 lane 0 issues the TMA loads of a three-stage ring (and runs
// ahead into the next mainloop while the epilogue drains), warp 9 lane 0
// issues the MMAs and commits each stage back to the producer, warps 0-7 read
// the accumulators (warp w: TMEM lanes 32 (w % 4) .. +31, 64 columns each)
// and hand the tensor memory back to the MMA warp as soon as it is in
// registers.  Every wait on
// an mbarrier is bounded (about one second of SM clock); a wait that runs
// out marks the items' status and the CTA frees its tensor memory and returns.
//
// Reference: the complex products this replaces are the zgemm calls of
// prealloc_mult (src/sparsekit_drv.F90:1896-2081) and cu_ZmultMat
// (src/gpuroutines.cu:395-446); libNEGF has no reduced-precision product
// of its own besides the TF32 switch of cu_Zdecimation (:794-797).
#include <cuda.h>   // CUtensorMap and its enums only; the encoder comes from the runtime's driver entry point
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "ozaki.cuh"

namespace negf {
namespace {

constexpr long long kSpinCycles = 2000000000LL;   // bound of one mbarrier wait (~1 s)
constexpr int kPlaneBytes = kOzTileM * kOzKChunk;  // one digit plane of a 128-row tile (A and B alike)
static_assert(kOzTileM == kOzTileN, "A and B tiles share the plane size");
constexpr int kOzGroup = 4;                        // level accumulators held in TMEM at a time

__device__ __forceinline__ uint32_t s32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s32(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(s32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the completion of the phase with the given parity; false (and
// *fail set) if it does not complete within kSpinCycles or another thread of
// the CTA has already given up.
__device__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* fail) {
  const long long t0 = clock64();
  while (!mbar_test(b, parity)) {
    if (*fail) return false;
    if (clock64() - t0 > kSpinCycles) {
      *fail = 1;
      return false;
    }
  }
  return true;
}

// ---------------------------------------------------------------- TMA
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(s32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(s32(bar))
      : "memory");
}

// ---------------------------------------------------------------- tcgen05
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory operand descriptor: K-major, 32-byte swizzle, rows of 32 bytes
// (one K step), 8-row groups 256 bytes apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}

// D[tmem] (+)= A[smem] * B[smem]^T, int8 x int8 -> int32, M = 128, N = 128, K = 32
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

constexpr uint32_t kTmemCols = 512;

// instruction descriptor: D s32, A/B signed int8, both K-major, N = 128, M = 128
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kOzTileN >> 3) << 17) |
                              ((uint32_t)(kOzTileM >> 4) << 24);

// ---------------------------------------------------------------- splitting
// Digits: x = a 2^-e in (-1, 1); d_0 = rint(64 x), then d_t = rint(128 r) of
// the remainder r in [-1/2, 1/2]: every digit lies in [-64, 64] and
// x = sum_t d_t 2^(-6-7t) + r 2^(-6-7(S-1)).  Rounding to nearest leaves the
// cut-off remainders zero-mean.  A digit pair (t, u) has the weight
// 2^(-12-7(t+u)), exact as a double.
__device__ __forceinline__ double level_weight(int l) { return __longlong_as_double((long long)(1023 - 12 - 7 * l) << 52); }

template <int S>
__device__ __forceinline__ void digits(double x, int8_t (&d)[S]) {
  double y = x * 64.0;
  double r = rint(y);
  d[0] = (int8_t)r;
  x = y - r;
#pragma unroll
  for (int t = 1; t < S; ++t) {
    y = x * 128.0;
    r = rint(y);
    d[t] = (int8_t)r;
    x = y - r;
  }
}

// levels kept: digit pairs (t, u) with t + u < levels(S); one TMEM accumulator each
__host__ __device__ constexpr int oz_levels(int S) { return S + 1 < 8 ? S + 1 : 8; }

// Rows of A (M x K, column major, lda = M): exponent per row, digit planes
// of Ar, Ai, -Ai with K contiguous (row pitch kp bytes).  Block: 32 rows.
template <int S>
__global__ void __launch_bounds__(256) k_split_rows(int m, int k, int kp, const double2* A, int64_t sA, int8_t* qa,
                                                   int* ea, int* flag, const int* item_map) {
  __shared__ double smax[8][32];
  __shared__ int sexp[32];
  __shared__ int sbad;
  __shared__ __align__(16) int8_t sq[3][S][32][32];
  const int item = blockIdx.y;
  const int m0 = blockIdx.x * 32;
  const int r = threadIdx.x & 31, g = threadIdx.x >> 5;
  const double2* Ab = A + (int64_t)(item_map ? item_map[item] : item) * sA;
  if (threadIdx.x == 0) sbad = 0;
  __syncthreads();
  double mx = 0.0;
  bool bad = false;
  if (m0 + r < m)
    for (int kk = g; kk < k; kk += 8) {
      const double2 v = Ab[(int64_t)(m0 + r) + (int64_t)kk * m];
      bad |= !(isfinite(v.x) && isfinite(v.y));
      mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
    }
  smax[g][r] = mx;
  if (bad) sbad = 1;
  __syncthreads();
  if (g == 0) {
    double t = smax[0][r];
#pragma unroll
    for (int q = 1; q < 8; ++q) t = fmax(t, smax[q][r]);
    int e = 0;
    if (t > 0.0 && isfinite(t)) frexp(t, &e);   // t = f 2^e, f in [0.5, 1): |row| < 2^e
    sexp[r] = e;
    if (m0 + r < m) ea[(int64_t)item * m + m0 + r] = e;
  }
  __syncthreads();
  if (sbad && threadIdx.x == 0) atomicOr(flag + item, 1);
  const int e = sexp[r];
  const int64_t plane = (int64_t)m * kp;
  for (int k0 = 0; k0 < kp; k0 += 32) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int kk = k0 + 4 * g + j;
      double2 v = make_double2(0.0, 0.0);
      if (m0 + r < m && kk < k) v = Ab[(int64_t)(m0 + r) + (int64_t)kk * m];
      int8_t dr[S], di[S];
      digits<S>(ldexp(v.x, -e), dr);
      digits<S>(ldexp(v.y, -e), di);
#pragma unroll
      for (int t = 0; t < S; ++t) {
        sq[0][t][r][4 * g + j] = dr[t];
        sq[1][t][r][4 * g + j] = di[t];
        sq[2][t][r][4 * g + j] = (int8_t)(-di[t]);
      }
    }
    __syncthreads();
    // 3 * S planes x 32 rows x 2 segments of 16 bytes
    for (int idx = threadIdx.x; idx < 3 * S * 64; idx += 256) {
      const int seg = idx & 1, row = (idx >> 1) & 31, pt = idx >> 6;   // pt = arr * S + t
      const int arr = pt / S, t = pt % S;
      if (m0 + row < m && k0 + 16 * seg < kp) {
        int8_t* dst = qa + ((int64_t)(item * 3 + arr) * S + t) * plane + (int64_t)(m0 + row) * kp + k0 + 16 * seg;
        *reinterpret_cast<int4*>(dst) = *reinterpret_cast<const int4*>(&sq[arr][t][row][16 * seg]);
      }
    }
    __syncthreads();
  }
}

// Columns of B (K x N, column major, ldb = K): exponent per column, digit
// planes of Br, Bi with K contiguous.  One warp per column.
template <int S>
__global__ void __launch_bounds__(256) k_split_cols(int k, int n, int kp, const double2* B, int64_t sB, int8_t* qb,
                                                   int* eb, int* flag, const int* item_map) {
  const int item = blockIdx.y;
  const int c = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= n) return;
  const double2* col = B + (int64_t)(item_map ? item_map[item] : item) * sB + (int64_t)c * k;
  double mx = 0.0;
  bool bad = false;
  for (int kk = lane; kk < k; kk += 32) {
    const double2 v = col[kk];
    bad |= !(isfinite(v.x) && isfinite(v.y));
    mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  bad = __any_sync(0xffffffffu, bad);
  int e = 0;
  if (mx > 0.0 && isfinite(mx)) frexp(mx, &e);
  if (lane == 0) {
    eb[(int64_t)item * n + c] = e;
    if (bad) atomicOr(flag + item, 1);
  }
  const int64_t plane = (int64_t)n * kp;
  int8_t* q0 = qb + (int64_t)(item * 2) * S * plane + (int64_t)c * kp;
  for (int kk = lane; kk < kp; kk += 32) {
    double2 v = make_double2(0.0, 0.0);
    if (kk < k) v = col[kk];
    int8_t dr[S], di[S];
    digits<S>(ldexp(v.x, -e), dr);
    digits<S>(ldexp(v.y, -e), di);
#pragma unroll
    for (int t = 0; t < S; ++t) {
      q0[(int64_t)t * plane + kk] = dr[t];
      q0[(int64_t)(S + t) * plane + kk] = di[t];
    }
  }
}

// ---------------------------------------------------------------- product
struct OzArgs {
  int m, n, k, nkc;   // nkc: K chunks of kOzKChunk bytes per half of the concatenated K
  int batch;
  double2 alpha, beta;
  double2* C;
  int64_t sC;
  const int* item_map;   // launch item -> problem index for C / maxabs / status (null = identity)
  const int* ea;
  const int* eb;
  const int* flag;
  double* t0;            // FP64 real part of C, m x n per launch item (read back for the final combine)
  double* maxabs;
  int* status;
};

// Warp roles: warps 0-7 read the accumulators (warp w owns TMEM lanes
// 32 (w % 4) .. +31, i.e. rows m0 + 32 (w % 4) + lane, and the 64 columns
// 64 (w / 4) .. +63), warp 8 lane 0 issues the TMA loads, warp 9 lane 0 the
// MMAs.
constexpr int kOzEpiWarps = 8;
constexpr int kOzWarps = kOzEpiWarps + 2;
constexpr int kOzEpiCols = kOzTileN / 2;   // columns per epilogue thread

// int32 -> double without the conversion unit: 2^52 + 2^31 + v assembled from
// bits (exact for every int32), minus 2^52 + 2^31 (exact): one FP64 add.
__device__ __forceinline__ double i2d(uint32_t v) {
  return __hiloint2double(0x43300000, (int)(v ^ 0x80000000u)) - 4503601774854144.0;
}

// 2^e as a double for the normal range, ldexp outside it
__device__ __forceinline__ double pow2(int e) {
  return (e > -1022 && e < 1023) ? __longlong_as_double((long long)(1023 + e) << 52) : ldexp(1.0, e);
}

template <int S>
__global__ void __launch_bounds__(kOzWarps * 32, 1)
    k_ozaki(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, OzArgs a) {
  constexpr int kLevels = oz_levels(S);
  constexpr int kStage = 2 * S * kPlaneBytes;   // S planes of A and S of B
  static_assert(kOzGroup * kOzTileN <= (int)kTmemCols, "a level group must fit the tensor memory");
  static_assert(kLevels > kOzGroup && kLevels <= 2 * kOzGroup, "two level groups");
  extern __shared__ __align__(1024) uint8_t oz_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(oz_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full[kOzStages], empty[kOzStages], accb, tfree;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int fail;
  __shared__ int issued[kOzStages];
  __shared__ double col_scale[kOzTileN];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_m = (a.m + kOzTileM - 1) / kOzTileM, tiles_n = (a.n + kOzTileN - 1) / kOzTileN;
  const int per_item = tiles_m * tiles_n;
  const int ntiles = per_item * a.batch;
  const int nchunk = 2 * a.nkc;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kOzStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
      issued[i] = 0;
    }
    mbar_init(&accb, 1);
    mbar_init(&tfree, kOzEpiWarps);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s32(&tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_base;

  if (warp == kOzEpiWarps) {
    // ---------------- producer: digit planes of every (tile, part, group, chunk)
    if (lane == 0) {
      int g = 0;
      for (int tile = blockIdx.x; tile < ntiles && !fail; tile += gridDim.x) {
        const int item = tile / per_item, tt = tile % per_item;
        const int m0 = (tt / tiles_n) * kOzTileM, n0 = (tt % tiles_n) * kOzTileN;
        for (int mi = 0; mi < 4 && !fail; ++mi) {
          const int part = mi >> 1, grp = mi & 1;
          // planes used by the group: digits t < 4 (levels 0-3) or all S
          const int np = grp == 0 ? kOzGroup : S;
          for (int c = 0; c < nchunk; ++c, ++g) {
            const int st = g % kOzStages, use = g / kOzStages;
            if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1, &fail)) break;
            uint8_t* sa = sm + st * kStage;
            uint8_t* sb = sa + S * kPlaneBytes;
            const int h = c / a.nkc, k0 = (c % a.nkc) * kOzKChunk;
            // real part: [Ar | -Ai] x [Br ; Bi]; imaginary part: [Ai | Ar] x [Br ; Bi]
            const int arr_a = (part == 0) ? (h == 0 ? 0 : 2) : (h == 0 ? 1 : 0);
            mbar_arrive_tx(&full[st], (uint32_t)(2 * np * kPlaneBytes));
            for (int t = 0; t < np; ++t) {
              tma_load_3d(sa + t * kPlaneBytes, &tA, &full[st], k0, m0, (item * 3 + arr_a) * S + t);
              tma_load_3d(sb + t * kPlaneBytes, &tB, &full[st], k0, n0, (item * 2 + h) * S + t);
            }
            issued[st] = use + 1;
          }
        }
      }
    }
  } else if (warp == kOzEpiWarps + 1) {
    // ---------------- MMA issuer: the digit pairs of one level group per mainloop
    if (lane == 0) {
      int g = 0, ml = 0;
      for (int tile = blockIdx.x; tile < ntiles && !fail; tile += gridDim.x) {
        for (int mi = 0; mi < 4 && !fail; ++mi, ++ml) {
          const int l0 = (mi & 1) * kOzGroup;
          // the accumulators are free once the epilogue has read the previous mainloop
          if (ml > 0 && !mbar_wait(&tfree, (ml - 1) & 1, &fail)) break;
          tc_fence_after();
          for (int c = 0; c < nchunk; ++c, ++g) {
            const int st = g % kOzStages, use = g / kOzStages;
            if (!mbar_wait(&full[st], use & 1, &fail)) break;
            tc_fence_after();
            const uint32_t sa = s32(sm + st * kStage), sb = sa + S * kPlaneBytes;
#pragma unroll
            for (int t = 0; t < S; ++t) {
#pragma unroll
              for (int u = 0; u < S; ++u) {
                const int l = t + u;
                if (l < l0 || l >= l0 + kOzGroup || l >= kLevels) continue;
                // the first pair of a level (smallest t) in a mainloop overwrites its accumulator
                const int first_t = (l > S - 1) ? l - (S - 1) : 0;
                const uint32_t acc = (c > 0 || t > first_t) ? 1u : 0u;
                umma_i8(tbase + (uint32_t)((l - l0) * kOzTileN), sdesc(sa + t * kPlaneBytes),
                        sdesc(sb + u * kPlaneBytes), kIdescI8, acc);
              }
            }
            umma_commit(&empty[st]);   // the stage is free once these MMAs have read it
          }
          umma_commit(&accb);          // this group's level accumulators are complete
        }
      }
    }
  } else {
    // ---------------- epilogue: warps 0-7
    const int quarter = warp & 3, cw = kOzEpiCols * (warp >> 2);
    const uint32_t tlane = (uint32_t)(32 * quarter) << 16;
    constexpr int nlev1 = kLevels - kOzGroup;
    const double w0 = level_weight(kOzGroup - 1);   // units of the level-0..3 Horner sum
    const double w1 = level_weight(kLevels - 1);    // units of the level-4.. Horner sum
    int ml = 0;
    double part0[kOzEpiCols];                       // levels 0-3 of the current part, exact
    for (int tile = blockIdx.x; tile < ntiles && !fail; tile += gridDim.x) {
      const int item = tile / per_item, tt = tile % per_item;
      const int prob = a.item_map ? a.item_map[item] : item;
      const int m0 = (tt / tiles_n) * kOzTileM, n0 = (tt % tiles_n) * kOzTileN;
      const int r = m0 + 32 * quarter + lane;
      const bool row_ok = r < a.m;
      const double rs = row_ok ? pow2(a.ea[(int64_t)item * a.m + r]) : 0.0;
      const bool nonfinite = a.flag[item] != 0;
      // column scales of this tile (the epilogue warps' named barrier 1)
      asm volatile("bar.sync 1, %0;" ::"n"(kOzEpiWarps * 32));
      if (threadIdx.x < kOzTileN) {
        const int c = n0 + threadIdx.x;
        col_scale[threadIdx.x] = (c < a.n) ? pow2(a.eb[(int64_t)item * a.n + c]) : 0.0;
      }
      asm volatile("bar.sync 1, %0;" ::"n"(kOzEpiWarps * 32));
      double* T0 = a.t0 + (int64_t)item * a.m * a.n;
      double local_max = 0.0;
      bool any_bad = false;
      for (int mi = 0; mi < 4; ++mi, ++ml) {
        const int part = mi >> 1, grp = mi & 1;
        if (!mbar_wait(&accb, ml & 1, &fail)) break;
        tc_fence_after();
        // pass 1: every accumulator of the group into registers, combined to
        // one double per element (group 0: the exact level-0..3 Horner sum;
        // group 1: the part's value, scaled), then the tensor memory goes
        // back to the MMA warp before any global memory is touched
#pragma unroll
        for (int j8 = 0; j8 < kOzEpiCols / 8; ++j8) {
          uint32_t v[kOzGroup][8];
          const uint32_t col = (uint32_t)(cw + 8 * j8);
          if (grp == 0) {
#pragma unroll
            for (int l = 0; l < kOzGroup; ++l) tmem_ld8(tbase + tlane + (uint32_t)(l * kOzTileN) + col, v[l]);
          } else {
#pragma unroll
            for (int l = 0; l < nlev1; ++l) tmem_ld8(tbase + tlane + (uint32_t)(l * kOzTileN) + col, v[l]);
          }
          tmem_wait_ld();
          if (grp == 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              // exact: |acc| < 2^26, four levels 2^7 apart stay below 2^48
              double x = i2d(v[0][j]);
#pragma unroll
              for (int l = 1; l < kOzGroup; ++l) x = fma(x, 128.0, i2d(v[l][j]));
              part0[8 * j8 + j] = x;
            }
          } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              double y = i2d(v[0][j]);
#pragma unroll
              for (int l = 1; l < nlev1; ++l) y = fma(y, 128.0, i2d(v[l][j]));
              part0[8 * j8 + j] = fma(part0[8 * j8 + j], w0, y * w1) * rs * col_scale[col + j];
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tfree);
        if (grp == 0 || !row_ok) continue;
        // pass 2 (group 1, the part complete): global memory while the next mainloop runs
#pragma unroll
        for (int j8 = 0; j8 < kOzEpiCols / 8; ++j8) {
          const uint32_t col = (uint32_t)(cw + 8 * j8);
          const double* val = part0 + 8 * j8;
          const int c0 = n0 + (int)col;
          if (part == 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
              if (c0 + j < a.n) T0[(int64_t)r + (int64_t)(c0 + j) * a.m] = val[j];
            continue;
          }
          double pr[8];
          double2 old[8];
          const bool use_beta = (a.beta.x != 0.0 || a.beta.y != 0.0);
          double2* Cp = a.C + (int64_t)prob * a.sC;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int64_t o = (int64_t)r + (int64_t)(c0 + j) * a.m;
            const bool ok = c0 + j < a.n;
            pr[j] = ok ? T0[o] : 0.0;
            old[j] = (ok && use_beta) ? Cp[o] : make_double2(0.0, 0.0);
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (c0 + j >= a.n) continue;
            const double pi = val[j];
            double2 out = make_double2(a.alpha.x * pr[j] - a.alpha.y * pi, a.alpha.x * pi + a.alpha.y * pr[j]);
            out.x += a.beta.x * old[j].x - a.beta.y * old[j].y;
            out.y += a.beta.x * old[j].y + a.beta.y * old[j].x;
            if (nonfinite) {
              const double qnan = __longlong_as_double(0x7ff8000000000000LL);
              out = make_double2(qnan, qnan);
            }
            Cp[(int64_t)r + (int64_t)(c0 + j) * a.m] = out;
            if (a.maxabs) {
              const double h = hypot(out.x, out.y);
              local_max = fmax(local_max, h);
              any_bad |= !(h <= 1.7976931348623157e308);   // NaN or Inf
            }
          }
        }
      }
      if (fail) break;
      if (a.maxabs) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) local_max = fmax(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
        // a NaN or Inf element makes the maximum NaN (fmax drops it), which stays
        // above every finite bit pattern under atomicMax: a convergence test on it fails
        if (__any_sync(0xffffffffu, any_bad)) local_max = __longlong_as_double(0x7ff8000000000000LL);
        if (lane == 0 && !(local_max <= 0.0))
          atomicMax(reinterpret_cast<unsigned long long*>(a.maxabs + prob),
                    (unsigned long long)__double_as_longlong(local_max));
      }
      if (nonfinite && threadIdx.x == 0 && a.status && tt == 0) a.status[prob] = 3;
    }
  }

  __syncthreads();
  if (fail) {
    // let every TMA load this CTA issued land before its shared memory is released
    if (threadIdx.x == 0)
      for (int st = 0; st < kOzStages; ++st)
        if (issued[st] > 0) {
          const long long t0 = clock64();
          while (!mbar_test(&full[st], (issued[st] - 1) & 1) && clock64() - t0 < kSpinCycles) {
          }
        }
    if (threadIdx.x == 0 && a.status)
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int item = tile / per_item;
        a.status[a.item_map ? a.item_map[item] : item] = 7;
      }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTmemCols)
                              : "memory");
}

// ---------------------------------------------------------------- host
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// 3-D map over digit planes: x = K byte (inner), y = row, z = plane
bool make_map(CUtensorMap* map, void* base, int k, int rows, int kp, int planes, int box_rows) {
  EncodeTiledFn fn = encoder();
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)k, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)kp, (cuuint64_t)kp * (cuuint64_t)rows};
  const cuuint32_t box[3] = {(cuuint32_t)kOzKChunk, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int num_sms() {
  static int n[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!n[dev] && cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    n[dev] = 148;
  }
  return n[dev];
}

template <int S>
cudaError_t run(const OzakiLayout& L, double2 alpha, const double2* A, int64_t sA, const double2* B, int64_t sB,
                double2 beta, double2* C, int64_t sC, uint8_t* w, double* maxabs, int* status, cudaStream_t s,
                const int* item_map) {
  int8_t* qa = reinterpret_cast<int8_t*>(w + L.qa_off);
  int8_t* qb = reinterpret_cast<int8_t*>(w + L.qb_off);
  int* ea = reinterpret_cast<int*>(w + L.ea_off);
  int* eb = reinterpret_cast<int*>(w + L.eb_off);
  int* flag = reinterpret_cast<int*>(w + L.flag_off);
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int) * (size_t)L.batch, s);
  if (e != cudaSuccess) return e;
  k_split_rows<S><<<dim3((L.m + 31) / 32, L.batch), 256, 0, s>>>(L.m, L.k, L.kp, A, sA, qa, ea, flag, item_map);
  k_split_cols<S><<<dim3((L.n + 7) / 8, L.batch), 256, 0, s>>>(L.k, L.n, L.kp, B, sB, qb, eb, flag, item_map);
  CUtensorMap ta, tb;
  if (!make_map(&ta, qa, L.k, L.m, L.kp, L.batch * 3 * S, kOzTileM) ||
      !make_map(&tb, qb, L.k, L.n, L.kp, L.batch * 2 * S, kOzTileN))
    return cudaErrorInvalidValue;
  OzArgs a;
  a.m = L.m; a.n = L.n; a.k = L.k; a.nkc = (L.k + kOzKChunk - 1) / kOzKChunk;
  a.batch = L.batch;
  a.alpha = alpha; a.beta = beta; a.C = C; a.sC = sC; a.item_map = item_map;
  a.ea = ea; a.eb = eb; a.flag = flag;
  a.t0 = reinterpret_cast<double*>(w + L.t0_off);
  a.maxabs = maxabs; a.status = status;
  const size_t smem = (size_t)kOzStages * 2 * S * kPlaneBytes + 1024;
  static std::mutex mu;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
      e = cudaFuncSetAttribute(k_ozaki<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
  }
  const long long tiles = (long long)((L.m + kOzTileM - 1) / kOzTileM) * ((L.n + kOzTileN - 1) / kOzTileN) * L.batch;
  const int grid = (int)(tiles < num_sms() ? tiles : num_sms());
  k_ozaki<S><<<grid, kOzWarps * 32, smem, s>>>(ta, tb, a);
  return cudaGetLastError();
}

}  // namespace

OzakiLayout ozaki_layout(int batch, int m, int n, int k, int slices) {
  OzakiLayout L;
  L.batch = batch; L.m = m; L.n = n; L.k = k; L.slices = slices;
  L.kp = (k + 15) & ~15;
  size_t off = 0;
  L.qa_off = off; off = align256(off + (size_t)batch * 3 * slices * m * L.kp);
  L.qb_off = off; off = align256(off + (size_t)batch * 2 * slices * n * L.kp);
  L.ea_off = off; off = align256(off + sizeof(int) * (size_t)batch * m);
  L.eb_off = off; off = align256(off + sizeof(int) * (size_t)batch * n);
  L.flag_off = off; off = align256(off + sizeof(int) * (size_t)batch);
  L.t0_off = off; off = align256(off + sizeof(double) * (size_t)batch * m * n);
  L.total = off;
  return L;
}

cudaError_t launch_ozaki_zgemm(int batch, int m, int n, int k, double2 alpha, const double2* A, int64_t sA,
                               const double2* B, int64_t sB, double2 beta, double2* C, int64_t sC, int slices,
                               void* work, double* maxabs, int* status, cudaStream_t s, const int* item_map) {
  if (batch <= 0 || m <= 0 || n <= 0) return cudaSuccess;
  if (k <= 0 || k > 1024 || batch > 65535 || slices < kOzMinSlices || slices > kOzMaxSlices || !work ||
      (reinterpret_cast<uintptr_t>(work) & 255))
    return cudaErrorInvalidValue;
  const OzakiLayout L = ozaki_layout(batch, m, n, k, slices);
  uint8_t* w = static_cast<uint8_t*>(work);
  switch (slices) {
    case 4: return run<4>(L, alpha, A, sA, B, sB, beta, C, sC, w, maxabs, status, s, item_map);
    case 5: return run<5>(L, alpha, A, sA, B, sB, beta, C, sC, w, maxabs, status, s, item_map);
    case 6: return run<6>(L, alpha, A, sA, B, sB, beta, C, sC, w, maxabs, status, s, item_map);
    case 7: return run<7>(L, alpha, A, sA, B, sB, beta, C, sC, w, maxabs, status, s, item_map);
    default: return run<8>(L, alpha, A, sA, B, sB, beta, C, sC, w, maxabs, status, s, item_map);
  }
}

}  // namespace negf
