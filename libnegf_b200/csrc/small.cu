// Small-order block operations for the lock-step FP64 form (small.cuh): one
// CTA per product (operands staged in shared memory), one warp per
// inversion (lane i holding row i).  Reference operations replaced: the zgemm of prealloc_mult
// (src/sparsekit_drv.F90:1896-2081) and zinv = zgetrf + zgetrs against the
// identity (src/inversions.F90:807-839), at orders n <= 32.
#include <cuda_runtime.h>

#include <mutex>

#include "cta_ops.cuh"
#include "small.cuh"

namespace negf {
namespace {

constexpr int kWarps = 4;                  // problems per CTA
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int batch_limit(int batch, const int* count) {
  return count ? min(*count, batch) : batch;
}

// One CTA (4 warps) per problem: A and B staged in shared memory by
// coalesced loads (one memory latency per operand), then warp w computes
// columns [w CW, (w + 1) CW) of C and lane i row i: A's column k is read
// conflict-free, B's row k by broadcast.
template <int N>
__global__ void __launch_bounds__(kWarps * 32)
    k_small_zgemm(int batch, int n, double2 alpha, const double2* __restrict__ A, const double2* __restrict__ B,
                  double2 beta, double2* C, int64_t Q, const int* map, const int* count, double* maxabs) {
  constexpr int CW = N / kWarps;   // columns per warp
  __shared__ double2 sA[N * N], sB[N * N];
  __shared__ double smx[kWarps];
  __shared__ int sbad[kWarps];
  const int b = blockIdx.x;
  if (b >= batch_limit(batch, count)) return;
  const int p = map ? map[b] : b;
  const int nn = n * n;
  const double2* Ap = A + p * Q;
  const double2* Bp = B + p * Q;
  {
    constexpr int R = (N * N + kWarps * 32 - 1) / (kWarps * 32);
    double2 va[R], vb[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int q = threadIdx.x + i * kWarps * 32;
      if (q < nn) {
        va[i] = __ldg(Ap + q);
        vb[i] = __ldg(Bp + q);
      }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int q = threadIdx.x + i * kWarps * 32;
      if (q < nn) {
        sA[q] = va[i];
        sB[q] = vb[i];
      }
    }
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j0 = w * CW;
  double2 acc[CW];
#pragma unroll
  for (int jj = 0; jj < CW; ++jj) acc[jj] = make_double2(0.0, 0.0);
  if (lane < n) {
    for (int k = 0; k < n; ++k) {
      const double2 a = sA[lane + k * n];
#pragma unroll
      for (int jj = 0; jj < CW; ++jj) {
        const int j = j0 + jj;
        if (j < n) {
          const double2 bv = sB[k + j * n];
          acc[jj].x = fma(a.x, bv.x, acc[jj].x);
          acc[jj].x = fma(-a.y, bv.y, acc[jj].x);
          acc[jj].y = fma(a.x, bv.y, acc[jj].y);
          acc[jj].y = fma(a.y, bv.x, acc[jj].y);
        }
      }
    }
  }
  const bool use_beta = beta.x != 0.0 || beta.y != 0.0;
  double mx = 0.0;
  bool bad = false;
  if (lane < n) {
    double2* Cp = C + p * Q;
#pragma unroll
    for (int jj = 0; jj < CW; ++jj) {
      const int j = j0 + jj;
      if (j < n) {
        double2* el = Cp + lane + (int64_t)j * n;
        double2 v = cmul(alpha, acc[jj]);
        if (use_beta) v = cadd(v, cmul(beta, *el));
        *el = v;
        const double h = hypot(v.x, v.y);
        mx = fmax(mx, h);
        bad |= !(h <= 1.7976931348623157e308);   // NaN or Inf
      }
    }
  }
  if (maxabs) {
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(kFull, mx, o));
    bad = __any_sync(kFull, bad);
    if (lane == 0) {
      smx[w] = mx;
      sbad[w] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      bool any = false;
      for (int q = 0; q < kWarps; ++q) {
        mx = fmax(mx, smx[q]);
        any |= sbad[q] != 0;
      }
      // a non-finite element makes the maximum NaN (fmax would drop it): the
      // positive quiet NaN is above every finite bit pattern, so it stays
      if (any) mx = __longlong_as_double(0x7ff8000000000000LL);
      atomicMax(reinterpret_cast<unsigned long long*>(maxabs + p), (unsigned long long)__double_as_longlong(mx));
    }
  }
}

// In-place Gauss-Jordan, one CTA (4 warps) per matrix: lane i holds row i,
// warp w the columns [w CW, (w + 1) CW).  Rows never move between lanes:
// each lane carries the logical (pivot-order) index of its row, identical in
// every warp.  Per step the warp owning column k picks the pivot (the unused
// row with the largest |Re|+|Im|, lowest logical index on a tie: izamax) by
// integer warp reductions on the bit pattern and publishes column k and the
// pivot's lane in shared memory (double-buffered by step parity: one barrier
// per step); every warp then updates its columns, taking the pivot row's
// entries from the pivot lane by shuffle.  The pivot row becomes row * d
// (d = 1 / pivot, entry k = d), every other row r - (r_k d) * row (entry
// k = -(r_k d)), the update order of the engine's Gauss-Jordan.  The column
// interchanges that undo the row order are applied to the store addresses.
template <int N>
__global__ void __launch_bounds__(kWarps * 32)
    k_small_zinv(int batch, int n, const double2* A, double2* X, int64_t Q, const int* map, const int* count,
                 int* info, int* status, int singular_code) {
  constexpr int CW = N / kWarps;
  __shared__ double2 colk[2][32];  // one entry per lane: rows >= N exist as lanes too
  __shared__ int sbl[2];
  __shared__ int sidx[N];
  __shared__ int scm[N];
  const int b = blockIdx.x;
  if (b >= batch_limit(batch, count)) return;
  const int p = map ? map[b] : b;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double2* Ap = A + p * Q;
  double2 r[CW];
#pragma unroll
  for (int cc = 0; cc < CW; ++cc) {
    const int c = w * CW + cc;
    r[cc] = (lane < n && c < n) ? Ap[lane + (int64_t)c * n] : make_double2(0.0, 0.0);
  }
  int lg = lane;
  bool used = lane >= n;
  int inf = 0;
  for (int k = 0; k < n; ++k) {
    const int ow = k / CW, ck = k % CW, par = k & 1;
    if (w == ow) {
      double2 rk = r[0];
#pragma unroll
      for (int cc = 1; cc < CW; ++cc)
        if (cc == ck) rk = r[cc];
      // |Re|+|Im| orders as its bit pattern; + 1 puts an unused row with a zero entry
      // above the used rows (key 0); NaN ranks highest so all lanes see one order
      double v = cabs1(rk);
      if (v != v) v = __longlong_as_double(0x7ff0000000000000LL);
      const unsigned long long key = used ? 0ull : (unsigned long long)__double_as_longlong(v) + 1ull;
      const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
      const unsigned mhi = __reduce_max_sync(kFull, hi);
      const unsigned mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
      const bool cand = hi == mhi && lo == mlo;
      const int blg = (int)__reduce_min_sync(kFull, cand ? (unsigned)lg : 0xffffffffu);
      const int bl = __ffs(__ballot_sync(kFull, cand && lg == blg)) - 1;
      colk[par][lane] = rk;
      if (lane == 0) {
        sbl[par] = bl;
        sidx[k] = blg;
      }
    }
    __syncthreads();
    const int bl = sbl[par];
    const int blg = sidx[k];
    const double2 pv = colk[par][bl];
    if (pv.x == 0.0 && pv.y == 0.0 && inf == 0) inf = k + 1;
    const double2 d = crecip(pv);
    const double2 fd = cmul(colk[par][lane], d);
    // both candidate values for every lane, then selects: no divergent path for the pivot lane
    const bool isp = lane == bl;
#pragma unroll
    for (int cc = 0; cc < CW; ++cc) {
      const int c = w * CW + cc;
      double2 pc;
      pc.x = __shfl_sync(kFull, r[cc].x, bl);
      pc.y = __shfl_sync(kFull, r[cc].y, bl);
      const double2 prow = cmul(pc, d);
      const double2 upd = csub(r[cc], cmul(fd, pc));
      double2 v = isp ? prow : (c < n ? upd : r[cc]);
      if (c == k) v = isp ? d : make_double2(-fd.x, -fd.y);
      r[cc] = v;
    }
    if (lg == k) lg = blg;
    if (lane == bl) {
      lg = k;
      used = true;
    }
  }
  // column interchanges in reverse pivot order: output column dest[c] takes internal column c
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 0; j < n; ++j) scm[j] = j;
    for (int l = n - 1; l >= 0; --l) {
      const int il = sidx[l];
      if (il != l) {
        const int t = scm[il];
        scm[il] = scm[l];
        scm[l] = t;
      }
    }
    for (int j = 0; j < n; ++j) sidx[scm[j]] = j;
  }
  __syncthreads();
  if (lane < n) {
    double2* Xp = X + p * Q;
#pragma unroll
    for (int cc = 0; cc < CW; ++cc) {
      const int c = w * CW + cc;
      if (c < n) Xp[lg + (int64_t)sidx[c] * n] = r[cc];
    }
  }
  if (threadIdx.x == 0) {
    if (info) info[p] = inf;
    if (status && inf != 0 && status[p] == 0) status[p] = singular_code;
  }
}

// ---------------------------------------------------------------- decimation steps
// Row `lane` of columns [w CW, (w + 1) CW) of A B, A and B n x n in shared
// memory (the product of k_small_zgemm, for the fused decimation iteration below).
template <int N>
__device__ __forceinline__ void mm_rows(int n, const double2* sA, const double2* sB, double2 (&acc)[N / kWarps]) {
  constexpr int CW = N / kWarps;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int jj = 0; jj < CW; ++jj) acc[jj] = make_double2(0.0, 0.0);
  if (lane >= n) return;
  for (int k = 0; k < n; ++k) {
    const double2 a = sA[lane + k * n];
#pragma unroll
    for (int jj = 0; jj < CW; ++jj) {
      const int j = w * CW + jj;
      if (j < n) {
        const double2 bv = sB[k + j * n];
        acc[jj].x = fma(a.x, bv.x, acc[jj].x);
        acc[jj].x = fma(-a.y, bv.y, acc[jj].x);
        acc[jj].y = fma(a.x, bv.y, acc[jj].y);
        acc[jj].y = fma(a.y, bv.x, acc[jj].y);
      }
    }
  }
}

// Three n x n operands into shared memory: every thread issues all of its
// global loads before its first shared store (one memory latency, not three).
template <int N>
__device__ __forceinline__ void stage3(int n, double2* d0, const double2* s0, double2* d1, const double2* s1,
                                       double2* d2, const double2* s2) {
  constexpr int R = (N * N + kWarps * 32 - 1) / (kWarps * 32);
  const int nn = n * n;
  double2 v0[R], v1[R], v2[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int q = threadIdx.x + i * kWarps * 32;
    if (q < nn) {
      v0[i] = __ldg(s0 + q);
      v1[i] = __ldg(s1 + q);
      v2[i] = __ldg(s2 + q);
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int q = threadIdx.x + i * kWarps * 32;
    if (q < nn) {
      d0[q] = v0[i];
      d1[q] = v1[i];
      d2[q] = v2[i];
    }
  }
}

// One decimation iteration (src/contselfenergy.F90:271-340) for the points
// list[b], b < *count, one CTA each, with Go, Co and Bo staged in shared
// memory once: X = Go Co, C1 = Co X, the CPU convergence rule on max|C1| (a
// point is done on its second consecutive max|C1| <= tol: ncyc = it; the
// others go on to next[]), and for the points that go on Self = Bo X,
// Ao -= Self, Aos -= Self, then Y = Go Bo (in X's place), B1 = Bo Y,
// Ao -= Co Y.
template <int N>
__global__ void __launch_bounds__(kWarps * 32)
    k_small_dec(int n, const int* list, const int* count, int P, const double2* Go, const double2* Co,
                const double2* Bo, double2* C1, double2* B1, double2* Ao, double2* Aos, int64_t Q, int* ok,
                int* ncyc_c, double tol, int it, int* next, int* next_count, int* redo) {
  constexpr int CW = N / kWarps;
  extern __shared__ __align__(16) double2 sdec[];
  double2* sG = sdec;
  double2* sC = sG + N * N;
  double2* sB = sC + N * N;
  double2* sX = sB + N * N;
  __shared__ double smx[kWarps];
  __shared__ int sgo;
  const int b = blockIdx.x;
  if (b >= min(*count, P)) return;
  const int p = list[b];
  const int64_t o = p * Q;
  stage3<N>(n, sG, Go + o, sC, Co + o, sB, Bo + o);
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 acc[CW];
  mm_rows<N>(n, sG, sC, acc);                      // X = Go Co
  if (lane < n)
#pragma unroll
    for (int jj = 0; jj < CW; ++jj)
      if (w * CW + jj < n) sX[lane + (w * CW + jj) * n] = acc[jj];
  __syncthreads();
  mm_rows<N>(n, sC, sX, acc);                      // C1 = Co X
  double mx = 0.0;
  bool bad = false;
  if (lane < n)
#pragma unroll
    for (int jj = 0; jj < CW; ++jj) {
      const int j = w * CW + jj;
      if (j < n) {
        C1[o + lane + j * n] = acc[jj];
        const double h = hypot(acc[jj].x, acc[jj].y);
        mx = fmax(mx, h);
        bad |= !(h <= 1.7976931348623157e308);
      }
    }
  for (int s = 16; s > 0; s >>= 1) mx = fmax(mx, __shfl_xor_sync(kFull, mx, s));
  if (__any_sync(kFull, bad)) mx = __longlong_as_double(0x7ff8000000000000LL);
  if (lane == 0) smx[w] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = smx[0];
    for (int q = 1; q < kWarps; ++q) m = (m != m || smx[q] != smx[q]) ? m + smx[q] : fmax(m, smx[q]);
    bool go = true;
    if (!(m <= 1.7976931348623157e308)) {   // Inf / NaN: will not converge; run it again
      go = false;
      ncyc_c[p] = it;
      if (redo) redo[p] = 1;
    } else if (m <= tol) {
      if (ok[p]) {
        go = false;
        ncyc_c[p] = it;
      }
      ok[p] = 1;
    } else {
      ok[p] = 0;
    }
    if (go) next[atomicAdd(next_count, 1)] = p;
    sgo = go;
  }
  __syncthreads();
  if (!sgo) return;
  mm_rows<N>(n, sB, sX, acc);                      // Self = Bo X
  if (lane < n)
#pragma unroll
    for (int jj = 0; jj < CW; ++jj) {
      const int j = w * CW + jj;
      if (j < n) {
        const int64_t q = o + lane + j * n;
        Ao[q] = csub(Ao[q], acc[jj]);
        Aos[q] = csub(Aos[q], acc[jj]);
      }
    }
  __syncthreads();                                 // X is read; Y takes its place
  mm_rows<N>(n, sG, sB, acc);                      // Y = Go Bo
  if (lane < n)
#pragma unroll
    for (int jj = 0; jj < CW; ++jj)
      if (w * CW + jj < n) sX[lane + (w * CW + jj) * n] = acc[jj];
  __syncthreads();
  mm_rows<N>(n, sB, sX, acc);                      // B1 = Bo Y
  if (lane < n)
#pragma unroll
    for (int jj = 0; jj < CW; ++jj)
      if (w * CW + jj < n) B1[o + lane + (w * CW + jj) * n] = acc[jj];
  mm_rows<N>(n, sC, sX, acc);                      // Ao -= Co Y
  if (lane < n)
#pragma unroll
    for (int jj = 0; jj < CW; ++jj) {
      const int j = w * CW + jj;
      if (j < n) Ao[o + lane + j * n] = csub(Ao[o + lane + j * n], acc[jj]);
    }
}

// Dynamic shared memory above the 48 KB default needs an opt-in per device.
template <typename K>
cudaError_t opt_in(K kernel, size_t smem, bool (&done)[64], std::mutex& mu) {
  if (smem <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

// Residual probe of the inverse X of A and up to two Newton steps
// X <- X + X (I - A X) where it exceeds kInvProbeTol (cta_inv_probe, the
// engine's refine block), one CTA per problem with A, X and I - A X staged
// in shared memory.  A problem whose probe passes costs two matrix-vector
// products and leaves X untouched.
template <int N>
__global__ void __launch_bounds__(kWarps * 32)
    k_small_refine(int batch, int n, const double2* A, double2* X, int64_t Q, const int* map, const int* count,
                   int* sens) {
  extern __shared__ __align__(16) double2 sref[];
  double2* sA = sref;
  double2* sX = sA + N * N;
  double2* sR = sX + N * N;
  double2* y = sR + N * N;
  __shared__ double red[kWarps], redk[kWarps];
  const int b = blockIdx.x;
  if (b >= batch_limit(batch, count)) return;
  const int p = map ? map[b] : b;
  const int nn = n * n;
  const double2* Ap = A + p * Q;
  double2* Xp = X + p * Q;
  for (int q = threadIdx.x; q < nn; q += kWarps * 32) {
    sA[q] = Ap[q];
    sX[q] = Xp[q];
  }
  __syncthreads();
  bool changed = false;
  for (int round = 0; round < 2; ++round) {
    // probe: y = X v, then max |A y - v|
    for (int r = threadIdx.x; r < n; r += kWarps * 32) {
      double2 acc = make_double2(0.0, 0.0);
      for (int c = 0; c < n; ++c) acc = cadd(acc, cmul(sX[r + c * n], probe_v(c)));
      y[r] = acc;
    }
    __syncthreads();
    double e = 0.0, kap = 0.0;
    for (int r = threadIdx.x; r < n; r += kWarps * 32) {
      double2 acc = make_double2(0.0, 0.0);
      double sa = 0.0;
      for (int c = 0; c < n; ++c) {
        acc = cadd(acc, cmul(sA[r + c * n], y[c]));
        sa += cabs1(sA[r + c * n]) * cabs1(y[c]);
      }
      const double d = cabs(csub(acc, probe_v(r)));
      e = (d <= 1.7976931348623157e308) ? fmax(e, d) : __longlong_as_double(0x7ff0000000000000LL);
      kap = fmax(kap, sa);
    }
    for (int o = 16; o > 0; o >>= 1) {
      e = fmax(e, __shfl_xor_sync(kFull, e, o));
      kap = fmax(kap, __shfl_xor_sync(kFull, kap, o));
    }
    if ((threadIdx.x & 31) == 0) {
      red[threadIdx.x >> 5] = e;
      redk[threadIdx.x >> 5] = kap;
    }
    __syncthreads();
    double em = 0.0, km = 0.0;
    for (int q = 0; q < kWarps; ++q) {
      em = fmax(em, red[q]);
      km = fmax(km, redk[q]);
    }
    __syncthreads();
    // the condition estimate of the unrefined inverse marks a nearly singular matrix
    if (round == 0 && km > kSensitiveCond && sens && threadIdx.x == 0) sens[p] = 1;
    if (!(em > kInvProbeTol) || !(em <= 1.7976931348623157e308)) break;
    // R = I - A X
    for (int q = threadIdx.x; q < nn; q += kWarps * 32) {
      const int i = q % n, j = q / n;
      double2 acc = make_double2(i == j ? 1.0 : 0.0, 0.0);
      for (int k = 0; k < n; ++k) acc = csub(acc, cmul(sA[i + k * n], sX[k + j * n]));
      sR[q] = acc;
    }
    __syncthreads();
    // X + X R, element by element into registers, then back into sX
    double2 nx[N * N / (kWarps * 32) + 1];
    int cnt = 0;
    for (int q = threadIdx.x; q < nn; q += kWarps * 32, ++cnt) {
      const int i = q % n, j = q / n;
      double2 acc = sX[q];
      for (int k = 0; k < n; ++k) acc = cadd(acc, cmul(sX[i + k * n], sR[k + j * n]));
      nx[cnt] = acc;
    }
    __syncthreads();
    cnt = 0;
    for (int q = threadIdx.x; q < nn; q += kWarps * 32, ++cnt) sX[q] = nx[cnt];
    __syncthreads();
    changed = true;
  }
  if (changed)
    for (int q = threadIdx.x; q < nn; q += kWarps * 32) Xp[q] = sX[q];
}

}  // namespace

cudaError_t launch_small_refine(int batch, int n, const double2* A, double2* X, int64_t Q, const int* map,
                                const int* count, cudaStream_t s, int* sens) {
  if (batch <= 0) return cudaSuccess;
  if (n < 1 || n > kSmallMax) return cudaErrorInvalidValue;
  if (n <= 16) {
    const size_t smem = (3 * 16 * 16 + 16) * sizeof(double2);
    k_small_refine<16><<<batch, kWarps * 32, smem, s>>>(batch, n, A, X, Q, map, count, sens);
  } else {
    const size_t smem = (3 * 32 * 32 + 32) * sizeof(double2);   // above the 48 KB default: opt in per device
    static std::mutex mu;
    static bool attr[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64 || !attr[dev]) {
      cudaError_t e = cudaFuncSetAttribute(k_small_refine<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    k_small_refine<32><<<batch, kWarps * 32, smem, s>>>(batch, n, A, X, Q, map, count, sens);
  }
  return cudaGetLastError();
}

cudaError_t launch_small_dec(int P, int n, const int* list, const int* count, const double2* Go, const double2* Co,
                             const double2* Bo, double2* C1, double2* B1, double2* Ao, double2* Aos, int64_t Q, int* ok,
                             int* ncyc_c, double tol, int it, int* next, int* next_count, int* redo, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  if (n < 1 || n > kSmallMax) return cudaErrorInvalidValue;
  static std::mutex mu;
  static bool done16[64] = {false}, done32[64] = {false};
  if (n <= 16) {
    const size_t smem = 4 * 16 * 16 * sizeof(double2);
    cudaError_t e = opt_in(k_small_dec<16>, smem, done16, mu);
    if (e != cudaSuccess) return e;
    k_small_dec<16><<<P, kWarps * 32, smem, s>>>(n, list, count, P, Go, Co, Bo, C1, B1, Ao, Aos, Q, ok, ncyc_c, tol,
                                                 it, next, next_count, redo);
  } else {
    const size_t smem = 4 * 32 * 32 * sizeof(double2);
    cudaError_t e = opt_in(k_small_dec<32>, smem, done32, mu);
    if (e != cudaSuccess) return e;
    k_small_dec<32><<<P, kWarps * 32, smem, s>>>(n, list, count, P, Go, Co, Bo, C1, B1, Ao, Aos, Q, ok, ncyc_c, tol,
                                                 it, next, next_count, redo);
  }
  return cudaGetLastError();
}

cudaError_t launch_small_zgemm(int batch, int n, double2 alpha, const double2* A, const double2* B, double2 beta,
                               double2* C, int64_t Q, const int* map, const int* count, double* maxabs,
                               cudaStream_t s) {
  if (batch <= 0) return cudaSuccess;
  if (n < 1 || n > kSmallMax) return cudaErrorInvalidValue;
  if (n <= 16)
    k_small_zgemm<16><<<batch, kWarps * 32, 0, s>>>(batch, n, alpha, A, B, beta, C, Q, map, count, maxabs);
  else
    k_small_zgemm<32><<<batch, kWarps * 32, 0, s>>>(batch, n, alpha, A, B, beta, C, Q, map, count, maxabs);
  return cudaGetLastError();
}

cudaError_t launch_small_zinv(int batch, int n, const double2* A, double2* X, int64_t Q, const int* map,
                              const int* count, int* info, int* status, int singular_code, cudaStream_t s) {
  if (batch <= 0) return cudaSuccess;
  if (n < 1 || n > kSmallMax) return cudaErrorInvalidValue;
  if (n <= 16)
    k_small_zinv<16><<<batch, kWarps * 32, 0, s>>>(batch, n, A, X, Q, map, count, info, status, singular_code);
  else
    k_small_zinv<32><<<batch, kWarps * 32, 0, s>>>(batch, n, A, X, Q, map, count, info, status, singular_code);
  return cudaGetLastError();
}

}  // namespace negf
