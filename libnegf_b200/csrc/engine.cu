// Persistent per-energy-point engine for sm_100a.
//
// One CTA owns one (energy, k) point at a time and runs its complete solve:
// Sancho-Rubio decimation per contact, contact self-energies, the backward
// gsmr sweep, Gr(1,1), then (by mode) the Caroli transmission, the full
// retarded sweep with the diagonal spectral density, or the elastic
// dephasing SCBA loop with the lesser sweep, Meir-Wingreen and layer
// currents.  CTAs pull points from a global queue, so all energy x k points
// of a call (and all SCBA iterations of each point) run in one launch with
// no host synchronisation; per-point convergence (decimation, SCBA) is
// decided on the device.
//
// Reference routines (libNEGF): decimation src/contselfenergy.F90:271-340,
// contact self-energy :445-491/:552-566, build_ESH src/iterative.F90:1956,
// gsmr/Gr/Gn sweeps src/iterative_cpu.F90:51-372, transmissions :399-583,
// DOS src/iterative.F90:1821-1952, elastic SCBA :289-363 with
// src/elphdd.F90:108-276 and src/scba.F90:120-147, Meir-Wingreen and layer
// current src/iterative.F90:382-461.
#include <mutex>

#include "program.cuh"

namespace negf {

static_assert(kGemmSmemBytes + (int)sizeof(GemmDesc) <= kSmemMain,
              "GEMM staging ring and descriptor must fit the main shared-memory region");
static_assert((kSmallInvMax * kSmallInvMax + 3 * kSmallInvMax + 1) * 16 <= kSmemMain,
              "small inversion must fit the main shared-memory region");

size_t engine_smem_bytes(int nmax) { return smem_bytes_for(nmax); }

// ---------------------------------------------------------------- helpers (primitive kernels)
__device__ __forceinline__ void gemm(int M, int N, int K, Operand A, Operand B, double2* C, int ldc,
                                     double2 alpha, double2 beta, SmemMap& sm, bool want_max = false) {
  long long t0 = sm.tr.start();
  Epilogue e = epi_store(C, ldc, alpha, beta);
  if (want_max) {
    if (threadIdx.x == 0) *sm.maxv = 0.0;
    __syncthreads();
    e.maxabs = sm.maxv;
  }
  cta_gemm(M, N, K, A, B, e, sm.main);
  sm.tr.stop(TR_GEMM, t0);
}

__device__ __forceinline__ int zinv(int n, const double2* A, double2* out, double2* ws, SmemMap& sm) {
  return cta_zinv(n, A, out, ws, sm.main, sm.inv);
}

// zinv, then the residual probe and up to two Newton steps
// X <- X + X (I - A X) where the probe exceeds kInvProbeTol (the engine's
// refine block); R and Xn are n x n scratch (R null: no probe).
// *nearly_singular (optional): the probe's condition estimate exceeds
// kSensitiveCond.
__device__ __noinline__ int zinv_refined(int n, const double2* A, double2* X, double2* ws, double2* R, double2* Xn,
                                         SmemMap& sm, bool* nearly_singular = nullptr) {
  const int bad = zinv(n, A, X, ws, sm);
  if (nearly_singular) *nearly_singular = false;
  const double2 one = make_double2(1, 0), mone = make_double2(-1, 0);
  const int nn = n * n;
  for (int k = 0; k < 2 && R; ++k) {
    double kap = 0.0;
    const double e = cta_inv_probe(n, A, X, sm.main, sm.red, &kap);
    if (k == 0 && nearly_singular && kap > kSensitiveCond) *nearly_singular = true;
    if (!(e > kInvProbeTol) || !(e <= 1.7976931348623157e308)) break;
    for (int q = threadIdx.x; q < nn; q += blockDim.x) R[q] = make_double2((q % n) == (q / n) ? 1.0 : 0.0, 0.0);
    __syncthreads();
    gemm(n, n, n, opN(A, n), opN(X, n), R, n, mone, one, sm);     // R = I - A X
    cta_copy(Xn, X, nn);
    __syncthreads();
    gemm(n, n, n, opN(X, n), opN(R, n), Xn, n, one, one, sm);     // X + X R
    cta_copy(X, Xn, nn);
    __syncthreads();
  }
  return bad;
}

// Sancho-Rubio decimation (src/contselfenergy.F90:271-340), CTA-cooperative.
// In: Ao, Bo, Co in slot 0, 2, 3 (consumed).  Out: surface GF in *go_out
// (one of the slots).  Returns a status.
__device__ __noinline__ int cta_decimation(int L, const Ws& w, double tol, int max_iter, int& ncyc, double2** go_out,
                              SmemMap& sm) {
  double2* Ao = w.slot(0);
  double2* Aos = w.slot(1);
  double2* Bo = w.slot(2);
  double2* Co = w.slot(3);
  double2* Go = w.slot(4);
  double2* X = w.slot(5);
  double2* Sf = w.slot(6);
  double2* C1 = w.slot(7);
  const int nn = L * L;
  int st = ST_OK;
  cta_copy(Aos, Ao, nn);
  __syncthreads();
  bool ok = false, done = false;
  int it;
  const double2 one = cz(1, 0), zero = cz(0, 0), mone = cz(-1, 0);
  for (it = 1; it <= max_iter; ++it) {
    if (zinv_refined(L, Ao, Go, w.inv(), w.slot(8), w.slot(9), sm)) st = ST_SINGULAR;
    gemm(L, L, L, opN(Go, L), opN(Co, L), X, L, one, zero, sm);            // GoXCo
    gemm(L, L, L, opN(Co, L), opN(X, L), C1, L, one, zero, sm, true);      // C1 = Co GoXCo
    const double mx = *sm.maxv;
    if (!(mx <= 1.7976931348623157e308)) break;   // Inf / NaN: will not converge (NOT_CONVERGED)
    if (mx <= tol) {
      if (ok) { done = true; break; }
      ok = true;
    } else {
      ok = false;
    }
    gemm(L, L, L, opN(Bo, L), opN(X, L), Sf, L, one, zero, sm);            // Self = Bo GoXCo
    for (int q = threadIdx.x; q < nn; q += blockDim.x) {
      Aos[q] = csub(Aos[q], Sf[q]);
      Ao[q] = csub(Ao[q], Sf[q]);
    }
    __syncthreads();
    gemm(L, L, L, opN(Go, L), opN(Bo, L), Sf, L, one, zero, sm);            // GoXBo
    gemm(L, L, L, opN(Bo, L), opN(Sf, L), X, L, one, zero, sm);             // B1 = Bo GoXBo
    gemm(L, L, L, opN(Co, L), opN(Sf, L), Ao, L, mone, one, sm);            // Ao -= Co GoXBo
    double2* t = Bo; Bo = X; X = t;                                         // Bo = B1
    t = Co; Co = C1; C1 = t;                                                // Co = C1
  }
  ncyc = done ? it : max_iter + 1;
  if (!done && st == ST_OK) st = ST_NOT_CONVERGED;
  if (zinv_refined(L, Aos, Go, w.inv(), w.slot(8), w.slot(9), sm)) st = ST_SINGULAR;
  *go_out = Go;
  return st;
}

// ---------------------------------------------------------------- engine kernel
// Persistent: each CTA pulls points from the queue inside engine_step() and
// runs the heavy steps it returns.  The product loop is inlined here and the
// kernel keeps nothing in registers across engine_step() (its state is in
// local memory, the shared-memory map in shared memory), so the loop is
// register-allocated as in a kernel of its own.  The inversion leaves are
// separately compiled routines (leaf_dev.cu).
__global__ void __launch_bounds__(kThreads, 2) k_engine(EngineArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ SmemMap smap;
  if (threadIdx.x == 0) {
    smap = map_smem(smem_raw, a.nmax);
    if (!a.trace) smap.tr.acc = nullptr;
    smap.inv.tr = smap.tr;
  }
  __syncthreads();
  if (a.trace && threadIdx.x < TR_NPHASE) smap.tr.acc[threadIdx.x] = 0;
  __syncthreads();
  const long long t_all = a.trace ? clock64() : 0;
  EngineCtl c;
  c.prog.pc = 0;
  c.in_inv = 0;
  c.open = -1;
  for (;;) {
    const int st = engine_step(a, c, smap);
    if (st == STEP_DONE) break;
    if (st == STEP_GEMM) {
      cta_gemm_body<OP_RT, OP_RT, EPI_RT>(reinterpret_cast<const GemmDesc*>(smap.main + kGemmDescOffset), smap.main);
    } else if (st == STEP_ROWS) {
      rows_run(c.ip, smap.main, smap.inv);
    } else if (c.ip.rpt == 1) {
      leaf_run_r1(c.ip.X, c.ip.n, c.ip.c0, c.ip.w, smap.main, smap.inv);
    } else if (c.ip.rpt == 2) {
      leaf_run_r2(c.ip.X, c.ip.n, c.ip.c0, c.ip.w, smap.main, smap.inv);
    } else {
      leaf_run_r4(c.ip.X, c.ip.n, c.ip.c0, c.ip.w, smap.main, smap.inv);
    }
  }
  if (a.trace) {
    if (threadIdx.x == 0) smap.tr.acc[TR_TOTAL] += clock64() - t_all;
    __syncthreads();
    if (threadIdx.x < TR_NPHASE) atomicAdd(a.trace + threadIdx.x, (unsigned long long)smap.tr.acc[threadIdx.x]);
  }
}

int64_t engine_slots(int mode, int nbl_max, int ncont_max) {
  int64_t s = S_SIG + ncont_max;
  if (mode == MODE_T || mode == MODE_DOS) s += nbl_max + ncont_max;   // gsmr, Gr(cb,cb)
  else if (mode == MODE_RHO) s += nbl_max + 2 * ncont_max;             // + gs per contact
  else s += 8 * (int64_t)nbl_max + ncont_max;                     // GN arrays, gs per contact
  return s;
}

int64_t engine_ws_elems(int mode, int nbl_max, int ncont_max, int nmax) {
  const int64_t Q = (int64_t)nmax * nmax;
  int64_t e = engine_slots(mode, nbl_max, ncont_max) * Q;
  if (mode == MODE_GN) e += 2 * (int64_t)nbl_max * nmax + 16;  // sigma_r, sigma_n vectors
  return e;
}

cudaError_t launch_engine(const EngineArgs& a, int grid, cudaStream_t s) {
  // the shared-memory opt-in is raised once per device and size (not per launch), so
  // a launch is a stream operation only and can be captured into a CUDA graph
  static std::mutex mu;
  static int set_bytes[64] = {0};
  const size_t smem = engine_smem_bytes(a.nmax);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64 || set_bytes[dev] < (int)smem) {
      // every size up to the largest block order, so that later launches never need it
      const int want = (int)engine_smem_bytes(kMaxOrder);
      e = cudaFuncSetAttribute(k_engine, cudaFuncAttributeMaxDynamicSharedMemorySize, want);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) set_bytes[dev] = want;
    }
  }
  k_engine<<<grid, kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- primitives
__global__ void __launch_bounds__(kThreads, 2)
    k_zgemm_batched(int m, int n, int k, double2 alpha, const double2* A, int64_t sA, const double2* B,
                    int64_t sB, double2 beta, double2* C, int64_t sC, int dagger) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemMap sm = map_smem(smem_raw, 1);
  sm.tr.acc = nullptr;
  const int b = blockIdx.x;
  Operand Ao = (dagger == 1) ? opC(A + b * sA, k) : opN(A + b * sA, m);
  Operand Bo = (dagger == 2) ? opC(B + b * sB, n) : opN(B + b * sB, k);
  const GemmDesc* d = gemm_desc_publish(m, n, k, Ao, Bo, epi_store(C + b * sC, m, alpha, beta), sm.main);
  cta_gemm_body<OP_RT, OP_RT, EPI_RT>(d, sm.main);
}

cudaError_t launch_zgemm_batched(int batch, int m, int n, int k, double2 alpha, const double2* A, int64_t sA,
                                 const double2* B, int64_t sB, double2 beta, double2* C, int64_t sC,
                                 int dagger, cudaStream_t s) {
  const size_t smem = engine_smem_bytes(1);
  cudaError_t e = cudaFuncSetAttribute(k_zgemm_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_zgemm_batched<<<batch, kThreads, smem, s>>>(m, n, k, alpha, A, sA, B, sB, beta, C, sC, dagger);
  return cudaGetLastError();
}

// per matrix: the inversion's own buffers, then two n x n refinement buffers
size_t zinv_batched_work_elems(int n) { return zinv_ws_elems(n, kSmemMain) + 2 * (size_t)n * n; }

__global__ void __launch_bounds__(kThreads, 2)
    k_zinv_batched(int n, const double2* A, double2* Ainv, int* info, double2* work, int64_t wstride) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemMap sm = map_smem(smem_raw, n);
  sm.tr.acc = nullptr;
  const int b = blockIdx.x;
  const int64_t nn = (int64_t)n * n;
  double2* wb = work ? work + b * wstride : nullptr;
  double2* R = work ? wb + zinv_ws_elems(n, kSmemMain) : nullptr;
  int inf = zinv_refined(n, A + b * nn, Ainv + b * nn, wb, R, R ? R + nn : nullptr, sm);
  if (threadIdx.x == 0 && info) info[b] = inf;
}

cudaError_t launch_zinv_batched(int batch, int n, const double2* A, double2* Ainv, int* info, double2* work,
                                cudaStream_t s) {
  const size_t smem = engine_smem_bytes(n);
  cudaError_t e = cudaFuncSetAttribute(k_zinv_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_zinv_batched<<<batch, kThreads, smem, s>>>(n, A, Ainv, info, work, (int64_t)zinv_batched_work_elems(n));
  return cudaGetLastError();
}

// Inverses of the problems map[b], b < batch (map null: b), matrices sA / sX
// complex elements apart; work holds batch slots of zinv_batched_work_elems(n).
// info[map[b]] gets the zgetrf-style singular column (0 = none).
__global__ void __launch_bounds__(kThreads, 2)
    k_zinv_mapped(int n, const double2* A, int64_t sA, double2* X, int64_t sX, const int* map, int* info,
                  double2* work, int64_t wstride, int* sens) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemMap sm = map_smem(smem_raw, n);
  sm.tr.acc = nullptr;
  const int b = blockIdx.x;
  const int p = map ? map[b] : b;
  double2* wb = work + (int64_t)b * wstride;
  double2* R = wb + zinv_ws_elems(n, kSmemMain);
  bool near_sing = false;
  int inf = zinv_refined(n, A + (int64_t)p * sA, X + (int64_t)p * sX, wb, R, R + (int64_t)n * n, sm, &near_sing);
  if (threadIdx.x == 0 && info) info[p] = inf;
  if (threadIdx.x == 0 && sens && near_sing) sens[p] = 1;
}

cudaError_t launch_zinv_mapped(int batch, int n, const double2* A, int64_t sA, double2* X, int64_t sX,
                               const int* map, int* info, double2* work, cudaStream_t s, int* sens) {
  if (batch <= 0) return cudaSuccess;
  const size_t smem = engine_smem_bytes(n);
  cudaError_t e = cudaFuncSetAttribute(k_zinv_mapped, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_zinv_mapped<<<batch, kThreads, smem, s>>>(n, A, sA, X, sX, map, info, work,
                                              (int64_t)zinv_batched_work_elems(n), sens);
  return cudaGetLastError();
}

__host__ __device__ inline size_t dec_work_elems(int n) { return (size_t)(S_INV + 3) * n * n; }
size_t decimation_batched_work_elems(int n) { return dec_work_elems(n); }

__global__ void __launch_bounds__(kThreads, 2)
    k_decimation_batched(int n, const double2* Ao, const double2* Bo, const double2* Co, double2* Go, int* ncyc,
                         double tol, int max_iter, double2* work) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemMap sm = map_smem(smem_raw, n);
  sm.tr.acc = nullptr;
  const int b = blockIdx.x;
  const int64_t nn = (int64_t)n * n;
  Ws w;
  w.base = work + (int64_t)b * dec_work_elems(n);
  w.Q = nn;
  w.ncont = 0;
  cta_copy(w.slot(0), Ao + b * nn, (int)nn);
  cta_copy(w.slot(2), Bo + b * nn, (int)nn);
  cta_copy(w.slot(3), Co + b * nn, (int)nn);
  __syncthreads();
  int nc = 0;
  double2* gs = nullptr;
  cta_decimation(n, w, tol, max_iter, nc, &gs, sm);
  cta_copy(Go + b * nn, gs, (int)nn);
  if (threadIdx.x == 0 && ncyc) ncyc[b] = nc;
}

cudaError_t launch_decimation_batched(int batch, int n, const double2* Ao, const double2* Bo, const double2* Co,
                                      double2* Go, int* ncyc, double tol, int max_iter, double2* work,
                                      cudaStream_t s) {
  const size_t smem = engine_smem_bytes(n);
  cudaError_t e =
      cudaFuncSetAttribute(k_decimation_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_decimation_batched<<<batch, kThreads, smem, s>>>(n, Ao, Bo, Co, Go, ncyc, tol, max_iter, work);
  return cudaGetLastError();
}

}  // namespace negf
