// Mixed-precision transmission solve (north-star precision form): the
// 2-contact fast path of calculate_transmissions (src/iterative.F90:1697-1713)
// for a batch of (E, k) points moved through the same steps together, so
// that every block product is one batched product on the integer tensor
// cores (launch_ozaki_zgemm: int8 digits, exact int32 accumulation, FP64
// recombination) and every block inverse one batched FP64 Gauss-Jordan
// inversion (launch_zinv_mapped).  FP64 throughout outside the products: the
// decimation's convergence test on max|C1|, the inverses, and the Caroli
// trace (whose two products are FP64 tensor-core products).
//
// Steps per batch, following the reference routine by routine:
//   surface_green + decimation      src/contselfenergy.F90:184-210, 271-340
//     (lock step over the points still iterating; a point leaves the active
//     set on its second consecutive max|C1| <= SGFACC, as the CPU rule)
//   compute_contacts / SelfEnergy   src/contselfenergy.F90:445-491, 552-566
//   build_ESH (ESH at the real E)   src/iterative.F90:1956-1982
//   calculate_gsmr_blocks(nbl, 2)   src/iterative_cpu.F90:51-124
//   Gr(1,1)                         src/iterative_cpu.F90:134-170
//   calculate_single_transmission_2_contacts   src/iterative_cpu.F90:399-470
#include <algorithm>
#include <vector>

#include "../../include/negf_b200.h"
#include "mixed.cuh"
#include "ozaki.cuh"
#include "small.cuh"

namespace negf {
namespace {

constexpr int kBlocks = 14;   // n x n complex work blocks per point (the 14th: a kept surface GF)

__device__ __forceinline__ double2 cmulm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conjm(double2 a) { return make_double2(a.x, -a.y); }

// Ao = Ec S00 - H00, Aos = Ao, Bo = Ec S01 - H01, Co = (conj(Ec) S01 - H01)^dag,
// Ec = (E + i eta) scale, for the points map[b] (map null: b)
__global__ void k_lead_init(int n, int c, const int* ids, const double* E, double eta, double scale, const int* map,
                            const DevDesc* descs, double2* Ao, double2* Aos, double2* Bo, double2* Co, int64_t Q) {
  const int p = map ? map[blockIdx.y] : blockIdx.y;
  const DevDesc& d = descs[ids[p]];
  const double2 ec = make_double2(E[p] * scale, eta * scale);
  const int64_t ol = d.olead[c], nn = (int64_t)n * n;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nn; q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % n), j = (int)(q / n);
    const int64_t qt = j + (int64_t)i * n;   // element (j, i)
    const double2 s00 = d.has_s00 ? d.s00[ol + q] : make_double2(i == j ? 1.0 : 0.0, 0.0);
    const double2 h00 = d.h00[ol + q];
    const double2 s01 = d.has_s01 ? d.s01[ol + q] : make_double2(0.0, 0.0);
    const double2 h01 = d.h01[ol + q];
    const double2 s01t = d.has_s01 ? d.s01[ol + qt] : make_double2(0.0, 0.0);
    const double2 h01t = d.h01[ol + qt];
    double2 a = cmulm(ec, s00);
    a.x -= h00.x; a.y -= h00.y;
    double2 b = cmulm(ec, s01);
    b.x -= h01.x; b.y -= h01.y;
    double2 ct = cmulm(conjm(ec), s01t);
    ct.x -= h01t.x; ct.y -= h01t.y;
    Ao[p * Q + q] = a;
    Aos[p * Q + q] = a;
    Bo[p * Q + q] = b;
    Co[p * Q + q] = conjm(ct);
  }
}

// Ao -= Self, Aos -= Self for the points of the list (its first *count
// entries when count is given)
__global__ void k_sub_self(int64_t nn, const int* list, const int* count, const double2* Self, double2* Ao,
                           double2* Aos, int64_t Q) {
  if (count && (int)blockIdx.y >= *count) return;
  const int p = list[blockIdx.y];
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nn; q += (int64_t)gridDim.x * blockDim.x) {
    const double2 s = Self[p * Q + q];
    double2 a = Ao[p * Q + q], b = Aos[p * Q + q];
    a.x -= s.x; a.y -= s.y;
    b.x -= s.x; b.y -= s.y;
    Ao[p * Q + q] = a;
    Aos[p * Q + q] = b;
  }
}

// The CPU convergence rule (src/contselfenergy.F90:300-310): a point is done
// on its second consecutive max|C1| <= tol.  Builds the list of the points
// that go on (and zeroes their max for the next iteration).  One CTA.  The
// list's length is na, or *count when count is given.
__global__ void k_dec_check(int na, const int* count, const int* list, double* mx, int* ok, int* ncyc_c, double tol,
                            int it, int* next, int* next_count, int* redo) {
  __shared__ int cnt;
  if (count) na = *count;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int b = threadIdx.x; b < na; b += blockDim.x) {
    const int p = list[b];
    const double m = mx[p];
    bool go = true;
    if (!(m <= 1.7976931348623157e308)) {   // Inf / NaN: this decimation will not converge; run it again
      go = false;
      ncyc_c[p] = it;
      redo[p] = 1;
    } else if (m <= tol) {
      if (ok[p]) {
        go = false;
        ncyc_c[p] = it;
      }
      ok[p] = 1;
    } else {
      ok[p] = 0;
    }
    if (go) {
      next[atomicAdd(&cnt, 1)] = p;
      mx[p] = 0.0;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *next_count = cnt;
}

__global__ void k_info_to_status(int nb, const int* count, const int* list, const int* info, int* status, int code) {
  if (count) nb = min(nb, *count);
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int p = list ? list[b] : b;
    if (info[p] != 0 && status[p] == 0) status[p] = code;
  }
}

// Tlc = Ec SMC - HMC (n x L), Tcl = (conj(Ec) SMC - HMC)^dag (L x n); here L = n
__global__ void k_tlc(int n, int c, const int* ids, const double* E, double eta, const DevDesc* descs,
                      double2* Tlc, double2* Tcl, int64_t Q) {
  const int p = blockIdx.y;
  const DevDesc& d = descs[ids[p]];
  const double2 ec = make_double2(E[p], eta);
  const int64_t om = d.omc[c], nn = (int64_t)n * n;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nn; q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % n), j = (int)(q / n);
    const int64_t qt = j + (int64_t)i * n;
    const double2 smc = d.has_smc ? d.smc[om + q] : make_double2(0.0, 0.0);
    const double2 hmc = d.hmc[om + q];
    double2 t = cmulm(ec, smc);
    t.x -= hmc.x; t.y -= hmc.y;
    const double2 smct = d.has_smc ? d.smc[om + qt] : make_double2(0.0, 0.0);
    const double2 hmct = d.hmc[om + qt];
    double2 u = cmulm(conjm(ec), smct);
    u.x -= hmct.x; u.y -= hmct.y;
    Tlc[p * Q + q] = t;
    Tcl[p * Q + q] = conjm(u);
  }
}

// ESH blocks at the real energy: which 0 = (i,i) minus sig (if given),
// 1 = (i,i+1), 2 = (i+1,i); i 0-based
__global__ void k_esh(int n, int which, int i, const int* ids, const double* E, const DevDesc* descs,
                      const double2* sig, double2* out, int64_t Q) {
  const int p = blockIdx.y;
  const DevDesc& d = descs[ids[p]];
  const double e = E[p];
  const int64_t nn = (int64_t)n * n;
  const int64_t off = (which == 0) ? d.od[i] : d.oo[i];
  const double2* H = (which == 0) ? d.hd : (which == 1 ? d.hu : d.hl);
  const double2* S = (which == 0) ? d.sd : (which == 1 ? d.su : d.sl);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nn; q += (int64_t)gridDim.x * blockDim.x) {
    const double2 h = H[off + q];
    double2 v;
    if (d.has_s) {
      const double2 sv = S[off + q];
      v = make_double2(e * sv.x - h.x, e * sv.y - h.y);
    } else {
      v = make_double2(-h.x, -h.y);
      if (which == 0 && (q % n) == (q / n)) v.x += e;
    }
    if (sig) {
      const double2 sg = sig[p * Q + q];
      v.x -= sg.x; v.y -= sg.y;
    }
    out[p * Q + q] = v;
  }
}

// The three ESH blocks of one sweep step in one pass: U = ESH(i,i+1),
// L = ESH(i+1,i), W = ESH(i,i) - sig (sig may be null)
__global__ void k_esh_step(int n, int i, const int* ids, const double* E, const DevDesc* descs, const double2* sig,
                           double2* U, double2* Lo, double2* W, int64_t Q) {
  const int p = blockIdx.y;
  const DevDesc& d = descs[ids[p]];
  const double e = E[p];
  const int64_t nn = (int64_t)n * n;
  const int64_t od = d.od[i], oo = d.oo[i];
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nn; q += (int64_t)gridDim.x * blockDim.x) {
    const double2 hu = d.hu[oo + q], hl = d.hl[oo + q], hd = d.hd[od + q];
    double2 u, l, w;
    if (d.has_s) {
      const double2 su = d.su[oo + q], sl = d.sl[oo + q], sd = d.sd[od + q];
      u = make_double2(e * su.x - hu.x, e * su.y - hu.y);
      l = make_double2(e * sl.x - hl.x, e * sl.y - hl.y);
      w = make_double2(e * sd.x - hd.x, e * sd.y - hd.y);
    } else {
      u = make_double2(-hu.x, -hu.y);
      l = make_double2(-hl.x, -hl.y);
      w = make_double2(-hd.x, -hd.y);
      if ((q % n) == (q / n)) w.x += e;
    }
    if (sig) {
      const double2 sg = sig[p * Q + q];
      w.x -= sg.x; w.y -= sg.y;
    }
    U[p * Q + q] = u;
    Lo[p * Q + q] = l;
    W[p * Q + q] = w;
  }
}

// Gamma = i (Sigma - Sigma^dag)   (zspectral_dns, src/sparsekit_drv.F90:2870-2890)
__global__ void k_gamma(int n, const double2* Sig, double2* Gam, int64_t Q) {
  const int p = blockIdx.y;
  const int64_t nn = (int64_t)n * n;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nn; q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % n), j = (int)(q / n);
    const double2 a = Sig[p * Q + q], b = Sig[p * Q + j + (int64_t)i * n];
    // i * (a - conj(b))
    Gam[p * Q + q] = make_double2(-(a.y + b.y), a.x - b.x);
  }
}

// T = |Re Tr[Gam i(G - G^dag)] - Re Tr[Gam G Gam G^dag]|
//   Tr[Gam A]            = sum_ij Gam_ij i (G_ji - conj(G_ij))
//   Tr[Gam G Gam G^dag]  = sum_ij M_ij conj(N_ij),  M = Gam G, N = G Gam
// (calculate_single_transmission_2_contacts, src/iterative_cpu.F90:424-464).
// One CTA per point; FP64.
__global__ void k_trace(int n, const double2* Gam, const double2* G, const double2* M, const double2* N, double* T,
                        int64_t Q) {
  const int p = blockIdx.x;
  const int64_t nn = (int64_t)n * n;
  double t1 = 0.0, t2 = 0.0;
  for (int64_t q = threadIdx.x; q < nn; q += blockDim.x) {
    const int i = (int)(q % n), j = (int)(q / n);
    const double2 g = Gam[p * Q + q];
    const double2 gji = G[p * Q + j + (int64_t)i * n], gij = G[p * Q + q];
    // A_ji = i (G_ji - conj(G_ij))
    const double2 aji = make_double2(-(gji.y + gij.y), gji.x - gij.x);
    t1 += g.x * aji.x - g.y * aji.y;
    const double2 m = M[p * Q + q], nq = N[p * Q + q];
    t2 += m.x * nq.x + m.y * nq.y;   // Re(m conj(n))
  }
  __shared__ double r1[32], r2[32];
  for (int o = 16; o > 0; o >>= 1) {
    t1 += __shfl_xor_sync(0xffffffffu, t1, o);
    t2 += __shfl_xor_sync(0xffffffffu, t2, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { r1[w] = t1; r2[w] = t2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s1 = 0.0, s2 = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { s1 += r1[k]; s2 += r2[k]; }
    T[p] = fabs(s1 - s2);
  }
}

// Points whose surface Green's function left the retarded solution: the
// diagonal of -Im gs must be >= 0 (up to 1e-6 of the largest |gs_ii|); a
// converged fixed point of the wrong kind, or one that is not finite, marks
// the point for the engine (redo[p] = 1).  One CTA per point.
__global__ void k_retarded_check(int n, const double2* gs, int64_t Q, const int* map, int* redo) {
  const int p = map ? map[blockIdx.x] : blockIdx.x;
  double lo = 1.7976931348623157e308, hi = 0.0;
  int bad = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double2 g = gs[p * Q + (int64_t)i * (n + 1)];
    const double v = -g.y, h = sqrt(g.x * g.x + g.y * g.y);
    if (!(h <= 1.7976931348623157e308)) bad = 1;
    else {
      lo = fmin(lo, v);
      hi = fmax(hi, h);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  bad = __any_sync(0xffffffffu, bad);
  __shared__ double slo[32], shi[32];
  __shared__ int sbad[32];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { slo[w] = lo; shi[w] = hi; sbad[w] = bad; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      lo = fmin(lo, slo[q]);
      hi = fmax(hi, shi[q]);
      bad |= sbad[q];
    }
    if (bad || (hi > 0.0 && lo < -1e-6 * hi)) redo[p] = 1;
  }
}

// Start of a decimation for the points map[b], b < nsub (map null: b):
// ok = 0, max = 0, ncyc = 0, sensitivity 0, the active list = the points,
// its count.
__global__ void k_dec_start(int nsub, const int* map, int* ok, double* mx, int* ncyc_c, int* list, int* count,
                            int* sens) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nsub; b += gridDim.x * blockDim.x) {
    const int p = map ? map[b] : b;
    ok[p] = 0;
    sens[p] = 0;
    mx[p] = 0.0;
    ncyc_c[p] = 0;
    list[b] = p;
  }
  if (count && blockIdx.x == 0 && threadIdx.x == 0) *count = nsub;
}

// kept_p = gs_p for the points map[b], b < nsub; one CTA per point.
__global__ void k_keep(int64_t nn, const int* map, const double2* gs, double2* kept, int64_t Q) {
  const int p = map[blockIdx.x];
  for (int64_t q = threadIdx.x; q < nn; q += blockDim.x) kept[p * Q + q] = gs[p * Q + q];
}

// agree[p] = max |gs_p - kept_p| <= tol max |kept_p| for the points map[b]; one CTA per point.
__global__ void k_agree(int64_t nn, const int* map, const double2* gs, const double2* kept, int64_t Q, double tol,
                        int* agree) {
  const int p = map[blockIdx.x];
  double d = 0.0, m = 0.0;
  for (int64_t q = threadIdx.x; q < nn; q += blockDim.x) {
    const double2 a = gs[p * Q + q], b = kept[p * Q + q];
    d = fmax(d, hypot(a.x - b.x, a.y - b.y));
    m = fmax(m, hypot(b.x, b.y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  __shared__ double sd[32], sm[32];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { sd[w] = d; sm[w] = m; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) { d = fmax(d, sd[q]); m = fmax(m, sm[q]); }
    agree[p] = (d <= tol * m) ? 1 : 0;
  }
}

// Points still flagged after the last retry: NOT_CONVERGED, ncyc = cap + 1.
__global__ void k_flag_unresolved(int P, const int* redo, int* ncyc_c, int* status, int max_iter) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
    if (redo[p]) {
      ncyc_c[p] = max_iter + 1;
      if (status[p] == 0) status[p] = NEGF_B200_ERR_NOT_CONVERGED;
    }
}


size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Carver {
  char* p;
  size_t off = 0;
  template <typename T>
  T* take(size_t n) {
    T* r = p ? reinterpret_cast<T*>(p + off) : nullptr;
    off = align256(off + n * sizeof(T));
    return r;
  }
};

struct Ws {
  double2* blk[kBlocks];
  double* mx;
  int *ok, *ncl, *ncr, *list0, *list1, *count, *info, *pst, *redo, *sub, *sens, *agree;
  double* tb;
  double2* zwork;
  void* oz;
};

Ws carve(void* base, int P, int n, int slices, size_t* total) {
  Carver c{static_cast<char*>(base)};
  Ws w;
  const size_t Q = (size_t)n * n;
  for (int b = 0; b < kBlocks; ++b) w.blk[b] = c.take<double2>((size_t)P * Q);
  w.mx = c.take<double>(P);
  w.ok = c.take<int>(P);
  w.ncl = c.take<int>(P);
  w.ncr = c.take<int>(P);
  w.list0 = c.take<int>(P);
  w.list1 = c.take<int>(P);
  w.count = c.take<int>(4);
  w.info = c.take<int>(P);
  w.pst = c.take<int>(P);
  w.tb = c.take<double>(P);
  w.redo = c.take<int>(P);
  w.sub = c.take<int>(P);
  w.sens = c.take<int>(P);
  w.agree = c.take<int>(P);
  const bool small = slices == 0;        // the lock-step FP64 form: one-warp kernels, no splitting
  w.zwork = c.take<double2>(small ? 1 : (size_t)P * zinv_batched_work_elems(n) + 1);
  w.oz = small ? nullptr : c.take<uint8_t>(ozaki_layout(P, n, n, n, slices).total);
  *total = c.off + 256;
  return w;
}

__global__ void k_finish(int P, const int* ncl, const int* ncr, const int* pst, const double* Tb, double* T,
                         int* ncyc, int* status) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    T[p] = Tb[p];
    if (ncyc) ncyc[p] = ncl[p] + ncr[p];
    // a non-finite T that no step flagged (NaN in the device blocks) is reported as such
    if (status) status[p] = (pst[p] == 0 && !isfinite(Tb[p])) ? NEGF_B200_ERR_NONFINITE : pst[p];
  }
}

__global__ void k_not_converged(int na, const int* count, const int* list, int* ncyc_c, int* pst, int max_iter) {
  if (count) na = min(na, *count);
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < na; b += gridDim.x * blockDim.x) {
    const int p = list[b];
    ncyc_c[p] = max_iter + 1;
    if (pst[p] == 0) pst[p] = NEGF_B200_ERR_NOT_CONVERGED;
  }
}

}  // namespace

size_t mixed_ws_bytes(int batch, int n, int slices) {
  size_t t = 0;
  carve(nullptr, batch, n, slices, &t);
  return t;
}

int mixed_batch_for(size_t bytes, int n, int slices) {
  int lo = 0, hi = 1 << 14;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (mixed_ws_bytes(mid, n, slices) <= bytes) lo = mid; else hi = mid - 1;
  }
  return lo;
}

int mixed_run(const MixedArgs& a, void* ws, int batch, cudaStream_t s, std::string* err) {
  const int n = a.n;
  const int64_t Q = (int64_t)n * n;
  const double2 one = make_double2(1, 0), zero = make_double2(0, 0), mone = make_double2(-1, 0);
  const bool small = a.slices == 0;
  size_t tot = 0;
  Ws w = carve(ws, batch, n, a.slices, &tot);
  double2** B = w.blk;
  const dim3 eb(256);
  const int gx = (int)std::min<int64_t>(64, (Q + 255) / 256);
  auto ck = [&](cudaError_t e, const char* what) -> int {
    if (e == cudaSuccess) return 0;
    if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
    return NEGF_B200_ERR_CUDA;
  };
#define MCK(x, what)             \
  do {                           \
    int r_ = ck((x), what);      \
    if (r_) return r_;           \
  } while (0)
  // products and inverses of the problems map[b], b < nb (or b < *count)
  uint64_t nl = 0;                 // kernels launched (reported through a.launches)
  auto prod = [&](int nb, const int* map, const int* count, double2 alpha, const double2* A, const double2* Bm,
                  double2 beta, double2* C, double* maxabs) -> cudaError_t {
    if (small) {
      ++nl;
      return launch_small_zgemm(nb, n, alpha, A, Bm, beta, C, Q, map, count, maxabs, s);
    }
    nl += 3;                       // digit split of A, of B, the product
    return launch_ozaki_zgemm(nb, n, n, n, alpha, A, Q, Bm, Q, beta, C, Q, a.slices, w.oz, maxabs, w.pst, s, map);
  };
  auto inv = [&](int nb, const int* map, const int* count, const double2* A, double2* X) -> cudaError_t {
    ++nl;
    if (small) {
      // the one-warp inversion, then its residual probe and Newton steps where needed
      cudaError_t e = launch_small_zinv(nb, n, A, X, Q, map, count, w.info, w.pst, NEGF_B200_ERR_SINGULAR, s);
      if (e != cudaSuccess) return e;
      ++nl;
      return launch_small_refine(nb, n, A, X, Q, map, count, s, w.sens);
    }
    return launch_zinv_mapped(nb, n, A, Q, X, Q, map, w.info, w.zwork, s, w.sens);   // probe and refinement inside
  };
  // FP64 products of the trace (the one-warp kernel at small orders, else the DMMA product)
  auto prod64 = [&](int nb, const double2* A, const double2* Bm, double2* C) -> cudaError_t {
    ++nl;
    if (small) return launch_small_zgemm(nb, n, one, A, Bm, zero, C, Q, nullptr, nullptr, nullptr, s);
    return launch_zgemm_batched(nb, n, n, n, one, A, Q, Bm, Q, zero, C, Q, 0, s);
  };
  // the small form runs the decimation without a host round trip per
  // iteration: the kernels read the active count on the device, and the host
  // looks at it every kPoll iterations
  constexpr int kPoll = 8;

  for (int p0 = 0; p0 < a.npts; p0 += batch) {
    const int P = std::min(batch, a.npts - p0);
    const int* ids = a.d_ids + p0;
    const double* E = a.d_E + p0;
    MCK(cudaMemsetAsync(w.pst, 0, sizeof(int) * P, s), "memset status");
    // ---- surface Green's function of each contact (B9 left, B10 right)
    // decimation of contact `side` for the points sub[b], b < nsub (sub null:
    // all P), the contact energy scaled by `scale`; then gs = Aos^-1 and the
    // retarded-branch check (redo[p] = 1 where it fails)
    auto decimate = [&](int side, const int* sub, int nsub, double scale) -> int {
      const int c = side == 0 ? a.left : a.right;
      int* ncyc_c = side == 0 ? w.ncl : w.ncr;
      double2 *Ao = B[0], *Aos = B[1], *Bo = B[2], *Co = B[3], *Go = B[4], *X = B[5], *C1 = B[6], *Y = B[7],
              *B1 = B[8];
      k_lead_init<<<dim3(gx, nsub), eb, 0, s>>>(n, c, ids, E, a.eta, scale, sub, a.d_descs, Ao, Aos, Bo, Co, Q);
      ++nl;
      MCK(cudaGetLastError(), "lead init");
      int* cnt_cur = small ? w.count : nullptr;        // device active counts (small form)
      int* cnt_nxt = small ? w.count + 1 : nullptr;
      k_dec_start<<<(nsub + 255) / 256, 256, 0, s>>>(nsub, sub, w.ok, w.mx, ncyc_c, w.list0, cnt_cur, w.sens);
      ++nl;
      int na = nsub;                                   // host bound of the active list
      int* cur = w.list0;
      int* nxt = w.list1;
      int it = 1;
      for (; it <= a.sgf_max_iter && na > 0; ++it) {
        MCK(inv(na, cur, cnt_cur, Ao, Go), "zinv");
        if (small) {
          // the rest of the iteration in one fused launch, one CTA per point
          MCK(cudaMemsetAsync(cnt_nxt, 0, sizeof(int), s), "memset count");
          MCK(launch_small_dec(na, n, cur, cnt_cur, Go, Co, Bo, C1, B1, Ao, Aos, Q, w.ok, ncyc_c, a.sgf_tol, it,
                               nxt, cnt_nxt, w.redo, s), "decimation");
          ++nl;
          std::swap(cur, nxt);
          std::swap(cnt_cur, cnt_nxt);
          std::swap(B[2], B[8]);
          std::swap(B[3], B[6]);
          Bo = B[2]; Co = B[3]; B1 = B[8]; C1 = B[6];
          if (it % kPoll == 0) {
            MCK(cudaMemcpyAsync(&na, cnt_cur, sizeof(int), cudaMemcpyDeviceToHost, s), "count");
            MCK(cudaStreamSynchronize(s), "sync");
          }
          continue;
        }
        // the mixed form: one batched product per step, the active list compacted on the host
        k_info_to_status<<<(na + 255) / 256, 256, 0, s>>>(na, nullptr, cur, w.info, w.pst, NEGF_B200_ERR_SINGULAR);
        ++nl;
        MCK(prod(na, cur, nullptr, one, Go, Co, zero, X, nullptr), "GoXCo");
        MCK(prod(na, cur, nullptr, one, Co, X, zero, C1, w.mx), "C1");
        k_dec_check<<<1, 1024, 0, s>>>(na, nullptr, cur, w.mx, w.ok, ncyc_c, a.sgf_tol, it, nxt, w.count, w.redo);
        ++nl;
        MCK(cudaGetLastError(), "check");
        std::swap(cur, nxt);
        {
          int h_count = 0;
          MCK(cudaMemcpyAsync(&h_count, w.count, sizeof(int), cudaMemcpyDeviceToHost, s), "count");
          MCK(cudaStreamSynchronize(s), "sync");
          na = h_count;
          if (na == 0) break;
        }
        MCK(prod(na, cur, nullptr, one, Bo, X, zero, B1, nullptr), "Self");
        k_sub_self<<<dim3(gx, na), eb, 0, s>>>(Q, cur, nullptr, B1, Ao, Aos, Q); ++nl;
        MCK(prod(na, cur, nullptr, one, Go, Bo, zero, Y, nullptr), "GoXBo");
        MCK(prod(na, cur, nullptr, one, Bo, Y, zero, B1, nullptr), "B1");
        MCK(prod(na, cur, nullptr, mone, Co, Y, one, Ao, nullptr), "Ao update");
        // Bo = B1, Co = C1 for every point still iterating (the others are done with them)
        std::swap(B[2], B[8]);
        std::swap(B[3], B[6]);
        Bo = B[2]; Co = B[3]; B1 = B[8]; C1 = B[6];
      }
      if (small && na > 0) {         // the loop ran to the cap: how many are left
        MCK(cudaMemcpyAsync(&na, cnt_cur, sizeof(int), cudaMemcpyDeviceToHost, s), "count");
        MCK(cudaStreamSynchronize(s), "sync");
      }
      if (na > 0) {
        k_not_converged<<<(na + 255) / 256, 256, 0, s>>>(na, cnt_cur, cur, ncyc_c, w.pst, a.sgf_max_iter);
        ++nl;
      }
      MCK(inv(nsub, sub, nullptr, Aos, B[9 + side]), "gs");
      if (!small) {
        k_info_to_status<<<(nsub + 255) / 256, 256, 0, s>>>(nsub, nullptr, sub, w.info, w.pst,
                                                              NEGF_B200_ERR_SINGULAR);
        ++nl;
      }
      if (a.eta > 0.0) {
        k_retarded_check<<<nsub, 128, 0, s>>>(n, B[9 + side], Q, sub, w.redo);
        ++nl;
      }
      return 0;
    };
    for (int side = 0; side < 2; ++side) {
      MCK(cudaMemsetAsync(w.redo, 0, sizeof(int) * P, s), "memset redo");
      if (int r = decimate(side, nullptr, P, 1.0)) return r;
      if (!(a.eta > 0.0)) continue;
      // Decimations that reached another fixed point (or ran off to Inf / NaN) run
      // again, in lock step over just those points, from the contact energy times
      // 1 + k 2^-50.  A sensitive decimation (one of its inverses needed a Newton
      // step: a nearly singular Ao) is accepted once two attempts reach the same gs.
      std::vector<int> hredo(P), hsens(P), hagree(P), kept(P, 0), done(P, 0), cur_sub, again, cmp, keep;
      cur_sub.resize(P);
      for (int p = 0; p < P; ++p) cur_sub[p] = p;
      double2* gs = B[9 + side];
      for (int att = 1;; ++att) {
        MCK(cudaMemcpyAsync(hredo.data(), w.redo, sizeof(int) * P, cudaMemcpyDeviceToHost, s), "redo");
        MCK(cudaMemcpyAsync(hsens.data(), w.sens, sizeof(int) * P, cudaMemcpyDeviceToHost, s), "sens");
        MCK(cudaStreamSynchronize(s), "sync");
        cmp.clear();
        for (int p : cur_sub)
          if (!hredo[p] && hsens[p] && kept[p]) cmp.push_back(p);
        if (!cmp.empty()) {
          MCK(cudaMemcpyAsync(w.sub, cmp.data(), sizeof(int) * cmp.size(), cudaMemcpyHostToDevice, s), "cmp");
          k_agree<<<(int)cmp.size(), 256, 0, s>>>(Q, w.sub, gs, B[13], Q, 1e-2, w.agree); ++nl;
          MCK(cudaMemcpyAsync(hagree.data(), w.agree, sizeof(int) * P, cudaMemcpyDeviceToHost, s), "agree");
          MCK(cudaStreamSynchronize(s), "sync");
        }
        again.clear();
        keep.clear();
        for (int p : cur_sub) {
          if (hredo[p]) { again.push_back(p); continue; }                  // wrong fixed point: run again
          if (!hsens[p]) continue;                                          // settled
          if (kept[p] && hagree[p]) continue;                               // two attempts agree
          keep.push_back(p);                                                // keep this gs, run again
          again.push_back(p);
        }
        if (again.empty()) break;
        if (att > kDecRetries) {
          for (int p : again) hredo[p] = 1;
          MCK(cudaMemcpyAsync(w.redo, hredo.data(), sizeof(int) * P, cudaMemcpyHostToDevice, s), "redo");
          k_flag_unresolved<<<(P + 255) / 256, 256, 0, s>>>(P, w.redo, side == 0 ? w.ncl : w.ncr, w.pst,
                                                              a.sgf_max_iter);
          ++nl;
          MCK(cudaStreamSynchronize(s), "sync");
          break;
        }
        if (!keep.empty()) {
          MCK(cudaMemcpyAsync(w.sub, keep.data(), sizeof(int) * keep.size(), cudaMemcpyHostToDevice, s), "keep");
          k_keep<<<(int)keep.size(), 256, 0, s>>>(Q, w.sub, gs, B[13], Q); ++nl;
          for (int p : keep) kept[p] = 1;
        }
        MCK(cudaMemcpyAsync(w.sub, again.data(), sizeof(int) * again.size(), cudaMemcpyHostToDevice, s), "sub");
        MCK(cudaMemsetAsync(w.redo, 0, sizeof(int) * P, s), "memset redo");
        if (int r = decimate(side, w.sub, (int)again.size(), 1.0 + att * 0x1p-50)) return r;
        cur_sub = again;
        MCK(cudaStreamSynchronize(s), "sync");   // the host vectors above are reused next round
      }
    }
    // ---- self-energies Sigma_c = Tlc gs Tcl (B11 left, B12 right)
    for (int side = 0; side < 2; ++side) {
      const int c = side == 0 ? a.left : a.right;
      k_tlc<<<dim3(gx, P), eb, 0, s>>>(n, c, ids, E, a.eta, a.d_descs, B[0], B[1], Q); ++nl;
      MCK(cudaGetLastError(), "tlc");
      MCK(prod(P, nullptr, nullptr, one, B[0], B[9 + side], zero, B[2], nullptr), "Tlc gs");
      MCK(prod(P, nullptr, nullptr, one, B[2], B[1], zero, B[11 + side], nullptr), "Sigma");
    }
    // ---- gsmr sweep from block nbl down to 2, then Gr(1,1)
    double2 *g = B[4], *X = B[5], *W = B[6], *U = B[7], *Lb = B[8];
    k_esh<<<dim3(gx, P), eb, 0, s>>>(n, 0, a.nbl - 1, ids, E, a.d_descs, B[12], W, Q); ++nl;
    MCK(inv(P, nullptr, nullptr, W, g), "gsmr N");
    if (!small) {
      k_info_to_status<<<(P + 255) / 256, 256, 0, s>>>(P, nullptr, nullptr, w.info, w.pst, NEGF_B200_ERR_SINGULAR);
      ++nl;
    }
    for (int i = a.nbl - 2; i >= 0; --i) {
      // W = ESH(i,i) - ESH(i,i+1) gsmr(i+1) ESH(i+1,i)  (block i 0-based; Sigma_left on block 0)
      k_esh_step<<<dim3(gx, P), eb, 0, s>>>(n, i, ids, E, a.d_descs, i == 0 ? B[11] : nullptr, U, Lb, W, Q); ++nl;
      MCK(cudaGetLastError(), "esh");
      MCK(prod(P, nullptr, nullptr, one, U, g, zero, X, nullptr), "U g");
      MCK(prod(P, nullptr, nullptr, mone, X, Lb, one, W, nullptr), "W");
      MCK(inv(P, nullptr, nullptr, W, g), "gsmr");
      if (!small) {
        k_info_to_status<<<(P + 255) / 256, 256, 0, s>>>(P, nullptr, nullptr, w.info, w.pst, NEGF_B200_ERR_SINGULAR);
        ++nl;
      }
    }
    // g = Gr(1,1).  Trace with Gamma of the contact on block 1 (FP64 products)
    k_gamma<<<dim3(gx, P), eb, 0, s>>>(n, B[11], B[0], Q); ++nl;
    MCK(prod64(P, B[0], g, B[1]), "Gam G");
    MCK(prod64(P, g, B[0], B[2]), "G Gam");
    k_trace<<<P, 512, 0, s>>>(n, B[0], g, B[1], B[2], w.tb, Q); ++nl;
    MCK(cudaGetLastError(), "trace");
    k_finish<<<(P + 255) / 256, 256, 0, s>>>(P, w.ncl, w.ncr, w.pst, w.tb, a.d_T + p0,
                                             a.d_ncyc ? a.d_ncyc + p0 : nullptr,
                                             a.d_status ? a.d_status + p0 : nullptr); ++nl;
    MCK(cudaGetLastError(), "finish");
  }
#undef MCK
  if (a.launches) *a.launches += nl;
  return NEGF_B200_OK;
}

}  // namespace negf
