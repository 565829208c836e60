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
#include "cta_ops.cuh"
#include "engine.cuh"

namespace negf {

static_assert(kGemmSmemBytes <= kSmemMain, "GEMM staging ring must fit the main shared-memory region");
static_assert((kSmallInvMax * kSmallInvMax + 3 * kSmallInvMax) * 16 <= kSmemMain,
              "small inversion must fit the main shared-memory region");

// ---------------------------------------------------------------- smem map
struct SmemMap {
  double2* main;
  InvScratch inv;
  double* red;
  double* maxv;
  int* item;
  Trace tr;
};

__device__ __forceinline__ SmemMap map_smem(char* base, int nmax) {
  SmemMap m;
  m.main = reinterpret_cast<double2*>(base);
  char* p = base + kSmemMain;
  m.red = reinterpret_cast<double*>(p); p += 32 * sizeof(double);
  m.maxv = reinterpret_cast<double*>(p); p += 2 * sizeof(double);
  m.inv.redv = reinterpret_cast<double*>(p); p += 32 * sizeof(double);
  m.inv.redi = reinterpret_cast<int*>(p); p += 32 * sizeof(int);
  m.inv.flag = reinterpret_cast<int*>(p); p += 4 * sizeof(int);
  m.item = reinterpret_cast<int*>(p); p += 4 * sizeof(int);
  m.inv.piv = reinterpret_cast<int*>(p); p += nmax * sizeof(int);
  m.inv.perm = reinterpret_cast<int*>(p); p += nmax * sizeof(int);
  m.inv.cperm = reinterpret_cast<int*>(p); p += nmax * sizeof(int);
  p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 7) & ~uintptr_t(7));
  m.tr.acc = reinterpret_cast<long long*>(p);   // TR_NPHASE entries; enabled by the caller
  m.inv.tr.acc = nullptr;
  return m;
}

size_t engine_smem_bytes(int nmax) {
  return kSmemMain + 32 * 8 + 2 * 8 + 32 * 8 + 32 * 4 + 4 * 4 + 4 * 4 + 3 * (size_t)nmax * 4 + 8 +
         TR_NPHASE * 8;
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double2 cz(double re, double im) { return make_double2(re, im); }

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
  return cta_zinv(n, A, out, ws, sm.main, kSmemMain, sm.inv);
}

// Slots of the per-CTA workspace
enum : int {
  S_DEC0 = 0,       // 8 decimation buffers (also sweep scratch 0..11)
  S_SCR = 0,
  N_SCR = 12,
  S_INV = 12,       // 3 slots of inversion workspace
  S_SIG = 15,       // kMaxCont contact self-energies follow
};

struct Ws {
  double2* base;
  int64_t Q;
  int ncont;
  __device__ double2* slot(int k) const { return base + (int64_t)k * Q; }
  __device__ double2* inv() const { return slot(S_INV); }
  __device__ double2* sig(int c) const { return slot(S_SIG + c); }
  __device__ double2* layer(int arr, int i, int nbl) const {  // arr-th per-layer array
    return slot(S_SIG + ncont + arr * nbl + i);
  }
};

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
    if (zinv(L, Ao, Go, w.inv(), sm)) st = ST_SINGULAR;
    gemm(L, L, L, opN(Go, L), opN(Co, L), X, L, one, zero, sm);            // GoXCo
    gemm(L, L, L, opN(Co, L), opN(X, L), C1, L, one, zero, sm, true);      // C1 = Co GoXCo
    const double mx = *sm.maxv;
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
  if (zinv(L, Aos, Go, w.inv(), sm)) st = ST_SINGULAR;
  *go_out = Go;
  return st;
}

// ESH(i,i) = ec*S(i,i) - H(i,i) - Sigma_c (contacts on block i) - diag(sigr)
__device__ void esh_diag(const DevDesc& d, int i, double2 ec, double2* dst, const Ws& w, bool with_sigma,
                         const double2* sigr, const Trace& tr) {
  long long t0 = tr.start();
  const int n = d.pl[i];
  const double2* H = d.hd + d.od[i];
  const double2* S = d.has_s ? d.sd + d.od[i] : nullptr;
  const double2* sub = nullptr;
  int first = -1;
  if (with_sigma)
    for (int c = 0; c < d.ncont; ++c)
      if (d.cblk[c] == i + 1) { first = c; sub = w.sig(c); break; }
  cta_esh(dst, n, n, H, S, ec, true, sub, sigr ? sigr + d.pstart[i] : nullptr, OP_N);
  __syncthreads();
  if (first >= 0)
    for (int c = first + 1; c < d.ncont; ++c)
      if (d.cblk[c] == i + 1) {
        const double2* sg = w.sig(c);
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) dst[q] = csub(dst[q], sg[q]);
        __syncthreads();
      }
  tr.stop(TR_ELEM, t0);
}
// ESH(i,i+1): n_i x n_{i+1}
__device__ void esh_up(const DevDesc& d, int i, double2 ec, double2* dst) {
  cta_esh(dst, d.pl[i], d.pl[i + 1], d.hu + d.oo[i], d.has_s ? d.su + d.oo[i] : nullptr, ec, false, nullptr,
          nullptr, OP_N);
}
// ESH(i+1,i): n_{i+1} x n_i
__device__ void esh_lo(const DevDesc& d, int i, double2 ec, double2* dst) {
  cta_esh(dst, d.pl[i + 1], d.pl[i], d.hl + d.oo[i], d.has_s ? d.sl + d.oo[i] : nullptr, ec, false, nullptr,
          nullptr, OP_N);
}

// Contact surface GFs and self-energies (compute_contacts_dns,
// src/contselfenergy.F90:445-491).  Sigma_c -> w.sig(c).  ncyc_max receives
// the total decimation iterations over all contacts (the reference prints
// their average, src/integrations.F90:1751).
__device__ __noinline__ int contacts(const DevDesc& d, double2 ec, const Ws& w, double tol, int max_iter, int& ncyc_max,
                        SmemMap& sm) {
  int st = ST_OK;
  ncyc_max = 0;
  const double2 ecc = cconj(ec);
  const double2 one = cz(1, 0), zero = cz(0, 0);
  for (int c = 0; c < d.ncont; ++c) {
    const int L = d.L[c];
    const int ncb = d.pl[d.cblk[c] - 1];
    const double2* h00 = d.h00 + d.olead[c];
    const double2* h01 = d.h01 + d.olead[c];
    const double2* s00 = d.has_s00 ? d.s00 + d.olead[c] : nullptr;
    const double2* s01 = d.has_s01 ? d.s01 + d.olead[c] : nullptr;
    cta_esh(w.slot(0), L, L, h00, s00, ec, true, nullptr, nullptr, OP_N);    // Ao
    cta_esh(w.slot(2), L, L, h01, s01, ec, false, nullptr, nullptr, OP_N);   // Bo
    cta_esh(w.slot(3), L, L, h01, s01, ecc, false, nullptr, nullptr, OP_C);  // Co = (E* S01 - H01)^dag
    __syncthreads();
    int ncyc = 0;
    double2* gs = nullptr;
    int s1 = cta_decimation(L, w, tol, max_iter, ncyc, &gs, sm);
    if (st == ST_OK) st = s1;
    ncyc_max += ncyc;   // total over contacts
    // Tlc = E*SMC - HMC (ncb x L), Tcl = (E^* SMC - HMC)^dag (L x ncb)
    const double2* hmc = d.hmc + d.omc[c];
    const double2* smc = d.has_smc ? d.smc + d.omc[c] : nullptr;
    double2* Tlc = w.slot(0);
    double2* Tcl = w.slot(1);
    double2* TG = w.slot(2);
    cta_esh(Tlc, ncb, L, hmc, smc, ec, false, nullptr, nullptr, OP_N);
    cta_esh(Tcl, L, ncb, hmc, smc, ecc, false, nullptr, nullptr, OP_C);
    __syncthreads();
    gemm(ncb, L, L, opN(Tlc, ncb), opN(gs, L), TG, ncb, one, zero, sm);
    gemm(ncb, ncb, L, opN(TG, ncb), opN(Tcl, L), w.sig(c), ncb, one, zero, sm);
  }
  return st;
}

// gsmr(N-1 .. lo) backward sweep (calculate_gsmr_blocks).  If keep, gsmr(i)
// goes to w.layer(0, i); else the last one computed is returned in *gout.
// ec: energy of ES-H; sigr: dephasing sigma_r (or null).
__device__ __noinline__ int gsmr_sweep(const DevDesc& d, double2 ec, const Ws& w, int lo, bool keep, const double2* sigr,
                          double2** gout, SmemMap& sm) {
  const int N = d.nbl;
  int st = ST_OK;
  double2* E0 = w.slot(0);
  double2* E1 = w.slot(1);
  double2* E2 = w.slot(2);
  double2* W = w.slot(3);
  double2* G[2] = {w.slot(4), w.slot(5)};
  const double2 one = cz(1, 0), zero = cz(0, 0), mone = cz(-1, 0);
  esh_diag(d, N - 1, ec, E0, w, true, sigr, sm.tr);
  double2* gnext = keep ? w.layer(0, N - 1, N) : G[0];
  if (zinv(d.pl[N - 1], E0, gnext, w.inv(), sm)) st = ST_SINGULAR;
  int pp = 1;
  for (int i = N - 2; i >= lo; --i) {
    const int ni = d.pl[i], nj = d.pl[i + 1];
    esh_up(d, i, ec, E1);
    esh_lo(d, i, ec, E2);
    esh_diag(d, i, ec, E0, w, true, sigr, sm.tr);   // ends with a barrier
    gemm(ni, nj, nj, opN(E1, ni), opN(gnext, nj), W, ni, mone, zero, sm);      // -ESH(i,i+1) gsmr(i+1)
    gemm(ni, ni, nj, opN(W, ni), opN(E2, nj), E0, ni, one, one, sm);           // ESH(i,i) + W ESH(i+1,i)
    double2* gcur = keep ? w.layer(0, i, N) : G[pp];
    pp ^= 1;
    if (zinv(ni, E0, gcur, w.inv(), sm)) st = ST_SINGULAR;
    gnext = gcur;
  }
  *gout = gnext;
  return st;
}

// Gr(1,1) = [ESH(1,1) - ESH(1,2) gsmr(2) ESH(2,1)]^-1 -> out
__device__ __noinline__ int gr_first(const DevDesc& d, double2 ec, const Ws& w, const double2* g2, const double2* sigr,
                        double2* out, SmemMap& sm) {
  const int n0 = d.pl[0];
  double2* E0 = w.slot(0);
  double2* E1 = w.slot(1);
  double2* E2 = w.slot(2);
  double2* W = w.slot(3);
  const double2 one = cz(1, 0), zero = cz(0, 0), mone = cz(-1, 0);
  esh_diag(d, 0, ec, E0, w, true, sigr, sm.tr);
  if (d.nbl > 1) {
    const int n1 = d.pl[1];
    esh_up(d, 0, ec, E1);
    esh_lo(d, 0, ec, E2);
    __syncthreads();
    gemm(n0, n1, n1, opN(E1, n0), opN(g2, n1), W, n0, one, zero, sm);
    gemm(n0, n0, n1, opN(W, n0), opN(E2, n1), E0, n0, mone, one, sm);
  }
  return zinv(n0, E0, out, w.inv(), sm) ? ST_SINGULAR : ST_OK;
}

// One forward step of the retarded sweep (calculate_Gr_tridiag_blocks):
// Gr(i,i-1) -> gl (if non-null), Gr(i-1,i) -> gu (if non-null),
// Gr(i,i) -> gd.  E1/E2/X/W2/GL scratch from slots 0..4 (not the inputs).
__device__ __noinline__ void gr_step(const DevDesc& d, double2 ec, int i, const double2* gsm_i, const double2* gprev,
                        double2* gd, double2* gu, double2* gl_out, const Ws& w, SmemMap& sm) {
  const int ni = d.pl[i], np = d.pl[i - 1];
  double2* E1 = w.slot(0);   // ESH(i-1,i)  np x ni
  double2* E2 = w.slot(1);   // ESH(i,i-1)  ni x np
  double2* X = w.slot(2);
  double2* W2 = w.slot(3);
  double2* GL = gl_out ? gl_out : w.slot(6);
  const double2 one = cz(1, 0), zero = cz(0, 0), mone = cz(-1, 0);
  esh_up(d, i - 1, ec, E1);
  esh_lo(d, i - 1, ec, E2);
  __syncthreads();
  gemm(ni, np, ni, opN(gsm_i, ni), opN(E2, ni), X, ni, one, zero, sm);         // gsmr(i) ESH(i,i-1)
  gemm(ni, np, np, opN(X, ni), opN(gprev, np), GL, ni, mone, zero, sm);       // Gr(i,i-1)
  gemm(np, ni, ni, opN(E1, np), opN(gsm_i, ni), W2, np, one, zero, sm);        // ESH(i-1,i) gsmr(i)
  if (gu) gemm(np, ni, np, opN(gprev, np), opN(W2, np), gu, np, mone, zero, sm);  // Gr(i-1,i)
  cta_copy(gd, gsm_i, ni * ni);
  __syncthreads();
  gemm(ni, ni, np, opN(GL, ni), opN(W2, np), gd, ni, mone, one, sm);           // Gr(i,i)
}

// |Re Tr[Gam1 i(G - G^dag) - Gam1 G Gam1 G^dag]|  (2-contact form)
__device__ __noinline__ double trans2(int n, const double2* sig1, const double2* G, const Ws& w, SmemMap& sm) {
  // scratch avoids slots 6, 9, 10, 11 (where G may live) and 12-14 (inversion)
  double2* Gam = w.slot(7);
  double2* W1 = w.slot(8);
  double2* W2 = w.slot(2);
  double2* A = w.slot(3);
  const double2 one = cz(1, 0), zero = cz(0, 0);
  cta_spectral(Gam, sig1, n);
  cta_spectral(A, G, n);
  __syncthreads();
  gemm(n, n, n, opN(Gam, n), opN(G, n), W1, n, one, zero, sm);
  gemm(n, n, n, opN(W1, n), opN(Gam, n), W2, n, one, zero, sm);
  double t2 = cta_re_trace_prod(W2, G, n, OP_C, sm.red);   // Tr(Gam G Gam G^dag)
  double t1 = cta_re_trace_prod(Gam, A, n, OP_N, sm.red);  // Tr(Gam A)
  return fabs(t1 - t2);
}

// |Re Tr[Gam2 G21 Gam1 G21^dag]|  (N-contact form)
__device__ __noinline__ double transN(int n2, int n1, const double2* sig2, const double2* sig1, const double2* G21,
                         const Ws& w, SmemMap& sm) {
  // scratch avoids slots 6 and 9 (where G21 may live)
  double2* Gam1 = w.slot(7);
  double2* Gam2 = w.slot(8);
  double2* W1 = w.slot(2);
  double2* W2 = w.slot(3);
  const double2 one = cz(1, 0), zero = cz(0, 0);
  cta_spectral(Gam1, sig1, n1);
  cta_spectral(Gam2, sig2, n2);
  __syncthreads();
  gemm(n2, n1, n2, opN(Gam2, n2), opN(G21, n2), W1, n2, one, zero, sm);
  gemm(n2, n1, n1, opN(W1, n2), opN(Gam1, n1), W2, n2, one, zero, sm);
  // Tr(W2 G21^dag): W2 is n2 x n1, G21^dag is n1 x n2
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < n2 * n1; idx += blockDim.x) {
    const int r = idx % n2, c = idx / n2;     // W2(r,c) * conj(G21(r,c))
    double2 x = W2[idx], y = G21[(size_t)r + (size_t)c * n2];
    acc += x.x * y.x + x.y * y.y;
  }
  return fabs(cta_sum(acc, sm.red));
}

// Complex trace of X*op(Y): X is n x m, op(Y) is m x n
__device__ double2 cta_trace_prod_c(const double2* X, const double2* Y, int n, int m, int opY, double* red) {
  double re = 0.0, im = 0.0;
  for (int idx = threadIdx.x; idx < n * m; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;   // X(i,j) * opY(j,i)
    double2 x = X[idx];
    double2 y = (opY == OP_C) ? cconj(Y[(size_t)i + (size_t)j * n]) : Y[(size_t)j + (size_t)i * m];
    re += x.x * y.x - x.y * y.y;
    im += x.x * y.y + x.y * y.x;
  }
  re = cta_sum(re, red);
  im = cta_sum(im, red);
  return cz(re, im);
}

__device__ void put_status(int* st, int s) { if (*st == ST_OK) *st = s; }

// ---------------------------------------------------------------- point solves
__device__ __noinline__ void solve_T(const EngineArgs& a, const DevDesc& d, double E, int p, const Ws& w, SmemMap& sm) {
  int st = ST_OK, ncyc = 0;
  const double2 ec_sig = cz(E, a.eta);
  const double2 ec = (a.mode == MODE_DOS) ? cz(E, a.dos_delta) : cz(E, 0.0);
  put_status(&st, contacts(d, ec_sig, w, a.sgf_tol, a.sgf_max_iter, ncyc, sm));
  const int N = d.nbl;
  double T = 0.0;
  const int ni = a.ni - 1, nf = a.nf - 1;
  const int cbi = d.cblk[ni], cbf = d.cblk[nf];
  const int ct1 = (cbi < cbf) ? ni : nf;
  const int ct2 = (cbi < cbf) ? nf : ni;
  const int bl1 = d.cblk[ct1], bl2 = d.cblk[ct2];
  const bool fast = (a.mode == MODE_T) && d.ncont == 2 && min(cbi, cbf) == 1;
  double2* G11 = w.slot(11);
  if (d.ncont == 1 && a.mode == MODE_T) {
    T = 0.0;
  } else if (fast) {
    double2* g2 = nullptr;
    if (N > 1) put_status(&st, gsmr_sweep(d, ec, w, 1, false, nullptr, &g2, sm));
    put_status(&st, gr_first(d, ec, w, g2, nullptr, G11, sm));
    T = trans2(d.pl[0], w.sig(ct1), G11, w, sm);
  } else {
    // gsmr kept for every layer; retarded sweep as far as needed
    double2* g2 = nullptr;
    if (N > 1) put_status(&st, gsmr_sweep(d, ec, w, 1, true, nullptr, &g2, sm));
    double2* Gd[2] = {w.slot(11), w.slot(10)};   // ping-pong Gr(i,i); slot 10 free until trans*
    double2* Gkeep = w.slot(9);
    put_status(&st, gr_first(d, ec, w, g2, nullptr, Gd[0], sm));
    int cur = 0;
    const int last = (a.mode == MODE_DOS) ? N - 1 : bl1 - 1;
    const double pi = 3.14159265358979323846;
    for (int i = 0; i <= last; ++i) {
      if (i > 0) {
        gr_step(d, ec, i, w.layer(0, i, N), Gd[cur], Gd[cur ^ 1], nullptr, nullptr, w, sm);
        cur ^= 1;
      }
      if (a.mode == MODE_DOS && a.dos) {
        const int n = d.pl[i];
        for (int k = threadIdx.x; k < n; k += blockDim.x)
          a.dos[(int64_t)p * a.dos_stride + d.pstart[i] + k] = -(1.0 / pi) * Gd[cur][(size_t)k + (size_t)k * n].y;
      }
      if (i == bl1 - 1) {
        cta_copy(Gkeep, Gd[cur], d.pl[i] * d.pl[i]);
        __syncthreads();
      }
    }
    if (d.ncont == 1) {
      T = 0.0;
    } else if (a.mode == MODE_DOS && d.ncont == 2) {
      T = trans2(d.pl[bl1 - 1], w.sig(ct1), Gkeep, w, sm);
    } else {
      // column sweep Gr(i,bl1), i = bl1+1..bl2 (src/iterative_cpu.F90:507-538)
      double2* col[2] = {Gkeep, w.slot(6)};
      int cc = 0;
      bool tiny = false;
      const double2 one = cz(1, 0), zero = cz(0, 0), mone = cz(-1, 0);
      for (int i = bl1; i <= bl2 - 1 && !tiny; ++i) {   // 0-based row block i
        const int nr = d.pl[i], np = d.pl[i - 1], nc = d.pl[bl1 - 1];
        // max|Gr(i-1,bl1)| < EPS -> T = EPS^2
        double mx = 0.0;
        for (int q = threadIdx.x; q < np * nc; q += blockDim.x) mx = fmax(mx, cabs(col[cc][q]));
        mx = cta_max(mx, sm.red);
        if (mx < a.eps) { tiny = true; break; }
        double2* E2 = w.slot(0);
        double2* X = w.slot(1);
        esh_lo(d, i - 1, ec, E2);
        __syncthreads();
        gemm(nr, np, nr, opN(w.layer(0, i, N), nr), opN(E2, nr), X, nr, mone, zero, sm);
        gemm(nr, nc, np, opN(X, nr), opN(col[cc], np), col[cc ^ 1], nr, one, zero, sm);
        cc ^= 1;
      }
      if (tiny) T = a.eps * a.eps;
      else T = transN(d.pl[bl2 - 1], d.pl[bl1 - 1], w.sig(ct2), w.sig(ct1), col[cc], w, sm);
    }
  }
  if (!isfinite(T)) put_status(&st, ST_NONFINITE);
  if (threadIdx.x == 0) {
    if (a.T) a.T[p] = T;
    if (a.ncyc) a.ncyc[p] = ncyc;
    if (a.status) a.status[p] = st;
  }
}

// Elastic dephasing SCBA + Meir-Wingreen + layer currents (MODE_GN).
// Per-layer arrays: 0 gsmr, 1 Gr(i,i), 2 Gr(i,i+1), 3 Sigma_n(i,i),
// 4/5 Gn(i,i) (ping-pong), 6/7 Gn(i,i+1) (ping-pong).
__device__ __noinline__ void solve_GN(const EngineArgs& a, const DevDesc& d, double E, int p, const Ws& w,
                         double2* vec, SmemMap& sm) {
  int st = ST_OK, ncyc = 0;
  const int N = d.nbl, norb = d.norb, ncont = d.ncont;
  const double2 ec = cz(E, 0.0);
  put_status(&st, contacts(d, cz(E, a.eta), w, a.sgf_tol, a.sgf_max_iter, ncyc, sm));
  const double2 one = cz(1, 0), zero = cz(0, 0), mone = cz(-1, 0);
  double2* sigr = vec;            // norb
  double2* sign = vec + norb;     // norb
  const double* cpl = a.coupling;
  const double* frm = a.frm + (int64_t)p * a.frm_stride;
  int it = 0;
  bool conv = false, have_old = false;
  double err = 0.0;
  int par = 0;
  while (!conv && it <= a.scba_niter) {
    const double2* sr = (it > 0 && cpl) ? sigr : nullptr;
    double2* g2 = nullptr;
    put_status(&st, gsmr_sweep(d, ec, w, 1, true, sr, &g2, sm));
    put_status(&st, gr_first(d, ec, w, g2, sr, w.layer(1, 0, N), sm));
    for (int i = 1; i < N; ++i)
      gr_step(d, ec, i, w.layer(0, i, N), w.layer(1, i - 1, N), w.layer(1, i, N), w.layer(2, i - 1, N),
              nullptr, w, sm);
    // set_Gr: sigma_r = D * diag(Gr)
    if (cpl) {
      for (int i = 0; i < N; ++i) {
        const int n = d.pl[i];
        const double2* G = w.layer(1, i, N);
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
          const double c = cpl[d.pstart[i] + k];
          sigr[d.pstart[i] + k] = cscale(c * c, G[(size_t)k + (size_t)k * n]);
        }
      }
    }
    // Sigma_n(i,i): dephasing (it > 0) + contacts (f_c - f_ref) Gam_c, f_ref = 0
    for (int i = 0; i < N; ++i) {
      const int n = d.pl[i];
      double2* Sn = w.layer(3, i, N);
      for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int r = q % n, c = q / n;
        Sn[q] = (it > 0 && cpl && r == c) ? sign[d.pstart[i] + r] : zero;
      }
    }
    __syncthreads();
    for (int c = 0; c < ncont; ++c) {
      const double fd = frm[c];
      if (fabs(fd) > a.eps) {
        const int cb = d.cblk[c] - 1, n = d.pl[cb];
        double2* Sn = w.layer(3, cb, N);
        const double2* sg = w.sig(c);
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
          const int r = q % n, cc = q / n;
          double2 a1 = sg[q], b1 = cconj(sg[(size_t)cc + (size_t)r * n]);
          double2 gam = cz(-(a1.y - b1.y), a1.x - b1.x);   // i (S - S^dag)
          Sn[q] = cadd(Sn[q], cscale(fd, gam));
        }
        __syncthreads();
      }
    }
    // upward fold of Sigma_n (calculate_sigma_n); off-diagonal Sigma_n are 0
    double2* gns = w.slot(6);
    double2* T1 = w.slot(7);
    double2* E1 = w.slot(8);
    {
      const int n = d.pl[N - 1];
      gemm(n, n, n, opN(w.layer(0, N - 1, N), n), opN(w.layer(3, N - 1, N), n), T1, n, one, zero, sm);
      gemm(n, n, n, opN(T1, n), opC(w.layer(0, N - 1, N), n), gns, n, one, zero, sm);
    }
    for (int i = N - 2; i >= 0; --i) {
      const int ni = d.pl[i], nj = d.pl[i + 1];
      esh_up(d, i, ec, E1);
      __syncthreads();
      gemm(ni, nj, nj, opN(E1, ni), opN(gns, nj), T1, ni, one, zero, sm);
      gemm(ni, ni, nj, opN(T1, ni), opC(E1, ni), w.layer(3, i, N), ni, one, one, sm);
      if (i > 0) {
        gemm(ni, ni, ni, opN(w.layer(0, i, N), ni), opN(w.layer(3, i, N), ni), T1, ni, one, zero, sm);
        gemm(ni, ni, ni, opN(T1, ni), opC(w.layer(0, i, N), ni), gns, ni, one, zero, sm);
      }
    }
    // Gn(1,1) = Gr(1,1) Sigma_n(1,1) Gr(1,1)^dag
    double2* gnd0 = w.layer(4 + par, 0, N);
    {
      const int n = d.pl[0];
      gemm(n, n, n, opN(w.layer(3, 0, N), n), opC(w.layer(1, 0, N), n), T1, n, one, zero, sm);
      gemm(n, n, n, opN(w.layer(1, 0, N), n), opN(T1, n), gnd0, n, one, zero, sm);
    }
    double2* E2 = w.slot(9);
    for (int i = 0; i + 1 < N; ++i) {
      const int ni = d.pl[i], nj = d.pl[i + 1];
      double2* gnl = w.slot(10);                      // Gn(i+1,i)
      double2* gnu = w.layer(6 + par, i, N);          // Gn(i,i+1)
      double2* gdi = w.layer(4 + par, i, N);
      double2* gdj = w.layer(4 + par, i + 1, N);
      esh_lo(d, i, ec, E2);
      __syncthreads();
      // W1 = Sn(i+1,i+1) Gr(i,i+1)^dag - ESH(i+1,i) Gn(i,i)
      gemm(nj, ni, nj, opN(w.layer(3, i + 1, N), nj), opC(w.layer(2, i, N), ni), T1, nj, one, zero, sm);
      gemm(nj, ni, ni, opN(E2, nj), opN(gdi, ni), T1, nj, mone, one, sm);
      gemm(nj, ni, nj, opN(w.layer(0, i + 1, N), nj), opN(T1, nj), gnl, nj, one, zero, sm);
      // Gn(i,i+1) = Gn(i+1,i)^dag
      for (int q = threadIdx.x; q < ni * nj; q += blockDim.x) {
        const int r = q % ni, c = q / ni;
        gnu[q] = cconj(gnl[(size_t)c + (size_t)r * nj]);
      }
      __syncthreads();
      // W1 = Sn(i+1,i+1) Gr(i+1,i+1)^dag - ESH(i+1,i) Gn(i,i+1)
      gemm(nj, nj, nj, opN(w.layer(3, i + 1, N), nj), opC(w.layer(1, i + 1, N), nj), T1, nj, one, zero, sm);
      gemm(nj, nj, ni, opN(E2, nj), opN(gnu, ni), T1, nj, mone, one, sm);
      gemm(nj, nj, nj, opN(w.layer(0, i + 1, N), nj), opN(T1, nj), gdj, nj, one, zero, sm);
    }
    // set_Gn: sigma_n = D * diag(Gn); SCBA error on the S pattern
    double e = 0.0;
    for (int i = 0; i < N; ++i) {
      const int n = d.pl[i];
      const double2* G = w.layer(4 + par, i, N);
      const double2* Go = w.layer(4 + (par ^ 1), i, N);
      if (have_old) {
        if (!d.has_s) {
          for (int k = threadIdx.x; k < n; k += blockDim.x)
            e = fmax(e, cabs(csub(G[(size_t)k * (n + 1)], Go[(size_t)k * (n + 1)])));
        } else {
          const double2* S = d.sd + d.od[i];
          for (int q = threadIdx.x; q < n * n; q += blockDim.x)
            if (S[q].x != 0.0 || S[q].y != 0.0) e = fmax(e, cabs(csub(G[q], Go[q])));
          if (i + 1 < N) {
            const int nj = d.pl[i + 1];
            const double2* U = w.layer(6 + par, i, N);
            const double2* Uo = w.layer(6 + (par ^ 1), i, N);
            const double2* Su = d.su + d.oo[i];
            const double2* Sl = d.sl + d.oo[i];
            for (int q = threadIdx.x; q < n * nj; q += blockDim.x) {
              const int r = q % n, c = q / n;
              const double diff = cabs(csub(U[q], Uo[q]));   // |Gn(i,i+1)| diff == |Gn(i+1,i)| diff at (c,r)
              if (Su[q].x != 0.0 || Su[q].y != 0.0) e = fmax(e, diff);
              const double2 sl = Sl[(size_t)c + (size_t)r * nj];
              if (sl.x != 0.0 || sl.y != 0.0) e = fmax(e, diff);
            }
          }
        }
      }
      if (cpl)
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
          const double c = cpl[d.pstart[i] + k];
          sign[d.pstart[i] + k] = cscale(c * c, G[(size_t)k * (n + 1)]);
        }
    }
    e = cta_max(e, sm.red);
    if (have_old) {
      err = e;
      conv = e < a.scba_tol;
    }
    have_old = true;
    par ^= 1;
    ++it;
  }
  par ^= 1;  // parity of the last computed Gn
  // Meir-Wingreen: I_c = -Re Tr[Gam_c Gn(cb,cb) - f_c Gam_c A(cb,cb)]
  if (a.curr) {
    double2* Gam = w.slot(7);
    double2* A = w.slot(8);
    for (int c = 0; c < ncont; ++c) {
      const int cb = d.cblk[c] - 1, n = d.pl[cb];
      cta_spectral(Gam, w.sig(c), n);
      cta_spectral(A, w.layer(1, cb, N), n);
      __syncthreads();
      const double t1 = cta_re_trace_prod(Gam, w.layer(4 + par, cb, N), n, OP_N, sm.red);
      const double t2 = cta_re_trace_prod(Gam, A, n, OP_N, sm.red);
      if (threadIdx.x == 0) a.curr[(int64_t)p * a.curr_stride + c] = -(t1 - frm[c] * t2);
    }
  }
  // layer currents J_{i,i+1} = Re[i Tr(ESH(i,i+1) Gn(i+1,i) - Gn(i,i+1) ESH(i+1,i))], densities Tr Gn(i,i)
  if (a.lcurr || a.ldens) {
    double2* E1 = w.slot(8);
    double2* E2 = w.slot(9);
    for (int i = 0; i < N; ++i) {
      const int ni = d.pl[i];
      if (a.ldens) {
        double tr = 0.0;
        const double2* G = w.layer(4 + par, i, N);
        for (int k = threadIdx.x; k < ni; k += blockDim.x) tr += G[(size_t)k * (ni + 1)].x;
        tr = cta_sum(tr, sm.red);
        if (threadIdx.x == 0) a.ldens[(int64_t)p * a.ldens_stride + i] = tr;
      }
      if (a.lcurr && i + 1 < N) {
        const int nj = d.pl[i + 1];
        esh_up(d, i, ec, E1);
        esh_lo(d, i, ec, E2);
        __syncthreads();
        const double2* U = w.layer(6 + par, i, N);   // Gn(i,i+1); Gn(i+1,i) = U^dag
        double2 t1 = cta_trace_prod_c(E1, U, ni, nj, OP_C, sm.red);   // Tr(ESH(i,i+1) Gn(i+1,i))
        double2 t2 = cta_trace_prod_c(U, E2, ni, nj, OP_N, sm.red);   // Tr(Gn(i,i+1) ESH(i+1,i))
        // Re(i z) = -Im z
        if (threadIdx.x == 0) a.lcurr[(int64_t)p * a.lcurr_stride + i] = -(t1.y - t2.y);
      }
    }
  }
  if (threadIdx.x == 0) {
    if (a.scba_iter) a.scba_iter[p] = it;
    if (a.scba_err) a.scba_err[p] = err;
    if (a.ncyc) a.ncyc[p] = ncyc;
    if (a.status) a.status[p] = st;
  }
}

// ---------------------------------------------------------------- kernels
__global__ void __launch_bounds__(kThreads, 2) k_engine(EngineArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemMap sm = map_smem(smem_raw, a.nmax);
  if (a.trace) {
    if (threadIdx.x < TR_NPHASE) sm.tr.acc[threadIdx.x] = 0;
    sm.inv.tr = sm.tr;
  } else {
    sm.tr.acc = nullptr;
  }
  __syncthreads();
  const long long t_all = sm.tr.start();
  Ws w;
  w.base = a.ws + (int64_t)blockIdx.x * a.ws_per_cta;
  w.Q = a.Q;
  w.ncont = a.ncont_max;
  for (;;) {
    if (threadIdx.x == 0) *sm.item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int p = *sm.item;
    __syncthreads();
    if (p >= a.npts) break;
    const DevDesc& d = a.devs[a.dev_id[p]];
    const double E = a.energy[p];
    if (a.mode == MODE_GN) {
      double2* vec = w.slot(S_SIG + a.ncont_max + 8 * a.nbl_max);
      solve_GN(a, d, E, p, w, vec, sm);
    } else {
      solve_T(a, d, E, p, w, sm);
    }
    if (sm.tr.acc && threadIdx.x == 0) sm.tr.acc[TR_POINTS] += 1;
    __syncthreads();
  }
  sm.tr.stop(TR_TOTAL, t_all);
  __syncthreads();
  if (a.trace && threadIdx.x < TR_NPHASE)
    atomicAdd(a.trace + threadIdx.x, (unsigned long long)sm.tr.acc[threadIdx.x]);
}

int64_t engine_slots(int mode, int nbl_max, int ncont_max) {
  int64_t s = S_SIG + ncont_max;
  if (mode == MODE_T || mode == MODE_DOS) s += nbl_max;          // gsmr
  else s += 8 * (int64_t)nbl_max;                                 // GN arrays
  return s;
}

int64_t engine_ws_elems(int mode, int nbl_max, int ncont_max, int nmax) {
  const int64_t Q = (int64_t)nmax * nmax;
  int64_t e = engine_slots(mode, nbl_max, ncont_max) * Q;
  if (mode == MODE_GN) e += 2 * (int64_t)nbl_max * nmax + 16;  // sigma_r, sigma_n vectors
  return e;
}

cudaError_t launch_engine(const EngineArgs& a, int grid, cudaStream_t s) {
  const size_t smem = engine_smem_bytes(a.nmax);
  cudaError_t e = cudaFuncSetAttribute(k_engine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
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
  gemm(m, n, k, Ao, Bo, C + b * sC, m, alpha, beta, sm);
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

size_t zinv_batched_work_elems(int n) { return zinv_ws_elems(n, kSmemMain); }

__global__ void __launch_bounds__(kThreads, 2)
    k_zinv_batched(int n, const double2* A, double2* Ainv, int* info, double2* work, int64_t wstride) {
  extern __shared__ __align__(16) char smem_raw[];
  SmemMap sm = map_smem(smem_raw, n);
  sm.tr.acc = nullptr;
  const int b = blockIdx.x;
  const int64_t nn = (int64_t)n * n;
  int inf = zinv(n, A + b * nn, Ainv + b * nn, work + b * wstride, sm);
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
