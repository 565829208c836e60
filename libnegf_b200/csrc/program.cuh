// The per-point program of the persistent engine, written as a resumable
// generator.
//
// A CTA's work alternates between control (which block operation comes
// next, convergence decisions, bookkeeping) and the block operations
// themselves (GEMM on the FP64 tensor pipe, Gauss-Jordan inversion, ES-H
// assembly, traces).  Calling the block operations from deep inside the
// control code made every heavy routine run under the register pressure of
// its callers.  Here the control code is a generator: next_op() runs until
// it has filled one Op descriptor and returns; the kernel's top level then
// executes the op with exec_op() in a clean register context and calls
// next_op() again, which resumes where it stopped.  The generator keeps all
// state that must survive an op in a Prog struct (local memory), switch-
// based resumption points (PT_EMIT) mark where it yields.  Op results the
// control code needs (max|C1|, pivot info, traces) come back in shared
// memory.  All threads of the CTA run the generator identically.
//
// The operation sequence is the one of libNEGF's per-point solve:
// decimation src/contselfenergy.F90:271-340, contact self-energies :445-491,
// build_ESH src/iterative.F90:1956, gsmr/Gr/Gn sweeps
// src/iterative_cpu.F90:51-372, transmissions :399-583, DOS
// src/iterative.F90:1821-1952, elastic SCBA :289-363 with
// src/elphdd.F90:108-276 and src/scba.F90:120-147, Meir-Wingreen and layer
// currents src/iterative.F90:382-461.
#pragma once
#include "cta_ops.cuh"
#include "engine.cuh"

namespace negf {

// ---------------------------------------------------------------- smem map
struct SmemMap {
  double2* main;
  InvScratch inv;
  double* red;
  double* maxv;
  double* res;      // op results read by the control code
  int* ires;
  int* item;
  Trace tr;
};

__device__ __forceinline__ SmemMap map_smem(char* base, int nmax) {
  SmemMap m;
  m.main = reinterpret_cast<double2*>(base);
  char* p = base + kSmemMain;
  m.red = reinterpret_cast<double*>(p); p += 32 * sizeof(double);
  m.maxv = reinterpret_cast<double*>(p); p += 2 * sizeof(double);
  m.res = reinterpret_cast<double*>(p); p += 12 * sizeof(double);
  m.inv.redv = reinterpret_cast<double*>(p); p += 32 * sizeof(double);
  m.inv.redi = reinterpret_cast<int*>(p); p += 32 * sizeof(int);
  m.inv.flag = reinterpret_cast<int*>(p); p += 4 * sizeof(int);
  m.item = reinterpret_cast<int*>(p); p += 4 * sizeof(int);
  m.ires = reinterpret_cast<int*>(p); p += 4 * sizeof(int);
  m.inv.piv = reinterpret_cast<int*>(p); p += nmax * sizeof(int);
  m.inv.perm = reinterpret_cast<int*>(p); p += nmax * sizeof(int);
  m.inv.cperm = reinterpret_cast<int*>(p); p += nmax * sizeof(int);
  p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 7) & ~uintptr_t(7));
  m.tr.acc = reinterpret_cast<long long*>(p);   // TR_NPHASE entries; enabled by the caller
  m.inv.tr.acc = nullptr;
  return m;
}

inline size_t smem_bytes_for(int nmax) {
  return kSmemMain + 32 * 8 + 2 * 8 + 12 * 8 + 32 * 8 + 32 * 4 + 4 * 4 + 4 * 4 + 4 * 4 + 3 * (size_t)nmax * 4 + 8 +
         TR_NPHASE * 8;
}

__device__ __forceinline__ double2 cz(double re, double im) { return make_double2(re, im); }

// Workspace slots: 0..11 scratch (0..7 also the decimation buffers),
// 12..14 inversion workspace, 15.. one self-energy per contact, then the
// per-layer arrays.
enum : int { S_INV = 12, S_SIG = 15 };

struct Ws {
  double2* base;
  int64_t Q;
  int ncont;
  int nbl_max;
  __device__ double2* slot(int k) const { return base + (int64_t)k * Q; }
  __device__ double2* inv() const { return slot(S_INV); }
  __device__ double2* sig(int c) const { return slot(S_SIG + c); }
  __device__ double2* layer(int arr, int i, int nbl) const { return slot(S_SIG + ncont + arr * nbl + i); }
  // T / DOS: Gr(cb,cb) kept at the block of contact c during the forward sweep
  __device__ double2* keep(int c) const { return slot(S_SIG + ncont + nbl_max + c); }
  // density: the surface GF of contact c, kept for the outer blocks
  __device__ double2* gskeep(int c) const { return slot(S_SIG + 2 * ncont + nbl_max + c); }
  // GN: the same, after the eight layer arrays
  __device__ double2* gnkeep(int c) const { return slot(S_SIG + ncont + 8 * nbl_max + c); }
};

// ---------------------------------------------------------------- ops
enum OpKind : int {
  K_NONE = 0,
  K_GEMM,      // C = alpha op(A) op(B) + beta C   (flag: reduce max|C| into sm.maxv)
  K_ZINV,      // C = A^-1, order n                 (info -> ires[0])
  K_ESH,       // C (m x n) = s_e S - H - sub - diag(subdiag)   (A = H, X = S, Y = sub, V = subdiag)
  K_COPY,      // C = A, m elements
  K_SUB,       // C -= A, m elements
  K_DECUPD,    // C -= A and D -= A, m elements (decimation Ao_s, Ao update)
  K_SPECTRAL,  // C = i (A - A^dag), order m
  K_TRACE,     // res[slot] = Re Tr(A op(B)), order m (diagonal entries k with mask[k], if mask)
  K_TRACEC,    // res[slot], res[slot+1] = Tr(A op(B)), A m x n
  K_TRACEN,    // res[slot] = Re Tr(A B^dag), A and B m x n (rows k with mask[k], if mask)
  K_DOS,       // out[k] = -Im A_kk / pi, k < m
  K_SIGDIAG,   // C[k] = cpl[k]^2 A_kk, k < m; flag 1: scal cpl^2 A_kk + (1-scal) C[k]; flag 2: scal cpl^2 A_kk
  K_SNINIT,    // C (m x m) = diag(A) or 0
  K_SNGAMMA,   // C += scal * i (A - A^dag), order m
  K_DAGGER,    // C (m x n) = A^dag, A is n x m
  K_ERRDIAG,   // res[slot] = max(res[slot], max_k |A_kk - B_kk|), order m
  K_ERRPAT,    // res[slot] = max(res[slot], max_{X(q) != 0} |A(q) - B(q)|), m x n;
               //   Y (n x m) adds the pattern of Y at transposed positions
  K_MAXABS,    // res[slot] = max |A(q)|, m elements
  K_TRDIAG,    // res[slot] = Re Tr A, order m
  K_LDOS,      // out[k] = sum over LDOS set k of dos[i-1] (A = dos row as doubles, device sets)
  K_ACCUM,     // C[q] += alpha * A[q], q < m (atomic: C is shared by all CTAs)
  K_SUBCOPY,   // C(flag + r, flag + c) = A(r, c), A m x m, C leading dimension ldc
  K_RESPROBE,  // res[slot] = max_i |(A (B v))_i - v_i|, res[8] = the condition estimate, order m (cta_inv_probe)
  K_EYE,       // C = identity, order m
  K_RETCHECK,  // res[slot] = min_i s Im A_ii / max_i |A_ii|, order m, s = -sign of the energy's imaginary part
  K_RELDIFF,   // res[slot] = max |A(q) - B(q)| / max |B(q)|, m elements
};

// The retarded surface Green's function has a negative semidefinite
// anti-Hermitian part, so -Im gs_ii >= 0 on every diagonal entry (checked
// to 1e-6 of the largest |gs_ii|, far above rounding).  At a
// nearly singular decimation (a lead resonance at small eta) FP64 rounding
// can steer Sancho-Rubio to another fixed point of its equation, with
// diagonal entries of the wrong sign; the decimation is then run again from
// inputs moved by a few units in the last place (the energy times
// 1 + k 2^-50, k = 1..kDecRetries, engine.cuh), which keeps its result
// within the FP64 scatter of the reference path.
constexpr double kRetardedTol = 1e-6;


struct Op {
  int kind;
  int m, n, k;
  int opa, opb, flag, slot;
  int lda, ldb, ldc, pad;
  const double2* A;
  const double2* B;
  double2* C;
  double2* D;
  const double2* X;
  const double2* Y;
  const double2* V;
  const double* cpl;
  double* out;
  const unsigned char* mask;   // K_TRACE / K_TRACEN projection, or null
  const DevDesc* dd;           // K_LDOS
  double2 alpha, beta;
  double scal;
};

__device__ __forceinline__ void set_gemm(Op& o, int M, int N, int K, const double2* A, int lda, int opa,
                                         const double2* B, int ldb, int opb, double2* C, int ldc, double2 al,
                                         double2 be, int want_max = 0) {
  o.kind = K_GEMM; o.m = M; o.n = N; o.k = K; o.A = A; o.lda = lda; o.opa = opa; o.B = B; o.ldb = ldb;
  o.opb = opb; o.C = C; o.ldc = ldc; o.alpha = al; o.beta = be; o.flag = want_max;
}

__device__ __forceinline__ void set_esh(Op& o, double2* D, int rows, int cols, const double2* H, const double2* S,
                                        double2 se, int diag, const double2* sub, const double2* subdiag, int opm) {
  o.kind = K_ESH; o.C = D; o.m = rows; o.n = cols; o.A = H; o.X = S; o.alpha = se; o.flag = diag; o.Y = sub;
  o.V = subdiag; o.opa = opm;
}

__device__ __forceinline__ void set_simple(Op& o, int kind, int m, const double2* A, double2* C) {
  o.kind = kind; o.m = m; o.A = A; o.C = C;
}

// ---------------------------------------------------------------- executor
// The light operations (everything but products and inversions), executed
// inside engine_step.
__device__ __forceinline__ void exec_light(const Op& o, SmemMap& sm) {
  const int tid = threadIdx.x;
  long long t0 = sm.tr.start();
  switch (o.kind) {
    case K_ESH:
      cta_esh(o.C, o.m, o.n, o.A, o.X, o.alpha, o.flag != 0, o.Y, o.V, o.opa);
      break;
    case K_COPY:
      cta_copy(o.C, o.A, o.m);
      break;
    case K_SUB:
      for (int q = tid; q < o.m; q += blockDim.x) o.C[q] = csub(o.C[q], o.A[q]);
      break;
    case K_DECUPD:
      for (int q = tid; q < o.m; q += blockDim.x) {
        const double2 s = o.A[q];
        o.C[q] = csub(o.C[q], s);
        o.D[q] = csub(o.D[q], s);
      }
      break;
    case K_SPECTRAL:
      cta_spectral(o.C, o.A, o.m);
      break;
    case K_TRACE: {
      const double r = cta_re_trace_prod(o.A, o.B, o.m, o.opb, sm.red, o.mask);
      if (tid == 0) sm.res[o.slot] = r;
      break;
    }
    case K_TRACEC: {
      const int n = o.m, m = o.n;   // A is n x m, op(B) is m x n
      double re = 0.0, im = 0.0;
      for (int idx = tid; idx < n * m; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;   // A(i,j) * opB(j,i)
        const double2 x = o.A[idx];
        const double2 y = (o.opb == OP_C) ? cconj(o.B[(size_t)i + (size_t)j * n]) : o.B[(size_t)j + (size_t)i * m];
        re += x.x * y.x - x.y * y.y;
        im += x.x * y.y + x.y * y.x;
      }
      re = cta_sum(re, sm.red);
      im = cta_sum(im, sm.red);
      if (tid == 0) { sm.res[o.slot] = re; sm.res[o.slot + 1] = im; }
      break;
    }
    case K_TRACEN: {
      const int n2 = o.m, n1 = o.n;
      double acc = 0.0;
      for (int idx = tid; idx < n2 * n1; idx += blockDim.x) {
        if (o.mask && !o.mask[idx % n2]) continue;
        const double2 x = o.A[idx], y = o.B[idx];   // W2(r,c) * conj(G21(r,c))
        acc += x.x * y.x + x.y * y.y;
      }
      acc = cta_sum(acc, sm.red);
      if (tid == 0) sm.res[o.slot] = acc;
      break;
    }
    case K_DOS: {
      const double pi = 3.14159265358979323846;
      for (int k = tid; k < o.m; k += blockDim.x) o.out[k] = -(1.0 / pi) * o.A[(size_t)k * (o.m + 1)].y;
      break;
    }
    case K_SIGDIAG:
      for (int k = tid; k < o.m; k += blockDim.x) {
        const double c = o.cpl[k];
        const double2 v = cscale(c * c, o.A[(size_t)k * (o.m + 1)]);
        if (o.flag == 0) o.C[k] = v;
        else if (o.flag == 1) o.C[k] = cadd(cscale(o.scal, v), cscale(1.0 - o.scal, o.C[k]));
        else o.C[k] = cscale(o.scal, v);
      }
      break;
    case K_SNINIT:
      for (int q = tid; q < o.m * o.m; q += blockDim.x) {
        const int r = q % o.m, c = q / o.m;
        o.C[q] = (o.A && r == c) ? o.A[r] : cz(0.0, 0.0);
      }
      break;
    case K_SNGAMMA:
      for (int q = tid; q < o.m * o.m; q += blockDim.x) {
        const int r = q % o.m, c = q / o.m;
        const double2 a1 = o.A[q], b1 = cconj(o.A[(size_t)c + (size_t)r * o.m]);
        const double2 gam = cz(-(a1.y - b1.y), a1.x - b1.x);   // i (S - S^dag)
        o.C[q] = cadd(o.C[q], cscale(o.scal, gam));
      }
      break;
    case K_DAGGER:
      for (int q = tid; q < o.m * o.n; q += blockDim.x) {
        const int r = q % o.m, c = q / o.m;
        o.C[q] = cconj(o.A[(size_t)c + (size_t)r * o.n]);
      }
      break;
    case K_ERRDIAG: {
      double e = 0.0;
      for (int k = tid; k < o.m; k += blockDim.x)
        e = fmax(e, cabs(csub(o.A[(size_t)k * (o.m + 1)], o.B[(size_t)k * (o.m + 1)])));
      e = cta_max(e, sm.red);
      if (tid == 0) sm.res[o.slot] = fmax(sm.res[o.slot], e);
      break;
    }
    case K_ERRPAT: {
      double e = 0.0;
      for (int q = tid; q < o.m * o.n; q += blockDim.x) {
        const int r = q % o.m, c = q / o.m;
        const double diff = cabs(csub(o.A[q], o.B[q]));
        const double2 sp = o.X[q];
        if (sp.x != 0.0 || sp.y != 0.0) e = fmax(e, diff);
        if (o.Y) {
          const double2 st = o.Y[(size_t)c + (size_t)r * o.n];
          if (st.x != 0.0 || st.y != 0.0) e = fmax(e, diff);
        }
      }
      e = cta_max(e, sm.red);
      if (tid == 0) sm.res[o.slot] = fmax(sm.res[o.slot], e);
      break;
    }
    case K_MAXABS: {
      double e = 0.0;
      for (int q = tid; q < o.m; q += blockDim.x) e = fmax(e, cabs(o.A[q]));
      e = cta_max(e, sm.red);
      if (tid == 0) sm.res[o.slot] = e;
      break;
    }
    case K_TRDIAG: {
      double tr = 0.0;
      for (int k = tid; k < o.m; k += blockDim.x) tr += o.A[(size_t)k * (o.m + 1)].x;
      tr = cta_sum(tr, sm.red);
      if (tid == 0) sm.res[o.slot] = tr;
      break;
    }
    case K_LDOS: {
      // set k summed in its index order, as the reference's accumulation
      // loop (src/iterative.F90:1931-1945); indices past the device skipped
      const double* dos = reinterpret_cast<const double*>(o.A);
      for (int k = tid; k < o.dd->nldos; k += blockDim.x) {
        double acc = 0.0;
        for (int q = o.dd->ldos_ptr[k]; q < o.dd->ldos_ptr[k + 1]; ++q) {
          const int i2 = o.dd->ldos_idx[q];
          if (i2 >= 1 && i2 <= o.dd->norb) acc += dos[i2 - 1];
        }
        o.out[k] = acc;
      }
      break;
    }
    case K_SUBCOPY:
      for (int q = tid; q < o.m * o.m; q += blockDim.x) {
        const int r = q % o.m, c = q / o.m;
        o.C[(int64_t)(o.flag + r) + (int64_t)(o.flag + c) * o.ldc] = o.A[q];
      }
      break;
    case K_RESPROBE: {
      double k = 0.0;
      const double e = cta_inv_probe(o.m, o.A, o.B, sm.main, sm.red, &k);
      if (tid == 0) {
        sm.res[o.slot] = e;
        sm.res[8] = k;
      }
      break;
    }
    case K_EYE:
      for (int q = tid; q < o.m * o.m; q += blockDim.x)
        o.C[q] = make_double2((q % o.m) == (q / o.m) ? 1.0 : 0.0, 0.0);
      break;
    case K_RETCHECK: {
      // -Inf when a diagonal entry is not finite
      double lo = 1.7976931348623157e308, hi = 0.0, bad = 0.0;
      for (int i = tid; i < o.m; i += blockDim.x) {
        const double2 a = o.A[(size_t)i * (o.m + 1)];
        const double v = o.scal * a.y, h = cabs(a);
        if (!(h <= 1.7976931348623157e308)) bad = 1.0;
        else {
          lo = fmin(lo, v);
          hi = fmax(hi, h);
        }
      }
      lo = -cta_max(-lo, sm.red);
      hi = cta_max(hi, sm.red);
      bad = cta_max(bad, sm.red);
      if (tid == 0)
        sm.res[o.slot] = (bad > 0.0) ? -__longlong_as_double(0x7ff0000000000000LL) : ((hi > 0.0) ? lo / hi : 0.0);
      break;
    }
    case K_RELDIFF: {
      double d = 0.0, b = 0.0;
      for (int q = tid; q < o.m; q += blockDim.x) {
        d = fmax(d, cabs(csub(o.A[q], o.B[q])));
        b = fmax(b, cabs(o.B[q]));
      }
      d = cta_max(d, sm.red);
      b = cta_max(b, sm.red);
      if (tid == 0) sm.res[o.slot] = (b > 0.0) ? d / b : d;
      break;
    }
    case K_ACCUM:
      for (int q = tid; q < o.m; q += blockDim.x) {
        const double2 v = cmul(o.alpha, o.A[q]);
        atomicAdd(&o.C[q].x, v.x);
        atomicAdd(&o.C[q].y, v.y);
      }
      break;
    default:
      break;
  }
  __syncthreads();
  sm.tr.stop(TR_ELEM, t0);
}

// ---------------------------------------------------------------- generator
struct Prog {
  int pc;
  int p;                // current point
  const DevDesc* d;
  double E;
  int st, ncyc;
  double2 ec, ecs;      // ES-H energy, contact energy
  // contacts / decimation
  int c, L, ncb, it, ok, done, ib, ix, ic, ic1;
  int att;              // decimation attempt (retarded-branch retries)
  int diverged;         // the attempt's max|C1| went Inf / NaN
  int sens;             // the attempt met a nearly singular Ao (condition estimate above kSensitiveCond)
  int kept;             // a previous sensitive attempt's gs is kept for comparison
  int in_dec;           // inside a decimation (refinements mark it sensitive)
  double2 ecd;          // contact energy of the attempt
  // inverse refinement (the `refine` block): matrix, its computed inverse, order, return point
  const double2* rA;
  double2* rX;
  int rm, rret, rk;
  // sweeps
  int i, j, sub_first, cur, cc, last, tiny, pp, lo;
  double2* gnext;
  double2* gsv;         // target of gr_first
  int keep;
  const double2* sr;    // dephasing sigma_r in effect (or null)
  // transmission bookkeeping (contact pair q of npairs)
  int fast, ct1, ct2, bl1, bl2, q, npairs;
  double T;
  // SCBA
  int sit, conv, have_old, par;
  double err, iold;     // SCBA error; contact-1 current of the previous sweep (scba_rule 1)
  double2* vec;
};

#define PT_EMIT(s) do { (s).pc = __LINE__; return true; case __LINE__:; } while (0)
// Runs the `refine` block on the inverse X_ of A_ (order m_) and resumes here.
#define PT_REFINE(s, A_, X_, m_)                                        \
  do {                                                                  \
    (s).rA = (A_); (s).rX = (X_); (s).rm = (m_); (s).rret = __LINE__;   \
    goto refine;                                                        \
    case __LINE__:;                                                     \
  } while (0)

__device__ __forceinline__ const double2* sig_on_block(const DevDesc* d, const Ws& w, int i, int& first) {
  first = -1;
  for (int c = 0; c < d->ncont; ++c)
    if (d->cblk[c] == i + 1) { first = c; return w.sig(c); }
  return nullptr;
}

// ESH(i,i) = ec S - H - Sigma_first - diag(sigr)
__device__ __forceinline__ void op_esh_diag(Op& o, const DevDesc* d, int i, double2 ec, double2* dst, const Ws& w,
                                            const double2* sigr, int& first) {
  const double2* sub = sig_on_block(d, w, i, first);
  set_esh(o, dst, d->pl[i], d->pl[i], d->hd + d->od[i], d->has_s ? d->sd + d->od[i] : nullptr, ec, 1, sub,
          sigr ? sigr + d->pstart[i] : nullptr, OP_N);
}
__device__ __forceinline__ void op_esh_up(Op& o, const DevDesc* d, int i, double2 ec, double2* dst) {
  set_esh(o, dst, d->pl[i], d->pl[i + 1], d->hu + d->oo[i], d->has_s ? d->su + d->oo[i] : nullptr, ec, 0, nullptr,
          nullptr, OP_N);
}
__device__ __forceinline__ void op_esh_lo(Op& o, const DevDesc* d, int i, double2 ec, double2* dst) {
  set_esh(o, dst, d->pl[i + 1], d->pl[i], d->hl + d->oo[i], d->has_s ? d->sl + d->oo[i] : nullptr, ec, 0, nullptr,
          nullptr, OP_N);
}

// With S = I the off-diagonal ES-H blocks are E*0 - H = -H: the products
// take the H block itself and the sign in their alpha (the negation is
// exact), so no assembly pass is run for them.  With S they take the
// assembled block in `slot`.
__device__ __forceinline__ const double2* esh_up_op(const DevDesc* d, int i, const double2* slot) {
  return d->has_s ? slot : d->hu + d->oo[i];
}
__device__ __forceinline__ const double2* esh_lo_op(const DevDesc* d, int i, const double2* slot) {
  return d->has_s ? slot : d->hl + d->oo[i];
}
__device__ __forceinline__ double2 esh_al(const DevDesc* d, double2 a) {
  return d->has_s ? a : make_double2(-a.x, -a.y);
}

__device__ __forceinline__ void put_status(int& st, int s) { if (st == ST_OK) st = s; }

// Contact pair q (0-based) of the call: ct1 is the contact on the smaller
// block (src/iterative_cpu.F90:421-427), ct2 the other; bl1/bl2 their blocks.
__device__ __forceinline__ void pair_of(const EngineArgs& a, Prog& s, int q) {
  const int ni = (a.npairs > 1 ? a.pair_ni[q] : a.ni) - 1, nf = (a.npairs > 1 ? a.pair_nf[q] : a.nf) - 1;
  const int cbi = s.d->cblk[ni < s.d->ncont ? ni : 0], cbf = s.d->cblk[nf < s.d->ncont ? nf : 0];
  s.ct1 = (cbi < cbf) ? ni : nf;
  s.ct2 = (cbi < cbf) ? nf : ni;
  s.bl1 = s.d->cblk[s.ct1 < s.d->ncont ? s.ct1 : 0];
  s.bl2 = s.d->cblk[s.ct2 < s.d->ncont ? s.ct2 : 0];
}

__device__ __forceinline__ const unsigned char* tun_mask_of(const DevDesc* d, int bl) {
  return d->tun_mask ? d->tun_mask + d->pstart[bl - 1] : nullptr;
}

// Fills `o` with the next block operation of this CTA and returns true, or
// returns false when the work queue is exhausted.
__device__ __forceinline__ bool next_op(const EngineArgs& a, Prog& s, SmemMap& sm, const Ws& w, Op& o) {
  const double2 one = cz(1, 0), zero = cz(0, 0), mone = cz(-1, 0);
  double mx;
dispatch:
  switch (s.pc) {
    case 0:
    for (;;) {
      // ---------------------------------------------------------- next point
      if (threadIdx.x == 0) *sm.item = atomicAdd(a.counter, 1);
      __syncthreads();
      s.p = *sm.item;
      __syncthreads();
      if (s.p >= a.npts) break;
      s.d = a.devs + a.dev_id[s.p];
      s.E = a.energy[s.p];
      s.st = ST_OK;
      s.ncyc = 0;
      s.T = 0.0;
      s.ecs = cz(s.E, a.eta);
      s.ec = (a.mode == MODE_DOS) ? cz(s.E, a.dos_delta) : cz(s.E, 0.0);
      if (a.mode == MODE_RHO) {   // compute_Gr (src/integrations.F90:2287-2340): contacts and ES-H at Ec
        s.ec = cz(s.E, a.energy_im[s.p]);
        s.ecs = s.ec;
      }
      if (threadIdx.x == 0 && sm.tr.acc) sm.tr.acc[TR_POINTS] += 1;

      // ------------------------------------------ contacts (compute_contacts_dns)
      for (s.c = 0; s.c < s.d->ncont; ++s.c) {
        s.L = s.d->L[s.c];
        s.ncb = s.d->pl[s.d->cblk[s.c] - 1];
        if (a.sgf_in && a.sgf_in[(int64_t)s.p * a.ncont_max + s.c] >= 0) {
          // cached surface GF (surface_green's retrieve, src/contselfenergy.F90:262-264): no decimation
          set_simple(o, K_COPY, s.L * s.L, a.sgf_arena + a.sgf_in[(int64_t)s.p * a.ncont_max + s.c], w.slot(4));
          PT_EMIT(s);
          goto sgf_ready;
        }
        s.att = 0;
        s.kept = 0;
      decimation_attempt:
        s.ecd = (s.att == 0) ? s.ecs : cscale(1.0 + s.att * 0x1p-50, s.ecs);
        s.sens = 0;
        s.in_dec = 1;
        set_esh(o, w.slot(0), s.L, s.L, s.d->h00 + s.d->olead[s.c], s.d->has_s00 ? s.d->s00 + s.d->olead[s.c] : nullptr,
                s.ecd, 1, nullptr, nullptr, OP_N);                                          // Ao
        PT_EMIT(s);
        set_esh(o, w.slot(2), s.L, s.L, s.d->h01 + s.d->olead[s.c], s.d->has_s01 ? s.d->s01 + s.d->olead[s.c] : nullptr,
                s.ecd, 0, nullptr, nullptr, OP_N);                                          // Bo
        PT_EMIT(s);
        set_esh(o, w.slot(3), s.L, s.L, s.d->h01 + s.d->olead[s.c], s.d->has_s01 ? s.d->s01 + s.d->olead[s.c] : nullptr,
                cconj(s.ecd), 0, nullptr, nullptr, OP_C);                                   // Co = (E* S01 - H01)^dag
        PT_EMIT(s);
        // ---- decimation (src/contselfenergy.F90:271-340): Ao 0, Aos 1, Go 4, Sf 6
        set_simple(o, K_COPY, s.L * s.L, w.slot(0), w.slot(1));
        PT_EMIT(s);
        s.ok = 0; s.done = 0; s.diverged = 0; s.ib = 2; s.ix = 5; s.ic = 3; s.ic1 = 7;
        for (s.it = 1; s.it <= a.sgf_max_iter; ++s.it) {
          o.kind = K_ZINV; o.m = s.L; o.A = w.slot(0); o.C = w.slot(4);
          PT_EMIT(s);
          if (sm.ires[0]) put_status(s.st, ST_SINGULAR);
          PT_REFINE(s, w.slot(0), w.slot(4), s.L);
          set_gemm(o, s.L, s.L, s.L, w.slot(4), s.L, OP_N, w.slot(s.ic), s.L, OP_N, w.slot(s.ix), s.L, one, zero);
          PT_EMIT(s);                                                                    // GoXCo
          set_gemm(o, s.L, s.L, s.L, w.slot(s.ic), s.L, OP_N, w.slot(s.ix), s.L, OP_N, w.slot(s.ic1), s.L, one,
                   zero, 1);
          PT_EMIT(s);                                                                    // C1 = Co GoXCo
          mx = *sm.maxv;
          if (!(mx <= 1.7976931348623157e308)) {   // Inf / NaN: this iteration will not converge
            s.diverged = 1;
            break;
          }
          if (mx <= a.sgf_tol) {
            if (s.ok) { s.done = 1; break; }
            s.ok = 1;
          } else {
            s.ok = 0;
          }
          set_gemm(o, s.L, s.L, s.L, w.slot(s.ib), s.L, OP_N, w.slot(s.ix), s.L, OP_N, w.slot(6), s.L, one, zero);
          PT_EMIT(s);                                                                    // Self = Bo GoXCo
          o.kind = K_DECUPD; o.m = s.L * s.L; o.A = w.slot(6); o.C = w.slot(1); o.D = w.slot(0);
          PT_EMIT(s);                                                                    // Ao_s -= Self, Ao -= Self
          set_gemm(o, s.L, s.L, s.L, w.slot(4), s.L, OP_N, w.slot(s.ib), s.L, OP_N, w.slot(6), s.L, one, zero);
          PT_EMIT(s);                                                                    // GoXBo
          set_gemm(o, s.L, s.L, s.L, w.slot(s.ib), s.L, OP_N, w.slot(6), s.L, OP_N, w.slot(s.ix), s.L, one, zero);
          PT_EMIT(s);                                                                    // B1 = Bo GoXBo
          set_gemm(o, s.L, s.L, s.L, w.slot(s.ic), s.L, OP_N, w.slot(6), s.L, OP_N, w.slot(0), s.L, mone, one);
          PT_EMIT(s);                                                                    // Ao -= Co GoXBo
          { int t = s.ib; s.ib = s.ix; s.ix = t; t = s.ic; s.ic = s.ic1; s.ic1 = t; }   // Bo = B1, Co = C1
        }
        o.kind = K_ZINV; o.m = s.L; o.A = w.slot(1); o.C = w.slot(4);
        PT_EMIT(s);                                                                      // gs = Ao_s^-1
        if (sm.ires[0]) put_status(s.st, ST_SINGULAR);
        PT_REFINE(s, w.slot(1), w.slot(4), s.L);
        if (s.ecs.y != 0.0) {
          o.kind = K_RETCHECK; o.m = s.L; o.A = w.slot(4); o.slot = 6; o.scal = (s.ecs.y > 0.0) ? -1.0 : 1.0;
          PT_EMIT(s);
          // a converged fixed point of the wrong kind, or an iteration that ran off to Inf / NaN
          const bool wrong = (s.done && !(sm.res[6] >= -kRetardedTol)) || s.diverged ||
                             sm.res[6] == -__longlong_as_double(0x7ff0000000000000LL);
          if (wrong && s.att < kDecRetries) {
            ++s.att;
            goto decimation_attempt;
          }
          if (wrong) s.done = 0;   // no retarded solution reached: NOT_CONVERGED
          // a sensitive decimation (one of its inverses needed refinement) is accepted once
          // two attempts reach the same gs: a fixed point other than the retarded one can
          // pass the diagonal test, and the retarded one is the common outcome
          if (!wrong && s.sens) {
            if (s.kept) {
              o.kind = K_RELDIFF; o.m = s.L * s.L; o.A = w.slot(4); o.B = w.slot(10); o.slot = 5;
              PT_EMIT(s);
            }
            if (!s.kept || !(sm.res[5] <= 1e-2)) {
              if (s.att < kDecRetries) {
                set_simple(o, K_COPY, s.L * s.L, w.slot(4), w.slot(10));
                PT_EMIT(s);
                s.kept = 1;
                ++s.att;
                goto decimation_attempt;
              }
              s.done = 0;          // no two attempts agree: NOT_CONVERGED
            }
          }
        }
        s.in_dec = 0;
        if (!s.done) put_status(s.st, ST_NOT_CONVERGED);
        s.ncyc += s.done ? s.it : a.sgf_max_iter + 1;
        if (a.sgf_out && a.sgf_out[(int64_t)s.p * a.ncont_max + s.c] >= 0) {
          // surface_green's add (:251-256)
          set_simple(o, K_COPY, s.L * s.L, w.slot(4), a.sgf_arena + a.sgf_out[(int64_t)s.p * a.ncont_max + s.c]);
          PT_EMIT(s);
        }
      sgf_ready:
        if (s.d->surf[s.c] > 0) {
          // bound-surface block of surface_green (src/contselfenergy.F90:226-243): GS is the
          // inverse of E S - H over Surf + PL1 with the PL1 block replaced by gs^-1
          o.kind = K_ZINV; o.m = s.L; o.A = w.slot(4); o.C = w.slot(5);
          PT_EMIT(s);
          if (sm.ires[0]) put_status(s.st, ST_SINGULAR);
          PT_REFINE(s, w.slot(4), w.slot(5), s.L);
          set_esh(o, w.slot(0), s.L + s.d->surf[s.c], s.L + s.d->surf[s.c], s.d->hs + s.d->osurf[s.c],
                  s.d->has_ss ? s.d->ss + s.d->osurf[s.c] : nullptr, s.ecs, 1, nullptr, nullptr, OP_N);
          PT_EMIT(s);
          o.kind = K_SUBCOPY; o.m = s.L; o.ldc = s.L + s.d->surf[s.c]; o.flag = s.d->surf[s.c];
          o.A = w.slot(5); o.C = w.slot(0);
          PT_EMIT(s);
          s.L += s.d->surf[s.c];
          o.kind = K_ZINV; o.m = s.L; o.A = w.slot(0); o.C = w.slot(4);
          PT_EMIT(s);
          if (sm.ires[0]) put_status(s.st, ST_SINGULAR);
          PT_REFINE(s, w.slot(0), w.slot(4), s.L);
        }
        if (a.acc_lc && (a.mode == MODE_RHO || a.mode == MODE_GN)) {
          set_simple(o, K_COPY, s.L * s.L, w.slot(4), a.mode == MODE_RHO ? w.gskeep(s.c) : w.gnkeep(s.c));
          PT_EMIT(s);
        }
        // ---- self-energy: Tlc = E SMC - HMC, Tcl = (E^* SMC - HMC)^dag, Sigma = Tlc gs Tcl
        set_esh(o, w.slot(0), s.ncb, s.L, s.d->hmc + s.d->omc[s.c], s.d->has_smc ? s.d->smc + s.d->omc[s.c] : nullptr,
                s.ecs, 0, nullptr, nullptr, OP_N);
        PT_EMIT(s);
        set_esh(o, w.slot(1), s.L, s.ncb, s.d->hmc + s.d->omc[s.c], s.d->has_smc ? s.d->smc + s.d->omc[s.c] : nullptr,
                cconj(s.ecs), 0, nullptr, nullptr, OP_C);
        PT_EMIT(s);
        set_gemm(o, s.ncb, s.L, s.L, w.slot(0), s.ncb, OP_N, w.slot(4), s.L, OP_N, w.slot(2), s.ncb, one, zero);
        PT_EMIT(s);
        set_gemm(o, s.ncb, s.ncb, s.L, w.slot(2), s.ncb, OP_N, w.slot(1), s.L, OP_N, w.sig(s.c), s.ncb, one, zero);
        PT_EMIT(s);
      }

      // ------------------------------------------------ transmission bookkeeping
      // calculate_transmissions (src/iterative.F90:1669-1780): the 2-contact
      // fast path iff 2 contacts, one pair and that pair's smaller block is 1;
      // otherwise gsmr is kept and every pair takes the N-contact formula.
      // The forward sweep runs to the largest ct1 block over the pairs.
      s.npairs = a.npairs > 1 ? a.npairs : 1;
      s.last = 0;
      for (s.q = s.npairs - 1; s.q >= 0; --s.q) {
        pair_of(a, s, s.q);
        s.last = max(s.last, s.bl1 - 1);
      }
      s.q = 0;                              // pair_of(0) is in effect
      s.fast = (a.mode == MODE_T) && s.d->ncont == 2 && s.npairs == 1 && s.bl1 == 1;
      if (a.mode == MODE_T && s.d->ncont == 1) {
        if (threadIdx.x == 0 && a.T)
          for (int q = 0; q < s.npairs; ++q) a.T[(int64_t)s.p * s.npairs + q] = 0.0;
        goto point_done;
      }

      // ------------------------------------------------ SCBA loop (once for T / DOS)
      s.sit = 0; s.conv = 0; s.have_old = 0; s.err = 0.0; s.par = 0;
      s.vec = w.slot(S_SIG + 2 * a.ncont_max + 8 * a.nbl_max);   // after the layers and gnkeep
      for (;;) {
        if (a.mode == MODE_GN && (s.conv || s.sit > a.scba_niter)) break;
        s.sr = (a.mode == MODE_GN && s.sit > 0 && a.coupling) ? s.vec : nullptr;
        s.keep = !s.fast;
        // -------------------------------------- gsmr sweep (calculate_gsmr_blocks)
        if (s.d->nbl > 1) {
          op_esh_diag(o, s.d, s.d->nbl - 1, s.ec, w.slot(0), w, s.sr, s.sub_first);
          PT_EMIT(s);
          for (s.j = s.sub_first + 1; s.sub_first >= 0 && s.j < s.d->ncont; ++s.j)
            if (s.d->cblk[s.j] == s.d->nbl) {
              set_simple(o, K_SUB, s.d->pl[s.d->nbl - 1] * s.d->pl[s.d->nbl - 1], w.sig(s.j), w.slot(0));
              PT_EMIT(s);
            }
          s.gnext = s.keep ? w.layer(0, s.d->nbl - 1, s.d->nbl) : w.slot(4);
          o.kind = K_ZINV; o.m = s.d->pl[s.d->nbl - 1]; o.A = w.slot(0); o.C = s.gnext;
          PT_EMIT(s);
          if (sm.ires[0]) put_status(s.st, ST_SINGULAR);
          PT_REFINE(s, w.slot(0), s.gnext, s.d->pl[s.d->nbl - 1]);
          s.pp = 1;
          for (s.i = s.d->nbl - 2; s.i >= 1; --s.i) {
            if (s.d->has_s) {
              op_esh_up(o, s.d, s.i, s.ec, w.slot(1));
              PT_EMIT(s);
              op_esh_lo(o, s.d, s.i, s.ec, w.slot(2));
              PT_EMIT(s);
            }
            op_esh_diag(o, s.d, s.i, s.ec, w.slot(0), w, s.sr, s.sub_first);
            PT_EMIT(s);
            for (s.j = s.sub_first + 1; s.sub_first >= 0 && s.j < s.d->ncont; ++s.j)
              if (s.d->cblk[s.j] == s.i + 1) {
                set_simple(o, K_SUB, s.d->pl[s.i] * s.d->pl[s.i], w.sig(s.j), w.slot(0));
                PT_EMIT(s);
              }
            set_gemm(o, s.d->pl[s.i], s.d->pl[s.i + 1], s.d->pl[s.i + 1], esh_up_op(s.d, s.i, w.slot(1)), s.d->pl[s.i],
                     OP_N, s.gnext, s.d->pl[s.i + 1], OP_N, w.slot(3), s.d->pl[s.i], esh_al(s.d, mone),
                     zero);                                                          // -ESH(i,i+1) gsmr(i+1)
            PT_EMIT(s);
            set_gemm(o, s.d->pl[s.i], s.d->pl[s.i], s.d->pl[s.i + 1], w.slot(3), s.d->pl[s.i], OP_N,
                     esh_lo_op(s.d, s.i, w.slot(2)), s.d->pl[s.i + 1], OP_N, w.slot(0), s.d->pl[s.i],
                     esh_al(s.d, one), one);                                        // ESH(i,i) + W ESH(i+1,i)
            PT_EMIT(s);
            o.kind = K_ZINV; o.m = s.d->pl[s.i]; o.A = w.slot(0);
            o.C = s.keep ? w.layer(0, s.i, s.d->nbl) : w.slot(4 + s.pp);
            s.pp ^= 1;
            s.gnext = o.C;
            PT_EMIT(s);
            if (sm.ires[0]) put_status(s.st, ST_SINGULAR);
            PT_REFINE(s, w.slot(0), s.gnext, s.d->pl[s.i]);
          }
        }
        // -------------------------------------- Gr(1,1)
        s.gsv = (a.mode == MODE_GN) ? w.layer(1, 0, s.d->nbl) : w.slot(11);
        op_esh_diag(o, s.d, 0, s.ec, w.slot(0), w, s.sr, s.sub_first);
        PT_EMIT(s);
        for (s.j = s.sub_first + 1; s.sub_first >= 0 && s.j < s.d->ncont; ++s.j)
          if (s.d->cblk[s.j] == 1) {
            set_simple(o, K_SUB, s.d->pl[0] * s.d->pl[0], w.sig(s.j), w.slot(0));
            PT_EMIT(s);
          }
        if (s.d->nbl > 1) {
          if (s.d->has_s) {
            op_esh_up(o, s.d, 0, s.ec, w.slot(1));
            PT_EMIT(s);
            op_esh_lo(o, s.d, 0, s.ec, w.slot(2));
            PT_EMIT(s);
          }
          set_gemm(o, s.d->pl[0], s.d->pl[1], s.d->pl[1], esh_up_op(s.d, 0, w.slot(1)), s.d->pl[0], OP_N, s.gnext,
                   s.d->pl[1], OP_N, w.slot(3), s.d->pl[0], esh_al(s.d, one), zero);
          PT_EMIT(s);
          set_gemm(o, s.d->pl[0], s.d->pl[0], s.d->pl[1], w.slot(3), s.d->pl[0], OP_N, esh_lo_op(s.d, 0, w.slot(2)),
                   s.d->pl[1], OP_N, w.slot(0), s.d->pl[0], esh_al(s.d, mone), one);
          PT_EMIT(s);
        }
        o.kind = K_ZINV; o.m = s.d->pl[0]; o.A = w.slot(0); o.C = s.gsv;
        PT_EMIT(s);
        if (sm.ires[0]) put_status(s.st, ST_SINGULAR);
        PT_REFINE(s, w.slot(0), s.gsv, s.d->pl[0]);
        if (s.fast) {
          // ------------------------------------ 2-contact trace (iterative_cpu.F90:399-470)
          s.lo = s.d->pl[0];
          s.q = 0;
          goto trans2;
        }
        // -------------------------------------- forward retarded sweep
        // T / DOS: Gr(i,i) ping-pongs in slots 11/10, Gr(bl1,bl1) kept in slot 9.
        // GN: Gr(i,i) -> layer 1, Gr(i-1,i) -> layer 2.
        s.cur = 0;
        if (a.mode != MODE_T) s.last = s.d->nbl - 1;
        for (s.i = 0; s.i <= s.last; ++s.i) {
          if (s.i > 0) {
            // gr_step(i): E1 = ESH(i-1,i) slot 0, E2 = ESH(i,i-1) slot 1, X slot 2, W2 slot 3, GL slot 6
            if (s.d->has_s) {
              op_esh_up(o, s.d, s.i - 1, s.ec, w.slot(0));
              PT_EMIT(s);
              op_esh_lo(o, s.d, s.i - 1, s.ec, w.slot(1));
              PT_EMIT(s);
            }
            set_gemm(o, s.d->pl[s.i], s.d->pl[s.i - 1], s.d->pl[s.i], w.layer(0, s.i, s.d->nbl), s.d->pl[s.i], OP_N,
                     esh_lo_op(s.d, s.i - 1, w.slot(1)), s.d->pl[s.i], OP_N, w.slot(2), s.d->pl[s.i],
                     esh_al(s.d, one), zero);                                                     // gsmr(i) ESH(i,i-1)
            PT_EMIT(s);
            set_gemm(o, s.d->pl[s.i], s.d->pl[s.i - 1], s.d->pl[s.i - 1], w.slot(2), s.d->pl[s.i], OP_N,
                     (a.mode == MODE_GN) ? w.layer(1, s.i - 1, s.d->nbl) : w.slot(11 - s.cur), s.d->pl[s.i - 1], OP_N,
                     w.slot(6), s.d->pl[s.i], mone, zero);                                         // Gr(i,i-1)
            PT_EMIT(s);
            set_gemm(o, s.d->pl[s.i - 1], s.d->pl[s.i], s.d->pl[s.i], esh_up_op(s.d, s.i - 1, w.slot(0)),
                     s.d->pl[s.i - 1], OP_N, w.layer(0, s.i, s.d->nbl), s.d->pl[s.i], OP_N, w.slot(3),
                     s.d->pl[s.i - 1], esh_al(s.d, one), zero);                                   // ESH gsmr
            PT_EMIT(s);
            if (a.mode == MODE_GN) {
              set_gemm(o, s.d->pl[s.i - 1], s.d->pl[s.i], s.d->pl[s.i - 1], w.layer(1, s.i - 1, s.d->nbl),
                       s.d->pl[s.i - 1], OP_N, w.slot(3), s.d->pl[s.i - 1], OP_N, w.layer(2, s.i - 1, s.d->nbl),
                       s.d->pl[s.i - 1], mone, zero);                                              // Gr(i-1,i)
              PT_EMIT(s);
            }
            if (a.mode == MODE_RHO) {
              // Gr(i-1,i) = -Gr(i-1,i-1) ESH(i-1,i) gsmr(i); then w Gr(i,i-1), w Gr(i-1,i) into the sums
              set_gemm(o, s.d->pl[s.i - 1], s.d->pl[s.i], s.d->pl[s.i - 1], w.slot(11 - s.cur), s.d->pl[s.i - 1],
                       OP_N, w.slot(3), s.d->pl[s.i - 1], OP_N, w.slot(5), s.d->pl[s.i - 1], mone, zero);
              PT_EMIT(s);
              set_simple(o, K_ACCUM, s.d->pl[s.i] * s.d->pl[s.i - 1], w.slot(6), a.acc_l + s.d->oo[s.i - 1]);
              o.alpha = a.weight[s.p];
              PT_EMIT(s);
              set_simple(o, K_ACCUM, s.d->pl[s.i] * s.d->pl[s.i - 1], w.slot(5), a.acc_u + s.d->oo[s.i - 1]);
              o.alpha = a.weight[s.p];
              PT_EMIT(s);
            }
            set_simple(o, K_COPY, s.d->pl[s.i] * s.d->pl[s.i], w.layer(0, s.i, s.d->nbl),
                       (a.mode == MODE_GN) ? w.layer(1, s.i, s.d->nbl) : w.slot(11 - (s.cur ^ 1)));
            PT_EMIT(s);
            set_gemm(o, s.d->pl[s.i], s.d->pl[s.i], s.d->pl[s.i - 1], w.slot(6), s.d->pl[s.i], OP_N, w.slot(3),
                     s.d->pl[s.i - 1], OP_N,
                     (a.mode == MODE_GN) ? w.layer(1, s.i, s.d->nbl) : w.slot(11 - (s.cur ^ 1)), s.d->pl[s.i], mone,
                     one);                                                                         // Gr(i,i)
            PT_EMIT(s);
            s.cur ^= 1;
          }
          if (a.mode == MODE_RHO) {
            set_simple(o, K_ACCUM, s.d->pl[s.i] * s.d->pl[s.i], w.slot(11 - s.cur), a.acc_d + s.d->od[s.i]);
            o.alpha = a.weight[s.p];
            PT_EMIT(s);
          }
          if (a.mode == MODE_DOS && a.dos) {
            set_simple(o, K_DOS, s.d->pl[s.i], w.slot(11 - s.cur), nullptr);
            o.out = a.dos + (int64_t)s.p * a.dos_stride + s.d->pstart[s.i];
            PT_EMIT(s);
          }
          if (a.mode != MODE_GN)
            for (s.j = 0; s.j < s.d->ncont; ++s.j)
              if (s.d->cblk[s.j] == s.i + 1) {
                set_simple(o, K_COPY, s.d->pl[s.i] * s.d->pl[s.i], w.slot(11 - s.cur), w.keep(s.j));
                PT_EMIT(s);
              }
        }
        if (a.mode == MODE_RHO) {
          if (a.acc_lc)
            // calculate_Gr_outer, outer_blocks = 2 (src/iterative.F90:1463-1573): for every contact
            // -Gr(cb,cb) Tlc gs and -gs Tcl Gr(cb,cb), summed with the weight (masked on the host)
            for (s.c = 0; s.c < s.d->ncont; ++s.c) {
              s.L = s.d->L[s.c];
              s.ncb = s.d->pl[s.d->cblk[s.c] - 1];
              set_esh(o, w.slot(0), s.ncb, s.L, s.d->hmc + s.d->omc[s.c],
                      s.d->has_smc ? s.d->smc + s.d->omc[s.c] : nullptr, s.ecs, 0, nullptr, nullptr, OP_N);   // Tlc
              PT_EMIT(s);
              set_gemm(o, s.ncb, s.L, s.ncb, w.keep(s.c), s.ncb, OP_N, w.slot(0), s.ncb, OP_N, w.slot(2), s.ncb,
                       mone, zero);
              PT_EMIT(s);
              set_gemm(o, s.ncb, s.L, s.L, w.slot(2), s.ncb, OP_N, w.gskeep(s.c), s.L, OP_N, w.slot(3), s.ncb, one,
                       zero);
              PT_EMIT(s);
              set_simple(o, K_ACCUM, s.ncb * s.L, w.slot(3), a.acc_lc + s.d->omc[s.c]);
              o.alpha = a.weight[s.p];
              PT_EMIT(s);
              set_esh(o, w.slot(1), s.L, s.ncb, s.d->hmc + s.d->omc[s.c],
                      s.d->has_smc ? s.d->smc + s.d->omc[s.c] : nullptr, cconj(s.ecs), 0, nullptr, nullptr, OP_C);  // Tcl
              PT_EMIT(s);
              set_gemm(o, s.L, s.ncb, s.L, w.gskeep(s.c), s.L, OP_N, w.slot(1), s.L, OP_N, w.slot(2), s.L, mone,
                       zero);
              PT_EMIT(s);
              set_gemm(o, s.L, s.ncb, s.ncb, w.slot(2), s.L, OP_N, w.keep(s.c), s.ncb, OP_N, w.slot(3), s.L, one,
                       zero);
              PT_EMIT(s);
              set_simple(o, K_ACCUM, s.ncb * s.L, w.slot(3), a.acc_cl + s.d->omc[s.c]);
              o.alpha = a.weight[s.p];
              PT_EMIT(s);
            }
          goto point_done;
        }
        if (a.mode != MODE_GN) {
          if (a.mode == MODE_DOS && a.ldos && a.dos && s.d->nldos > 0) {
            o.kind = K_LDOS; o.A = reinterpret_cast<const double2*>(a.dos + (int64_t)s.p * a.dos_stride);
            o.out = a.ldos + (int64_t)s.p * a.ldos_stride; o.dd = s.d;
            PT_EMIT(s);
          }
          for (s.q = 0; s.q < s.npairs; ++s.q) {
            pair_of(a, s, s.q);
            if (s.d->ncont == 1) { s.T = 0.0; goto pair_done; }
            if (a.mode == MODE_DOS && s.d->ncont == 2) {
              s.lo = s.d->pl[s.bl1 - 1];
              s.gsv = w.keep(s.ct1);
              goto trans2;
            }
            // ---------------------------------- column sweep Gr(i,bl1) (iterative_cpu.F90:507-538)
            set_simple(o, K_COPY, s.d->pl[s.bl1 - 1] * s.d->pl[s.bl1 - 1], w.keep(s.ct1), w.slot(9));
            PT_EMIT(s);
            s.cc = 0;
            s.tiny = 0;
            for (s.i = s.bl1; s.i <= s.bl2 - 1; ++s.i) {
              set_simple(o, K_MAXABS, s.d->pl[s.i - 1] * s.d->pl[s.bl1 - 1], s.cc ? w.slot(6) : w.slot(9), nullptr);
              o.slot = 0;
              PT_EMIT(s);
              if (sm.res[0] < a.eps) { s.tiny = 1; break; }
              if (s.d->has_s) {
                op_esh_lo(o, s.d, s.i - 1, s.ec, w.slot(0));
                PT_EMIT(s);
              }
              set_gemm(o, s.d->pl[s.i], s.d->pl[s.i - 1], s.d->pl[s.i], w.layer(0, s.i, s.d->nbl), s.d->pl[s.i],
                       OP_N, esh_lo_op(s.d, s.i - 1, w.slot(0)), s.d->pl[s.i], OP_N, w.slot(1), s.d->pl[s.i],
                       esh_al(s.d, mone), zero);
              PT_EMIT(s);
              set_gemm(o, s.d->pl[s.i], s.d->pl[s.bl1 - 1], s.d->pl[s.i - 1], w.slot(1), s.d->pl[s.i], OP_N,
                       s.cc ? w.slot(6) : w.slot(9), s.d->pl[s.i - 1], OP_N, s.cc ? w.slot(9) : w.slot(6),
                       s.d->pl[s.i], one, zero);
              PT_EMIT(s);
              s.cc ^= 1;
            }
            if (s.tiny) { s.T = a.eps * a.eps; goto pair_done; }
            // ---------------------------------- N-contact trace |Re Tr[Gam2 G21 Gam1 G21^dag]|
            // Gam1 slot 7, Gam2 slot 8, W1 slot 2, W2 slot 3; G21 in slot 9 or 6
            set_simple(o, K_SPECTRAL, s.d->pl[s.bl1 - 1], w.sig(s.ct1), w.slot(7));
            PT_EMIT(s);
            set_simple(o, K_SPECTRAL, s.d->pl[s.bl2 - 1], w.sig(s.ct2), w.slot(8));
            PT_EMIT(s);
            set_gemm(o, s.d->pl[s.bl2 - 1], s.d->pl[s.bl1 - 1], s.d->pl[s.bl2 - 1], w.slot(8), s.d->pl[s.bl2 - 1],
                     OP_N, s.cc ? w.slot(6) : w.slot(9), s.d->pl[s.bl2 - 1], OP_N, w.slot(2), s.d->pl[s.bl2 - 1], one,
                     zero);
            PT_EMIT(s);
            set_gemm(o, s.d->pl[s.bl2 - 1], s.d->pl[s.bl1 - 1], s.d->pl[s.bl1 - 1], w.slot(2), s.d->pl[s.bl2 - 1],
                     OP_N, w.slot(7), s.d->pl[s.bl1 - 1], OP_N, w.slot(3), s.d->pl[s.bl2 - 1], one, zero);
            PT_EMIT(s);
            o.kind = K_TRACEN; o.m = s.d->pl[s.bl2 - 1]; o.n = s.d->pl[s.bl1 - 1]; o.A = w.slot(3);
            o.B = s.cc ? w.slot(6) : w.slot(9); o.slot = 0; o.mask = tun_mask_of(s.d, s.bl2);
            PT_EMIT(s);
            s.T = fabs(sm.res[0]);
            goto pair_done;
          trans2:
            // |Re Tr[Gam1 i(G - G^dag) - Gam1 G Gam1 G^dag]| over the tun_proj rows of block bl1;
            // G in s.gsv, order s.lo.  Gam slot 7, W1 slot 8, W2 slot 2, A slot 3
            set_simple(o, K_SPECTRAL, s.lo, w.sig(s.ct1), w.slot(7));
            PT_EMIT(s);
            set_simple(o, K_SPECTRAL, s.lo, s.gsv, w.slot(3));
            PT_EMIT(s);
            set_gemm(o, s.lo, s.lo, s.lo, w.slot(7), s.lo, OP_N, s.gsv, s.lo, OP_N, w.slot(8), s.lo, one, zero);
            PT_EMIT(s);
            set_gemm(o, s.lo, s.lo, s.lo, w.slot(8), s.lo, OP_N, w.slot(7), s.lo, OP_N, w.slot(2), s.lo, one, zero);
            PT_EMIT(s);
            o.kind = K_TRACE; o.m = s.lo; o.A = w.slot(2); o.B = s.gsv; o.opb = OP_C; o.slot = 0;  // Tr(Gam G Gam G^dag)
            o.mask = tun_mask_of(s.d, s.bl1);
            PT_EMIT(s);
            o.kind = K_TRACE; o.m = s.lo; o.A = w.slot(7); o.B = w.slot(3); o.opb = OP_N; o.slot = 1;  // Tr(Gam A)
            o.mask = tun_mask_of(s.d, s.bl1);
            PT_EMIT(s);
            s.T = fabs(sm.res[1] - sm.res[0]);
          pair_done:
            if (!isfinite(s.T)) put_status(s.st, ST_NONFINITE);
            if (threadIdx.x == 0 && a.T) a.T[(int64_t)s.p * s.npairs + s.q] = s.T;
            __syncthreads();
          }
          goto point_done;
        }
        // ================================== elastic SCBA: lesser sweep (GN)
        // sigma_r = D diag(Gr)
        if (a.coupling)
          for (s.i = 0; s.i < s.d->nbl; ++s.i) {
            set_simple(o, K_SIGDIAG, s.d->pl[s.i], w.layer(1, s.i, s.d->nbl), s.vec + s.d->pstart[s.i]);
            o.cpl = a.coupling + s.d->pstart[s.i];
            o.scal = a.scba_mix;
            o.flag = (a.scba_mix == 1.0) ? 0 : (s.sit > 0 ? 1 : 2);   // linear mixing from sigma = 0
            PT_EMIT(s);
          }
        // Sigma_n(i,i) = dephasing (it > 0) + contacts (f_c - f_ref) Gam_c, f_ref = 0
        for (s.i = 0; s.i < s.d->nbl; ++s.i) {
          set_simple(o, K_SNINIT, s.d->pl[s.i],
                     (s.sit > 0 && a.coupling) ? s.vec + s.d->norb + s.d->pstart[s.i] : nullptr,
                     w.layer(3, s.i, s.d->nbl));
          PT_EMIT(s);
        }
        for (s.c = 0; s.c < s.d->ncont; ++s.c) {
          if (fabs(a.frm[(int64_t)s.p * a.frm_stride + s.c]) > a.eps) {
            set_simple(o, K_SNGAMMA, s.d->pl[s.d->cblk[s.c] - 1], w.sig(s.c), w.layer(3, s.d->cblk[s.c] - 1, s.d->nbl));
            o.scal = a.frm[(int64_t)s.p * a.frm_stride + s.c];
            PT_EMIT(s);
          }
        }
        // upward fold of Sigma_n (calculate_sigma_n); gns slot 6, T1 slot 7, E1 slot 8
        s.i = s.d->nbl - 1;
        set_gemm(o, s.d->pl[s.i], s.d->pl[s.i], s.d->pl[s.i], w.layer(0, s.i, s.d->nbl), s.d->pl[s.i], OP_N,
                 w.layer(3, s.i, s.d->nbl), s.d->pl[s.i], OP_N, w.slot(7), s.d->pl[s.i], one, zero);
        PT_EMIT(s);
        set_gemm(o, s.d->pl[s.i], s.d->pl[s.i], s.d->pl[s.i], w.slot(7), s.d->pl[s.i], OP_N,
                 w.layer(0, s.i, s.d->nbl), s.d->pl[s.i], OP_C, w.slot(6), s.d->pl[s.i], one, zero);
        PT_EMIT(s);
        for (s.i = s.d->nbl - 2; s.i >= 0; --s.i) {
          if (s.d->has_s) {
            op_esh_up(o, s.d, s.i, s.ec, w.slot(8));
            PT_EMIT(s);
          }
          set_gemm(o, s.d->pl[s.i], s.d->pl[s.i + 1], s.d->pl[s.i + 1], esh_up_op(s.d, s.i, w.slot(8)), s.d->pl[s.i],
                   OP_N, w.slot(6), s.d->pl[s.i + 1], OP_N, w.slot(7), s.d->pl[s.i], esh_al(s.d, one), zero);
          PT_EMIT(s);
          set_gemm(o, s.d->pl[s.i], s.d->pl[s.i], s.d->pl[s.i + 1], w.slot(7), s.d->pl[s.i], OP_N,
                   esh_up_op(s.d, s.i, w.slot(8)), s.d->pl[s.i], OP_C, w.layer(3, s.i, s.d->nbl), s.d->pl[s.i],
                   esh_al(s.d, one), one);
          PT_EMIT(s);
          if (s.i > 0) {
            set_gemm(o, s.d->pl[s.i], s.d->pl[s.i], s.d->pl[s.i], w.layer(0, s.i, s.d->nbl), s.d->pl[s.i], OP_N,
                     w.layer(3, s.i, s.d->nbl), s.d->pl[s.i], OP_N, w.slot(7), s.d->pl[s.i], one, zero);
            PT_EMIT(s);
            set_gemm(o, s.d->pl[s.i], s.d->pl[s.i], s.d->pl[s.i], w.slot(7), s.d->pl[s.i], OP_N,
                     w.layer(0, s.i, s.d->nbl), s.d->pl[s.i], OP_C, w.slot(6), s.d->pl[s.i], one, zero);
            PT_EMIT(s);
          }
        }
        // Gn(1,1) = Gr(1,1) Sigma_n(1,1) Gr(1,1)^dag
        set_gemm(o, s.d->pl[0], s.d->pl[0], s.d->pl[0], w.layer(3, 0, s.d->nbl), s.d->pl[0], OP_N,
                 w.layer(1, 0, s.d->nbl), s.d->pl[0], OP_C, w.slot(7), s.d->pl[0], one, zero);
        PT_EMIT(s);
        set_gemm(o, s.d->pl[0], s.d->pl[0], s.d->pl[0], w.layer(1, 0, s.d->nbl), s.d->pl[0], OP_N, w.slot(7),
                 s.d->pl[0], OP_N, w.layer(4 + s.par, 0, s.d->nbl), s.d->pl[0], one, zero);
        PT_EMIT(s);
        // downward sweep; E2 slot 9, Gn(i+1,i) slot 10
        for (s.i = 0; s.i + 1 < s.d->nbl; ++s.i) {
          if (s.d->has_s) {
            op_esh_lo(o, s.d, s.i, s.ec, w.slot(9));
            PT_EMIT(s);
          }
          set_gemm(o, s.d->pl[s.i + 1], s.d->pl[s.i], s.d->pl[s.i + 1], w.layer(3, s.i + 1, s.d->nbl),
                   s.d->pl[s.i + 1], OP_N, w.layer(2, s.i, s.d->nbl), s.d->pl[s.i], OP_C, w.slot(7), s.d->pl[s.i + 1],
                   one, zero);
          PT_EMIT(s);
          set_gemm(o, s.d->pl[s.i + 1], s.d->pl[s.i], s.d->pl[s.i], esh_lo_op(s.d, s.i, w.slot(9)), s.d->pl[s.i + 1],
                   OP_N, w.layer(4 + s.par, s.i, s.d->nbl), s.d->pl[s.i], OP_N, w.slot(7), s.d->pl[s.i + 1],
                   esh_al(s.d, mone), one);
          PT_EMIT(s);
          set_gemm(o, s.d->pl[s.i + 1], s.d->pl[s.i], s.d->pl[s.i + 1], w.layer(0, s.i + 1, s.d->nbl),
                   s.d->pl[s.i + 1], OP_N, w.slot(7), s.d->pl[s.i + 1], OP_N, w.slot(10), s.d->pl[s.i + 1], one, zero);
          PT_EMIT(s);
          o.kind = K_DAGGER; o.m = s.d->pl[s.i]; o.n = s.d->pl[s.i + 1]; o.A = w.slot(10);
          o.C = w.layer(6 + s.par, s.i, s.d->nbl);
          PT_EMIT(s);
          set_gemm(o, s.d->pl[s.i + 1], s.d->pl[s.i + 1], s.d->pl[s.i + 1], w.layer(3, s.i + 1, s.d->nbl),
                   s.d->pl[s.i + 1], OP_N, w.layer(1, s.i + 1, s.d->nbl), s.d->pl[s.i + 1], OP_C, w.slot(7),
                   s.d->pl[s.i + 1], one, zero);
          PT_EMIT(s);
          set_gemm(o, s.d->pl[s.i + 1], s.d->pl[s.i + 1], s.d->pl[s.i], esh_lo_op(s.d, s.i, w.slot(9)),
                   s.d->pl[s.i + 1], OP_N, w.layer(6 + s.par, s.i, s.d->nbl), s.d->pl[s.i], OP_N, w.slot(7),
                   s.d->pl[s.i + 1], esh_al(s.d, mone), one);
          PT_EMIT(s);
          set_gemm(o, s.d->pl[s.i + 1], s.d->pl[s.i + 1], s.d->pl[s.i + 1], w.layer(0, s.i + 1, s.d->nbl),
                   s.d->pl[s.i + 1], OP_N, w.slot(7), s.d->pl[s.i + 1], OP_N, w.layer(4 + s.par, s.i + 1, s.d->nbl),
                   s.d->pl[s.i + 1], one, zero);
          PT_EMIT(s);
        }
        // set_Gn (sigma_n = D diag(Gn)) and the SCBA error on the S pattern
        if (threadIdx.x == 0) sm.res[1] = 0.0;
        __syncthreads();
        for (s.i = 0; s.i < s.d->nbl; ++s.i) {
          if (s.have_old && a.scba_rule == 0) {
            if (!s.d->has_s) {
              o.kind = K_ERRDIAG; o.m = s.d->pl[s.i]; o.A = w.layer(4 + s.par, s.i, s.d->nbl);
              o.B = w.layer(4 + (s.par ^ 1), s.i, s.d->nbl); o.slot = 1;
              PT_EMIT(s);
            } else {
              o.kind = K_ERRPAT; o.m = s.d->pl[s.i]; o.n = s.d->pl[s.i]; o.A = w.layer(4 + s.par, s.i, s.d->nbl);
              o.B = w.layer(4 + (s.par ^ 1), s.i, s.d->nbl); o.X = s.d->sd + s.d->od[s.i]; o.Y = nullptr; o.slot = 1;
              PT_EMIT(s);
              if (s.i + 1 < s.d->nbl) {
                o.kind = K_ERRPAT; o.m = s.d->pl[s.i]; o.n = s.d->pl[s.i + 1];
                o.A = w.layer(6 + s.par, s.i, s.d->nbl); o.B = w.layer(6 + (s.par ^ 1), s.i, s.d->nbl);
                o.X = s.d->su + s.d->oo[s.i]; o.Y = s.d->sl + s.d->oo[s.i]; o.slot = 1;
                PT_EMIT(s);
              }
            }
          }
          if (a.coupling) {
            set_simple(o, K_SIGDIAG, s.d->pl[s.i], w.layer(4 + s.par, s.i, s.d->nbl),
                       s.vec + s.d->norb + s.d->pstart[s.i]);
            o.cpl = a.coupling + s.d->pstart[s.i];
            o.scal = a.scba_mix;
            o.flag = (a.scba_mix == 1.0) ? 0 : (s.sit > 0 ? 1 : 2);
            PT_EMIT(s);
          }
        }
        if (a.scba_rule == 1) {
          // stopping rule 1: change of the contact-1 Meir-Wingreen current between sweeps
          // (the formula of the final currents below; Gam slot 7, A slot 8)
          set_simple(o, K_SPECTRAL, s.d->pl[s.d->cblk[0] - 1], w.sig(0), w.slot(7));
          PT_EMIT(s);
          set_simple(o, K_SPECTRAL, s.d->pl[s.d->cblk[0] - 1], w.layer(1, s.d->cblk[0] - 1, s.d->nbl), w.slot(8));
          PT_EMIT(s);
          o.kind = K_TRACE; o.m = s.d->pl[s.d->cblk[0] - 1]; o.A = w.slot(7);
          o.B = w.layer(4 + s.par, s.d->cblk[0] - 1, s.d->nbl); o.opb = OP_N; o.slot = 2; o.mask = nullptr;
          PT_EMIT(s);
          o.kind = K_TRACE; o.m = s.d->pl[s.d->cblk[0] - 1]; o.A = w.slot(7); o.B = w.slot(8); o.opb = OP_N;
          o.slot = 3; o.mask = nullptr;
          PT_EMIT(s);
          {
            const double icur = -(sm.res[2] - a.frm[(int64_t)s.p * a.frm_stride] * sm.res[3]);
            if (s.have_old) {
              s.err = fabs(icur - s.iold);
              s.conv = s.err < a.scba_tol;
            }
            s.iold = icur;
          }
          __syncthreads();
        } else if (s.have_old) {
          s.err = sm.res[1];
          s.conv = s.err < a.scba_tol;
        }
        s.have_old = 1;
        s.par ^= 1;
        ++s.sit;
      }
      s.par ^= 1;   // parity of the last computed Gn
      if (a.acc_d) {
        // real_axis_int (src/integrations.F90:1093-1176): w_p Gn(E_p) summed over the points
        for (s.i = 0; s.i < s.d->nbl; ++s.i) {
          set_simple(o, K_ACCUM, s.d->pl[s.i] * s.d->pl[s.i], w.layer(4 + s.par, s.i, s.d->nbl),
                     a.acc_d + s.d->od[s.i]);
          o.alpha = a.weight[s.p];
          PT_EMIT(s);
          if (s.i + 1 < s.d->nbl) {
            set_simple(o, K_ACCUM, s.d->pl[s.i] * s.d->pl[s.i + 1], w.layer(6 + s.par, s.i, s.d->nbl),
                       a.acc_u + s.d->oo[s.i]);                                     // Gn(i,i+1)
            o.alpha = a.weight[s.p];
            PT_EMIT(s);
            o.kind = K_DAGGER; o.m = s.d->pl[s.i + 1]; o.n = s.d->pl[s.i]; o.A = w.layer(6 + s.par, s.i, s.d->nbl);
            o.C = w.slot(10);                                                       // Gn(i+1,i)
            PT_EMIT(s);
            set_simple(o, K_ACCUM, s.d->pl[s.i] * s.d->pl[s.i + 1], w.slot(10), a.acc_l + s.d->oo[s.i]);
            o.alpha = a.weight[s.p];
            PT_EMIT(s);
          }
        }
        if (a.acc_lc)
          // calculate_Gn_outer, outer_blocks = 2 (src/iterative.F90:1576-1665): per contact
          // Gn(cb,c) = -Gn(cb,cb) Tlc gs^dag - (f_c - f_ref) Gr(cb,cb) Tlc i(gs - gs^dag), and
          // Gn(c,cb) = Gn(cb,c)^dag, summed with the weight (masked on the host)
          for (s.c = 0; s.c < s.d->ncont; ++s.c) {
            s.L = s.d->L[s.c];
            s.ncb = s.d->pl[s.d->cblk[s.c] - 1];
            set_esh(o, w.slot(0), s.ncb, s.L, s.d->hmc + s.d->omc[s.c],
                    s.d->has_smc ? s.d->smc + s.d->omc[s.c] : nullptr, s.ecs, 0, nullptr, nullptr, OP_N);   // Tlc
            PT_EMIT(s);
            set_gemm(o, s.ncb, s.L, s.L, w.slot(0), s.ncb, OP_N, w.gnkeep(s.c), s.L, OP_C, w.slot(2), s.ncb, one,
                     zero);                                                                                 // Tlc gA
            PT_EMIT(s);
            set_gemm(o, s.ncb, s.L, s.ncb, w.layer(4 + s.par, s.d->cblk[s.c] - 1, s.d->nbl), s.ncb, OP_N, w.slot(2),
                     s.ncb, OP_N, w.slot(3), s.ncb, mone, zero);
            PT_EMIT(s);
            if (fabs(a.frm[(int64_t)s.p * a.frm_stride + s.c]) > a.eps) {
              set_simple(o, K_SPECTRAL, s.L, w.gnkeep(s.c), w.slot(1));                 // i (gs - gs^dag)
              PT_EMIT(s);
              set_gemm(o, s.ncb, s.L, s.L, w.slot(0), s.ncb, OP_N, w.slot(1), s.L, OP_N, w.slot(2), s.ncb, one, zero);
              PT_EMIT(s);
              set_gemm(o, s.ncb, s.L, s.ncb, w.layer(1, s.d->cblk[s.c] - 1, s.d->nbl), s.ncb, OP_N, w.slot(2),
                       s.ncb, OP_N, w.slot(3), s.ncb, cz(-a.frm[(int64_t)s.p * a.frm_stride + s.c], 0.0), one);
              PT_EMIT(s);
            }
            set_simple(o, K_ACCUM, s.ncb * s.L, w.slot(3), a.acc_lc + s.d->omc[s.c]);
            o.alpha = a.weight[s.p];
            PT_EMIT(s);
            o.kind = K_DAGGER; o.m = s.L; o.n = s.ncb; o.A = w.slot(3); o.C = w.slot(2);      // L x ncb
            PT_EMIT(s);
            set_simple(o, K_ACCUM, s.ncb * s.L, w.slot(2), a.acc_cl + s.d->omc[s.c]);
            o.alpha = a.weight[s.p];
            PT_EMIT(s);
          }
      }
      // ------------------------------------ Meir-Wingreen (iterative.F90:382-414); Gam slot 7, A slot 8
      if (a.curr)
        for (s.c = 0; s.c < s.d->ncont; ++s.c) {
          set_simple(o, K_SPECTRAL, s.d->pl[s.d->cblk[s.c] - 1], w.sig(s.c), w.slot(7));
          PT_EMIT(s);
          set_simple(o, K_SPECTRAL, s.d->pl[s.d->cblk[s.c] - 1], w.layer(1, s.d->cblk[s.c] - 1, s.d->nbl), w.slot(8));
          PT_EMIT(s);
          o.kind = K_TRACE; o.m = s.d->pl[s.d->cblk[s.c] - 1]; o.A = w.slot(7);
          o.B = w.layer(4 + s.par, s.d->cblk[s.c] - 1, s.d->nbl); o.opb = OP_N; o.slot = 2; o.mask = nullptr;
          PT_EMIT(s);
          o.kind = K_TRACE; o.m = s.d->pl[s.d->cblk[s.c] - 1]; o.A = w.slot(7); o.B = w.slot(8); o.opb = OP_N;
          o.slot = 3; o.mask = nullptr;
          PT_EMIT(s);
          if (threadIdx.x == 0)
            a.curr[(int64_t)s.p * a.curr_stride + s.c] =
                -(sm.res[2] - a.frm[(int64_t)s.p * a.frm_stride + s.c] * sm.res[3]);
          __syncthreads();
        }
      // ------------------------------------ layer currents / densities (iterative.F90:427-461)
      if (a.lcurr || a.ldens)
        for (s.i = 0; s.i < s.d->nbl; ++s.i) {
          if (a.ldens) {
            o.kind = K_TRDIAG; o.m = s.d->pl[s.i]; o.A = w.layer(4 + s.par, s.i, s.d->nbl); o.slot = 2;
            PT_EMIT(s);
            if (threadIdx.x == 0) a.ldens[(int64_t)s.p * a.ldens_stride + s.i] = sm.res[2];
            __syncthreads();
          }
          if (a.lcurr && s.i + 1 < s.d->nbl) {
            op_esh_up(o, s.d, s.i, s.ec, w.slot(8));
            PT_EMIT(s);
            op_esh_lo(o, s.d, s.i, s.ec, w.slot(9));
            PT_EMIT(s);
            o.kind = K_TRACEC; o.m = s.d->pl[s.i]; o.n = s.d->pl[s.i + 1]; o.A = w.slot(8);
            o.B = w.layer(6 + s.par, s.i, s.d->nbl); o.opb = OP_C; o.slot = 2;   // Tr(ESH(i,i+1) Gn(i+1,i))
            PT_EMIT(s);
            o.kind = K_TRACEC; o.m = s.d->pl[s.i]; o.n = s.d->pl[s.i + 1]; o.A = w.layer(6 + s.par, s.i, s.d->nbl);
            o.B = w.slot(9); o.opb = OP_N; o.slot = 4;                           // Tr(Gn(i,i+1) ESH(i+1,i))
            PT_EMIT(s);
            if (threadIdx.x == 0) a.lcurr[(int64_t)s.p * a.lcurr_stride + s.i] = -(sm.res[3] - sm.res[5]);
            __syncthreads();
          }
        }
      if (threadIdx.x == 0) {
        if (a.scba_iter) a.scba_iter[s.p] = s.sit;
        if (a.scba_err) a.scba_err[s.p] = s.err;
      }
      goto point_done;

    point_done:
      if (threadIdx.x == 0) {
        if (a.ncyc) a.ncyc[s.p] = s.ncyc;
        if (a.status) a.status[s.p] = s.st;
      }
      __syncthreads();
    }
    goto program_end;

    refine:
      // residual probe of the inverse just formed; a Newton step where it failed
      for (s.rk = 0; s.rk < 2; ++s.rk) {
        o.kind = K_RESPROBE; o.m = s.rm; o.A = s.rA; o.B = s.rX; o.slot = 7;
        PT_EMIT(s);
        if (s.in_dec && s.rk == 0 && sm.res[8] > kSensitiveCond) s.sens = 1;
        if (!(sm.res[7] > kInvProbeTol) || !(sm.res[7] <= 1.7976931348623157e308)) break;   // fine, or non-finite
        o.kind = K_EYE; o.m = s.rm; o.C = w.slot(S_INV);
        PT_EMIT(s);
        set_gemm(o, s.rm, s.rm, s.rm, s.rA, s.rm, OP_N, s.rX, s.rm, OP_N, w.slot(S_INV), s.rm, mone, one);
        PT_EMIT(s);                                                                      // R = I - A X
        set_simple(o, K_COPY, s.rm * s.rm, s.rX, w.slot(S_INV + 1));
        PT_EMIT(s);
        set_gemm(o, s.rm, s.rm, s.rm, s.rX, s.rm, OP_N, w.slot(S_INV), s.rm, OP_N, w.slot(S_INV + 1), s.rm, one, one);
        PT_EMIT(s);                                                                      // X + X R
        set_simple(o, K_COPY, s.rm * s.rm, w.slot(S_INV + 1), s.rX);
        PT_EMIT(s);
      }
      s.pc = s.rret;
      goto dispatch;
  }
program_end:
  s.pc = -1;
  return false;
}

#undef PT_REFINE
#undef PT_EMIT

// ---------------------------------------------------------------- stepping
// State of a CTA between two heavy steps (local memory of the kernel).
struct EngineCtl {
  Prog prog;
  Op op;
  InvProg ip;
  int in_inv;       // an inversion is in progress (ip)
  int open;         // phase of the heavy step just run (TR_GEMM, TR_INV_PANEL) or -1
  long long t0;
};

enum StepKind : int { STEP_DONE = 0, STEP_GEMM = 1, STEP_LEAF = 2, STEP_ROWS = 3 };

// Runs the point program (generator, inversion driver, light operations)
// up to the next heavy step and returns it: STEP_GEMM (descriptor published
// at sm.main + kGemmDescOffset), STEP_LEAF (leaf of c.ip), STEP_ROWS
// (row-owner node update of c.ip) or STEP_DONE.
// The kernel runs the heavy step itself.  Compiled in program.cu, apart
// from the kernel, so that the product loop in the kernel is register-
// allocated without the control code around it.
__device__ int engine_step(const EngineArgs& a, EngineCtl& c, SmemMap& sm);

}  // namespace negf
