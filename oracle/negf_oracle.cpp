// Test infrastructure only -- the parity checker of this repository, never
// part of the product path.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load it.
//
// CPU restatement of libNEGF's per-energy-point transport solve, following
// the reference Fortran op for op and issuing the same LAPACK/BLAS sequence
// (zgetrf + zgetrs against the identity for every inverse, zgemm with the
// accumulate-if-allocated rule of prealloc_mult).  The reference itself
// cannot be compiled on this image (no Fortran compiler); its own golden
// T(E) files are git-LFS pointers that are absent, so the restatement is
// pinned by analytic known answers (perfect chain T = 1 in band, closed-form
// surface Green's function, the chain current of tests/f90elph_deph) and by
// an independent NumPy twin (oracle/twin.py).
//
// Reference files followed (paths inside the libNEGF tree):
//   src/inversions.F90:807-839            zinv
//   src/sparsekit_drv.F90:1896-2081       zmultdns / zmultdnss (prealloc_mult)
//   src/sparsekit_drv.F90:2870-2890       zspectral_dns
//   src/sparsekit_drv.F90:3200-3223       ztrace_dns
//   src/contselfenergy.F90:115-268        surface_green (surfdim = 0)
//   src/contselfenergy.F90:271-340        decimation
//   src/contselfenergy.F90:445-491        compute_contacts_dns
//   src/contselfenergy.F90:552-566        SelfEnergy_dns
//   src/iterative.F90:1956-1982           build_ESH
//   src/iterative_cpu.F90:51-124          calculate_gsmr_blocks
//   src/iterative_cpu.F90:134-224         calculate_Gr_tridiag_blocks
//   src/iterative_cpu.F90:230-372         calculate_Gn_tridiag_blocks
//   src/iterative_cpu.F90:399-470         calculate_single_transmission_2_contacts
//   src/iterative_cpu.F90:477-583         calculate_single_transmission_N_contacts
//   src/iterative_cpu.F90:586-618         get_tun_mask (tun_proj)
//   src/iterative.F90:1669-1780           calculate_transmissions
//   src/iterative.F90:1821-1952           calculate_transmissions_and_dos
//   src/iterative.F90:174-279, 289-363    calculate_Gn_neq_components, elastic SCBA
//   src/elphdd.F90:108-156, 227-276       local dephasing sigma_r / sigma_n
//   src/scba.F90:120-147                  check_Mat_convergence
//   src/iterative.F90:382-461             meir_wingreen / layer current kernels
//   src/distributions.F90:27-72           fermi_f
//   src/integrations.F90:2688-2830        integrate_el, integrate_el_meir_wingreen
//   src/integrations.F90:844-897, 2287    contour_int, compute_Gr (density matrix)
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/negf_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

using cplx = std::complex<double>;

extern "C" {
void scipy_zgemm_(const char* ta, const char* tb, const int* m, const int* n,
                  const int* k, const cplx* alpha, const cplx* a,
                  const int* lda, const cplx* b, const int* ldb,
                  const cplx* beta, cplx* c, const int* ldc, size_t, size_t);
void scipy_zgetrf_(const int* m, const int* n, cplx* a, const int* lda,
                   int* ipiv, int* info);
void scipy_zgetrs_(const char* t, const int* n, const int* nrhs,
                   const cplx* a, const int* lda, const int* ipiv, cplx* b,
                   const int* ldb, int* info, size_t);
void scipy_openblas_set_num_threads(int);
}

namespace {

const cplx I1(0.0, 1.0);

// type(z_DNS): allocated flag + column-major values (src/mat_def.F90:199-204)
struct Dns {
  int nr = 0, nc = 0;
  bool alloc = false;
  std::vector<cplx> v;
  void create(int r, int c) {
    nr = r; nc = c; alloc = true;
    v.assign((size_t)r * c, cplx(0.0, 0.0));
  }
  void destroy() { alloc = false; v.clear(); v.shrink_to_fit(); nr = nc = 0; }
  cplx& at(int i, int j) { return v[(size_t)j * nr + i]; }
  const cplx& at(int i, int j) const { return v[(size_t)j * nr + i]; }
};

struct Err {
  int code = NEGF_B200_OK;
  void set(int c) { if (code == NEGF_B200_OK) code = c; }
};

// prealloc_mult: C = s*A*B if C is not allocated (beta = 0), else C += s*A*B
// (zmultdns/zmultdnss, src/sparsekit_drv.F90:1896-2081).
void mult(const Dns& A, const Dns& B, Dns& C, cplx s = cplx(1.0, 0.0)) {
  int M = A.nr, N = B.nc, K = A.nc;
  cplx beta(0.0, 0.0);
  if (C.alloc) beta = cplx(1.0, 0.0); else C.create(M, N);
  if (M == 0 || N == 0) return;
  int lda = std::max(M, 1), ldb = std::max(B.nr, 1), ldc = std::max(M, 1);
  scipy_zgemm_("N", "N", &M, &N, &K, &s, A.v.data(), &lda, B.v.data(), &ldb,
               &beta, C.v.data(), &ldc, 1, 1);
}

// zinv: LU = A, zgetrf, identity, zgetrs (src/inversions.F90:807-839)
void zinv(Dns& inA, const Dns& A, Err& err) {
  int n = A.nr;
  Dns LU = A;
  std::vector<int> ipiv(std::max(n, 1));
  int info = 0;
  scipy_zgetrf_(&n, &n, LU.v.data(), &n, ipiv.data(), &info);
  if (info != 0) err.set(NEGF_B200_ERR_SINGULAR);
  inA.create(n, n);
  for (int i = 0; i < n; ++i) inA.at(i, i) = cplx(1.0, 0.0);
  scipy_zgetrs_("N", &n, &n, LU.v.data(), &n, ipiv.data(), inA.v.data(), &n,
                &info, 1);
}

void dagger(const Dns& A, Dns& Ad) {
  Ad.create(A.nc, A.nr);
  for (int j = 0; j < A.nc; ++j)
    for (int i = 0; i < A.nr; ++i) Ad.at(j, i) = std::conj(A.at(i, j));
}

// zspectral_dns(G, G, 0, A): A = i*(G - G^dag)
void spectral(const Dns& G, Dns& A) {
  Dns Ga;
  dagger(G, Ga);
  A.create(Ga.nr, Ga.nc);
  for (size_t i = 0; i < A.v.size(); ++i) A.v[i] = I1 * (G.v[i] - Ga.v[i]);
}

cplx trace(const Dns& M) {
  cplx t(0.0, 0.0);
  for (int i = 0; i < M.nr; ++i) t += M.at(i, i);
  return t;
}

// trace(M, mask) with the tun_proj mask of get_tun_mask
// (src/iterative_cpu.F90:586-618): mask[k] != 0 selects diagonal entry k;
// no mask = the whole diagonal.
cplx trace_mask(const Dns& M, const unsigned char* mask) {
  if (!mask) return trace(M);
  cplx t(0.0, 0.0);
  for (int i = 0; i < M.nr; ++i)
    if (mask[i]) t += M.at(i, i);
  return t;
}

double maxabs(const Dns& M) {
  double m = 0.0;
  for (const cplx& z : M.v) m = std::max(m, std::abs(z));
  return m;
}

Dns from_ptr(const double* p, int r, int c) {
  Dns d;
  d.create(r, c);
  if (p) std::memcpy(d.v.data(), p, sizeof(cplx) * (size_t)r * c);
  return d;
}

// ---------------------------------------------------------------------------
// Device description unpacked into dense blocks (CSR -> blocks is done by the
// caller, as zcsr2blk_sod would).
struct DeviceBlocks {
  int nbl = 0, ncont = 0;
  std::vector<int> n;           // PL sizes
  std::vector<Dns> Hd, Hu, Hl;  // H(i,i), H(i,i+1), H(i+1,i)
  std::vector<Dns> Sd, Su, Sl;
  bool s_id = true;
  std::vector<int> cblk, L;
  std::vector<Dns> H00, H01, S00, S01, HMC, SMC;
  std::vector<int> surf;          // bound surface orbitals per contact (surfdim)
  std::vector<Dns> HS, SS;        // H, S over Surf + PL1 (surf > 0 only)
  int norb = 0;
  std::vector<int> start;       // 0-based start orbital of each PL
};

DeviceBlocks unpack(const negf_b200_device* d) {
  DeviceBlocks B;
  B.nbl = d->nbl;
  B.ncont = d->ncont;
  B.n.assign(d->pl_size, d->pl_size + d->nbl);
  B.s_id = (d->s_diag == nullptr);
  size_t od = 0, oo = 0;
  B.start.resize(B.nbl);
  for (int i = 0; i < B.nbl; ++i) {
    B.start[i] = B.norb;
    B.norb += B.n[i];
    int ni = B.n[i];
    B.Hd.push_back(from_ptr(d->h_diag + 2 * od, ni, ni));
    if (!B.s_id) B.Sd.push_back(from_ptr(d->s_diag + 2 * od, ni, ni));
    od += (size_t)ni * ni;
    if (i + 1 < B.nbl) {
      int nj = B.n[i + 1];
      B.Hu.push_back(from_ptr(d->h_upper + 2 * oo, ni, nj));
      B.Hl.push_back(from_ptr(d->h_lower + 2 * oo, nj, ni));
      if (!B.s_id) {
        B.Su.push_back(from_ptr(d->s_upper + 2 * oo, ni, nj));
        B.Sl.push_back(from_ptr(d->s_lower + 2 * oo, nj, ni));
      }
      oo += (size_t)ni * nj;
    }
  }
  size_t ol = 0, om = 0, os = 0;
  for (int c = 0; c < B.ncont; ++c) {
    int L = d->lead_size[c];
    int cb = d->cblk[c];
    B.cblk.push_back(cb);
    B.L.push_back(L);
    const int n0 = d->surf_size ? d->surf_size[c] : 0;
    B.surf.push_back(n0);
    const int ngs = L + n0;
    if (n0 > 0) {
      B.HS.push_back(from_ptr(d->lead_hs + 2 * os, ngs, ngs));
      Dns ss = from_ptr(d->lead_ss ? d->lead_ss + 2 * os : nullptr, ngs, ngs);
      if (!d->lead_ss)
        for (int i = 0; i < ngs; ++i) ss.at(i, i) = 1.0;
      B.SS.push_back(ss);
      os += (size_t)ngs * ngs;
    } else {
      B.HS.push_back(Dns());
      B.SS.push_back(Dns());
    }
    int ncb = B.n[cb - 1];
    B.H00.push_back(from_ptr(d->lead_h00 + 2 * ol, L, L));
    B.H01.push_back(from_ptr(d->lead_h01 + 2 * ol, L, L));
    Dns s00 = from_ptr(d->lead_s00 ? d->lead_s00 + 2 * ol : nullptr, L, L);
    if (!d->lead_s00)
      for (int i = 0; i < L; ++i) s00.at(i, i) = 1.0;
    B.S00.push_back(s00);
    B.S01.push_back(from_ptr(d->lead_s01 ? d->lead_s01 + 2 * ol : nullptr, L, L));
    B.HMC.push_back(from_ptr(d->hmc + 2 * om, ncb, ngs));
    B.SMC.push_back(from_ptr(d->smc ? d->smc + 2 * om : nullptr, ncb, ngs));
    ol += (size_t)L * L;
    om += (size_t)ncb * ngs;
  }
  return B;
}

// ---------------------------------------------------------------------------
// decimation (src/contselfenergy.F90:271-340).  Ao, Bo, Co are overwritten.
void decimation(Dns& Go, Dns& Ao, Dns& Bo, Dns& Co, int n, int& ncyc,
                double sgf_acc, int max_iter, Err& err) {
  Dns Ao_s = Ao;
  bool okCo = false;
  int i1;
  for (i1 = 1; i1 <= max_iter; ++i1) {
    ncyc = i1;
    Go.destroy();
    zinv(Go, Ao, err);
    Dns GoXCo; mult(Go, Co, GoXCo);
    Dns C1; mult(Co, GoXCo, C1);
    if (maxabs(C1) <= sgf_acc) {
      if (okCo) break;
      okCo = true;
    } else {
      okCo = false;
    }
    Dns Self; mult(Bo, GoXCo, Self);
    for (size_t i = 0; i < Ao.v.size(); ++i) {
      Ao_s.v[i] -= Self.v[i];
      Ao.v[i] -= Self.v[i];
    }
    Dns GoXBo; mult(Go, Bo, GoXBo);
    Dns B1; mult(Bo, GoXBo, B1);
    Bo = B1;
    mult(Co, GoXBo, Ao, cplx(-1.0, 0.0));  // Ao = Ao - Co*GoXBo (beta = 1)
    Co = C1;
  }
  ncyc = i1;  // Fortran DO index after the loop: max_iter+1 if never exited
  if (ncyc > max_iter) err.set(NEGF_B200_ERR_NOT_CONVERGED);
  Go.destroy();
  zinv(Go, Ao_s, err);
  (void)n;
}

// The bound-surface block of surface_green (src/contselfenergy.F90:226-243):
// with n0 surface orbitals ahead of the periodic PLs, GS (n0+L square) is
// the inverse of E S - H over Surf + PL1 whose PL1 block is replaced by the
// inverse of the decimation's Go.
void bound_surface(cplx E, const DeviceBlocks& D, int c, Dns& GS, Err& err) {
  const int n0 = D.surf[c];
  if (n0 == 0) return;
  const int L = D.L[c], ngs = n0 + L;
  Dns Ginv;
  zinv(Ginv, GS, err);
  Dns gt;
  gt.create(ngs, ngs);
  for (size_t q = 0; q < gt.v.size(); ++q) gt.v[q] = E * D.SS[c].v[q] - D.HS[c].v[q];
  for (int j = 0; j < L; ++j)
    for (int i = 0; i < L; ++i) gt.at(n0 + i, n0 + j) = Ginv.at(i, j);
  GS.destroy();
  zinv(GS, gt, err);
}

// surface_green, no cache (src/contselfenergy.F90:115-268)
void surface_green(cplx E, const DeviceBlocks& D, int c, Dns& GS, int& ncyc,
                   double sgf_acc, int max_iter, Err& err) {
  int L = D.L[c];
  Dns Ao, Bo, Co, Ct;
  Ao.create(L, L); Bo.create(L, L); Ct.create(L, L);
  for (size_t i = 0; i < Ao.v.size(); ++i) {
    Ao.v[i] = E * D.S00[c].v[i] - D.H00[c].v[i];
    Bo.v[i] = E * D.S01[c].v[i] - D.H01[c].v[i];
    Ct.v[i] = std::conj(E) * D.S01[c].v[i] - D.H01[c].v[i];
  }
  dagger(Ct, Co);
  decimation(GS, Ao, Bo, Co, L, ncyc, sgf_acc, max_iter, err);
  bound_surface(E, D, c, GS, err);
}

// compute_contacts_dns (src/contselfenergy.F90:445-491) + SelfEnergy_dns
struct ContactParts {   // GS, Tlc, Tcl per contact (for calculate_Gr_outer)
  std::vector<Dns> GS, Tlc, Tcl;
};

void compute_contacts(cplx Ec, const DeviceBlocks& D, std::vector<Dns>& Sig,
                      int& ncyc_max, double sgf_acc, int max_iter, Err& err,
                      ContactParts* parts = nullptr) {
  Sig.assign(D.ncont, Dns());
  ncyc_max = 0;
  if (parts) {
    parts->GS.assign(D.ncont, Dns());
    parts->Tlc.assign(D.ncont, Dns());
    parts->Tcl.assign(D.ncont, Dns());
  }
  for (int c = 0; c < D.ncont; ++c) {
    Dns GS;
    int ncyc = 0;
    surface_green(Ec, D, c, GS, ncyc, sgf_acc, max_iter, err);
    ncyc_max += ncyc;  // total over contacts
    const Dns& HMC = D.HMC[c];
    const Dns& SMC = D.SMC[c];
    Dns Tlc, TpMt, Tcl;
    Tlc.create(HMC.nr, HMC.nc);
    TpMt.create(HMC.nr, HMC.nc);
    for (size_t i = 0; i < HMC.v.size(); ++i) {
      Tlc.v[i] = -HMC.v[i] + Ec * SMC.v[i];
      TpMt.v[i] = -HMC.v[i] + std::conj(Ec) * SMC.v[i];
    }
    dagger(TpMt, Tcl);
    Dns TG;
    mult(Tlc, GS, TG);
    mult(TG, Tcl, Sig[c]);
    if (parts) {
      parts->GS[c] = GS;
      parts->Tlc[c] = Tlc;
      parts->Tcl[c] = Tcl;
    }
  }
}

// ESH blocks: tridiagonal ES-H (zcsr2blk_sod layout); index (i,j) 0-based.
struct Trid {
  int nbl;
  std::vector<Dns> d, u, l;  // (i,i), (i,i+1), (i+1,i)
  explicit Trid(int n = 0) : nbl(n), d(n), u(n > 0 ? n - 1 : 0), l(n > 0 ? n - 1 : 0) {}
};

// build_ESH (src/iterative.F90:1956-1982): ES - H, then ESH(cb,cb) -= Sigma_c
void build_ESH(cplx Ec, const DeviceBlocks& D, const std::vector<Dns>* Sig,
               Trid& ESH) {
  ESH = Trid(D.nbl);
  for (int i = 0; i < D.nbl; ++i) {
    int ni = D.n[i];
    ESH.d[i].create(ni, ni);
    for (size_t q = 0; q < ESH.d[i].v.size(); ++q) {
      cplx s = D.s_id ? cplx(0.0, 0.0) : D.Sd[i].v[q];
      ESH.d[i].v[q] = Ec * s - D.Hd[i].v[q];
    }
    if (D.s_id)
      for (int k = 0; k < ni; ++k) ESH.d[i].at(k, k) += Ec;
    if (i + 1 < D.nbl) {
      ESH.u[i].create(D.Hu[i].nr, D.Hu[i].nc);
      ESH.l[i].create(D.Hl[i].nr, D.Hl[i].nc);
      for (size_t q = 0; q < ESH.u[i].v.size(); ++q) {
        cplx su = D.s_id ? cplx(0.0, 0.0) : D.Su[i].v[q];
        cplx sl = D.s_id ? cplx(0.0, 0.0) : D.Sl[i].v[q];
        ESH.u[i].v[q] = Ec * su - D.Hu[i].v[q];
        ESH.l[i].v[q] = Ec * sl - D.Hl[i].v[q];
      }
    }
  }
  if (Sig)
    for (int c = 0; c < D.ncont; ++c) {
      Dns& B = ESH.d[D.cblk[c] - 1];
      for (size_t q = 0; q < B.v.size(); ++q) B.v[q] -= (*Sig)[c].v[q];
    }
}

// calculate_gsmr_blocks(ESH, sbl, ebl, gsmr, keep) -- 1-based sbl/ebl
void gsmr_blocks(const Trid& ESH, int sbl, int ebl, std::vector<Dns>& gsmr,
                 bool keep, Err& err) {
  if (sbl < ebl) return;
  int nbl = ESH.nbl;
  if (nbl == 1) return;
  gsmr[sbl - 1].destroy();
  zinv(gsmr[sbl - 1], ESH.d[sbl - 1], err);
  for (int i = sbl - 1; i >= ebl; --i) {
    Dns work1, work2;
    mult(ESH.u[i - 1], gsmr[i], work1, cplx(-1.0, 0.0));  // ESH(i,i+1) gsmr(i+1)
    if (!keep) gsmr[i].destroy();
    mult(work1, ESH.l[i - 1], work2);                      // * ESH(i+1,i)
    Dns w;
    w.create(work2.nr, work2.nc);
    for (size_t q = 0; q < w.v.size(); ++q) w.v[q] = ESH.d[i - 1].v[q] + work2.v[q];
    gsmr[i - 1].destroy();
    zinv(gsmr[i - 1], w, err);
  }
}

// Gr storage: diagonal, Gr(i,i-1) and Gr(i-1,i), plus column blocks Gr(i,bl1)
struct GrBlocks {
  std::vector<Dns> d, l, u;  // l[i] = Gr(i+1,i), u[i] = Gr(i,i+1) (0-based)
  explicit GrBlocks(int nbl = 0) : d(nbl), l(nbl > 0 ? nbl - 1 : 0), u(nbl > 0 ? nbl - 1 : 0) {}
};

// calculate_Gr_tridiag_blocks(ESH, gsmr, Gr, sbl) -- Gr(sbl,sbl) only
void Gr_first(const Trid& ESH, const std::vector<Dns>& gsmr, GrBlocks& Gr,
              int sbl, Err& err) {
  int nbl = ESH.nbl;
  int s = sbl - 1;
  if (nbl == 1) {
    Gr.d[s].destroy();
    zinv(Gr.d[s], ESH.d[s], err);
    return;
  }
  Dns work1 = ESH.d[s];
  if (sbl + 1 <= nbl) {
    Dns work2, work3;
    mult(ESH.u[s], gsmr[s + 1], work2);
    mult(work2, ESH.l[s], work3);
    for (size_t q = 0; q < work1.v.size(); ++q) work1.v[q] = work1.v[q] - work3.v[q];
  }
  Gr.d[s].destroy();
  zinv(Gr.d[s], work1, err);
}

// calculate_Gr_tridiag_blocks(ESH, gsmr, Gr, sbl, ebl), sbl > 1
void Gr_sweep(const Trid& ESH, const std::vector<Dns>& gsmr, GrBlocks& Gr,
              int sbl, int ebl) {
  for (int i = sbl; i <= ebl; ++i) {
    int k = i - 1;  // 0-based block i
    Dns work1, work2;
    mult(gsmr[k], ESH.l[k - 1], work1);                       // gsmr(i) ESH(i,i-1)
    mult(work1, Gr.d[k - 1], Gr.l[k - 1], cplx(-1.0, 0.0));   // Gr(i,i-1)
    work1.destroy();
    mult(ESH.u[k - 1], gsmr[k], work2);                       // ESH(i-1,i) gsmr(i)
    mult(Gr.d[k - 1], work2, Gr.u[k - 1], cplx(-1.0, 0.0));   // Gr(i-1,i)
    mult(Gr.l[k - 1], work2, work1, cplx(-1.0, 0.0));
    Gr.d[k].create(gsmr[k].nr, gsmr[k].nc);
    for (size_t q = 0; q < work1.v.size(); ++q) Gr.d[k].v[q] = gsmr[k].v[q] + work1.v[q];
  }
}

// calculate_single_transmission_2_contacts (src/iterative_cpu.F90:399-470)
double transmission_2(int ni, int nf, const std::vector<Dns>& Sig,
                      const std::vector<int>& cblk, const GrBlocks& Gr,
                      const unsigned char* tmask = nullptr, const std::vector<int>* start = nullptr) {
  int ct1 = (cblk[ni - 1] < cblk[nf - 1]) ? ni : nf;
  int bl1 = cblk[ct1 - 1];
  const Dns& G = Gr.d[bl1 - 1];
  Dns GA, GAM1, work1, work2, AA, TRS;
  dagger(G, GA);
  spectral(Sig[ct1 - 1], GAM1);
  mult(GAM1, G, work1);
  mult(work1, GAM1, work2);
  work1.destroy();
  mult(work2, GA, work1);
  work2.destroy();
  AA.create(GA.nr, GA.nc);
  for (size_t q = 0; q < AA.v.size(); ++q) AA.v[q] = I1 * (G.v[q] - GA.v[q]);
  mult(GAM1, AA, work2);
  TRS.create(work1.nr, work1.nc);
  for (size_t q = 0; q < TRS.v.size(); ++q) TRS.v[q] = work2.v[q] - work1.v[q];
  return std::abs(std::real(trace_mask(TRS, tmask ? tmask + (*start)[bl1 - 1] : nullptr)));
}

// calculate_single_transmission_N_contacts (src/iterative_cpu.F90:477-583)
double transmission_N(int ni, int nf, const Trid& ESH, const std::vector<Dns>& Sig,
                      const std::vector<int>& cblk, const std::vector<Dns>& gsmr,
                      GrBlocks& Gr, double eps, const unsigned char* tmask = nullptr,
                      const std::vector<int>* start = nullptr) {
  int ct1, ct2;
  if (cblk[ni - 1] < cblk[nf - 1]) { ct1 = ni; ct2 = nf; } else { ct1 = nf; ct2 = ni; }
  int bl1 = cblk[ct1 - 1], bl2 = cblk[ct2 - 1];
  int nblc = (int)cblk.size();
  // column blocks Gr(i,bl1), i = bl1..bl2 (0-based storage by row index)
  std::vector<Dns> col(ESH.nbl);
  col[bl1 - 1] = Gr.d[bl1 - 1];
  if (bl2 > bl1) col[bl1] = Gr.l[bl1 - 1];  // Gr(bl1+1,bl1) from the tridiagonal sweep
  if (nblc > 1 && (bl2 - bl1) > 1) {
    for (int i = bl1 + 1; i <= bl2; ++i) {
      double mx = maxabs(col[i - 2]);
      if (mx < eps) return eps * eps;
      if (!col[i - 1].alloc) {
        Dns work1;
        mult(gsmr[i - 1], ESH.l[i - 2], work1, cplx(-1.0, 0.0));
        mult(work1, col[i - 2], col[i - 1]);
      }
    }
  }
  const Dns& G21 = col[bl2 - 1];
  Dns GAM1, GAM2, work1, work2, GA, TRS;
  spectral(Sig[ct1 - 1], GAM1);
  spectral(Sig[ct2 - 1], GAM2);
  mult(GAM2, G21, work1);
  mult(work1, GAM1, work2);
  dagger(G21, GA);
  mult(work2, GA, TRS);
  return std::abs(std::real(trace_mask(TRS, tmask ? tmask + (*start)[bl2 - 1] : nullptr)));
}

struct Opts {
  double sgf_acc = 1e-9;
  int max_iter = 300;
  double eps = 0.0;
  // SCBA variants of the engine (not in the reference): linear mixing factor of the
  // dephasing self-energies (1 = overwrite, the reference) and stopping rule
  // (0 = max |dGn| on the S pattern, the reference; 1 = change of the contact-1 current)
  double scba_mix = 1.0;
  int scba_rule = 0;
};

// calculate_transmissions (src/iterative.F90:1669-1780) after
// compute_contacts(E + i*eta) (src/integrations.F90:1747)
double point_transmission(const DeviceBlocks& D, double E, double eta, int ni,
                          int nf, const Opts& o, int& ncyc, Err& err) {
  std::vector<Dns> Sig;
  compute_contacts(cplx(E, eta), D, Sig, ncyc, o.sgf_acc, o.max_iter, err);
  if (D.ncont == 1) return 0.0;
  Trid ESH;
  build_ESH(cplx(E, 0.0), D, &Sig, ESH);
  int nbl = D.nbl;
  int nt = std::min(D.cblk[ni - 1], D.cblk[nf - 1]);
  std::vector<Dns> gsmr(nbl);
  GrBlocks Gr(nbl);
  if (D.ncont == 2 && nt == 1) {
    gsmr_blocks(ESH, nbl, 2, gsmr, false, err);
    Gr_first(ESH, gsmr, Gr, 1, err);
    return transmission_2(ni, nf, Sig, D.cblk, Gr);
  }
  gsmr_blocks(ESH, nbl, 2, gsmr, true, err);
  int nt1 = std::max(D.cblk[ni - 1], D.cblk[nf - 1]);
  Gr_first(ESH, gsmr, Gr, 1, err);
  if (nt1 > 1) Gr_sweep(ESH, gsmr, Gr, 2, nt1);
  return transmission_N(ni, nf, ESH, Sig, D.cblk, gsmr, Gr, o.eps);
}

// calculate_transmissions_and_dos (src/iterative.F90:1821-1952); dos gets
// -Im(Gr_ii)/pi for every device orbital.
double point_transmission_dos(const DeviceBlocks& D, double E, double eta,
                              double dos_delta, int ni, int nf, const Opts& o,
                              double* dos, int& ncyc, Err& err) {
  std::vector<Dns> Sig;
  compute_contacts(cplx(E, eta), D, Sig, ncyc, o.sgf_acc, o.max_iter, err);
  Trid ESH;
  build_ESH(cplx(E, dos_delta), D, &Sig, ESH);
  int nbl = D.nbl;
  std::vector<Dns> gsmr(nbl);
  GrBlocks Gr(nbl);
  gsmr_blocks(ESH, nbl, 2, gsmr, true, err);
  Gr_first(ESH, gsmr, Gr, 1, err);
  if (nbl > 1) Gr_sweep(ESH, gsmr, Gr, 2, nbl);
  double tun = 0.0;
  if (D.ncont == 2)
    tun = transmission_2(ni, nf, Sig, D.cblk, Gr);
  else if (D.ncont > 2)
    tun = transmission_N(ni, nf, ESH, Sig, D.cblk, gsmr, Gr, o.eps);
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < nbl; ++i)
    for (int k = 0; k < D.n[i]; ++k)
      dos[D.start[i] + k] = -(1.0 / pi) * std::imag(Gr.d[i].at(k, k));
  return tun;
}

// calculate_transmissions (src/iterative.F90:1669-1780) for the contact
// pairs ni(:), nf(:) with the tun_proj mask.  The reference frees gsmr
// inside its pair loop after the first pair (:1766-1767), so a later pair
// whose contacts are more than one block apart would read freed blocks; here
// gsmr stays valid for every pair, which is the result the loop is meant to
// give (identical wherever the reference's loop is well defined).
void point_transmissions(const DeviceBlocks& D, double E, double eta, int npairs,
                         const int* ni, const int* nf, const unsigned char* tmask,
                         const Opts& o, double* T, int& ncyc, Err& err) {
  std::vector<Dns> Sig;
  compute_contacts(cplx(E, eta), D, Sig, ncyc, o.sgf_acc, o.max_iter, err);
  if (D.ncont == 1) {
    for (int q = 0; q < npairs; ++q) T[q] = 0.0;
    return;
  }
  Trid ESH;
  build_ESH(cplx(E, 0.0), D, &Sig, ESH);
  int nbl = D.nbl;
  int nt = std::min(D.cblk[ni[0] - 1], D.cblk[nf[0] - 1]);
  std::vector<Dns> gsmr(nbl);
  GrBlocks Gr(nbl);
  if (D.ncont == 2 && npairs == 1 && nt == 1) {
    gsmr_blocks(ESH, nbl, 2, gsmr, false, err);
    Gr_first(ESH, gsmr, Gr, 1, err);
    T[0] = transmission_2(ni[0], nf[0], Sig, D.cblk, Gr, tmask, &D.start);
    return;
  }
  gsmr_blocks(ESH, nbl, 2, gsmr, true, err);
  for (int q = 0; q < npairs; ++q) {
    int nt1 = std::max(D.cblk[ni[q] - 1], D.cblk[nf[q] - 1]);
    if (q == 0) {
      nt = nt1;
      Gr_first(ESH, gsmr, Gr, 1, err);
      if (nt > 1) Gr_sweep(ESH, gsmr, Gr, 2, nt);
    } else if (nt1 > nt) {
      Gr_sweep(ESH, gsmr, Gr, nt + 1, nt1);
      nt = nt1;
    }
    T[q] = transmission_N(ni[q], nf[q], ESH, Sig, D.cblk, gsmr, Gr, o.eps, tmask, &D.start);
  }
}

// calculate_transmissions_and_dos (src/iterative.F90:1821-1952) for the
// pairs and the LDOS index sets (dos_proj, 1-based orbital indices; set k
// holds idx[ptr[k]..ptr[k+1])); ledos[k] = sum over its indices of
// -Im Gr_ii / pi (indices past the device are skipped, :1936-1939).
void point_transmissions_ldos(const DeviceBlocks& D, double E, double eta, double dos_delta,
                              int npairs, const int* ni, const int* nf,
                              const unsigned char* tmask, int nsets, const int* ptr,
                              const int* idx, const Opts& o, double* T, double* ledos,
                              int& ncyc, Err& err) {
  std::vector<Dns> Sig;
  compute_contacts(cplx(E, eta), D, Sig, ncyc, o.sgf_acc, o.max_iter, err);
  Trid ESH;
  build_ESH(cplx(E, dos_delta), D, &Sig, ESH);
  int nbl = D.nbl;
  std::vector<Dns> gsmr(nbl);
  GrBlocks Gr(nbl);
  gsmr_blocks(ESH, nbl, 2, gsmr, true, err);
  Gr_first(ESH, gsmr, Gr, 1, err);
  if (nbl > 1) Gr_sweep(ESH, gsmr, Gr, 2, nbl);
  for (int q = 0; q < npairs; ++q) {
    if (D.ncont == 1) T[q] = 0.0;
    else if (D.ncont == 2) T[q] = transmission_2(ni[q], nf[q], Sig, D.cblk, Gr, tmask, &D.start);
    else T[q] = transmission_N(ni[q], nf[q], ESH, Sig, D.cblk, gsmr, Gr, o.eps, tmask, &D.start);
  }
  const double pi = 3.14159265358979323846;
  std::vector<double> diag(D.norb);
  for (int i = 0; i < nbl; ++i)
    for (int k = 0; k < D.n[i]; ++k)
      diag[D.start[i] + k] = -(1.0 / pi) * std::imag(Gr.d[i].at(k, k));
  for (int k = 0; k < nsets; ++k) {
    double acc = 0.0;
    for (int j = ptr[k]; j < ptr[k + 1]; ++j) {
      int i2 = idx[j];
      if (i2 >= 1 && i2 <= D.norb) acc += diag[i2 - 1];
    }
    ledos[k] = acc;
  }
}

// One contour point of contour_int (src/integrations.F90:844-897): Gr at the
// complex energy Ec (contacts and ES-H at Ec, compute_Gr :2287-2340 /
// calculate_Gr src/iterative.F90:90-148), all tridiagonal blocks.
void point_gr_blocks(const DeviceBlocks& D, cplx Ec, const Opts& o, GrBlocks& Gr, int& ncyc, Err& err,
                     ContactParts* parts = nullptr) {
  std::vector<Dns> Sig;
  compute_contacts(Ec, D, Sig, ncyc, o.sgf_acc, o.max_iter, err, parts);
  Trid ESH;
  build_ESH(Ec, D, &Sig, ESH);
  int nbl = D.nbl;
  std::vector<Dns> gsmr(nbl);
  gsmr_blocks(ESH, nbl, 2, gsmr, true, err);
  Gr_first(ESH, gsmr, Gr, 1, err);
  if (nbl > 1) Gr_sweep(ESH, gsmr, Gr, 2, nbl);
}

// calculate_Gn_tridiag_blocks (src/iterative_cpu.F90:230-372).
// Sigma_n holds the tridiagonal lesser self-energy (dephasing already added).
void Gn_blocks(const Trid& ESH, const std::vector<Dns>& Sig, const double* frm,
               int ref, const DeviceBlocks& D, const std::vector<Dns>& gsmr,
               const GrBlocks& Gr, Trid& Sn, Trid& Gn, double eps) {
  int nbl = D.nbl;
  for (int j = 1; j <= D.ncont; ++j) {
    double frmdiff = frm[j - 1] - frm[ref - 1];
    if (j != ref && std::abs(frmdiff) > eps) {
      int cb = D.cblk[j - 1];
      Dns Gam;
      spectral(Sig[j - 1], Gam);
      Dns& B = Sn.d[cb - 1];
      for (size_t q = 0; q < B.v.size(); ++q) B.v[q] += frmdiff * Gam.v[q];
    }
  }
  // calculate_sigma_n: upward fold
  if (nbl > 1) {
    Dns gsmrDag, work1, gns;
    dagger(gsmr[nbl - 1], gsmrDag);
    mult(gsmr[nbl - 1], Sn.d[nbl - 1], work1);
    mult(work1, gsmrDag, gns);
    for (int i = nbl - 1; i >= 1; --i) {
      int k = i - 1;  // 0-based block i
      Dns ESHdag, work;
      dagger(ESH.u[k], ESHdag);
      mult(ESH.u[k], gns, work);
      mult(work, ESHdag, Sn.d[k]);
      work.destroy(); gns.destroy();
      Dns gD;
      dagger(gsmr[k + 1], gD);
      mult(Sn.u[k], gD, work);
      mult(work, ESHdag, Sn.d[k], cplx(-1.0, 0.0));
      work.destroy();
      mult(ESH.u[k], gsmr[k + 1], work);
      mult(work, Sn.l[k], Sn.d[k], cplx(-1.0, 0.0));
      work.destroy();
      if (i > 1) {
        Dns gD2;
        dagger(gsmr[k], gD2);
        mult(gsmr[k], Sn.d[k], work);
        mult(work, gD2, gns);
      }
    }
  }
  {
    Dns Ga, work1;
    dagger(Gr.d[0], Ga);
    mult(Sn.d[0], Ga, work1);
    mult(Gr.d[0], work1, Gn.d[0]);
  }
  for (int i = 1; i <= nbl - 1; ++i) {
    int k = i - 1;
    Dns Ga, work1;
    dagger(Gr.d[k], Ga);
    mult(Sn.l[k], Ga, work1);
    dagger(Gr.u[k], Ga);
    mult(Sn.d[k + 1], Ga, work1);
    mult(ESH.l[k], Gn.d[k], work1, cplx(-1.0, 0.0));
    mult(gsmr[k + 1], work1, Gn.l[k]);
    work1.destroy();
    Gn.u[k].destroy();
    dagger(Gn.l[k], Gn.u[k]);
    dagger(Gr.l[k], Ga);
    mult(Sn.l[k], Ga, work1);
    dagger(Gr.d[k + 1], Ga);
    mult(Sn.d[k + 1], Ga, work1);
    mult(ESH.l[k], Gn.u[k], work1, cplx(-1.0, 0.0));
    mult(gsmr[k + 1], work1, Gn.d[k + 1]);
  }
}

void init_trid_zero(Trid& T, const Trid& like) {
  T = Trid(like.nbl);
  for (int i = 0; i < like.nbl; ++i) {
    T.d[i].create(like.d[i].nr, like.d[i].nc);
    if (i + 1 < like.nbl) {
      T.u[i].create(like.u[i].nr, like.u[i].nc);
      T.l[i].create(like.l[i].nr, like.l[i].nc);
    }
  }
}

// One energy point of meir_wingreen / layer_current with the elastic SCBA
// of calculate_elastic_scba (src/iterative.F90:289-363).
struct ScbaOut {
  int iters = 0;
  double err = 0.0;
};

void point_scba(const DeviceBlocks& D, double E, double eta, const double* frm,
                const double* coupling, int niter, double tol, const Opts& o,
                double* curr, double* lcurr, double* ldens, ScbaOut& so,
                int& ncyc, Err& err, Trid* gn_out = nullptr, ContactParts* parts = nullptr,
                std::vector<Dns>* grd_out = nullptr) {
  int nbl = D.nbl, ncont = D.ncont;
  std::vector<Dns> Sig;
  compute_contacts(cplx(E, eta), D, Sig, ncyc, o.sgf_acc, o.max_iter, err, parts);
  // meir_wingreen: ref = ncont+1 with f(ref) = 0 (src/integrations.F90:1833-1837)
  std::vector<double> frm_ext(frm, frm + ncont);
  frm_ext.push_back(0.0);
  int ref = ncont + 1;
  std::vector<double> D2(D.norb, 0.0);
  if (coupling)
    for (int q = 0; q < D.norb; ++q) D2[q] = coupling[q] * coupling[q];
  std::vector<cplx> sigma_r(D.norb, cplx(0.0, 0.0)), sigma_n(D.norb, cplx(0.0, 0.0));
  const double mix = o.scba_mix;
  // sigma <- D diag(G), or linear mixing from sigma = 0
  auto update = [&](cplx& sig, cplx g, double d2) {
    const cplx v = g * d2;
    sig = (mix == 1.0) ? v : mix * v + (1.0 - mix) * sig;
  };
  // iterative_meir_wingreen (src/iterative.F90:382-414) for contact c
  auto mw_current = [&](int c, const GrBlocks& Gr, const Trid& Gn) {
    int cb = D.cblk[c] - 1;
    Dns Gam, A, work1;
    spectral(Sig[c], Gam);
    mult(Gam, Gn.d[cb], work1);
    spectral(Gr.d[cb], A);
    mult(Gam, A, work1, cplx(-frm_ext[c], 0.0));
    return -std::real(trace(work1));
  };
  double iold = 0.0;
  // Mat_old pattern: S nonzeros inside the tridiagonal device blocks
  std::vector<cplx> old;
  bool have_old = false, converged = false;
  so.err = 0.0;
  int it = 0;
  Trid ESH, Gn;
  GrBlocks Gr(nbl);
  while (!converged && it <= niter) {
    build_ESH(cplx(E, 0.0), D, &Sig, ESH);
    if (it > 0 && coupling)
      for (int i = 0; i < nbl; ++i)
        for (int k = 0; k < D.n[i]; ++k) ESH.d[i].at(k, k) -= sigma_r[D.start[i] + k];
    std::vector<Dns> gsmr(nbl);
    gsmr_blocks(ESH, nbl, 2, gsmr, true, err);
    Gr = GrBlocks(nbl);
    Gr_first(ESH, gsmr, Gr, 1, err);
    if (nbl > 1) Gr_sweep(ESH, gsmr, Gr, 2, nbl);
    if (coupling && it <= niter)
      for (int i = 0; i < nbl; ++i)
        for (int k = 0; k < D.n[i]; ++k)
          update(sigma_r[D.start[i] + k], Gr.d[i].at(k, k), D2[D.start[i] + k]);
    Trid Sn;
    init_trid_zero(Sn, ESH);
    if (it > 0 && coupling)
      for (int i = 0; i < nbl; ++i)
        for (int k = 0; k < D.n[i]; ++k) Sn.d[i].at(k, k) += sigma_n[D.start[i] + k];
    init_trid_zero(Gn, ESH);
    Gn_blocks(ESH, Sig, frm_ext.data(), ref, D, gsmr, Gr, Sn, Gn, o.eps);
    if (coupling && it <= niter)
      for (int i = 0; i < nbl; ++i)
        for (int k = 0; k < D.n[i]; ++k)
          update(sigma_n[D.start[i] + k], Gn.d[i].at(k, k), D2[D.start[i] + k]);
    // blk2csr(Gn) on the S pattern + check_Mat_convergence
    std::vector<cplx> cur;
    for (int i = 0; i < nbl; ++i) {
      for (int q = 0; q < (int)Gn.d[i].v.size(); ++q) {
        bool nz = D.s_id ? (q % (D.n[i] + 1) == 0) : (D.Sd[i].v[q] != cplx(0.0, 0.0));
        if (nz) cur.push_back(Gn.d[i].v[q]);
      }
      if (!D.s_id && i + 1 < nbl) {
        for (size_t q = 0; q < Gn.u[i].v.size(); ++q)
          if (D.Su[i].v[q] != cplx(0.0, 0.0)) cur.push_back(Gn.u[i].v[q]);
        for (size_t q = 0; q < Gn.l[i].v.size(); ++q)
          if (D.Sl[i].v[q] != cplx(0.0, 0.0)) cur.push_back(Gn.l[i].v[q]);
      }
    }
    if (o.scba_rule == 1) {
      const double icur = mw_current(0, Gr, Gn);
      if (have_old) {
        so.err = std::abs(icur - iold);
        converged = so.err < tol;
      }
      iold = icur;
    } else if (have_old) {
      double e = 0.0;
      for (size_t q = 0; q < cur.size(); ++q) e = std::max(e, std::abs(cur[q] - old[q]));
      so.err = e;
      converged = e < tol;
    }
    old = cur;
    have_old = true;
    ++it;
  }
  so.iters = it;
  if (gn_out) *gn_out = Gn;
  if (grd_out) *grd_out = Gr.d;
  // iterative_meir_wingreen (src/iterative.F90:382-414)
  if (curr)
    for (int c = 0; c < ncont; ++c) curr[c] = mw_current(c, Gr, Gn);
  // iterative_layer_current (src/iterative.F90:427-461): ES-H without Sigma
  if (lcurr || ldens) {
    Trid E0;
    build_ESH(cplx(E, 0.0), D, nullptr, E0);
    for (int i = 0; i + 1 < nbl; ++i) {
      Dns work1;
      mult(E0.u[i], Gn.l[i], work1);
      mult(Gn.u[i], E0.l[i], work1, cplx(-1.0, 0.0));
      if (lcurr) lcurr[i] = std::real(I1 * trace(work1));
      if (ldens) ldens[i] = std::real(trace(Gn.d[i]));
    }
    if (ldens) ldens[nbl - 1] = std::real(trace(Gn.d[nbl - 1]));
  }
}

void set_threads(int nthreads) {
  scipy_openblas_set_num_threads(1);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}


// ---------------------------------------------------------------------------
// Independent-rounding restatements of the 2-contact T and T + DOS paths.
//
// The same steps as point_transmission / point_transmission_dos above
// (decimation with the two-consecutive max|C1| rule, compute_contacts,
// build_ESH, calculate_gsmr_blocks, Gr(1,1), the Gr sweep, the ct1 trace and
// -Im Gr_ii / pi), written over a real type R with their own unblocked LU
// (partial pivoting on max |Re|+|Im|, the izamax rule of zgetf2), triangular
// solves against the identity (zgetrs) and plain triple-loop products:
//   R = long double  (x87, 64-bit significand: unit roundoff 5.4e-20, about
//                     2000x below FP64) -- a near-exact solution of the same
//                     algorithm, used to measure how far each FP64 result
//                     (this oracle's, the GPU's) lies from it;
//   R = double       another FP64 rounding path than OpenBLAS's blocked
//                     kernels: two CPU FP64 implementations side by side.
namespace xp {

template <typename R>
struct C {
  R re, im;
};
template <typename R>
inline C<R> mk(R a, R b) { return C<R>{a, b}; }
template <typename R>
inline C<R> mul(C<R> a, C<R> b) { return mk<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
template <typename R>
inline C<R> add(C<R> a, C<R> b) { return mk<R>(a.re + b.re, a.im + b.im); }
template <typename R>
inline C<R> sub(C<R> a, C<R> b) { return mk<R>(a.re - b.re, a.im - b.im); }
template <typename R>
inline C<R> cj(C<R> a) { return mk<R>(a.re, -a.im); }
template <typename R>
inline C<R> rcp(C<R> z) {   // Smith's algorithm
  if (std::fabs(z.re) >= std::fabs(z.im)) {
    R r = z.im / z.re, d = z.re + z.im * r;
    return mk<R>(R(1) / d, -r / d);
  }
  R r = z.re / z.im, d = z.im + z.re * r;
  return mk<R>(r / d, R(-1) / d);
}

template <typename R>
struct Mat {
  int nr = 0, nc = 0;
  std::vector<C<R>> v;
  Mat() = default;
  Mat(int r, int c) : nr(r), nc(c), v((size_t)r * c, C<R>{0, 0}) {}
  C<R>& at(int i, int j) { return v[(size_t)j * nr + i]; }
  const C<R>& at(int i, int j) const { return v[(size_t)j * nr + i]; }
};

template <typename R>
Mat<R> from(const Dns& d) {
  Mat<R> m(d.nr, d.nc);
  for (size_t q = 0; q < d.v.size(); ++q) m.v[q] = mk<R>((R)d.v[q].real(), (R)d.v[q].imag());
  return m;
}

// C = s*A*B (acc = false) or C += s*A*B (acc = true): prealloc_mult
template <typename R>
void gemm(const Mat<R>& A, const Mat<R>& B, Mat<R>& Cm, C<R> s, bool acc) {
  if (!acc) Cm = Mat<R>(A.nr, B.nc);
  std::vector<C<R>> col(A.nr);
  for (int j = 0; j < B.nc; ++j) {
    for (int i = 0; i < A.nr; ++i) col[i] = C<R>{0, 0};
    for (int k = 0; k < A.nc; ++k) {
      const C<R> b = B.at(k, j);
      const C<R>* a = &A.v[(size_t)k * A.nr];
      for (int i = 0; i < A.nr; ++i) {
        col[i].re += a[i].re * b.re - a[i].im * b.im;
        col[i].im += a[i].re * b.im + a[i].im * b.re;
      }
    }
    for (int i = 0; i < A.nr; ++i) Cm.at(i, j) = add(Cm.at(i, j), mul(s, col[i]));
  }
}

// inverse by LU with partial pivoting + forward/backward solves against I
template <typename R>
int inv(const Mat<R>& A, Mat<R>& X) {
  const int n = A.nr;
  Mat<R> LU = A;
  std::vector<int> piv(n);
  int info = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    R best = -1;
    for (int i = k; i < n; ++i) {
      R a = std::fabs(LU.at(i, k).re) + std::fabs(LU.at(i, k).im);
      if (a > best) { best = a; p = i; }
    }
    piv[k] = p;
    if (best == 0) { if (!info) info = k + 1; continue; }
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(LU.at(k, j), LU.at(p, j));
    const C<R> r = rcp(LU.at(k, k));
    for (int i = k + 1; i < n; ++i) LU.at(i, k) = mul(LU.at(i, k), r);
    for (int j = k + 1; j < n; ++j) {
      const C<R> u = LU.at(k, j);
      for (int i = k + 1; i < n; ++i) LU.at(i, j) = sub(LU.at(i, j), mul(LU.at(i, k), u));
    }
  }
  X = Mat<R>(n, n);
  for (int i = 0; i < n; ++i) X.at(i, i) = C<R>{1, 0};
  for (int k = 0; k < n; ++k)   // row interchanges of the right-hand sides
    if (piv[k] != k)
      for (int j = 0; j < n; ++j) std::swap(X.at(k, j), X.at(piv[k], j));
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < n; ++k) {   // L y = b (unit diagonal)
      const C<R> y = X.at(k, j);
      for (int i = k + 1; i < n; ++i) X.at(i, j) = sub(X.at(i, j), mul(LU.at(i, k), y));
    }
    for (int k = n - 1; k >= 0; --k) {   // U x = y
      if (LU.at(k, k).re == 0 && LU.at(k, k).im == 0) continue;
      const C<R> x = mul(X.at(k, j), rcp(LU.at(k, k)));
      X.at(k, j) = x;
      for (int i = 0; i < k; ++i) X.at(i, j) = sub(X.at(i, j), mul(LU.at(i, k), x));
    }
  }
  return info;
}

// Gauss-Jordan inversion in place with partial pivoting (the same pivot
// rule), row interchanges recorded and undone as column interchanges at the
// end: the elimination order of the engine's inversion, unblocked.
template <typename R>
int inv_gj(const Mat<R>& A, Mat<R>& X) {
  const int n = A.nr;
  X = A;
  std::vector<int> piv(n);
  int info = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    R best = -1;
    for (int i = k; i < n; ++i) {
      R a = std::fabs(X.at(i, k).re) + std::fabs(X.at(i, k).im);
      if (a > best) { best = a; p = i; }
    }
    piv[k] = p;
    if (best == 0) { if (!info) info = k + 1; continue; }
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(X.at(k, j), X.at(p, j));
    const C<R> r = rcp(X.at(k, k));
    for (int j = 0; j < n; ++j) X.at(k, j) = (j == k) ? r : mul(X.at(k, j), r);
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      const C<R> f = X.at(i, k);
      for (int j = 0; j < n; ++j)
        if (j != k) X.at(i, j) = sub(X.at(i, j), mul(f, X.at(k, j)));
      X.at(i, k) = mul(mk<R>(-f.re, -f.im), r);
    }
  }
  for (int k = n - 1; k >= 0; --k)
    if (piv[k] != k)
      for (int i = 0; i < n; ++i) std::swap(X.at(i, k), X.at(i, piv[k]));
  return info;
}

// inversion used by the restatement: LU + solves, or Gauss-Jordan
inline int& inv_kind() { static thread_local int k = 0; return k; }
template <typename R>
int invert(const Mat<R>& A, Mat<R>& X) { return inv_kind() ? inv_gj(A, X) : inv(A, X); }

template <typename R>
Mat<R> dag(const Mat<R>& A) {
  Mat<R> D(A.nc, A.nr);
  for (int j = 0; j < A.nc; ++j)
    for (int i = 0; i < A.nr; ++i) D.at(j, i) = cj(A.at(i, j));
  return D;
}

template <typename R>
R maxabs(const Mat<R>& M) {
  R m = 0;
  for (const C<R>& z : M.v) m = std::max(m, (R)std::sqrt(z.re * z.re + z.im * z.im));
  return m;
}

// decimation (src/contselfenergy.F90:271-340)
template <typename R>
Mat<R> decimation(Mat<R> Ao, Mat<R> Bo, Mat<R> Co, R tol, int max_iter, int& ncyc, int& info) {
  Mat<R> Aos = Ao, Go, X, C1, Sf, Y, B1;
  const C<R> one{1, 0}, mone{-1, 0};
  bool ok = false;
  int it;
  for (it = 1; it <= max_iter; ++it) {
    if (invert(Ao, Go)) info = 1;
    gemm(Go, Co, X, one, false);
    gemm(Co, X, C1, one, false);
    if (maxabs(C1) <= tol) {
      if (ok) break;
      ok = true;
    } else {
      ok = false;
    }
    gemm(Bo, X, Sf, one, false);
    for (size_t q = 0; q < Ao.v.size(); ++q) {
      Aos.v[q] = sub(Aos.v[q], Sf.v[q]);
      Ao.v[q] = sub(Ao.v[q], Sf.v[q]);
    }
    gemm(Go, Bo, Y, one, false);
    gemm(Bo, Y, B1, one, false);
    gemm(Co, Y, Ao, mone, true);
    Bo = B1;
    Co = C1;
  }
  ncyc = it;
  if (invert(Aos, Go)) info = 1;
  return Go;
}

// one 2-contact point: T (dos == nullptr: ESH at E, gsmr down to block 2,
// Gr(1,1), trace) or T + DOS (ESH at E + i dos_delta, full Gr sweep)
template <typename R>
double point(const DeviceBlocks& D, double E, double eta, double dos_delta, double* dos, double tol,
             int max_iter, int& ncyc, int& info) {
  const C<R> one{1, 0}, mone{-1, 0};
  const C<R> Ec = mk<R>((R)E, (R)eta);
  ncyc = 0;
  std::vector<Mat<R>> Sig(D.ncont);
  for (int c = 0; c < D.ncont; ++c) {
    const int L = D.L[c];
    Mat<R> Ao(L, L), Bo(L, L), Ct(L, L);
    const Mat<R> H00 = from<R>(D.H00[c]), H01 = from<R>(D.H01[c]), S00 = from<R>(D.S00[c]),
                 S01 = from<R>(D.S01[c]), HMC = from<R>(D.HMC[c]), SMC = from<R>(D.SMC[c]);
    for (size_t q = 0; q < Ao.v.size(); ++q) {
      Ao.v[q] = sub(mul(Ec, S00.v[q]), H00.v[q]);
      Bo.v[q] = sub(mul(Ec, S01.v[q]), H01.v[q]);
      Ct.v[q] = sub(mul(cj(Ec), S01.v[q]), H01.v[q]);
    }
    int nc = 0;
    Mat<R> GS = decimation(Ao, Bo, dag(Ct), (R)tol, max_iter, nc, info);
    ncyc += nc;
    if (D.surf[c] > 0) {   // bound-surface block (src/contselfenergy.F90:226-243)
      const int n0 = D.surf[c], ngs = n0 + L;
      Mat<R> Ginv, gt(ngs, ngs);
      if (invert(GS, Ginv)) info = 1;
      const Mat<R> HS = from<R>(D.HS[c]), SS = from<R>(D.SS[c]);
      for (size_t q = 0; q < gt.v.size(); ++q) gt.v[q] = sub(mul(Ec, SS.v[q]), HS.v[q]);
      for (int j = 0; j < L; ++j)
        for (int i = 0; i < L; ++i) gt.at(n0 + i, n0 + j) = Ginv.at(i, j);
      if (invert(gt, GS)) info = 1;
    }
    Mat<R> Tlc(HMC.nr, HMC.nc), TpMt(HMC.nr, HMC.nc), TG;
    for (size_t q = 0; q < HMC.v.size(); ++q) {
      Tlc.v[q] = sub(mul(Ec, SMC.v[q]), HMC.v[q]);
      TpMt.v[q] = sub(mul(cj(Ec), SMC.v[q]), HMC.v[q]);
    }
    gemm(Tlc, GS, TG, one, false);
    gemm(TG, dag(TpMt), Sig[c], one, false);
  }
  const int nbl = D.nbl;
  const C<R> Ed = mk<R>((R)E, dos ? (R)dos_delta : (R)0);
  std::vector<Mat<R>> d(nbl), u(nbl > 0 ? nbl - 1 : 0), l(nbl > 0 ? nbl - 1 : 0);
  for (int i = 0; i < nbl; ++i) {
    const Mat<R> H = from<R>(D.Hd[i]);
    d[i] = Mat<R>(H.nr, H.nc);
    for (size_t q = 0; q < H.v.size(); ++q) {
      C<R> s = D.s_id ? C<R>{0, 0} : mk<R>((R)D.Sd[i].v[q].real(), (R)D.Sd[i].v[q].imag());
      d[i].v[q] = sub(mul(Ed, s), H.v[q]);
    }
    if (D.s_id)
      for (int k = 0; k < H.nr; ++k) d[i].at(k, k) = add(d[i].at(k, k), Ed);
    if (i + 1 < nbl) {
      const Mat<R> Hu = from<R>(D.Hu[i]), Hl = from<R>(D.Hl[i]);
      u[i] = Mat<R>(Hu.nr, Hu.nc);
      l[i] = Mat<R>(Hl.nr, Hl.nc);
      for (size_t q = 0; q < Hu.v.size(); ++q) {
        C<R> su = D.s_id ? C<R>{0, 0} : mk<R>((R)D.Su[i].v[q].real(), (R)D.Su[i].v[q].imag());
        C<R> sl = D.s_id ? C<R>{0, 0} : mk<R>((R)D.Sl[i].v[q].real(), (R)D.Sl[i].v[q].imag());
        u[i].v[q] = sub(mul(Ed, su), Hu.v[q]);
        l[i].v[q] = sub(mul(Ed, sl), Hl.v[q]);
      }
    }
  }
  for (int c = 0; c < D.ncont; ++c) {
    Mat<R>& B = d[D.cblk[c] - 1];
    for (size_t q = 0; q < B.v.size(); ++q) B.v[q] = sub(B.v[q], Sig[c].v[q]);
  }
  // gsmr(nbl) .. gsmr(2)
  std::vector<Mat<R>> g(nbl);
  if (nbl > 1) {
    if (invert(d[nbl - 1], g[nbl - 1])) info = 1;
    for (int i = nbl - 2; i >= 1; --i) {
      Mat<R> w1, w2;
      gemm(u[i], g[i + 1], w1, mone, false);
      gemm(w1, l[i], w2, one, false);
      for (size_t q = 0; q < w2.v.size(); ++q) w2.v[q] = add(d[i].v[q], w2.v[q]);
      if (invert(w2, g[i])) info = 1;
    }
  }
  // Gr(1,1)
  std::vector<Mat<R>> Gd(nbl);
  {
    Mat<R> w = d[0];
    if (nbl > 1) {
      Mat<R> w2, w3;
      gemm(u[0], g[1], w2, one, false);
      gemm(w2, l[0], w3, one, false);
      for (size_t q = 0; q < w.v.size(); ++q) w.v[q] = sub(w.v[q], w3.v[q]);
    }
    if (invert(w, Gd[0])) info = 1;
  }
  if (dos)
    for (int i = 1; i < nbl; ++i) {   // Gr(i,i) = gsmr_i - Gr(i,i-1) ESH(i-1,i) gsmr_i
      Mat<R> w1, Gl, w2, w3;
      gemm(g[i], l[i - 1], w1, one, false);
      gemm(w1, Gd[i - 1], Gl, mone, false);
      gemm(u[i - 1], g[i], w2, one, false);
      gemm(Gl, w2, w3, mone, false);
      Gd[i] = Mat<R>(g[i].nr, g[i].nc);
      for (size_t q = 0; q < w3.v.size(); ++q) Gd[i].v[q] = add(g[i].v[q], w3.v[q]);
    }
  // calculate_single_transmission_2_contacts with ct1 = the contact on block 1
  double tun = 0.0;
  if (D.ncont == 2) {
    const int ct1 = (D.cblk[0] < D.cblk[1]) ? 0 : 1;
    const Mat<R>& G = Gd[D.cblk[ct1] - 1];
    const Mat<R> GA = dag(G);
    Mat<R> GAM1(Sig[ct1].nr, Sig[ct1].nc);
    const Mat<R> SigA = dag(Sig[ct1]);
    for (size_t q = 0; q < GAM1.v.size(); ++q) GAM1.v[q] = mul(mk<R>(0, 1), sub(Sig[ct1].v[q], SigA.v[q]));
    Mat<R> w1, w2, w3, AA(G.nr, G.nc), w4;
    gemm(GAM1, G, w1, one, false);
    gemm(w1, GAM1, w2, one, false);
    gemm(w2, GA, w3, one, false);
    for (size_t q = 0; q < AA.v.size(); ++q) AA.v[q] = mul(mk<R>(0, 1), sub(G.v[q], GA.v[q]));
    gemm(GAM1, AA, w4, one, false);
    R tr = 0;
    for (int k = 0; k < G.nr; ++k) tr += w4.at(k, k).re - w3.at(k, k).re;
    tun = (double)std::fabs(tr);
  }
  if (dos) {
    const R pi = (R)3.14159265358979323846264338327950288L;
    for (int i = 0; i < nbl; ++i)
      for (int k = 0; k < D.n[i]; ++k) dos[D.start[i] + k] = (double)(-Gd[i].at(k, k).im / pi);
  }
  return tun;
}

}  // namespace xp

}  // namespace

extern "C" {

// decimation on host arrays; Ao/Bo/Co are copied (not modified).
int oracle_decimation(int n, const double* Ao, const double* Bo,
                      const double* Co, double tol, int max_iter, double* Go,
                      int* ncyc) {
  scipy_openblas_set_num_threads(1);
  Err err;
  Dns A = from_ptr(Ao, n, n), B = from_ptr(Bo, n, n), C = from_ptr(Co, n, n), G;
  decimation(G, A, B, C, n, *ncyc, tol, max_iter, err);
  std::memcpy(Go, G.v.data(), sizeof(cplx) * (size_t)n * n);
  return err.code;
}

// zinv on host arrays
int oracle_zinv(int n, const double* A, double* Ainv) {
  scipy_openblas_set_num_threads(1);
  Err err;
  Dns a = from_ptr(A, n, n), x;
  zinv(x, a, err);
  std::memcpy(Ainv, x.v.data(), sizeof(cplx) * (size_t)n * n);
  return err.code;
}

int oracle_transmission(const negf_b200_device* dev, int npts,
                        const double* energy, double eta, int ni, int nf,
                        double sgf_tol, int sgf_max_iter, double eps,
                        double* T, int* ncyc, int* status, int nthreads) {
  set_threads(nthreads);
  DeviceBlocks D = unpack(dev);
  Opts o;
  o.sgf_acc = sgf_tol; o.max_iter = sgf_max_iter; o.eps = eps;
  int first = 0;
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < npts; ++p) {
    Err err;
    int nc = 0;
    T[p] = point_transmission(D, energy[p], eta, ni, nf, o, nc, err);
    if (ncyc) ncyc[p] = nc;
    if (status) status[p] = err.code;
  }
  if (status)
    for (int p = 0; p < npts; ++p) if (status[p] && !first) first = status[p];
  return first;
}

int oracle_transmission_dos(const negf_b200_device* dev, int npts,
                            const double* energy, double eta, double dos_delta,
                            int ni, int nf, double sgf_tol, int sgf_max_iter,
                            double eps, double* T, double* dos, int* ncyc,
                            int* status, int nthreads) {
  set_threads(nthreads);
  DeviceBlocks D = unpack(dev);
  Opts o;
  o.sgf_acc = sgf_tol; o.max_iter = sgf_max_iter; o.eps = eps;
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < npts; ++p) {
    Err err;
    int nc = 0;
    T[p] = point_transmission_dos(D, energy[p], eta, dos_delta, ni, nf, o,
                                  dos + (size_t)p * D.norb, nc, err);
    if (ncyc) ncyc[p] = nc;
    if (status) status[p] = err.code;
  }
  int first = 0;
  if (status)
    for (int p = 0; p < npts; ++p) if (status[p] && !first) first = status[p];
  return first;
}

// calculate_transmissions / calculate_transmissions_and_dos over contact
// pairs, with the tun_proj mask (tun_mask: one byte per device orbital, or
// NULL) and, when ledos != NULL, the LDOS sets (dos_proj) of the DOS path.
// T is npts x npairs and ledos npts x nsets, point-major.
int oracle_transmissions(const negf_b200_device* dev, int npts, const double* energy,
                         double eta, double dos_delta, int npairs, const int* ni,
                         const int* nf, const unsigned char* tun_mask, int nsets,
                         const int* set_ptr, const int* set_idx, double sgf_tol,
                         int sgf_max_iter, double eps, double* T, double* ledos,
                         int* ncyc, int* status, int nthreads) {
  set_threads(nthreads);
  DeviceBlocks D = unpack(dev);
  Opts o;
  o.sgf_acc = sgf_tol; o.max_iter = sgf_max_iter; o.eps = eps;
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < npts; ++p) {
    Err err;
    int nc = 0;
    if (ledos)
      point_transmissions_ldos(D, energy[p], eta, dos_delta, npairs, ni, nf, tun_mask, nsets, set_ptr,
                               set_idx, o, T + (size_t)p * npairs, ledos + (size_t)p * nsets, nc, err);
    else
      point_transmissions(D, energy[p], eta, npairs, ni, nf, tun_mask, o, T + (size_t)p * npairs, nc, err);
    if (ncyc) ncyc[p] = nc;
    if (status) status[p] = err.code;
  }
  int first = 0;
  if (status)
    for (int p = 0; p < npts; ++p) if (status[p] && !first) first = status[p];
  return first;
}

// contour_int: TmpMt = sum_p w_p Gr(z_p) over the tridiagonal blocks (points
// in order), then rho = i (TmpMt - TmpMt^dag) (zspectral).  rho blocks in the
// layout of h_diag / h_upper / h_lower.
int oracle_density(const negf_b200_device* dev, int npts, const double* e_re, const double* e_im,
                   const double* weight, double sgf_tol, int sgf_max_iter, double* rho_d, double* rho_u,
                   double* rho_l, double* rho_dc, double* rho_cd, int* ncyc, int* status, int nthreads) {
  set_threads(nthreads);
  DeviceBlocks D = unpack(dev);
  Opts o;
  o.sgf_acc = sgf_tol; o.max_iter = sgf_max_iter;
  int nbl = D.nbl, ncont = D.ncont;
  std::vector<GrBlocks> G(npts, GrBlocks(nbl));
  std::vector<ContactParts> parts(npts);
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < npts; ++p) {
    Err err;
    int nc = 0;
    point_gr_blocks(D, cplx(e_re[p], e_im[p]), o, G[p], nc, err, &parts[p]);
    if (ncyc) ncyc[p] = nc;
    if (status) status[p] = err.code;
  }
  // calculate_Gr_outer, outer_blocks = 2 (src/iterative.F90:1463-1573):
  // Grlc = -Gr(cb,cb) Tlc gs on Tlc's pattern, Grcl = -gs Tcl Gr(cb,cb) on
  // Tcl's pattern, summed with the weights; then rho = i (T - T^dag) pairs
  // the device->contact block with the contact->device one.
  if (rho_dc || rho_cd) {
    size_t om = 0;
    for (int c = 0; c < ncont; ++c) {
      const int cb = D.cblk[c] - 1, n = D.n[cb], L = D.L[c];
      std::vector<cplx> Tlcs((size_t)n * L, cplx(0.0, 0.0)), Tcls((size_t)L * n, cplx(0.0, 0.0));
      for (int p = 0; p < npts; ++p) {
        const cplx w(weight[2 * p], weight[2 * p + 1]);
        const ContactParts& cp = parts[p];
        Dns work1, Grlc, work2, Grcl;
        mult(G[p].d[cb], cp.Tlc[c], work1, cplx(-1.0, 0.0));
        mult(work1, cp.GS[c], Grlc);
        mult(cp.GS[c], cp.Tcl[c], work2, cplx(-1.0, 0.0));
        mult(work2, G[p].d[cb], Grcl);
        for (size_t q = 0; q < Tlcs.size(); ++q)
          if (cp.Tlc[c].v[q] != cplx(0.0, 0.0)) Tlcs[q] += w * Grlc.v[q];
        for (size_t q = 0; q < Tcls.size(); ++q)
          if (cp.Tcl[c].v[q] != cplx(0.0, 0.0)) Tcls[q] += w * Grcl.v[q];
      }
      for (int j = 0; j < L; ++j)
        for (int r = 0; r < n; ++r) {
          const cplx v = I1 * (Tlcs[r + (size_t)j * n] - std::conj(Tcls[j + (size_t)r * L]));
          if (rho_dc) { rho_dc[2 * (om + r + (size_t)j * n)] = v.real(); rho_dc[2 * (om + r + (size_t)j * n) + 1] = v.imag(); }
          const cplx u = I1 * (Tcls[j + (size_t)r * L] - std::conj(Tlcs[r + (size_t)j * n]));
          if (rho_cd) { rho_cd[2 * (om + j + (size_t)r * L)] = u.real(); rho_cd[2 * (om + j + (size_t)r * L) + 1] = u.imag(); }
        }
      om += (size_t)n * L;
    }
  }
  size_t od = 0, oo = 0;
  for (int i = 0; i < nbl; ++i) {
    int n = D.n[i];
    std::vector<cplx> T((size_t)n * n, cplx(0.0, 0.0));
    for (int p = 0; p < npts; ++p) {
      cplx w(weight[2 * p], weight[2 * p + 1]);
      for (size_t q = 0; q < T.size(); ++q) T[q] += w * G[p].d[i].v[q];
    }
    for (int c = 0; c < n; ++c)
      for (int r = 0; r < n; ++r) {
        cplx v = I1 * (T[r + (size_t)c * n] - std::conj(T[c + (size_t)r * n]));
        rho_d[2 * (od + r + (size_t)c * n)] = v.real();
        rho_d[2 * (od + r + (size_t)c * n) + 1] = v.imag();
      }
    od += (size_t)n * n;
    if (i + 1 < nbl) {
      int m = D.n[i + 1];
      std::vector<cplx> U((size_t)n * m, cplx(0.0, 0.0)), Lw((size_t)m * n, cplx(0.0, 0.0));
      for (int p = 0; p < npts; ++p) {
        cplx w(weight[2 * p], weight[2 * p + 1]);
        for (size_t q = 0; q < U.size(); ++q) U[q] += w * G[p].u[i].v[q];
        for (size_t q = 0; q < Lw.size(); ++q) Lw[q] += w * G[p].l[i].v[q];
      }
      for (int c = 0; c < m; ++c)
        for (int r = 0; r < n; ++r) {
          cplx v = I1 * (U[r + (size_t)c * n] - std::conj(Lw[c + (size_t)r * m]));
          rho_u[2 * (oo + r + (size_t)c * n)] = v.real();
          rho_u[2 * (oo + r + (size_t)c * n) + 1] = v.imag();
        }
      for (int c = 0; c < n; ++c)
        for (int r = 0; r < m; ++r) {
          cplx v = I1 * (Lw[r + (size_t)c * m] - std::conj(U[c + (size_t)r * n]));
          rho_l[2 * (oo + r + (size_t)c * m)] = v.real();
          rho_l[2 * (oo + r + (size_t)c * m) + 1] = v.imag();
        }
      oo += (size_t)n * m;
    }
  }
  int first = 0;
  if (status)
    for (int p = 0; p < npts; ++p) if (status[p] && !first) first = status[p];
  return first;
}

int oracle_meir_wingreen(const negf_b200_device* dev, int npts,
                         const double* energy, double eta, const double* frm,
                         const double* coupling, int scba_niter,
                         double scba_tol, double scba_mix, int scba_rule, double sgf_tol, int sgf_max_iter,
                         double eps, double* curr, double* lcurr,
                         double* ldens, int* scba_iter, double* scba_err,
                         int* ncyc, int* status, int nthreads) {
  set_threads(nthreads);
  DeviceBlocks D = unpack(dev);
  Opts o;
  o.sgf_acc = sgf_tol; o.max_iter = sgf_max_iter; o.eps = eps;
  o.scba_mix = scba_mix; o.scba_rule = scba_rule;
  int nbl = D.nbl, ncont = D.ncont;
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < npts; ++p) {
    Err err;
    ScbaOut so;
    int nc = 0;
    point_scba(D, energy[p], eta, frm + (size_t)p * ncont, coupling,
               scba_niter, scba_tol, o,
               curr ? curr + (size_t)p * ncont : nullptr,
               lcurr ? lcurr + (size_t)p * (nbl - 1) : nullptr,
               ldens ? ldens + (size_t)p * nbl : nullptr, so, nc, err);
    if (scba_iter) scba_iter[p] = so.iters;
    if (scba_err) scba_err[p] = so.err;
    if (ncyc) ncyc[p] = nc;
    if (status) status[p] = err.code;
  }
  int first = 0;
  if (status)
    for (int p = 0; p < npts; ++p) if (status[p] && !first) first = status[p];
  return first;
}

// real_axis_int (src/integrations.F90:1093-1176): sum_p w_p Gn(E_p), Gn of
// compute_Gn with the occupations frm (reference contact already
// subtracted: Sigma^n = sum_c frm_c Gamma_c).  Blocks in the h_* layout.
// rho_dc / rho_cd (optional): calculate_Gn_outer with outer_blocks = 2
// (src/iterative.F90:1576-1665), summed with the weights.
int oracle_density_neq(const negf_b200_device* dev, int npts, const double* energy, double eta,
                       const double* weight, const double* frm, const double* coupling, int scba_niter,
                       double scba_tol, double sgf_tol, int sgf_max_iter, double* rho_d, double* rho_u,
                       double* rho_l, double* rho_dc, double* rho_cd, int* ncyc, int* status, int nthreads) {
  set_threads(nthreads);
  DeviceBlocks D = unpack(dev);
  Opts o;
  o.sgf_acc = sgf_tol; o.max_iter = sgf_max_iter;
  int nbl = D.nbl, ncont = D.ncont;
  std::vector<Trid> G(npts);
  std::vector<ContactParts> parts(npts);
  std::vector<std::vector<Dns>> grd(npts);
  const bool outer = rho_dc || rho_cd;
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < npts; ++p) {
    Err err;
    ScbaOut so;
    int nc = 0;
    point_scba(D, energy[p], eta, frm + (size_t)p * ncont, coupling, scba_niter, scba_tol, o, nullptr, nullptr,
               nullptr, so, nc, err, &G[p], outer ? &parts[p] : nullptr, outer ? &grd[p] : nullptr);
    if (ncyc) ncyc[p] = nc;
    if (status) status[p] = err.code;
  }
  if (outer) {
    size_t om = 0;
    for (int c = 0; c < ncont; ++c) {
      const int cb = D.cblk[c] - 1, n = D.n[cb], L = D.L[c];
      std::vector<cplx> lc((size_t)n * L, cplx(0.0, 0.0)), cl((size_t)L * n, cplx(0.0, 0.0));
      for (int p = 0; p < npts; ++p) {
        const cplx w(weight[2 * p], weight[2 * p + 1]);
        const ContactParts& cp = parts[p];
        Dns gA, work1, work2, work3;
        dagger(cp.GS[c], gA);
        mult(cp.Tlc[c], gA, work2);
        mult(G[p].d[cb], work2, work3, cplx(-1.0, 0.0));          // -Gn(cb,cb) Tlc gA
        const double f = frm[(size_t)p * ncont + c];
        if (std::abs(f) > o.eps) {
          Dns A, w2;
          spectral(cp.GS[c], A);
          mult(cp.Tlc[c], A, w2);
          mult(grd[p][cb], w2, work3, cplx(-f, 0.0));             // += (f_ref - f_c) Gr(cb,cb) Tlc A, accumulated
        }
        for (int j = 0; j < L; ++j)
          for (int r = 0; r < n; ++r) {
            const size_t q = r + (size_t)j * n;
            if (cp.Tlc[c].v[q] == cplx(0.0, 0.0)) continue;           // mask(Gn_lc, Tlc)
            lc[q] += w * work3.v[q];
            cl[j + (size_t)r * L] += w * std::conj(work3.v[q]);        // Gn(c,cb) = Gn(cb,c)^dag
          }
      }
      for (size_t q = 0; q < lc.size(); ++q) {
        if (rho_dc) { rho_dc[2 * (om + q)] = lc[q].real(); rho_dc[2 * (om + q) + 1] = lc[q].imag(); }
        if (rho_cd) { rho_cd[2 * (om + q)] = cl[q].real(); rho_cd[2 * (om + q) + 1] = cl[q].imag(); }
      }
      om += (size_t)n * L;
    }
  }
  size_t od = 0, oo = 0;
  for (int i = 0; i < nbl; ++i) {
    size_t nn = G.empty() ? 0 : G[0].d[i].v.size();
    for (size_t q = 0; q < nn; ++q) {
      cplx t(0.0, 0.0);
      for (int p = 0; p < npts; ++p) t += cplx(weight[2 * p], weight[2 * p + 1]) * G[p].d[i].v[q];
      rho_d[2 * (od + q)] = t.real(); rho_d[2 * (od + q) + 1] = t.imag();
    }
    od += (size_t)D.n[i] * D.n[i];
    if (i + 1 < nbl) {
      size_t nm = (size_t)D.n[i] * D.n[i + 1];
      for (size_t q = 0; q < nm; ++q) {
        cplx tu(0.0, 0.0), tl(0.0, 0.0);
        for (int p = 0; p < npts; ++p) {
          cplx w(weight[2 * p], weight[2 * p + 1]);
          tu += w * G[p].u[i].v[q];
          tl += w * G[p].l[i].v[q];
        }
        rho_u[2 * (oo + q)] = tu.real(); rho_u[2 * (oo + q) + 1] = tu.imag();
        rho_l[2 * (oo + q)] = tl.real(); rho_l[2 * (oo + q) + 1] = tl.imag();
      }
      oo += nm;
    }
  }
  int first = 0;
  if (status)
    for (int p = 0; p < npts; ++p) if (status[p] && !first) first = status[p];
  return first;
}

// fermi_f (src/distributions.F90:27-72)
double oracle_fermi(double E, double Ef, double kT) {
  if (kT == 0.0) return (E > Ef) ? 0.0 : 1.0;
  if (std::abs((E - Ef) / kT) > 30) {
    if (E > Ef) return std::exp(-(E - Ef) / kT);
    return 1.0;
  }
  return 1.0 / (std::exp((E - Ef) / kT) + 1.0);
}

// integrate_el (src/integrations.F90:2688-2770); Kb in the caller's units
double oracle_integrate_el(const double* tun, int ntun, double mu1, double mu2,
                           double kT1, double kT2, double emin, double emax,
                           double estep, double kb_1K) {
  (void)ntun;
  double curr = 0.0;
  int N = 0;
  double destep = 1.0e10;
  int Npoints = (int)std::lround((emax - emin) / estep);
  double kbT1 = (kT1 < kb_1K) ? kb_1K : kT1;
  double kbT2 = (kT2 < kb_1K) ? kb_1K : kT2;
  bool swapped = false;
  if (mu2 < mu1) {
    swapped = true;
    std::swap(mu1, mu2);
    std::swap(kbT1, kbT2);
  }
  for (int i = 0; i <= Npoints - 1; ++i) {
    double E1 = emin + estep * i;
    double TT1 = tun[i];
    double E2 = emin + estep * (i + 1);
    double TT2 = tun[i + 1];
    while (destep >= (kbT1 + kbT2) / 20.0) {
      N = N + 1;
      destep = (E2 - E1) / N;
    }
    for (int i1 = 0; i1 <= N - 1; ++i1) {
      double E3 = E1 + (E2 - E1) * i1 / N;
      double E4 = E3 + (E2 - E1) / N;
      double TT3 = (TT2 - TT1) * i1 / N + TT1;
      double TT4 = TT3 + (TT2 - TT1) / N;
      double c1 = (oracle_fermi(E3, mu2, kbT2) - oracle_fermi(E3, mu1, kbT1)) * TT3;
      double c2 = (oracle_fermi(E4, mu2, kbT2) - oracle_fermi(E4, mu1, kbT1)) * TT4;
      curr = curr + (c1 + c2) * (E4 - E3) / 2.0;
    }
  }
  if (swapped) curr = -1.0 * curr;
  return curr;
}

// Independent-rounding restatement of the 2-contact T (dos == null) or T +
// DOS path over `npts` energies: prec = 1 in long double (near-exact), 0 in
// double with its own unblocked LU and products, 2 in double with
// Gauss-Jordan inverses (the engine's elimination order, unblocked).  ncyc and status as in
// oracle_transmission; status 1 on a zero pivot.
int oracle_transmission_xp(const negf_b200_device* dev, int npts, const double* energy, double eta,
                           double dos_delta, double sgf_tol, int sgf_max_iter, int prec, double* T,
                           double* dos, int* ncyc, int* status, int nthreads) {
  set_threads(nthreads);
  DeviceBlocks D = unpack(dev);
  if (D.ncont != 2) return NEGF_B200_ERR_BAD_ARG;
  // the T-only path is the fast path of calculate_transmissions: Gr(1,1) only
  if (!dos && std::min(D.cblk[0], D.cblk[1]) != 1) return NEGF_B200_ERR_BAD_ARG;
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < npts; ++p) {
    int nc = 0, info = 0;
    double* dp = dos ? dos + (size_t)p * D.norb : nullptr;
    xp::inv_kind() = (prec == 2) ? 1 : 0;
    T[p] = (prec == 1) ? xp::point<long double>(D, energy[p], eta, dos_delta, dp, sgf_tol, sgf_max_iter, nc, info)
                       : xp::point<double>(D, energy[p], eta, dos_delta, dp, sgf_tol, sgf_max_iter, nc, info);
    if (ncyc) ncyc[p] = nc;
    if (status) status[p] = info;
  }
  return 0;
}

// Decimation restated over long double (prec 1) or double with its own LU
// (prec 0) or Gauss-Jordan inverses (prec 2); arguments as oracle_decimation.
int oracle_decimation_xp(int n, const double* Ao, const double* Bo, const double* Co, double tol, int max_iter,
                         int prec, double* Go, int* ncyc) {
  Dns A = from_ptr(Ao, n, n), B = from_ptr(Bo, n, n), C = from_ptr(Co, n, n);
  int info = 0, nc = 0;
  xp::inv_kind() = (prec == 2) ? 1 : 0;
  if (prec == 1) {
    xp::Mat<long double> G = xp::decimation<long double>(xp::from<long double>(A), xp::from<long double>(B),
                                                         xp::from<long double>(C), (long double)tol, max_iter, nc,
                                                         info);
    for (size_t q = 0; q < G.v.size(); ++q) { Go[2 * q] = (double)G.v[q].re; Go[2 * q + 1] = (double)G.v[q].im; }
  } else {
    xp::Mat<double> G = xp::decimation<double>(xp::from<double>(A), xp::from<double>(B), xp::from<double>(C), tol,
                                               max_iter, nc, info);
    for (size_t q = 0; q < G.v.size(); ++q) { Go[2 * q] = G.v[q].re; Go[2 * q + 1] = G.v[q].im; }
  }
  xp::inv_kind() = 0;
  if (ncyc) *ncyc = nc;
  return info;
}

}  // extern "C"
