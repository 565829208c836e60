// Persistent per-energy-point engine: shared declarations between the CUDA
// translation unit and the C-ABI host layer.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace negf {

constexpr int kMaxCont = 10;           // MAXNCONT (src/api/lnParams.h:10)
constexpr int kMaxOrder = 1024;        // largest PL / contact PL size supported
constexpr int kSmemMain = 100 * 1024;  // GEMM staging ring / inversion panel region
// A decimation that reaches a fixed point other than the retarded surface
// Green's function (or runs off to Inf / NaN) runs again from the contact
// energy times 1 + k 2^-50, k = 1..kDecRetries; after that the point
// reports NOT_CONVERGED.
constexpr int kDecRetries = 6;

enum Mode : int { MODE_T = 0, MODE_DOS = 1, MODE_GN = 2, MODE_RHO = 3 };

// Status codes (identical to include/negf_b200.h)
enum Status : int {
  ST_OK = 0, ST_SINGULAR = 1, ST_NOT_CONVERGED = 2, ST_NONFINITE = 3, ST_NOMEM = 4,
  ST_BAD_ARG = 5, ST_CUDA = 6, ST_TIMEOUT = 7, ST_ADMISSION = 8, ST_NO_GPU = 9,
  ST_SCBA_NOT_CONVERGED = 10,
};

// One uploaded device description, as the kernels see it (device memory).
struct DevDesc {
  int nbl, ncont, norb, has_s;
  int has_s00, has_s01, has_smc, pad;
  const int* pl;            // [nbl] PL sizes
  const int* pstart;        // [nbl] first orbital of each PL
  const int64_t* od;        // [nbl] element offset of block (i,i) in hd/sd
  const int64_t* oo;        // [nbl-1] element offset of block (i,i+1)/(i+1,i)
  const double2* hd; const double2* hu; const double2* hl;
  const double2* sd; const double2* su; const double2* sl;
  int cblk[kMaxCont];       // 1-based
  int L[kMaxCont];
  int64_t olead[kMaxCont];  // offset of lead blocks (L x L)
  int64_t omc[kMaxCont];    // offset of hmc/smc blocks (n_cb x L)
  const double2* h00; const double2* h01; const double2* s00; const double2* s01;
  const double2* hmc; const double2* smc;
  // projections (negf_b200_set_tun_proj / negf_b200_set_dos_proj)
  const unsigned char* tun_mask;   // [norb], 1 = orbital inside the transmission trace; null = all
  const int* ldos_ptr;             // [nldos+1] LDOS set k = ldos_idx[ldos_ptr[k] .. ldos_ptr[k+1])
  const int* ldos_idx;             // 1-based orbital indices
  int nldos, pad2;
  // bound surface layers (surfdim, src/contselfenergy.F90:226-243): surf[c] orbitals
  // ahead of the periodic PLs; H / S over Surf + PL1 at osurf[c] in hs / ss
  int surf[kMaxCont];
  int64_t osurf[kMaxCont];
  const double2* hs; const double2* ss;
  int has_ss, pad3;
};

struct EngineArgs {
  int mode;
  int npts;
  const int* dev_id;
  const double* energy;
  const DevDesc* devs;
  double eta, dos_delta;
  int ni, nf;                    // the contact pair when npairs <= 1 (1-based)
  int npairs;                    // >= 1: T is npts x npairs
  const int* pair_ni;            // [npairs] (device) when npairs > 1
  const int* pair_nf;
  double sgf_tol;
  int sgf_max_iter;
  double eps;
  // outputs
  double* T;
  double* dos; int64_t dos_stride;
  double* ldos; int ldos_stride;  // LDOS over the device's index sets (MODE_DOS; needs dos)
  // MODE_RHO (contour integration of Gr): complex energies E + i*energy_im and
  // complex weights; sum_p w_p Gr_p accumulated (atomically) into blocks laid
  // out like the device's H blocks (od / oo offsets)
  const double* energy_im;
  const double2* weight;
  double2* acc_d; double2* acc_u; double2* acc_l;
  double2* acc_lc; double2* acc_cl;   // outer blocks per contact (hmc layout), or null
  // surface Green's function cache (npts x ncont_max offsets into sgf_arena in
  // complex elements, -1 = none): read gs instead of the decimation / store it
  const int64_t* sgf_in;
  const int64_t* sgf_out;
  double2* sgf_arena;
  int* ncyc;
  int* status;
  // non-equilibrium (MODE_GN)
  const double* frm; int frm_stride;
  const double* coupling;       // norb (unsquared) or null
  int scba_niter; double scba_tol;
  double scba_mix; int scba_rule;  // linear mixing factor (1 = overwrite), stopping rule (0 Gn, 1 current)
  double* curr; int curr_stride;
  double* lcurr; int lcurr_stride;
  double* ldens; int ldens_stride;
  int* scba_iter; double* scba_err;
  // workspace
  double2* ws; int64_t ws_per_cta; int64_t Q;  // slot size in complex elements
  int nmax;                      // max PL/contact PL order over the launch
  int nbl_max;
  int ncont_max;                 // contacts per device, max over the launch
  int* counter;                  // work-queue head (zeroed before launch)
  unsigned long long* trace;     // TR_NPHASE phase cycle sums, or null (tracing off)
};

// Workspace slot counts of the engine for a launch
int64_t engine_slots(int mode, int nbl_max, int ncont_max);
int64_t engine_ws_elems(int mode, int nbl_max, int ncont_max, int nmax);
size_t engine_smem_bytes(int nmax);

cudaError_t launch_engine(const EngineArgs& a, int grid, cudaStream_t s);

// CSR -> dense blocks (csr.cu).  Indices 1-based as libNEGF's z_CSR; the
// outputs are zero-filled staging arrays in the negf_b200_device layout.
struct CsrScatter {
  int nrow, nnz, ndev, npl, ncont;
  const int* rowptr;            // nrow + 1
  const int* colind;            // nnz
  const double2* hv;            // nnz
  const double2* sv;            // nnz or null (S = I)
  const int* plstart;           // npl + 1, 0-based first orbital of each PL, plstart[npl] = ndev
  const int64_t* od;            // npl, offsets of H(i,i) in hd
  const int64_t* oo;            // npl - 1, offsets of H(i,i+1) / H(i+1,i)
  int j0[kMaxCont], L[kMaxCont], cb[kMaxCont];   // 0-based first contact orbital, PL size, cblk
  int64_t olead[kMaxCont], omc[kMaxCont];
  double2 *hd, *hu, *hl, *sd, *su, *sl, *h00, *h01, *s00, *s01, *hmc, *smc;
  int* bad;                     // set on an index outside the matrix
};
cudaError_t launch_csr_scatter(const CsrScatter& a, cudaStream_t s);
cudaError_t launch_zgemm_batched(int batch, int m, int n, int k, double2 alpha, const double2* A,
                                 int64_t sA, const double2* B, int64_t sB, double2 beta, double2* C,
                                 int64_t sC, int dagger, cudaStream_t s);
cudaError_t launch_zinv_batched(int batch, int n, const double2* A, double2* Ainv, int* info, double2* work,
                                cudaStream_t s);
size_t zinv_batched_work_elems(int n);
// sens (optional): sens[map[b]] = 1 where the matrix is nearly singular
// (its condition estimate from the residual probe exceeds kSensitiveCond)
cudaError_t launch_zinv_mapped(int batch, int n, const double2* A, int64_t sA, double2* X, int64_t sX,
                               const int* map, int* info, double2* work, cudaStream_t s, int* sens = nullptr);
cudaError_t launch_decimation_batched(int batch, int n, const double2* Ao, const double2* Bo, const double2* Co,
                                      double2* Go, int* ncyc, double tol, int max_iter, double2* work,
                                      cudaStream_t s);
size_t decimation_batched_work_elems(int n);

}  // namespace negf
