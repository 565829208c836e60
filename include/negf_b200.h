/*
 * negf_b200.h -- C-ABI of the B200 per-energy-point transport solve.
 *
 * Drop-in seam: libNEGF selects its RGF backend at build time
 * (src/iterative.F90:38-43: `use iterative_gpu` | `use iterative_cpu`) and
 * reaches CUDA through `bind(C)` interfaces (src/cudautils.F90:236-431) to the
 * `extern "C"` functions of src/gpuroutines.cu.  This header is the
 * replacement of that seam.  It keeps the reference's conventions:
 *
 *   - matrices are column-major complex128 (interleaved re,im doubles), the
 *     layout of `z_DNS%val` (src/mat_def.F90:199-204);
 *   - sizes are plain integers, pointers are plain pointers, no C++ types;
 *   - every function returns an `int` status (0 = OK), the convention of the
 *     `cu_*` functions (src/gpuroutines.cu:248-996), but never traps or exits:
 *     where the reference stops (`error stop`, `__trap()`), these functions
 *     return a NEGF_B200_ERR_* code and fill a per-point status array.
 *
 * Two levels are exported:
 *   1. batched per-energy-point solves over a device description that stays
 *      resident in HBM (the context API below) -- the hot path;
 *   2. device-pointer primitives that mirror the reference's cuBLAS/cuSOLVER
 *      wrappers one-for-one (cu_ZmultMat, cu_Zinverse, cu_Zdecimation).
 *
 * Energies are in the units of H (libNEGF does not rescale them).
 */
#ifndef NEGF_B200_H
#define NEGF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define NEGF_B200_OK 0
#define NEGF_B200_ERR_SINGULAR 1      /* exact zero pivot in a block inversion
                                         (zgetrf info>0, src/inversions.F90:823) */
#define NEGF_B200_ERR_NOT_CONVERGED 2 /* decimation reached the iteration cap
                                         (src/contselfenergy.F90:289) */
#define NEGF_B200_ERR_NONFINITE 3     /* NaN/Inf in an output */
#define NEGF_B200_ERR_NOMEM 4         /* device allocation failed */
#define NEGF_B200_ERR_BAD_ARG 5       /* shape / pointer / index error */
#define NEGF_B200_ERR_CUDA 6          /* CUDA runtime error */
#define NEGF_B200_ERR_TIMEOUT 7       /* a bounded device wait expired */
#define NEGF_B200_ERR_ADMISSION 8     /* request exceeds the HBM budget */
#define NEGF_B200_ERR_NO_GPU 9        /* no CUDA device / extension not built */
#define NEGF_B200_ERR_SCBA_NOT_CONVERGED 10 /* SCBA stopped at scba_niter
                                               (informational, results valid) */

#define NEGF_B200_MAXNCONT 10 /* src/api/lnParams.h:10 */

/* ---- device description ------------------------------------------------
 * The block-tridiagonal device of libNEGF after `zcsr2blk_sod`
 * (src/sparsekit_drv.F90:3409-3436) and the contact blocks after
 * `extract_cont` (src/ln_extract.F90:37-75).  All blocks are dense,
 * column-major complex128, concatenated in layer order.
 *
 *   h_diag : H(i,i),   n_i x n_i,       i = 0..nbl-1
 *   h_upper: H(i,i+1), n_i x n_{i+1},   i = 0..nbl-2
 *   h_lower: H(i+1,i), n_{i+1} x n_i,   i = 0..nbl-2
 *   s_*    : same for S; all three NULL means S = I (set_S_id,
 *            src/libnegf.F90:408).
 * Contacts (surfdim = 0, two principal layers per contact as in
 * src/contselfenergy.F90:184-207):
 *   cblk[c]      : 1-based device block the contact couples to (TStruct cblk)
 *   lead_size[c] : L_c, orbitals of one contact principal layer
 *   lead_h00/s00 : contact PL1 on-site block, L_c x L_c (concatenated over c)
 *   lead_h01/s01 : contact PL1 -> PL2 coupling, L_c x L_c
 *   hmc/smc      : device block cblk[c] -> contact PL1, n_cblk x L_c
 *   lead_s00/lead_s01/smc NULL means identity / zero overlap.
 * Bound surface layers (libNEGF's surfdim > 0, src/contselfenergy.F90:
 * 150-156, 226-243): a contact may start with n0_c orbitals ahead of its
 * periodic principal layers (Surf | PL1 | PL2).  Then
 *   surf_size[c] : n0_c (surf_size NULL = no surface anywhere)
 *   lead_hs/ss   : H and S over Surf followed by PL1, (n0_c + L_c)^2, for
 *                  the contacts with n0_c > 0 only, concatenated in contact
 *                  order (lead_ss NULL: S = I there); only the entries in a
 *                  Surf row or column are used (the PL1 block is the lead's)
 *   hmc/smc      : for such a contact n_cblk x (n0_c + L_c), device block
 *                  cblk[c] -> Surf and PL1
 * and the contact's surface Green's function is the inverse of
 * [E S - H over Surf+PL1 with the PL1 block replaced by gs^-1], gs the
 * decimation's (the bound-state block of surface_green).
 */
typedef struct negf_b200_device {
  int32_t nbl;
  const int32_t* pl_size;
  const double* h_diag;
  const double* h_upper;
  const double* h_lower;
  const double* s_diag;
  const double* s_upper;
  const double* s_lower;
  int32_t ncont;
  const int32_t* cblk;
  const int32_t* lead_size;
  const double* lead_h00;
  const double* lead_h01;
  const double* lead_s00;
  const double* lead_s01;
  const double* hmc;
  const double* smc;
  const int32_t* surf_size;
  const double* lead_hs;
  const double* lead_ss;
} negf_b200_device;

/* ---- solver options ------------------------------------------------------
 * Defaults (negf_b200_default_options) are the reference's:
 *   sgf_tol = SGFACC = 1e-9          src/ln_precision.F90:40
 *   sgf_max_iter = 300               src/contselfenergy.F90:289
 *   eps_drop = 0 (EPS is never set inside libNEGF, src/ln_precision.F90:36)
 *   scba_tol = 1e-7                  src/lib_param.F90:653
 *   scba_mix = 1, scba_rule = 0      (no mixing, the Gn convergence check)
 */
typedef struct negf_b200_options {
  double sgf_tol;
  int32_t sgf_max_iter;
  double eps_drop;
  double scba_tol;
  int32_t scba_niter;
  /* 0 = plain complex FP64 (the parity form).  4..8 = the mixed form for
   * 2-contact transmission solves (negf_b200_transmission, _dev): every
   * block product on the integer tensor cores with that many int8 digits
   * per operand element (negf_b200_zgemm_batched_i8; 7 digits carry about
   * the accuracy of an FP64 product, 8 a margin below it), the block
   * inverses, the decimation's convergence test and the Caroli trace in
   * FP64, all points of a call in lock step.  1 = the mixed form with 8
   * digits.  The mixed form needs two
   * contacts on blocks 1 and nbl, one PL size for every layer and both leads,
   * the same shape for every point of a call, a single contact pair and no
   * tun_proj; other solves return NEGF_B200_ERR_BAD_ARG under it.  It
   * neither reads nor fills the SGF cache (a context that keeps one still
   * runs it). */
  int32_t precision;
  /* Resident CTAs per SM for the persistent point engine (0 = auto). */
  int32_t ctas_per_sm;
  /* Elastic SCBA mixing and stopping rule.  scba_mix = 1 (default) is the
   * reference: the dephasing self-energies are overwritten by D diag(G)
   * each sweep (src/elphdd.F90:108-156, 227-276).  0 < scba_mix < 1 is
   * linear mixing from Sigma = 0: Sigma <- mix D diag(G) + (1-mix) Sigma.
   * scba_rule = 0 (default) stops when max |Gn - Gn_old| on the S pattern
   * is below scba_tol (src/scba.F90:120-147); scba_rule = 1 stops when the
   * Meir-Wingreen current of contact 1 changes by less than scba_tol
   * between sweeps.  Neither alternative exists in the reference. */
  double scba_mix;
  int32_t scba_rule;
  /* How the points of a 2-contact transmission solve (negf_b200_transmission,
   * _dev; single pair, no SGF cache) are scheduled under precision = 0:
   *   1 = the persistent engine: one CTA per point, its whole solve;
   *   2 = lock step: every point of the call through the same block
   *       operation at once, one CTA per point and operation (orders
   *       n <= 32; the call needs the shape rules of the mixed form);
   *   0 (default) = lock step when the call's points all fit it and n <= 32
   *       (for _dev calls: every device the context holds) and the stream is
   *       not capturing, else the engine.
   * Lock step synchronises its stream a few times per call (the
   * decimation's active count is read back), so a captured call takes the
   * engine (schedule 2 under capture: NEGF_B200_ERR_BAD_ARG).
   * Both compute the reference's operation sequence in complex FP64; their
   * last bits differ (summation order).  Under precision != 0 the mixed
   * form runs in lock step whatever this says. */
  int32_t schedule;
} negf_b200_options;

typedef struct negf_b200_ctx negf_b200_ctx;

void negf_b200_default_options(negf_b200_options* opt);

/* Library and build identification (never fails). */
const char* negf_b200_version(void);

/* Creates a context bound to CUDA device `cuda_device`: one stream, a
 * resident device arena and the persistent-kernel workspace.  Mirrors the
 * GPU part of init_negf (src/libnegf.F90:160-170). */
int negf_b200_ctx_create(int32_t cuda_device, negf_b200_ctx** ctx);
int negf_b200_ctx_destroy(negf_b200_ctx* ctx);
int negf_b200_set_options(negf_b200_ctx* ctx, const negf_b200_options* opt);
/* Last error message of this context (empty if none). */
const char* negf_b200_last_error(const negf_b200_ctx* ctx);
/* Kernels launched by this context's solve calls since it was created: one
 * per persistent-engine call, one per batched block operation of lock step
 * (three per product of the mixed form: two digit splits and the product). */
int negf_b200_launch_count(negf_b200_ctx* ctx, uint64_t* count);

/* Uploads a device description to HBM once (H/S blocks, contact blocks) and
 * returns a handle.  One description per k-point: libNEGF keeps one H(k),S(k)
 * pair per local k (negf%HS(iK), src/integrations.F90:1868-1870).  The host
 * arrays may be freed after the call. */
int negf_b200_upload_device(negf_b200_ctx* ctx, const negf_b200_device* dev,
                            int32_t* device_id);
/* The same from libNEGF's own input: the global H (and S; s_vals = NULL is
 * S = I, set_S_id) over device + contact orbitals as a 1-based z_CSR
 * (rowptr nrow+1, colind and values nnz, complex interleaved) and the
 * negf_init_structure arrays (src/api/libnegf_api.f90:146-185: plend per
 * PL, cblk / surfstart / surfend / contend per contact, 1-based).  The
 * dense blocks that zcsr2blk_sod (src/sparsekit_drv.F90:3409-3436) and
 * extract_cont (src/ln_extract.F90:37-75) take from the CSR on the host are
 * scattered from it on the GPU: the device's tridiagonal blocks, per
 * contact its first-PL block, the PL1 -> PL2 coupling and the coupling of
 * device PL cblk to PL1.  Surface blocks (surfend >= surfstart) are
 * rejected.  Temporary device memory: the CSR plus the dense blocks. */
int negf_b200_upload_csr(negf_b200_ctx* ctx, int32_t nrow, int32_t nnz,
                         const int32_t* rowptr, const int32_t* colind,
                         const double* h_vals, const double* s_vals,
                         int32_t npl, const int32_t* plend, int32_t ncont,
                         const int32_t* cblk, const int32_t* surfstart,
                         const int32_t* surfend, const int32_t* contend,
                         int32_t* device_id);
int negf_b200_release_device(negf_b200_ctx* ctx, int32_t device_id);
/* Bytes of HBM the device description holds. */
int negf_b200_device_bytes(const negf_b200_ctx* ctx, int32_t device_id,
                           size_t* bytes);

/* ---- batched per-energy-point solves (host buffers) ----------------------
 * A point is (device_id[p], energy[p]).  All points of one call run in one
 * persistent launch.  `status` (npts) receives a per-point NEGF_B200_* code;
 * the return value is the first non-OK point status (or a call error).
 * `ncyc` (npts, optional) receives the total decimation iteration count over
 * all contacts at that point (src/integrations.F90:1751 prints the average
 * over contacts).  Results of 1 MiB and more (DOS, LDOS, layer rows of large
 * calls) are read back through a pinned host staging buffer that the context
 * allocates on first use, sized to the largest such call, and frees in
 * negf_b200_ctx_destroy; the caller's arrays may be pageable. */

/* Coherent transmission T(E) between contacts ni -> nf (1-based).
 * Replaces compute_contacts(E+i*eta) + calculate_transmissions(E)
 * (src/integrations.F90:1747-1755, src/iterative.F90:1669-1780): contact
 * self-energies at E + i*eta, ES-H at real E, gsmr sweep, Caroli trace.
 * Uses the 2-contact fast path when the reference does (ncont == 2 and
 * min(cblk) == 1, src/iterative.F90:1697-1713), else the N-contact column
 * sweep (src/iterative_cpu.F90:477-583). */
int negf_b200_transmission(negf_b200_ctx* ctx, int32_t npts,
                           const int32_t* device_id, const double* energy,
                           double eta, int32_t ni, int32_t nf, double* T,
                           int32_t* ncyc, int32_t* status);

/* Transmission plus the diagonal spectral density -Im Gr_ii / pi of every
 * device orbital (dos: npts x norb, row-major by point).  Replaces
 * calculate_transmissions_and_dos(E + i*dos_delta) with contact
 * self-energies at E + i*eta (src/integrations.F90:1757-1770,
 * src/iterative.F90:1821-1952).  Projection on LDOS index sets is a host
 * reduction of `dos`. */
int negf_b200_transmission_dos(negf_b200_ctx* ctx, int32_t npts,
                               const int32_t* device_id, const double* energy,
                               double eta, double dos_delta, int32_t ni,
                               int32_t nf, double* T, double* dos,
                               int32_t* ncyc, int32_t* status);

/* Non-equilibrium solve with local elastic dephasing, one SCBA loop per
 * point (src/iterative.F90:289-363, src/elphdd.F90:108-276,
 * src/scba.F90:120-147), then the Meir-Wingreen contact currents
 * (src/iterative.F90:382-414) and the layer currents / layer densities
 * (src/iterative.F90:427-461).
 *   frm       : npts x ncont contact occupations f_c(E) (reference f = 0)
 *   coupling  : norb dephasing couplings (NOT squared; squared on device as
 *               in ElPhonDephD_init, src/elphdd.F90:95); NULL = no dephasing
 *   curr      : npts x ncont  I_c(E)   (optional)
 *   layer_curr: npts x (nbl-1) J_{i,i+1}(E) (optional)
 *   layer_dens: npts x nbl     Tr Gn_ii (optional)
 *   scba_iter : npts iterations run (optional); scba_err: npts last error */
int negf_b200_meir_wingreen(negf_b200_ctx* ctx, int32_t npts,
                            const int32_t* device_id, const double* energy,
                            double eta, const double* frm,
                            const double* coupling, double* curr,
                            double* layer_curr, double* layer_dens,
                            int32_t* scba_iter, double* scba_err,
                            int32_t* ncyc, int32_t* status);

/* Equilibrium density matrix by contour integration, the loop of contour_int
 * (src/integrations.F90:844-897) over the points of one device: at every
 * complex energy z_p = e_re[p] + i e_im[p] the contact self-energies and ES-H
 * are taken at z_p (compute_Gr, :2287-2340), the whole tridiagonal Gr is
 * solved (calculate_Gr, src/iterative.F90:90-148) and w_p Gr accumulated;
 * finally rho = i (T - T^dag) (zspectral, :893).  weight: npts complex
 * (interleaved re, im) -- the en_grid%wght of contour_int_def (times z_p for
 * the energy-weighted matrix, DorE = 'E').  rho_diag / rho_upper / rho_lower
 * receive the blocks in the layout of h_diag / h_upper / h_lower (NULL to
 * skip); restricting them to the sparsity of S (blk2csr,
 * src/iterative.F90:1375-1450) is left to the caller.  rho_dc / rho_cd
 * (NULL to skip) receive the outer blocks of calculate_Gr_outer with
 * outer_blocks = 2 (src/iterative.F90:1463-1573): device PL cblk[c] ->
 * contact c (n_cb x L_c, the hmc layout) and contact -> device (L_c x n_cb,
 * same offsets), kept on the pattern of E SMC - HMC.  Dephasing is not
 * included. */
int negf_b200_density(negf_b200_ctx* ctx, int32_t device_id, int32_t npts,
                      const double* e_re, const double* e_im,
                      const double* weight, double* rho_diag,
                      double* rho_upper, double* rho_lower, double* rho_dc,
                      double* rho_cd, int32_t* ncyc, int32_t* status);

/* Non-equilibrium part of the density matrix on the real axis, the loop of
 * real_axis_int (src/integrations.F90:1093-1176): at every real energy E_p
 * the Gn blocks (contacts at E_p + i*eta, ES-H at E_p, the elastic-dephasing
 * SCBA when coupling != NULL, as compute_Gn :2350-2395) are summed with the
 * complex weights w_p into rho_* (same layout as negf_b200_density; no
 * spectral combination, the reference adds this sum to rho as it is).
 * frm: npts x ncont occupations with the reference contact's subtracted
 * (f_c - f_ref, 0 for ref), the Sigma^n of calculate_Gn_neq_components.
 * rho_dc / rho_cd (NULL to skip) receive the outer blocks of
 * calculate_Gn_outer with outer_blocks = 2 (src/iterative.F90:1576-1665):
 * Gn(cb,c) = -Gn(cb,cb) Tlc gs^dag - (f_c - f_ref) Gr(cb,cb) Tlc i(gs - gs^dag)
 * kept on the pattern of E SMC - HMC, and Gn(c,cb) = Gn(cb,c)^dag, summed
 * with the weights (layouts as in negf_b200_density).
 * The device needs nbl >= 2. */
int negf_b200_density_neq(negf_b200_ctx* ctx, int32_t device_id, int32_t npts,
                          const double* energy, double eta,
                          const double* weight, const double* frm,
                          const double* coupling, double* rho_diag,
                          double* rho_upper, double* rho_lower,
                          double* rho_dc, double* rho_cd, int32_t* ncyc,
                          int32_t* status);

/* ---- projections and contact pairs ----------------------------------------
 * tun_proj of libNEGF (negf%tun_proj): the transmission trace runs over the
 * listed orbitals only (1-based global orbital indices; the mask of
 * get_tun_mask, src/iterative_cpu.F90:586-618, used by both transmission
 * formulas, :466 and :578).  nidx = 0 clears it (whole trace).  Indices
 * outside the device are ignored.  Kept with the device description. */
int negf_b200_set_tun_proj(negf_b200_ctx* ctx, int32_t device_id, int32_t nidx,
                           const int32_t* idx);

/* dos_proj of libNEGF (negf%dos_proj): nsets LDOS index sets, set k =
 * set_idx[set_ptr[k] .. set_ptr[k+1]) (1-based orbital indices, summed in
 * that order; indices past the device skipped), as the LDOS loop of
 * calculate_transmissions_and_dos (src/iterative.F90:1931-1945).  nsets = 0
 * clears it.  Kept with the device description. */
int negf_b200_set_dos_proj(negf_b200_ctx* ctx, int32_t device_id, int32_t nsets,
                           const int32_t* set_ptr, const int32_t* set_idx);

/* Transmissions between the contact pairs ni[q] -> nf[q], q < npairs (T:
 * npts x npairs, row-major by point), as calculate_transmissions
 * (src/iterative.F90:1669-1780): the 2-contact fast path iff the device has
 * 2 contacts, npairs == 1 and min(cblk) == 1, otherwise gsmr is kept and
 * every pair takes the N-contact formula.  The reference frees gsmr inside
 * its pair loop after the first pair (:1766-1767); here it stays valid for
 * every pair.  With ledos != NULL this is calculate_transmissions_and_dos
 * (:1821-1952) at E + i*dos_delta instead, and ledos (npts x nsets, nsets =
 * the largest dos_proj set count over the points' devices) gets the LDOS of
 * the sets given by negf_b200_set_dos_proj.  Both honour tun_proj. */
int negf_b200_transmissions(negf_b200_ctx* ctx, int32_t npts,
                            const int32_t* device_id, const double* energy,
                            double eta, double dos_delta, int32_t npairs,
                            const int32_t* ni, const int32_t* nf, double* T,
                            double* ledos, int32_t* ncyc, int32_t* status);

/* Caps the engine workspace of this context at `bytes` (0 = no cap): a launch
 * whose resident CTAs would need more runs with fewer CTAs, and one whose
 * single CTA does not fit returns NEGF_B200_ERR_ADMISSION.  A serving loop
 * admits requests against this budget. */
int negf_b200_set_workspace_limit(negf_b200_ctx* ctx, size_t bytes);

/* ---- surface Green's function cache ----------------------------------------
 * The counterpart of libNEGF's surface_green_cache (src/ln_cache.F90, used
 * by surface_green, src/contselfenergy.F90:146-167, 251-264): the surface
 * Green's function of every contact at every solved point is kept in a
 * device arena of `bytes`, and a later host-buffer solve at the same
 * (device, contact, E, eta, SGF tolerance, iteration cap) reads it instead
 * of running the decimation (ncyc then counts 0 for that contact, as the
 * reference's load path).
 *   mode 0: off (frees the arena); 1: load if cached, else compute and store
 *   (ReadOldSGF = 0); 2: compute and overwrite (ReadOldSGF = 2).
 * When the misses of a call do not fit, they are computed without being
 * stored and the next call that finds the arena full starts afresh.
 * Releasing a device drops its entries.  The _dev solves do not use it. */
int negf_b200_set_sgf_cache(negf_b200_ctx* ctx, int32_t mode, size_t bytes);
/* Disk copy of the cache, for reuse across runs: the counterpart of
 * TMatrixCacheDisk (src/ln_cache.F90:154-511), which writes each surface GF
 * to its own file and reads it back when ReadOldSGF = 0
 * (src/contselfenergy.F90:161-167).  _save writes every cached gs with a
 * fingerprint of its lead (L and the H00, H01, S00, S01 blocks), the energy,
 * broadening, tolerance and iteration cap to one file; *entries = number
 * written.  _load (cache enabled) adds the file's entries for every
 * uploaded device whose contact has a lead with that fingerprint, as far as
 * the arena has room; *entries = number of file entries used.  Device ids
 * need not match between runs. */
int negf_b200_sgf_cache_save(negf_b200_ctx* ctx, const char* path,
                             int64_t* entries);
int negf_b200_sgf_cache_load(negf_b200_ctx* ctx, const char* path,
                             int64_t* entries);
int negf_b200_sgf_cache_stats(const negf_b200_ctx* ctx, int64_t* hits,
                              int64_t* misses, int64_t* entries,
                              size_t* bytes_used);

/* ---- batched solves on device buffers ------------------------------------
 * Same as negf_b200_transmission / _transmission_dos with every per-point
 * array already resident in HBM (device pointers) and no host
 * synchronisation: the launch is enqueued on `stream` (NULL = the context's
 * stream) and the call returns.  Workspace sizing covers every uploaded
 * device.  `dos_stride` is the row stride of d_dos in doubles. */
int negf_b200_transmission_dev(negf_b200_ctx* ctx, int32_t npts,
                               const int32_t* d_device_id,
                               const double* d_energy, double eta, int32_t ni,
                               int32_t nf, double* d_T, int32_t* d_ncyc,
                               int32_t* d_status, void* stream);
int negf_b200_transmission_dos_dev(negf_b200_ctx* ctx, int32_t npts,
                                   const int32_t* d_device_id,
                                   const double* d_energy, double eta,
                                   double dos_delta, int32_t ni, int32_t nf,
                                   double* d_T, double* d_dos,
                                   int64_t dos_stride, int32_t* d_ncyc,
                                   int32_t* d_status, void* stream);
/* negf_b200_meir_wingreen on device buffers (the SCBA energy loop of
 * meir_wingreen, src/integrations.F90:1855-1930, with every per-point array
 * in HBM).  Row strides: d_frm and d_curr rows hold cont_stride doubles,
 * d_layer_curr and d_layer_dens rows hold layer_stride doubles (at least
 * the largest ncont / nbl over the uploaded devices; every uploaded device
 * needs nbl >= 2).  d_device_id, d_energy, d_frm, d_scba_iter, d_scba_err
 * and d_status are required; d_coupling (no dephasing), d_curr,
 * d_layer_curr, d_layer_dens and d_ncyc may be NULL. */
int negf_b200_meir_wingreen_dev(negf_b200_ctx* ctx, int32_t npts,
                                const int32_t* d_device_id,
                                const double* d_energy, double eta,
                                const double* d_frm, const double* d_coupling,
                                double* d_curr, double* d_layer_curr,
                                double* d_layer_dens, int32_t* d_scba_iter,
                                double* d_scba_err, int32_t* d_ncyc,
                                int32_t* d_status, int32_t cont_stride,
                                int32_t layer_stride, void* stream);

/* ---- tracing ---------------------------------------------------------------
 * libNEGF times phases with a stack of host wall clocks (src/clock.F90:35-93,
 * printed when verbose > 70).  Here every CTA of the persistent engine
 * accumulates SM cycles per phase; negf_b200_get_trace synchronises the
 * device, returns the sums over all CTAs since the previous call and resets
 * them.  Phases:
 *   0 block products (decimation, self-energies, sweeps)
 *   1 inversion panel factorisation (pivot search, row exchanges)
 *   2 inversion trailing update
 *   3 inversion copies / final column permutation
 *   4 ES-H assembly and elementwise passes
 *   5 whole kernel (per CTA)      6 points processed (a count)   7 unused */
#define NEGF_B200_TRACE_NPHASE 8
int negf_b200_set_tracing(negf_b200_ctx* ctx, int32_t enable);
int negf_b200_get_trace(negf_b200_ctx* ctx, uint64_t* cycles);

/* ---- device-pointer primitives (mirror src/gpuroutines.cu) ---------------
 * All pointers are device pointers, `stream` is a cudaStream_t (NULL =
 * legacy default stream); `batch` independent problems, problem b of an
 * operand starting b * stride doubles (2 per complex element) after its
 * pointer.  No allocation inside except where stated. */

/* C = alpha*op(A)*op(B) + beta*C, complex128.  dagger: 0 = (N,N),
 * 1 = (C,N), 2 = (N,C) -- the `dagger` argument of cu_ZmultMat
 * (src/gpuroutines.cu:395-446).  alpha/beta are {re, im}. */
int negf_b200_zgemm_batched(int32_t batch, int32_t m, int32_t n, int32_t k,
                            const double* alpha, const double* A,
                            int64_t strideA, const double* B, int64_t strideB,
                            const double* beta, double* C, int64_t strideC,
                            int32_t dagger, void* stream);

/* C = alpha*A*B + beta*C, complex128, no transposes, on the integer tensor
 * cores: every row of A and column of B is scaled by a power of two and cut
 * into `slices` signed 7-bit digits (int8); the digit products accumulate
 * exactly in int32 (tcgen05.mma kind::i8, accumulators in tensor memory)
 * and are recombined in FP64.  The result carries about 7*slices - 1 bits
 * relative to the row / column scales (slices = 7: within a few units of
 * the rounding of an FP64 product; 4 <= slices <= 8).  Replaces, at FP64
 * accuracy, the zgemm of prealloc_mult (src/sparsekit_drv.F90:1896-2081)
 * and cu_ZmultMat with dagger = 0 (src/gpuroutines.cu:395-446).
 * k <= 1024.  C may alias A or B.  `work` holds
 * negf_b200_zgemm_i8_work_bytes(batch, m, n, k, slices) bytes; status
 * (device, batch entries, may be NULL) gets NEGF_B200_ERR_NONFINITE for an
 * operand with a NaN / Inf (C is NaN) and NEGF_B200_ERR_TIMEOUT if a
 * pipeline wait inside the kernel ran out; other entries are left as they
 * are. */
size_t negf_b200_zgemm_i8_work_bytes(int32_t batch, int32_t m, int32_t n, int32_t k,
                                     int32_t slices);
int negf_b200_zgemm_batched_i8(int32_t batch, int32_t m, int32_t n, int32_t k,
                               const double* alpha, const double* A,
                               int64_t strideA, const double* B, int64_t strideB,
                               const double* beta, double* C, int64_t strideC,
                               int32_t slices, void* work, int32_t* status,
                               void* stream);

/* Ainv = A^-1 (n x n) by Gauss-Jordan elimination with partial pivoting
 * (pivot = max |Re|+|Im|, the izamax rule of zgetrf).  Replaces cu_Zinverse
 * = cusolverDnZgetrf + Zgetrs against the identity (src/gpuroutines.cu:
 * 449-523) and zinv (src/inversions.F90:807-839).  `work` is a device buffer
 * of negf_b200_zinv_work_bytes(batch, n) bytes; info[b] = 0 or the 1-based
 * column of the first zero pivot.  Gauss-Jordan is not backward stable: each
 * inverse is checked by a residual probe, max |A (X v) - v| for a fixed v,
 * and gets up to two Newton steps X + X (I - A X) where it exceeds 1e-5
 * (well-conditioned inverses probe at 1e-14 .. 1e-7; a Gauss-Jordan inverse
 * of a matrix of condition 1e8 and up can reach 1e-4).  For n <= 64 `work` may be NULL:
 * the probe is then skipped. */
size_t negf_b200_zinv_work_bytes(int32_t batch, int32_t n);
int negf_b200_zinv_batched(int32_t batch, int32_t n, const double* A,
                           double* Ainv, int32_t* info, void* work,
                           void* stream);

/* Sancho-Rubio decimation, batched, device-side convergence: replaces
 * cu_Zdecimation (src/gpuroutines.cu:742-986) with the CPU rule of
 * decimation (src/contselfenergy.F90:271-340): converged when
 * max|C1| <= tol on two consecutive iterations, at most max_iter
 * iterations.  Ao/Bo/Co/Go: batch x n x n; ncyc: batch (as in the
 * reference, max_iter+1 when the cap is reached).  `work` holds
 * negf_b200_decimation_work_bytes(batch, n) bytes. */
size_t negf_b200_decimation_work_bytes(int32_t batch, int32_t n);
int negf_b200_decimation_batched(int32_t batch, int32_t n, const double* Ao,
                                 const double* Bo, const double* Co,
                                 double* Go, int32_t* ncyc, double tol,
                                 int32_t max_iter, void* work, void* stream);

/* Same as negf_b200_decimation_batched, but allocates no device memory and
 * takes no work buffer.  It has no counterpart in the reference.
 * For callers that cannot allocate: codes whose device memory belongs to
 * another allocator (a framework's caching pool, a host that passes only
 * the arrays it owns) and solver loops that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree.  Ao/Bo/Co/Go/ncyc are still the
 * caller's device buffers.
 * Scratch comes from one fixed 64 MiB array compiled into the library:
 * batch * 15 * n * n * 16 bytes must fit (e.g. up to 4 problems of order
 * 256, 68 of order 64); larger requests return NEGF_B200_ERR_ADMISSION and
 * print the limit.  The first call on each device resolves the array's
 * address for that device (again after a device reset, when the CUDA
 * context has changed); make it before any stream capture.  All calls
 * share the array: calls that can overlap on the GPU race, so serialise
 * them. */
int negf_b200_decimation_noalloc(int32_t batch, int32_t n, const double* Ao,
                                 const double* Bo, const double* Co,
                                 double* Go, int32_t* ncyc, double tol,
                                 int32_t max_iter, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NEGF_B200_H */
