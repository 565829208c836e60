/* A C caller of the C-ABI (include/negf_b200.h), the counterpart of
 * libNEGF's C interface test (tests/c_int): it fills a negf_b200_device from
 * a binary file, solves the transmission through negf_b200_transmission and
 * writes T, the decimation counts and the per-point status to a file.  The
 * pytest in test_c_abi.py writes the device, builds this program with gcc
 * and compares its output with the CPU oracle.
 *
 * device file: int32 nbl, ncont, has_s; int32 pl_size[nbl], cblk[ncont],
 *   lead_size[ncont]; then float64 (re, im) arrays in this order: h_diag,
 *   h_upper, h_lower, [s_diag, s_upper, s_lower], lead_h00, lead_h01,
 *   [lead_s00, lead_s01], hmc, [smc]  (bracketed ones when has_s)
 * energy file: int32 npts; float64 eta; float64 E[npts]
 * output file: float64 T[npts]; int32 ncyc[npts]; int32 status[npts]
 * Exit code 0 when every call returned as expected. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "negf_b200.h"

static double* read_doubles(FILE* f, size_t n) {
  double* p = (double*)malloc(n * sizeof(double) + 16);
  if (!p || fread(p, sizeof(double), n, f) != n) {
    fprintf(stderr, "short device file\n");
    exit(3);
  }
  return p;
}

int main(int argc, char** argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: %s device.bin energies.bin out.bin\n", argv[0]);
    return 2;
  }
  FILE* fd = fopen(argv[1], "rb");
  FILE* fe = fopen(argv[2], "rb");
  if (!fd || !fe) return 2;
  int32_t hdr[3];
  if (fread(hdr, 4, 3, fd) != 3) return 3;
  const int32_t nbl = hdr[0], ncont = hdr[1], has_s = hdr[2];
  int32_t* pl = (int32_t*)malloc(4 * (size_t)nbl);
  int32_t* cblk = (int32_t*)malloc(4 * (size_t)ncont);
  int32_t* lead = (int32_t*)malloc(4 * (size_t)ncont);
  if (fread(pl, 4, nbl, fd) != (size_t)nbl || fread(cblk, 4, ncont, fd) != (size_t)ncont ||
      fread(lead, 4, ncont, fd) != (size_t)ncont)
    return 3;
  size_t nd = 0, no = 0, nl = 0, nm = 0;
  for (int i = 0; i < nbl; ++i) {
    nd += (size_t)pl[i] * pl[i];
    if (i + 1 < nbl) no += (size_t)pl[i] * pl[i + 1];
  }
  for (int c = 0; c < ncont; ++c) {
    nl += (size_t)lead[c] * lead[c];
    nm += (size_t)pl[cblk[c] - 1] * lead[c];
  }
  negf_b200_device d;
  memset(&d, 0, sizeof(d));
  d.nbl = nbl;
  d.pl_size = pl;
  d.h_diag = read_doubles(fd, 2 * nd);
  d.h_upper = read_doubles(fd, 2 * no);
  d.h_lower = read_doubles(fd, 2 * no);
  if (has_s) {
    d.s_diag = read_doubles(fd, 2 * nd);
    d.s_upper = read_doubles(fd, 2 * no);
    d.s_lower = read_doubles(fd, 2 * no);
  }
  d.ncont = ncont;
  d.cblk = cblk;
  d.lead_size = lead;
  d.lead_h00 = read_doubles(fd, 2 * nl);
  d.lead_h01 = read_doubles(fd, 2 * nl);
  if (has_s) {
    d.lead_s00 = read_doubles(fd, 2 * nl);
    d.lead_s01 = read_doubles(fd, 2 * nl);
  }
  d.hmc = read_doubles(fd, 2 * nm);
  if (has_s) d.smc = read_doubles(fd, 2 * nm);
  fclose(fd);

  int32_t npts;
  double eta;
  if (fread(&npts, 4, 1, fe) != 1 || fread(&eta, 8, 1, fe) != 1) return 3;
  double* E = read_doubles(fe, (size_t)npts);
  fclose(fe);

  printf("negf_b200 %s\n", negf_b200_version());
  negf_b200_ctx* ctx = NULL;
  int rc = negf_b200_ctx_create(0, &ctx);
  if (rc != NEGF_B200_OK) {
    fprintf(stderr, "ctx_create: %d\n", rc);
    return 4;
  }
  negf_b200_options o;
  negf_b200_default_options(&o);
  o.sgf_tol = 1e-9;
  if (negf_b200_set_options(ctx, &o) != NEGF_B200_OK) return 5;
  int32_t id = -1;
  rc = negf_b200_upload_device(ctx, &d, &id);
  if (rc != NEGF_B200_OK) {
    fprintf(stderr, "upload: %d %s\n", rc, negf_b200_last_error(ctx));
    return 6;
  }
  int32_t* ids = (int32_t*)malloc(4 * (size_t)npts);
  int32_t* ncyc = (int32_t*)malloc(4 * (size_t)npts);
  int32_t* st = (int32_t*)malloc(4 * (size_t)npts);
  double* T = (double*)malloc(8 * (size_t)npts);
  for (int p = 0; p < npts; ++p) ids[p] = id;
  rc = negf_b200_transmission(ctx, npts, ids, E, eta, 1, 2, T, ncyc, st);
  if (rc != NEGF_B200_OK && rc != NEGF_B200_ERR_NOT_CONVERGED) {
    fprintf(stderr, "transmission: %d %s\n", rc, negf_b200_last_error(ctx));
    return 7;
  }
  /* a contact index outside 1..ncont is an argument error with a message, not a trap */
  rc = negf_b200_transmission(ctx, npts, ids, E, eta, 1, ncont + 1, T + 0, ncyc, st);
  if (rc != NEGF_B200_ERR_BAD_ARG || strlen(negf_b200_last_error(ctx)) == 0) {
    fprintf(stderr, "expected BAD_ARG for a bad contact pair, got %d\n", rc);
    return 8;
  }
  /* the failed call must not have touched the outputs of the good one: solve again */
  rc = negf_b200_transmission(ctx, npts, ids, E, eta, 1, 2, T, ncyc, st);
  if (rc != NEGF_B200_OK && rc != NEGF_B200_ERR_NOT_CONVERGED) return 7;
  FILE* fo = fopen(argv[3], "wb");
  if (!fo) return 2;
  fwrite(T, 8, npts, fo);
  fwrite(ncyc, 4, npts, fo);
  fwrite(st, 4, npts, fo);
  fclose(fo);
  if (negf_b200_release_device(ctx, id) != NEGF_B200_OK) return 9;
  if (negf_b200_ctx_destroy(ctx) != NEGF_B200_OK) return 10;
  printf("ok %d points\n", npts);
  return 0;
}
