// Device-side extraction of the dense blocks from a global sparse H (and S)
// in CSR, the work of zcsr2blk_sod (src/sparsekit_drv.F90:3409-3436) for
// the device's tridiagonal blocks and of extract_cont (src/ln_extract.F90:
// 37-75) for the contact blocks, done once per upload on the GPU instead of
// on the host.  One thread per CSR row scatters that row's nonzeros into
// the zero-filled staging arrays (every block element comes from at most
// one nonzero, so there are no write conflicts).
#include "engine.cuh"

namespace negf {

__device__ __forceinline__ int pl_of(const int* plstart, int npl, int r) {
  int lo = 0, hi = npl - 1;   // largest i with plstart[i] <= r
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (plstart[mid] <= r) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void k_csr_scatter(CsrScatter a) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.nrow) return;
  const int q0 = a.rowptr[r] - 1, q1 = a.rowptr[r + 1] - 1;
  if (q0 < 0 || q1 < q0 || q1 > a.nnz) {
    atomicOr(a.bad, 1);
    return;
  }
  auto put = [&](double2* H, double2* S, int64_t idx, int q) {
    H[idx] = a.hv[q];
    if (S) S[idx] = a.sv[q];
  };
  if (r < a.ndev) {
    const int i = pl_of(a.plstart, a.npl, r);
    const int rr = r - a.plstart[i], ni = a.plstart[i + 1] - a.plstart[i];
    for (int q = q0; q < q1; ++q) {
      const int c = a.colind[q] - 1;
      if (c < 0 || c >= a.nrow) { atomicOr(a.bad, 1); continue; }
      if (c < a.ndev) {
        const int j = pl_of(a.plstart, a.npl, c);
        const int cc = c - a.plstart[j];
        if (j == i) put(a.hd, a.sd, a.od[i] + rr + (int64_t)cc * ni, q);
        else if (j == i + 1) put(a.hu, a.su, a.oo[i] + rr + (int64_t)cc * ni, q);
        else if (j == i - 1) put(a.hl, a.sl, a.oo[j] + rr + (int64_t)cc * ni, q);
      } else {
        for (int k = 0; k < a.ncont; ++k)
          if (a.cb[k] - 1 == i && c >= a.j0[k] && c < a.j0[k] + a.L[k])
            put(a.hmc, a.smc, a.omc[k] + rr + (int64_t)(c - a.j0[k]) * ni, q);
      }
    }
  } else {
    for (int k = 0; k < a.ncont; ++k) {
      if (r < a.j0[k] || r >= a.j0[k] + a.L[k]) continue;   // only the contact's first PL rows
      const int rr = r - a.j0[k], L = a.L[k];
      for (int q = q0; q < q1; ++q) {
        const int c = a.colind[q] - 1;
        if (c < 0 || c >= a.nrow) { atomicOr(a.bad, 1); continue; }
        if (c >= a.j0[k] && c < a.j0[k] + L) put(a.h00, a.s00, a.olead[k] + rr + (int64_t)(c - a.j0[k]) * L, q);
        else if (c >= a.j0[k] + L && c < a.j0[k] + 2 * L)
          put(a.h01, a.s01, a.olead[k] + rr + (int64_t)(c - a.j0[k] - L) * L, q);
      }
    }
  }
}

cudaError_t launch_csr_scatter(const CsrScatter& a, cudaStream_t s) {
  if (a.nrow <= 0) return cudaSuccess;
  k_csr_scatter<<<(a.nrow + 255) / 256, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace negf
