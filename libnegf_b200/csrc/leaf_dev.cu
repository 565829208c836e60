// Gauss-Jordan leaf factorisations (gj_leaf2), compiled in a translation
// unit of their own (see gemm_run in cta_ops.cuh).
#include "cta_ops.cuh"

namespace negf {

__device__ void leaf_run_r1(double2* X, int n, int c0, int w, double2* sh, InvScratch& s) {
  gj_leaf2<1, 8>(X, n, c0, w, sh, s);
}
__device__ void leaf_run_r2(double2* X, int n, int c0, int w, double2* sh, InvScratch& s) {
  gj_leaf2<2, 4>(X, n, c0, w, sh, s);
}
__device__ void leaf_run_r4(double2* X, int n, int c0, int w, double2* sh, InvScratch& s) {
  gj_leaf2<4, 2>(X, n, c0, w, sh, s);
}

}  // namespace negf
