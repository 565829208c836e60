// Gauss-Jordan leaf factorisations (gj_leaf4) and row-owner node updates
// (gj_rows_update), compiled in a translation
// unit of their own (see gemm_run in cta_ops.cuh).
#include "cta_ops.cuh"

namespace negf {

__device__ void leaf_run_r1(double2* X, int n, int c0, int w, double2* sh, InvScratch& s) {
  gj_leaf4<1, 8>(X, n, c0, w, sh, s);
}
__device__ void leaf_run_r2(double2* X, int n, int c0, int w, double2* sh, InvScratch& s) {
  gj_leaf4<2, 4>(X, n, c0, w, sh, s);
}
__device__ void leaf_run_r4(double2* X, int n, int c0, int w, double2* sh, InvScratch& s) {
  gj_leaf4<4, 2>(X, n, c0, w, sh, s);
}

__device__ void rows_run_t2(const double2* X, double2* Y, const double2* Wm, int n, int N, int k0, int K,
                            const int* perm, double2* stage) {
  gj_rows_update<1, 2, 8>(X, Y, Wm, n, N, k0, K, perm, stage);
}
__device__ void rows_run_r1(const double2* X, double2* Y, const double2* Wm, int n, int N, int k0, int K,
                            const int* perm, double2* stage) {
  gj_rows_update<1, 1, 16>(X, Y, Wm, n, N, k0, K, perm, stage);
}
__device__ void rows_run_r2(const double2* X, double2* Y, const double2* Wm, int n, int N, int k0, int K,
                            const int* perm, double2* stage) {
  gj_rows_update<2, 1, 16>(X, Y, Wm, n, N, k0, K, perm, stage);
}
__device__ void rows_run_r4(const double2* X, double2* Y, const double2* Wm, int n, int N, int k0, int K,
                            const int* perm, double2* stage) {
  gj_rows_update<4, 1, 8>(X, Y, Wm, n, N, k0, K, perm, stage);
}

}  // namespace negf
