// The CTA product loop, compiled in a translation unit of its own (see
// gemm_run in cta_ops.cuh): operand and epilogue modes are read from the
// descriptor, so one routine serves every product of the engine and of the
// primitive kernels.
#include "cta_ops.cuh"

namespace negf {

__device__ void gemm_run(const GemmDesc* d, double2* smem) { cta_gemm_body<OP_RT, OP_RT, EPI_RT>(d, smem); }

}  // namespace negf
