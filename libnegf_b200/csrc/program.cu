// The control side of the persistent engine: the point program, the
// inversion driver and the light block operations, compiled apart from the
// kernel (relocatable device code).  The kernel in engine.cu calls
// engine_step() and runs the heavy step it returns.
#include "program.cuh"

namespace negf {

__device__ int engine_step(const EngineArgs& a, EngineCtl& c, SmemMap& sm) {
  const int tid = threadIdx.x;
  if (c.open >= 0) {   // close the timing of the heavy step the kernel just ran
    sm.tr.stop(c.open, c.t0);
    c.open = -1;
  }
  Ws w;
  w.base = a.ws + (int64_t)blockIdx.x * a.ws_per_cta;
  w.Q = a.Q;
  w.ncont = a.ncont_max;
  w.nbl_max = a.nbl_max;
  for (;;) {
    if (c.in_inv) {
      const int st = inv_next(c.ip, sm.main, sm.inv);
      if (st == INV_LEAF) {
        c.open = TR_INV_PANEL;
        c.t0 = sm.tr.start();
        return STEP_LEAF;
      }
      if (st == INV_APPLY) return STEP_GEMM;   // timed by inv_next
      if (st == INV_ROWS) return STEP_ROWS;    // likewise
      inv_end(c.ip, sm.inv);
      c.in_inv = 0;
      if (tid == 0) sm.ires[0] = *sm.inv.flag;
      __syncthreads();
      continue;
    }
    if (!next_op(a, c.prog, sm, w, c.op)) return STEP_DONE;
    const Op& o = c.op;
    if (o.kind == K_GEMM) {
      Epilogue e = epi_store(o.C, o.ldc, o.alpha, o.beta);
      if (o.flag) {
        if (tid == 0) *sm.maxv = 0.0;
        __syncthreads();
        e.maxabs = sm.maxv;
      }
      c.t0 = sm.tr.start();
      gemm_desc_publish(o.m, o.n, o.k, Operand{o.A, o.lda, o.opa, nullptr}, Operand{o.B, o.ldb, o.opb, nullptr}, e,
                        sm.main);
      c.open = TR_GEMM;
      return STEP_GEMM;
    }
    if (o.kind == K_ZINV) {
      if (inv_begin(c.ip, o.m, o.A, o.C, w.inv(), sm.main, sm.inv)) {   // small order: done
        if (tid == 0) sm.ires[0] = *sm.inv.flag;
        __syncthreads();
      } else {
        c.in_inv = 1;
      }
      continue;
    }
    exec_light(o, sm);
  }
}

}  // namespace negf
