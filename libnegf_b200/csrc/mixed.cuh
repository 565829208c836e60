// Mixed-precision transmission: the 2-contact Caroli solve of a batch of
// (E, k) points in lock step, with every block product on the integer
// tensor cores (ozaki.cuh) and the block inverses, the decimation's
// convergence test and the Caroli trace in FP64.
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "engine.cuh"

namespace negf {

struct MixedArgs {
  int npts;
  const int* d_ids;          // device index of each point (into d_descs)
  const double* d_E;         // real energies
  double eta;                // contact broadening: the contacts see E + i eta, the device E
  const DevDesc* d_descs;
  int n;                     // PL size of every layer and lead (uniform)
  int nbl;                   // layers (>= 2), the same for every point
  int left, right;           // 0-based contact indices on block 1 and on block nbl
  double sgf_tol;
  int sgf_max_iter;
  int slices;                // int8 digits per operand element (4..8); 0 = the small-order FP64 form (n <= 32)
  double* d_T;
  int* d_ncyc;               // decimation iterations summed over the contacts
  int* d_status;
  uint64_t* launches = nullptr;  // host counter of kernels launched (may be null)
};

// bytes of workspace for a batch of `batch` points of order n
size_t mixed_ws_bytes(int batch, int n, int slices);
// the largest batch that fits `bytes` (0 if none)
int mixed_batch_for(size_t bytes, int n, int slices);

// Runs the solve in batches of `batch` points on stream s (synchronises with
// the host once per decimation iteration to shrink the active set).
// Returns 0 or a NEGF_B200 status, with a message in *err.
int mixed_run(const MixedArgs& a, void* ws, int batch, cudaStream_t s, std::string* err);

}  // namespace negf
