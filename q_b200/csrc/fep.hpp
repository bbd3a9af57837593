// fep.hpp -- internal interface of the free-energy analysis (fep.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "qb_fep.h"

namespace qb {

// Where the per-state energy records live on the device: record p of file f,
// state st, component c is at base[foff[f] + p*rec_stride + st*15 + c].
struct FepSource {
  const double *base = nullptr;
  std::vector<long long> foff;   // per file, in doubles
  int rec_stride = 0;            // doubles per record
  std::vector<int> npts;         // records per file
  int nstates = 0;
  // r_xy of record p of file f (EVB): rbase[rfoff[f] + p*r_stride]
  const double *rbase = nullptr;
  std::vector<long long> rfoff;
  int r_stride = 0;
};

// Runs the analysis on `stream` and fills `out` (host buffers).  Throws
// qb::Error on invalid input or CUDA failure.
void fep_run(const FepSource &src, const qb_fep_params &p, int device, cudaStream_t stream, qb_fep_result *out);

}  // namespace qb
