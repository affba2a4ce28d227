// phl_runner.h -- interface between the runtime (phl_runtime.cu) and the per-configuration
// kernel launchers, which live in two translation units: the FP64 path (compiled without FMA
// contraction, reference rounding) and the FP32 split-precision path (phl_split.cu).
#pragma once
#include <cuda_runtime.h>
#include "phl_kernels.cuh"

namespace phl {

struct Runner {
  virtual ~Runner() {}
  // one RK stage (all kernels of the stage)
  virtual void stage(const Prm &P, cudaStream_t s) = 0;
  // FP64 runners (phl_runtime.cu) only: the standalone CFL maximum over the FP64 primitive
  // state and the step-0 thermodynamics.  A split-precision context runs these two through the
  // FP64 runner of its option set, so each of these kernels is compiled once, with the FP64
  // unit's reference rounding.
  virtual void dt(const Prm &, cudaStream_t) {}
  virtual void init_thermo(const Prm &, cudaStream_t) {}
  // split path only: FP64 primitives -> (U, FP32 deviations) and back
  virtual void split_from_prim(const Prm &, cudaStream_t) {}
  virtual void split_to_prim(const Prm &, cudaStream_t) {}
};

// factory of the FP32 split-precision runners (phl_split.cu); nullptr when not built
Runner *make_split_runner(int dim, int nv, bool mhd, bool helm, bool strat, int riem, bool fast, int rec, bool sf);

}  // namespace phl
