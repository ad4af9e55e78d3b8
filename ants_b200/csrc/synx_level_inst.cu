// One translation unit per CC radius of the persistent level kernel (the build compiles this
// file once per radius with -DSYNX_RCC=r, so the instantiations compile in parallel).
// the level kernel reads data its own blocks wrote earlier in the launch: coherent loads throughout
#define SYNX_COHERENT_LOADS 1
#include "synx_level_body.cuh"

#ifndef SYNX_RCC
#error "compile with -DSYNX_RCC=<CC radius>"
#endif

#define SYNX_CAT2(a, b) a##b
#define SYNX_CAT(a, b) SYNX_CAT2(a, b)

namespace synx {

void* SYNX_CAT(level_kernel_r, SYNX_RCC)(int dim, bool batch) {
  if (batch) return dim == 3 ? (void*)k_level_batch<3, SYNX_RCC> : (void*)k_level_batch<2, SYNX_RCC>;
  return dim == 3 ? (void*)k_level<3, SYNX_RCC> : (void*)k_level<2, SYNX_RCC>;
}

}  // namespace synx
