// FP32 instantiations of the hot-path kernels (mixed-precision path). This
// unit is compiled with FMA contraction; the FP64 unit is not.
#define CANARD_F32_EXTERN
#include "kernels_f32.h"

#ifdef CANARD_TRACE
// Trace builds only: this unit's copy of the per-CTA stamp buffer pointer (the
// kernels of each translation unit see their own).
extern "C" int canard_trace_buffer_fma(void* dev) {
  return cudaMemcpyToSymbol(canard::g_trace, &dev, sizeof(dev)) == cudaSuccess ? 0 : 2;
}
#endif
