// FP32 instantiations of the hot-path kernels (mixed-precision path). This
// unit is compiled with FMA contraction; the FP64 unit is not.
#define CANARD_F32_EXTERN
#include "kernels_f32.h"
