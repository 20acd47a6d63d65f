// The instantiations of the kernel launchers that are compiled with FMA
// contraction: the FP32 kernels of the mixed-precision path and the FP64
// split solves of the fast FP64 mode. kernels_f32.cu defines them
// (CANARD_F32_EXTERN empty) in a translation unit compiled with FMA
// contraction; every other unit declares them extern, so it neither
// instantiates nor compiles these kernels itself.
#pragma once
#include "kernels.cuh"

#ifndef CANARD_F32_EXTERN
#define CANARD_F32_EXTERN extern
#endif

namespace canard {

CANARD_F32_EXTERN template void launch_prim<float>(dim3, cudaStream_t, const BlockDev*, const CaseConst*, int);
CANARD_F32_EXTERN template void launch_dtmax<float>(dim3, cudaStream_t, const BlockDev*, const StageParams*,
                                                    const CaseConst*, unsigned long long*, int*);
CANARD_F32_EXTERN template void launch_copy_mu<float>(dim3, cudaStream_t, const BlockDev*);
CANARD_F32_EXTERN template void launch_viscous_assemble<float>(dim3, cudaStream_t, const BlockDev*);
CANARD_F32_EXTERN template void launch_flux<float>(dim3, cudaStream_t, const BlockDev*, const StageParams*,
                                                   const CaseConst*);
CANARD_F32_EXTERN template void launch_flux_visc<float>(dim3, cudaStream_t, const BlockDev*, const StageParams*,
                                                        const CaseConst*);
CANARD_F32_EXTERN template void launch_flux_sum<float>(dim3, cudaStream_t, const BlockDev*);
CANARD_F32_EXTERN template void launch_rk<float>(dim3, cudaStream_t, const BlockDev*, const StageParams*);
CANARD_F32_EXTERN template void launch_rk_next<float>(dim3, cudaStream_t, const BlockDev*, const StageParams*,
                                                      const CaseConst*, int, int, int);
CANARD_F32_EXTERN template void launch_rk_faces<float>(int, cudaStream_t, const BlockDev*, const StageParams*,
                                                       const int*, const long long*, int);
CANARD_F32_EXTERN template void launch_prim_points<float>(int, cudaStream_t, const BlockDev*, const CaseConst*,
                                                          const int*, const long long*, int);
CANARD_F32_EXTERN template void launch_gcbc_setup<float>(int, cudaStream_t, const BlockDev*, const GcbcTask*,
                                                         const int*, int, int, const StageParams*);
CANARD_F32_EXTERN template void launch_gcbc_update<float>(int, cudaStream_t, const BlockDev*, const GcbcTask*,
                                                          const int*, int, int, const StageParams*);
CANARD_F32_EXTERN template void launch_sponge<float>(int, cudaStream_t, const BlockDev*, const SpongeTask*,
                                                     const int*, int, int);
CANARD_F32_EXTERN template void launch_face_copy<float>(dim3, cudaStream_t, const void* const*, void* const*,
                                                        const int*, int);
CANARD_F32_EXTERN template void launch_mpigo_t<float>(int, cudaStream_t, const FaceTask*, const int*, int, int);

#define CANARD_F32_LINE(DIR, OP, TT)                                                                      \
  CANARD_F32_EXTERN template void launch_line2_t<DIR, OP, TT>(int, size_t, cudaStream_t, const LineTask*,   \
                                                              const int*, int, const CUtensorMap*, int*);   \
  CANARD_F32_EXTERN template cudaError_t line2_smem_limit<DIR, OP, TT>(int);
// split solves: derivatives on FP32 fields; filter of the FP64 state with an FP32 elimination
CANARD_F32_LINE(1, 0, float)
CANARD_F32_LINE(2, 0, float)
CANARD_F32_LINE(3, 0, float)
CANARD_F32_LINE(1, 1, double)
CANARD_F32_LINE(2, 1, double)
CANARD_F32_LINE(3, 1, double)
#undef CANARD_F32_LINE
// split solves in FP64 with FMA contraction: the fast FP64 mode (not
// bit-identical to the reference's order; held to its tolerance)
#define CANARD_F64S_LINE(DIR, OP)                                                                              \
  CANARD_F32_EXTERN template void launch_line2_t<DIR, OP, double, double>(int, size_t, cudaStream_t,            \
                                                                          const LineTask*, const int*, int,    \
                                                                          const CUtensorMap*, int*);           \
  CANARD_F32_EXTERN template cudaError_t line2_smem_limit<DIR, OP, double, double>(int);
CANARD_F64S_LINE(1, 0)
CANARD_F64S_LINE(2, 0)
CANARD_F64S_LINE(3, 0)
CANARD_F64S_LINE(1, 1)
CANARD_F64S_LINE(2, 1)
CANARD_F64S_LINE(3, 1)
#undef CANARD_F64S_LINE
// two-ended solves (two warps per 32 lines): FP64 with FMA for the fast
// mode, FP32 derivatives and FP32 filter eliminations for the mixed path
#define CANARD_TWIST_LINE(DIR, OP, TT, RS)                                                                     \
  CANARD_F32_EXTERN template void launch_line2t_t<DIR, OP, TT, RS>(int, size_t, cudaStream_t, const LineTask*, \
                                                                   const int*, int, const CUtensorMap*, int*); \
  CANARD_F32_EXTERN template cudaError_t line2t_smem_limit<DIR, OP, TT, RS>(int);
CANARD_TWIST_LINE(1, 0, double, double)
CANARD_TWIST_LINE(2, 0, double, double)
CANARD_TWIST_LINE(3, 0, double, double)
CANARD_TWIST_LINE(1, 1, double, double)
CANARD_TWIST_LINE(2, 1, double, double)
CANARD_TWIST_LINE(3, 1, double, double)
CANARD_TWIST_LINE(1, 0, float, float)
CANARD_TWIST_LINE(2, 0, float, float)
CANARD_TWIST_LINE(3, 0, float, float)
CANARD_TWIST_LINE(1, 1, double, float)
CANARD_TWIST_LINE(2, 1, double, float)
CANARD_TWIST_LINE(3, 1, double, float)
#undef CANARD_TWIST_LINE
// quad split derivatives (four lanes per line): FP64 for the fast mode, FP32
// for the mixed path
#define CANARD_QUAD_LINE(DIR, TT)                                                                              \
  CANARD_F32_EXTERN template void launch_line4_t<DIR, TT, TT>(int, size_t, cudaStream_t, const LineTask*,        \
                                                              const int*, int, const CUtensorMap*, int*);       \
  CANARD_F32_EXTERN template cudaError_t line4_smem_limit<DIR, TT, TT>(int);
CANARD_QUAD_LINE(1, double)
CANARD_QUAD_LINE(2, double)
CANARD_QUAD_LINE(3, double)
CANARD_QUAD_LINE(1, float)
CANARD_QUAD_LINE(2, float)
CANARD_QUAD_LINE(3, float)
#undef CANARD_QUAD_LINE
// one-lane sweeps with an FP32 elimination (the autotuner's alternative)
#define CANARD_F32_LINE1(DIR, OP, TT)                                                                         \
  CANARD_F32_EXTERN template void launch_line_t<DIR, OP, TT, float>(int, size_t, cudaStream_t, const LineTask*, \
                                                                    const int*, int, const CUtensorMap*, int*); \
  CANARD_F32_EXTERN template cudaError_t line_smem_limit<DIR, OP, TT, float>(int);
CANARD_F32_LINE1(1, 0, float)
CANARD_F32_LINE1(2, 0, float)
CANARD_F32_LINE1(3, 0, float)
CANARD_F32_LINE1(1, 1, double)
CANARD_F32_LINE1(2, 1, double)
CANARD_F32_LINE1(3, 1, double)
#undef CANARD_F32_LINE1
// the filter of the FP64 state streamed into FP32 right-hand sides (split FP32 solve)
#define CANARD_F32_FILT(DIR)                                                                              \
  CANARD_F32_EXTERN template void launch_filt2s_t<DIR>(int, size_t, cudaStream_t, const LineTask*, const int*, \
                                                       int, int*);                                        \
  CANARD_F32_EXTERN template cudaError_t filt2s_smem_limit<DIR>(int);
CANARD_F32_FILT(1)
CANARD_F32_FILT(2)
CANARD_F32_FILT(3)
#undef CANARD_F32_FILT

}  // namespace canard
