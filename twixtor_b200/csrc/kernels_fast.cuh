// The fast mode's variants of the solver kernels: fused.cu, solver.cu and coarse.cu compiled a second
// time with TW_FAST_VARIANT (FMA contraction, approximate division and square root, denormals
// flushed to zero). Same signatures as the strict kernels in kernels.cuh; namespace tw::fast.
#pragma once
#include "kernels.cuh"

namespace tw {
namespace fast {

__global__ void k_resample(const float* __restrict__ src, int sw, int sh, float* __restrict__ dst, int dw, int dh);
__global__ void k_range_any(const float* __restrict__ fu, const float* __restrict__ fv, int w, int h,
                            int* __restrict__ any_in_range);
__global__ void k_bm_rows(const float* __restrict__ A, const float* __restrict__ B, const float* __restrict__ fu,
                          const float* __restrict__ fv, int w, int h, float* __restrict__ uT, float* __restrict__ vT);
__global__ void k_bm_cols(const float* __restrict__ AT, const float* __restrict__ BT, const float* __restrict__ uT,
                          const float* __restrict__ vT, int w, int h, float* fu, float* fv);
__global__ void k_transpose2(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ at,
                             float* __restrict__ bt, int w, int h);
__global__ void k_blur5_band(const float* __restrict__ orig, const void* __restrict__ luma_src, int fmt, int luma_mode,
                             int w, int h, bool above_first, float* __restrict__ tmp_out, float* __restrict__ band_out,
                             float* __restrict__ band_t_out);
__global__ void k_level_init(const float* __restrict__ img, int w, int h, Taps g7, bool above_first,
                             float* __restrict__ gxo, float* __restrict__ gyo, float* __restrict__ a0o,
                             float* __restrict__ a1o, float* __restrict__ a2o, const float* __restrict__ mask,
                             const float* __restrict__ fu, const float* __restrict__ fv, const float* __restrict__ i0,
                             const float* __restrict__ mask_y, float* __restrict__ b_out, int bp, long bplane);
__global__ void k_calc_b_pitched(const float* __restrict__ i1, const float* __restrict__ i0,
                                 const float* __restrict__ gx, const float* __restrict__ gy,
                                 const float* __restrict__ fu, const float* __restrict__ fv, int w, int h,
                                 const float* __restrict__ mask_y, float* __restrict__ b_out, int bp, long bplane);
__global__ void k_apply_upsample(const float* __restrict__ su, const float* __restrict__ sv, int sw, int sh,
                                 const int* __restrict__ any, int l, int start, bool damp_now, float damp,
                                 float* __restrict__ du, float* __restrict__ dv, int dw, int dh);
__global__ void k_apply_negate(const float* __restrict__ fu, const float* __restrict__ fv, long n,
                               const int* __restrict__ any, int start, bool damp_now, float damp,
                               float* __restrict__ out, int* __restrict__ nan_flag);
__global__ void k_solve_coarse(CoarseJob job);
#define TW_DECLARE_LEVEL_ITER(TX, TY)                                                                                 \
    __global__ void k_level_iter_##TX##x##TY(                                                                       \
        const float* __restrict__ b_in, int bp, long bplane, const float* __restrict__ i1,                          \
        const float* __restrict__ i0, const float* __restrict__ gx, const float* __restrict__ gy,                    \
        const float* __restrict__ a0, const float* __restrict__ a1, const float* __restrict__ a2,                    \
        const float* __restrict__ fu, const float* __restrict__ fv, int w, int h, Taps g7, Taps g5,                  \
        bool above_first, float* __restrict__ fu_out, float* __restrict__ fv_out, const float* __restrict__ mask_y,  \
        float* __restrict__ b_out);
TW_DECLARE_LEVEL_ITER(32, 32)
TW_DECLARE_LEVEL_ITER(64, 32)
TW_DECLARE_LEVEL_ITER(64, 64)
#undef TW_DECLARE_LEVEL_ITER

}  // namespace fast
}  // namespace tw
