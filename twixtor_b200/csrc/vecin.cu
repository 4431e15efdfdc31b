// Vectors In on the device: the flow of an encoded vector image (decode, the hole flags of its
// alpha, Vec Scale), the two steps around the forward warp of the flow inversion, and the matte
// step of the layered loaders. Every kernel is one pass over the pixels (HBM bound); the hole fill
// between them is the engine's (fill_dev with FILL_FLOW).
#include "kernels.cuh"
#include "strict.cuh"

namespace tw {

namespace {

// vectors.rs:525-528: ((c * 2) / den - 1) * scale in double precision, one narrowing to single
__device__ __forceinline__ float dec_int(double c, double den, double scale) {
    return __double2float_rn(__dmul_rn(__dsub_rn(__ddiv_rn(__dmul_rn(c, 2.0), den), 1.0), scale));
}

// holefill.rs:22-31: the thresholds of the hole test `!(eps > (double)m)`
__device__ __forceinline__ double u8_eps() { return __longlong_as_double(0x20202020202020fcll); }
__device__ __forceinline__ double wide_eps() { return __longlong_as_double(0x3f0040bfe3b03e21ll); }

}  // namespace

__global__ void k_vec_decode(const void* __restrict__ vec, int fmt, float md, float2* __restrict__ flow,
                             uint8_t* __restrict__ holes, long n, int* __restrict__ any_hole) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool hole = false;
    if (i < n) {
        float2 o;
        double mdd = (double)md;
        if (fmt == 0) {
            uchar4 p = ((const uchar4*)vec)[i];  // A, R, G, B
            if (p.x == 0) o = make_float2(0.0f, 0.0f);
            else o = make_float2(dec_int((double)p.y, 254.0, mdd), dec_int((double)p.z, 254.0, mdd));
            hole = !(u8_eps() > (double)(uint8_t)(0xffu - p.x));
        } else if (fmt == 1) {
            ushort4 p = ((const ushort4*)vec)[i];
            if (p.x == 0) o = make_float2(0.0f, 0.0f);
            else o = make_float2(dec_int((double)p.y, 65534.0, mdd), dec_int((double)p.z, 65534.0, mdd));
            hole = !(wide_eps() > (double)(uint16_t)(0xffffu - p.x));
        } else {
            float4 p = ((const float4*)vec)[i];
            if (p.x == 0.0f) o = make_float2(0.0f, 0.0f);
            else o = make_float2(__fmul_rn(__fsub_rn(__fmul_rn(p.y, 2.0f), 1.0f), md),
                                 __fmul_rn(__fsub_rn(__fmul_rn(p.z, 2.0f), 1.0f), md));
            hole = !(wide_eps() > (double)__fsub_rn(1.0f, p.x));
        }
        flow[i] = o;
        holes[i] = hole ? 1 : 0;
    }
    if (__syncthreads_or(hole) && threadIdx.x == 0) atomicOr(any_hole, 1);
}

__global__ void k_vec_scale(float2* __restrict__ flow, long n, float sx, float sy) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float2 v = flow[i];
    flow[i] = make_float2(__fmul_rn(sx, v.x), __fmul_rn(sy, v.y));
}

__global__ void k_invert_prep(const float2* __restrict__ flow, float4* __restrict__ t, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float2 f = flow[i];
    float m = __fmul_rn(-1.0f, 1.0f);
    t[i] = make_float4(m, __fmul_rn(-1.0f, f.x), __fmul_rn(-1.0f, f.y), m);
}

__global__ void k_invert_take(const float4* __restrict__ pushed, const uint8_t* __restrict__ cov,
                              float2* __restrict__ flow, uint8_t* __restrict__ holes, long n, int* __restrict__ any_hole) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool hole = false;
    if (i < n) {
        float4 p = pushed[i];
        flow[i] = make_float2(p.y, p.z);
        hole = (uint8_t)(0xffu - cov[i]) != 0;
        holes[i] = hole ? 1 : 0;
    }
    if (__syncthreads_or(hole) && threadIdx.x == 0) atomicOr(any_hole, 1);
}

namespace {
// Rust's saturating `f32 as i64` followed by the clamp to 0..white
__device__ __forceinline__ int sat_unit(float v, int white) {
    if (v != v) return 0;
    if (v <= 0.0f) return 0;
    if (v >= (float)white) return white;
    return (int)v;  // in (0, white): the truncation
}
}  // namespace

__global__ void k_matte_step(void* __restrict__ img, int fmt, const float* __restrict__ matte, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = matte[i];
    if (fmt == 0) {
        uint8_t* a = (uint8_t*)img + i * 4;
        int c = sat_unit(__fadd_rn(__fmul_rn(v, 255.0f), 0.5f), 255);
        if (c < *a) *a = (uint8_t)c;
    } else if (fmt == 1) {
        uint16_t* a = (uint16_t*)img + i * 4;
        int c = sat_unit(__fadd_rn(__fmul_rn(v, 65535.0f), 0.5f), 65535);
        if (c < *a) *a = (uint16_t)c;
    } else {
        float* a = (float*)img + i * 4;
        if (v < *a) *a = v;
    }
}

}  // namespace tw
