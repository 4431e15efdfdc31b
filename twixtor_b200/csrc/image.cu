// Image boundary, luma, inverse warps and blends, strict mode. Each kernel cites the reference
// function (plugins/retime-engine/src/...) whose per-element arithmetic it repeats.
#include "kernels.cuh"
#include "luma.cuh"
#include "warp.cuh"
#include "blend.cuh"

namespace tw {

// ---- wire -> engine (image.rs:178-206, premultiply :276-303) ----------------------------------------

__global__ void k_from_frame_u8(const uint8_t* __restrict__ wire, uint8_t* __restrict__ eng, int w, int h, bool flip) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long n = (long)w * h;
    if (i >= n) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    long si = (long)(flip ? h - 1 - y : y) * w + x;
    uchar4 p = reinterpret_cast<const uchar4*>(wire)[si];  // r, g, b, a
    float a = (float)p.w * inv_255();
    uchar4 o;
    o.x = p.w;
    o.y = (uint8_t)qround((float)p.x * a);
    o.z = (uint8_t)qround((float)p.y * a);
    o.w = (uint8_t)qround((float)p.z * a);
    reinterpret_cast<uchar4*>(eng)[i] = o;
}

__global__ void k_from_frame_u16(const uint16_t* __restrict__ wire, uint16_t* __restrict__ eng, int w, int h, bool flip) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long n = (long)w * h;
    if (i >= n) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    long si = (long)(flip ? h - 1 - y : y) * w + x;
    ushort4 p = reinterpret_cast<const ushort4*>(wire)[si];
    uint16_t A = u16_to_q15(p.w), R = u16_to_q15(p.x), G = u16_to_q15(p.y), Bc = u16_to_q15(p.z);
    float a = (float)A * premul16_color();
    ushort4 o;
    o.x = (uint16_t)qround((float)A * premul16_alpha());
    o.y = (uint16_t)qround((float)R * a);
    o.z = (uint16_t)qround((float)G * a);
    o.w = (uint16_t)qround((float)Bc * a);
    reinterpret_cast<ushort4*>(eng)[i] = o;
}

__global__ void k_from_frame_f32(const float* __restrict__ wire, float* __restrict__ eng, int w, int h, bool flip) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long n = (long)w * h;
    if (i >= n) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    long si = (long)(flip ? h - 1 - y : y) * w + x;
    // planes G, B, R, A
    float g = wire[si], b = wire[n + si], r = wire[2 * n + si], a = wire[3 * n + si];
    float o1 = a * r, o2 = a * g, o3 = a * b;
    if (isnan(o1) || isnan(o2) || isnan(o3) || isnan(a)) {
        o1 = nr::mul(a, r);
        o2 = nr::mul(a, g);
        o3 = nr::mul(a, b);
    }
    reinterpret_cast<float4*>(eng)[i] = make_float4(a, o1, o2, o3);
}

// ---- engine -> wire (image.rs:213-245, unpremultiply :306-351) --------------------------------------

__device__ __forceinline__ uchar4 unpremul_u8(uchar4 p) {  // -> r, g, b, a
    if (p.x == 0) return make_uchar4(p.y, p.z, p.w, p.x);
    float s = 255.0f / (float)p.x;
    auto f = [&](uint8_t c) {
        float v = (float)c * s;
        if (v > 255.0f) v = 255.0f;
        return (uint8_t)qround(v);
    };
    return make_uchar4(f(p.y), f(p.z), f(p.w), p.x);
}

__device__ __forceinline__ ushort4 unpremul_u16(ushort4 p) {  // -> wire r, g, b, a
    ushort4 o;
    if (p.x == 0) {
        o = make_ushort4(p.y, p.z, p.w, p.x);
    } else {
        float a = (float)p.x;
        float s = 32768.0f / a;
        o = make_ushort4((uint16_t)qround((float)p.y * s), (uint16_t)qround((float)p.z * s),
                         (uint16_t)qround((float)p.w * s), (uint16_t)qround(a * unpremul16_alpha()));
    }
    return make_ushort4(q15_to_u16(o.x), q15_to_u16(o.y), q15_to_u16(o.z), q15_to_u16(o.w));
}

__device__ __forceinline__ float4 unpremul_f32(float4 p) {  // -> a, r, g, b (engine order)
    if ((double)p.x < 1e-12) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // `1.0 / a` keeps a NaN alpha's payload as the x86 divide does (the quieted NaN operand)
    float inv = nr::div(1.0f, p.x);
    float r = p.y * inv, g = p.z * inv, b = p.w * inv;
    if (isnan(r) || isnan(g) || isnan(b) || isnan(p.x)) {
        r = nr::mul(p.y, inv);
        g = nr::mul(p.z, inv);
        b = nr::mul(p.w, inv);
    }
    return make_float4(p.x, r, g, b);
}

__global__ void k_to_frame_u8(const uint8_t* __restrict__ eng, uint8_t* __restrict__ wire, int w, int h, bool flip) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long n = (long)w * h;
    if (i >= n) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    long si = (long)(flip ? h - 1 - y : y) * w + x;
    reinterpret_cast<uchar4*>(wire)[i] = unpremul_u8(reinterpret_cast<const uchar4*>(eng)[si]);
}

__global__ void k_to_frame_u16(const uint16_t* __restrict__ eng, uint16_t* __restrict__ wire, int w, int h, bool flip) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long n = (long)w * h;
    if (i >= n) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    long si = (long)(flip ? h - 1 - y : y) * w + x;
    reinterpret_cast<ushort4*>(wire)[i] = unpremul_u16(reinterpret_cast<const ushort4*>(eng)[si]);
}

__global__ void k_to_frame_f32(const float* __restrict__ eng, float* __restrict__ wire, int w, int h, bool flip) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long n = (long)w * h;
    if (i >= n) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    long si = (long)(flip ? h - 1 - y : y) * w + x;
    float4 o = unpremul_f32(reinterpret_cast<const float4*>(eng)[si]);
    wire[i] = o.z;          // G
    wire[n + i] = o.w;      // B
    wire[2 * n + i] = o.y;  // R
    wire[3 * n + i] = o.x;  // A
}

// ---- luma (prep.rs:168-235) ------------------------------------------------------------------------

__global__ void k_luma(const void* __restrict__ eng, int fmt, float* __restrict__ out, int w, int h, bool track_alpha,
                       bool video_range) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long n = (long)w * h;
    if (i >= n) return;
    out[i] = luma_px(eng, fmt, i, (track_alpha ? LUMA_TRACK_ALPHA : 0) | (video_range ? LUMA_VIDEO_RANGE : 0));
}

template <typename P>
__device__ __forceinline__ void inv_warp_px(const WarpParams& p, void* out, uint8_t* cov, int w, int h, int* bad) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    P o[4];
    bool b = false;
    uint8_t c = warp_pixel<P>(p, x, y, w, h, o, b);
    P* dst = (P*)out + ((long)y * w + x) * 4;
#pragma unroll
    for (int k = 0; k < 4; k++) dst[k] = o[k];
    if (cov) cov[(long)y * w + x] = c;
    if (b) atomicOr(bad, 1);
}

__global__ void k_inv_warp(WarpParams p, int fmt, void* __restrict__ out, uint8_t* __restrict__ cov, int w, int h,
                           int* __restrict__ bad) {
    if (fmt == 0) inv_warp_px<uint8_t>(p, out, cov, w, h, bad);
    else if (fmt == 1) inv_warp_px<uint16_t>(p, out, cov, w, h, bad);
    else inv_warp_px<float>(p, out, cov, w, h, bad);
}

// ---- blend and lerp (blend.rs) -----------------------------------------------------------------------

__global__ void k_blend(const void* __restrict__ a, const void* __restrict__ b, void* __restrict__ out, int fmt,
                        long nsamples, float w) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsamples) return;
    if (fmt == 0) ((uint8_t*)out)[i] = blend_sample<uint8_t>(((const uint8_t*)a)[i], ((const uint8_t*)b)[i], w);
    else if (fmt == 1) ((uint16_t*)out)[i] = blend_sample<uint16_t>(((const uint16_t*)a)[i], ((const uint16_t*)b)[i], w);
    else ((float*)out)[i] = blend_sample<float>(((const float*)a)[i], ((const float*)b)[i], w);
}

template <typename P>
__device__ __forceinline__ void lerp_one(void* first, const void* second, long i, float w) {
    P f[4], s[4];
    P* fp = (P*)first + i * 4;
    const P* sp = (const P*)second + i * 4;
#pragma unroll
    for (int k = 0; k < 4; k++) { f[k] = fp[k]; s[k] = sp[k]; }
    lerp_px<P>(f, s, w);
#pragma unroll
    for (int k = 0; k < 4; k++) fp[k] = f[k];
}

__global__ void k_lerp(void* __restrict__ first, const void* __restrict__ second, int fmt, long npx, float w) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npx) return;
    if (fmt == 0) lerp_one<uint8_t>(first, second, i, w);
    else if (fmt == 1) lerp_one<uint16_t>(first, second, i, w);
    else lerp_one<float>(first, second, i, w);
}

// ---- the fused Blend composition of warping code 0 ---------------------------------------------------

template <typename P>
__device__ __forceinline__ void store_px(const P o[4], void* out, long i, bool to_wire, long npx);
template <>
__device__ __forceinline__ void store_px<uint8_t>(const uint8_t o[4], void* out, long i, bool to_wire, long npx) {
    uchar4 e = make_uchar4(o[0], o[1], o[2], o[3]);
    reinterpret_cast<uchar4*>(out)[i] = to_wire ? unpremul_u8(e) : e;
}
template <>
__device__ __forceinline__ void store_px<uint16_t>(const uint16_t o[4], void* out, long i, bool to_wire, long npx) {
    ushort4 e = make_ushort4(o[0], o[1], o[2], o[3]);
    reinterpret_cast<ushort4*>(out)[i] = to_wire ? unpremul_u16(e) : e;
}
template <>
__device__ __forceinline__ void store_px<float>(const float o[4], void* out, long i, bool to_wire, long npx) {
    float4 e = make_float4(o[0], o[1], o[2], o[3]);
    if (!to_wire) {
        reinterpret_cast<float4*>(out)[i] = e;
        return;
    }
    float4 u = unpremul_f32(e);
    float* wire = (float*)out;
    wire[i] = u.z;
    wire[npx + i] = u.w;
    wire[2 * npx + i] = u.y;
    wire[3 * npx + i] = u.x;
}

template <typename P>
__device__ __forceinline__ void compose_blend_px(const WarpParams& pa, const WarpParams& pb, float wblend, int mode,
                                                 void* out, int w, int h, bool to_wire, bool flip_out, int* bad) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    // the output pixel (x, y) of the engine image lands on wire row h-1-y when flip_out
    P ta[4], tb[4], o[4];
    bool b = false;
    if (mode != 2) warp_pixel<P>(pa, x, y, w, h, ta, b);
    if (mode != 1) warp_pixel<P>(pb, x, y, w, h, tb, b);
    float wl = (float)(1.0 - (double)wblend);
    blend_px<P>(ta, tb, wblend, wl, mode, o);
    int oy = flip_out ? h - 1 - y : y;
    store_px<P>(o, out, (long)oy * w + x, to_wire, (long)w * h);
    if (b) atomicOr(bad, 1);
}

__global__ void k_compose_blend(WarpParams pa, WarpParams pb, int fmt, float wblend, int blend_mode, void* __restrict__ out,
                                int w, int h, bool to_wire, bool flip_out, int* __restrict__ bad) {
    if (fmt == 0) compose_blend_px<uint8_t>(pa, pb, wblend, blend_mode, out, w, h, to_wire, flip_out, bad);
    else if (fmt == 1) compose_blend_px<uint16_t>(pa, pb, wblend, blend_mode, out, w, h, to_wire, flip_out, bad);
    else compose_blend_px<float>(pa, pb, wblend, blend_mode, out, w, h, to_wire, flip_out, bad);
}

// ---- the vector encoder (vectors.rs:57-130) ---------------------------------------------------------
// Per output pixel: the flow sampled with the warps' flow sampler (warp.rs:415-442) at (x sx, y sy),
// scaled by (kx, ky), then the depth's store; zero != 0 writes the zero vector image
// (vectors.rs:148-156). Writes the engine image (A, R, G, B).
__global__ void k_encode_vectors(const float* __restrict__ flow, int fw, int fh, void* __restrict__ out, int W, int H,
                                 int fmt, float sx, float sy, float kx, float ky, int zero) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    float a = 0.0f, b = 0.0f;
    if (!zero) {
        float px = (float)x * sx, py = (float)y * sy;
        int fw1 = fw - 1, fh1 = fh - 1;
        int ix = cvtt32(px), iy = cvtt32(py);
        float fx = px - (float)ix, fy = py - (float)iy;
        if (ix >= fw1) { ix = fw1 - 1; fx = 1.0f; }
        if (iy >= fh1) { iy = fh1 - 1; fy = 1.0f; }
        long i00 = ((long)iy * fw + ix) * 2, i01 = i00 + (long)fw * 2;
        // x86 arithmetic: a NaN vector (a NaN or infinite flow) keeps the reference's bits in the
        // float depth's output
        float o[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            float p00 = flow[i00 + k], p10 = flow[i00 + 2 + k], p01 = flow[i01 + k], p11 = flow[i01 + 2 + k];
            float top = x86::add(x86::mul(x86::sub(p10, p00), fx), p00);
            float bot = x86::add(x86::mul(x86::sub(p11, p01), fx), p01);
            o[k] = x86::add(x86::mul(x86::sub(bot, top), fy), top);
        }
        a = x86::mul(o[0], kx);
        b = x86::mul(o[1], ky);
    }
    long i = ((long)y * W + x) * 4;
    if (fmt == 2) {
        float* d = (float*)out + i;
        d[0] = 1.0f;
        d[1] = x86::mul(x86::add(a, 1.0f), 0.5f);
        d[2] = x86::mul(x86::add(b, 1.0f), 0.5f);
        d[3] = 0.0f;
        return;
    }
    if (a > 1.0f) a = 1.0f;  // vectors.rs:133-140: a NaN falls through
    else if (-1.0f > a) a = -1.0f;
    if (b > 1.0f) b = 1.0f;
    else if (-1.0f > b) b = -1.0f;
    a = a + 1.0f;
    b = b + 1.0f;
    if (fmt == 0) {
        uint8_t* d = (uint8_t*)out + i;
        d[0] = 0xff;
        d[1] = (uint8_t)cvtt64d((double)a * 127.0 + 0.5);
        d[2] = (uint8_t)cvtt64d((double)b * 127.0 + 0.5);
        d[3] = 0;
    } else {
        uint16_t* d = (uint16_t*)out + i;
        d[0] = 0xffff;
        d[1] = (uint16_t)cvtt64d((double)a * 32767.0 + 0.5);
        d[2] = (uint16_t)cvtt64d((double)b * 32767.0 + 0.5);
        d[3] = 0;
    }
}

}  // namespace tw
