// The per-sample blend and the per-pixel lerp of blend.rs, shared by the compositions (image.cu)
// and the Weighted Blend filters (filters.cu).
#pragma once
#include "kernels.cuh"

namespace tw {

// blend.rs:81-114, the common branch of one sample
template <typename P> __device__ __forceinline__ P blend_sample(P a, P b, float w);
template <> __device__ __forceinline__ uint8_t blend_sample<uint8_t>(uint8_t a, uint8_t b, float w) {
    float af = (float)a, bf = (float)b;
    return (uint8_t)cvtt64f((bf - af) * w + af + 0.5f);
}
template <> __device__ __forceinline__ uint16_t blend_sample<uint16_t>(uint16_t a, uint16_t b, float w) {
    float af = (float)a, bf = (float)b;
    return (uint16_t)cvtt64f((bf - af) * w + af + 0.5f);
}
template <> __device__ __forceinline__ float blend_sample<float>(float a, float b, float w) {
    float r = (b - a) * w + a + 0.0f;
    if (isnan(r)) r = nr::add(nr::add(nr::mul(nr::sub(b, a), w), a), 0.0f);
    return r;
}

// blend.rs:214-249 (lerp_pixel_int) and :182-211 (lerp_pixel_f32): first = second + (first - second) * w
template <typename P> __device__ __forceinline__ void lerp_px(P f[4], const P s[4], float w);
template <typename T>
__device__ __forceinline__ void lerp_px_int(T f[4], const T s[4], float w, float scale) {
    auto diff = [&](int i) { return (float)((int32_t)f[i] - (int32_t)s[i]); };
    auto sf = [&](int i) { return (float)(int32_t)s[i]; };
    float a = diff(0) * w + sf(0);
    float n = a / scale;
    if (!(n > 0.0f)) {
        T z = (T)cvtt64f(0.0f);
#pragma unroll
        for (int i = 0; i < 4; i++) f[i] = z;
        return;
    }
    float r = diff(1) * w + sf(1), g = diff(2) * w + sf(2), b = diff(3) * w + sf(3);
    if (n > 1.0f) { r = r / n; g = g / n; b = b / n; a = scale; }
    auto clamp = [&](float c) { return c > a ? a : (0.0f > c ? 0.0f : c); };
    r = clamp(r); g = clamp(g); b = clamp(b);
    f[1] = (T)cvtt64f(r + 0.5f);
    f[2] = (T)cvtt64f(g + 0.5f);
    f[3] = (T)cvtt64f(b + 0.5f);
    f[0] = (T)cvtt64f(a + 0.5f);
}
template <> __device__ __forceinline__ void lerp_px<uint8_t>(uint8_t f[4], const uint8_t s[4], float w) {
    lerp_px_int<uint8_t>(f, s, w, 255.0f);
}
template <> __device__ __forceinline__ void lerp_px<uint16_t>(uint16_t f[4], const uint16_t s[4], float w) {
    lerp_px_int<uint16_t>(f, s, w, 65535.0f);
}
template <> __device__ __forceinline__ void lerp_px<float>(float f[4], const float s[4], float w) {
    bool rule = false;
#pragma unroll
    for (int i = 0; i < 4; i++) rule = rule || isnan(f[i]) || isnan(s[i]);
    if (!rule) {  // the processor's arithmetic: a NaN made of infinities is x86's default NaN
        auto L = [](float a, float b, float w) { return x86::add(x86::mul(x86::sub(b, a), w), a); };
        float a = L(s[0], f[0], w);
        if (!(a > 0.0f)) { for (int i = 0; i < 4; i++) f[i] = 0.0f; return; }
        float r = L(s[1], f[1], w), g = L(s[2], f[2], w), b = L(s[3], f[3], w);
        if (a > 1.0f) { r = x86::div(r, a); g = x86::div(g, a); b = x86::div(b, a); a = 1.0f; }
        f[1] = x86::add(r, 0.0f); f[2] = x86::add(g, 0.0f); f[3] = x86::add(b, 0.0f); f[0] = x86::add(a, 0.0f);
    } else {
        auto L = [](float a, float b, float w) { return nr::add(nr::mul(nr::sub(b, a), w), a); };
        float a = L(s[0], f[0], w);
        if (!(a > 0.0f)) { for (int i = 0; i < 4; i++) f[i] = 0.0f; return; }
        float r = L(s[1], f[1], w), g = L(s[2], f[2], w), b = L(s[3], f[3], w);
        if (a > 1.0f) { r = nr::div(r, a); g = nr::div(g, a); b = nr::div(b, a); a = 1.0f; }
        f[1] = nr::add(r, 0.0f); f[2] = nr::add(g, 0.0f); f[3] = nr::add(b, 0.0f); f[0] = nr::add(a, 0.0f);
    }
}

// blend.rs:55-78 (blend with its branches) on one pixel: mode 0 common, 1 copy a, 2 copy b,
// 3 copy a then lerp(out, b, wl) with its w == 1 / w == 0 early outs
template <typename P>
__device__ __forceinline__ void blend_px(const P a[4], const P b[4], float w, float wl, int mode, P o[4]) {
    if (mode == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = blend_sample<P>(a[k], b[k], w);
    } else if (mode == 1) {
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = a[k];
    } else if (mode == 2) {
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = b[k];
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = a[k];
        if (wl == 1.0f) return;
        if (wl == 0.0f) {
#pragma unroll
            for (int k = 0; k < 4; k++) o[k] = b[k];
            return;
        }
        lerp_px<P>(o, b, wl);
    }
}

}  // namespace tw
