// The inverse warp of one output pixel (warp.rs:290-561), shared by the warp, Blend and Smart Blend
// kernels. Strict mode: single precision in the reference's order, the NaN rule repeat of the
// float depth, x86 truncations.
#pragma once
#include "kernels.cuh"

namespace tw {

template <typename P> struct Pix;
template <> struct Pix<uint8_t> {
    __device__ static float f(uint8_t v) { return (float)v; }
    __device__ static uint8_t store(float v) { return sat_u8(v); }
    // warp.rs:152-155: the stored sample scaled by the fade, the add in double
    __device__ static uint8_t faded(float v, float f) { return (uint8_t)cvtt64d((double)((float)sat_u8(v) * f) + 0.5); }
};
template <> struct Pix<uint16_t> {
    __device__ static float f(uint16_t v) { return (float)v; }
    __device__ static uint16_t store(float v) { return sat_u16(v); }
    __device__ static uint16_t faded(float v, float f) { return (uint16_t)cvtt64d((double)((float)sat_u16(v) * f) + 0.5); }
};
template <> struct Pix<float> {
    __device__ static float f(float v) { return v; }
    __device__ static float store(float v) { return v; }
    // a NaN sample keeps its payload through the fade product, as on x86
    __device__ static float faded(float v, float f) { return nr::mul(v, f); }
};

// warp.rs:178-215 (clip_to_rect), bounded like the reference
__device__ __forceinline__ bool clip_to_rect(float x, float y, float& ix, float& iy, float w1, float h1) {
#pragma unroll 1
    for (int it = 0; it < 4096; it++) {
        if (ix < 0.0f) {
            float dy = y - iy, dxs = x - ix, num = x - 0.0f;
            ix = 0.0f;
            iy = y - (num / dxs) * dy;
            continue;
        }
        if (ix > w1) {
            float dy = y - iy, dxs = x - ix, num = x - w1;
            ix = w1;
            iy = y - (num / dxs) * dy;
            continue;
        }
        if (iy < 0.0f) {
            float dyy = y - iy, num = y - 0.0f, dx = x - ix;
            ix = x - (num / dyy) * dx;
            iy = 0.0f;
            continue;
        }
        if (iy > h1) {
            float dyy = y - iy, num = y - h1, dx = x - ix;
            ix = x - (num / dyy) * dx;
            iy = h1;
            continue;
        }
        return true;
    }
    return false;
}

// warp.rs:290-360 (bilerp4 + mix4 with the NaN rule repeat of the float depth)
template <typename P>
__device__ __forceinline__ void bilerp4(const P* __restrict__ src, int w, int w1, int h1, float x, float y, float o[4]) {
    int ix = cvtt32(x), iy = cvtt32(y);
    float fx = x - (float)ix, fy = y - (float)iy;
    if (ix >= w1) { ix = w1 - 1; fx = 1.0f; }
    if (iy >= h1) { iy = h1 - 1; fy = 1.0f; }
    long i00 = ((long)iy * w + ix) * 4;
    long i01 = i00 + (long)w * 4;
    P a[4], b[4], c[4], d[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        a[k] = src[i00 + k];
        b[k] = src[i00 + 4 + k];
        c[k] = src[i01 + k];
        d[k] = src[i01 + 4 + k];
    }
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float p00 = Pix<P>::f(a[k]), p10 = Pix<P>::f(b[k]), p01 = Pix<P>::f(c[k]), p11 = Pix<P>::f(d[k]);
        float top = p00 + (p10 - p00) * fx;
        float bot = p01 + (p11 - p01) * fx;
        o[k] = top + (bot - top) * fy;
        any = any || isnan(o[k]);
    }
    if (any) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float p00 = Pix<P>::f(a[k]), p10 = Pix<P>::f(b[k]), p01 = Pix<P>::f(c[k]), p11 = Pix<P>::f(d[k]);
            float top = nr::add(p00, nr::mul(nr::sub(p10, p00), fx));
            float bot = nr::add(p01, nr::mul(nr::sub(p11, p01), fx));
            o[k] = nr::add(top, nr::mul(nr::sub(bot, top), fy));
        }
    }
}

// warp.rs:415-442 (Flow::bilerp) on a strided field
__device__ __forceinline__ void flow_bilerp(const WarpParams& p, float x, float y, float& du, float& dv) {
    int fw1 = p.fw - 1, fh1 = p.fh - 1;
    int ix = cvtt32(x), iy = cvtt32(y);
    float fx = x - (float)ix, fy = y - (float)iy;
    if (ix >= fw1) { ix = fw1 - 1; fx = 1.0f; }
    if (iy >= fh1) { iy = fh1 - 1; fy = 1.0f; }
    long i00 = ((long)iy * p.fw + ix) * p.fstride;
    long i01 = i00 + (long)p.fw * p.fstride;
    long s = p.fstride;
    const float* planes[2] = {p.fu, p.fv};
    float r[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float* d = planes[k];
        float p00 = __ldg(d + i00), p10 = __ldg(d + i00 + s), p01 = __ldg(d + i01), p11 = __ldg(d + i01 + s);
        float top = (p10 - p00) * fx + p00;
        float bot = (p11 - p01) * fx + p01;
        r[k] = (bot - top) * fy + top;
    }
    du = r[0];
    dv = r[1];
}

// One output pixel of the inverse warp (warp.rs:466-561, Kernel::row / pixel_hold / pixel_fade).
// Returns the coverage byte; sets bad for a coordinate the reference refuses.
template <typename P>
__device__ __forceinline__ uint8_t warp_pixel(const WarpParams& p, int x, int y, int w, int h, P o[4], bool& bad) {
    const P* src = (const P*)p.src;
    if (p.copy_only) {
        const P* s = src + ((long)y * w + x) * 4;
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = s[k];
        return 255;
    }
    int w1i = w - 1, h1i = h - 1;
    float rx = (float)(p.fw - 1) / (float)w1i;
    float ry = (float)(p.fh - 1) / (float)h1i;
    float sx = p.amount / rx, sy = p.amount / ry;
    float wf = (float)w, hf = (float)h, w1 = (float)w1i, h1 = (float)h1i;
    float xf = (float)x, yf = (float)y;
    float du, dv;
    flow_bilerp(p, xf * rx, yf * ry, du, dv);
    float ix = du * sx + xf;
    float iy = dv * sy + yf;
    float s[4];
    if (p.hold) {
        if (!clip_to_rect(xf, yf, ix, iy, w1, h1) || isnan(ix) || isnan(iy)) {
            bad = true;
#pragma unroll
            for (int k = 0; k < 4; k++) o[k] = P(0);
            return 255;
        }
        bilerp4<P>(src, w, w1i, h1i, ix, iy, s);
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = Pix<P>::store(s[k]);
        return 255;
    }
    if (!(ix > -1.0f && ix < wf && iy > -1.0f && iy < hf)) {
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = P(0);
        return 0;
    }
    if (ix >= 0.0f && ix <= w1 && iy >= 0.0f && iy <= h1) {
        bilerp4<P>(src, w, w1i, h1i, ix, iy, s);
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = Pix<P>::store(s[k]);
        return 255;
    }
    float f = ix < 0.0f ? ix + 1.0f : (ix <= w1 ? 1.0f : wf - ix);
    if (iy < 0.0f) f *= iy + 1.0f;
    else if (iy > h1) f *= hf - iy;
    if (!clip_to_rect(xf, yf, ix, iy, w1, h1) || isnan(ix) || isnan(iy)) {
        bad = true;
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = P(0);
        return 0;
    }
    bilerp4<P>(src, w, w1i, h1i, ix, iy, s);
#pragma unroll
    for (int k = 0; k < 4; k++) o[k] = Pix<P>::faded(s[k], f);
    float c = f * 255.0f + 0.5f;
    return c <= 255.0f ? (uint8_t)cvtt64d((double)c) : (uint8_t)255;
}

}  // namespace tw
