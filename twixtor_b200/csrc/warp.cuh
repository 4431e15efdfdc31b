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

// warp.rs:339-352 (mix4): the three lerps of four taps, repeated with the NaN rule when NaN
template <typename P>
__device__ __forceinline__ void mix4(const P* a, const P* b, const P* c, const P* d, float fx, float fy, float o[4]) {
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

// warp.rs:362-396 (bilerp360): the coordinates already in [0, W) x [0, H); the right neighbour of
// the last column is column 0, below the last row the taps are the last row's shifted by half the
// width
template <typename P>
__device__ __forceinline__ void bilerp360(const P* __restrict__ src, int w, int w1, int h1, float x, float y, float o[4]) {
    int ix = cvtt32(x), iy = cvtt32(y);
    float fx = x - (float)ix, fy = y - (float)iy;
    int x1 = ix + 1 > w1 ? 0 : ix + 1;
    int xc, xd, yc;
    if (iy + 1 > h1) {
        int half = w / 2;
        xc = (half + ix) % w;
        xd = (half + x1) % w;
        yc = h1;
    } else {
        xc = ix;
        xd = x1;
        yc = iy + 1;
    }
    int ya = min(iy, h1);
    xc = max(xc, 0);
    xd = max(xd, 0);
    auto at = [&](int xx, int yy) { return src + ((long)yy * w + xx) * 4; };
    mix4<P>(at(ix, ya), at(x1, ya), at(xc, yc), at(xd, yc), fx, fy, o);
}

// warp.rs:563-621 (pixel_360): wrapped by whole turns (at most 2^16 steps, else bad), an odd number
// of vertical wraps reflected over the pole, then the 360 sampler; the coverage stays 255
template <typename P>
__device__ __forceinline__ void pixel_360(const P* src, int w, int h, float ix, float iy, P o[4], bool& bad) {
    const uint32_t WRAP_LIMIT = 1u << 16;
    float wf = (float)w, hf = (float)h;
    uint32_t guard = 0, n = 0;
    while (ix < 0.0f) { ix += wf; if (++guard > WRAP_LIMIT) break; }
    while (wf <= ix) { ix -= wf; if (++guard > WRAP_LIMIT) break; }
    while (iy < 0.0f) { iy += hf; n++; if (++guard > WRAP_LIMIT) break; }
    while (hf <= iy) { iy -= hf; n++; if (++guard > WRAP_LIMIT) break; }
    if (guard > WRAP_LIMIT || !(ix >= 0.0f && ix < wf) || isnan(iy)) {
        bad = true;
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = P(0);
        return;
    }
    if (n & 1) {
        ix = wf * 0.5f + ix;
        if (ix >= wf) ix -= wf;
        if (iy != 0.0f) iy = hf - iy;
    }
    float s[4];
    bilerp360<P>(src, w, w - 1, h - 1, ix, iy, s);
#pragma unroll
    for (int k = 0; k < 4; k++) o[k] = Pix<P>::store(s[k]);
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
    const float rx = p.rx, ry = p.ry, sx = p.sx, sy = p.sy;  // formed on the host (warp_params)
    float wf = (float)w, hf = (float)h, w1 = (float)w1i, h1 = (float)h1i;
    float xf = (float)x, yf = (float)y;
    float du, dv;
    flow_bilerp(p, xf * rx, yf * ry, du, dv);
    float ix = du * sx + xf;
    float iy = dv * sy + yf;
    float s[4];
    if (p.is360) {
        pixel_360<P>(src, w, h, ix, iy, o, bad);
        return 255;
    }
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
