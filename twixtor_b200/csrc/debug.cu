// The Debug views of Create Vectors (debug.rs): per pixel Blend and Diff of W' against Y, the luma
// planes of the Detail and Edge views and their 3x3 measures fused with the overlay store. W' itself
// is two OVERs (k_over_pl) of Y and of the forward warp W onto a cleared image.
#include "kernels.cuh"
#include "blend.cuh"
#include "strict.cuh"

namespace tw {

namespace {

__device__ __forceinline__ int64_t sat64(double v) {  // Rust's saturating `f64 as i64`
    if (isnan(v)) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

// debug.rs:70-90: 1 / |1 - 0.6| and 1 / (1 - 0.6 / 2), each a double quotient narrowed to single
__device__ __forceinline__ float diff_gain() {
    float amount = __double2float_rn(__dsub_rn(1.0, (double)0.6f));
    return __double2float_rn(__ddiv_rn(1.0, (double)fabsf(amount)));
}
__device__ __forceinline__ float overlay_gain() {
    float amount = 0.6f;
    float half = __double2float_rn(__dmul_rn((double)amount, 0.5));
    float rest = __double2float_rn(__dsub_rn(1.0, (double)half));
    return __double2float_rn(__ddiv_rn(1.0, (double)rest));
}

template <typename P> __device__ __forceinline__ void load4(const void* p, long i, P o[4]) {
    const P* q = (const P*)p + i * 4;
#pragma unroll
    for (int c = 0; c < 4; c++) o[c] = q[c];
}
template <typename P> __device__ __forceinline__ void store4(void* p, long i, const P o[4]) {
    P* q = (P*)p + i * 4;
#pragma unroll
    for (int c = 0; c < 4; c++) q[c] = o[c];
}

// debug.rs:252-255: (0.29 R + 0.59 G) + 0.12 B in double precision, narrowed (x86's NaN bits)
__device__ __forceinline__ float diff_luma(double r, double g, double b) {
    return x86::narrow(x86::addd(x86::addd(x86::muld(r, 0.29), x86::muld(g, 0.59)), x86::muld(b, 0.12)));
}
template <typename P> __device__ __forceinline__ double wide(P v) { return (double)v; }
template <> __device__ __forceinline__ double wide<float>(float v) { return x86::widen(v); }

template <typename P> __device__ __forceinline__ void diff_px(const void* wp, const void* y, void* out, long i) {
    P a[4], b[4], o[4];
    load4<P>(wp, i, a);
    load4<P>(y, i, b);
    float l1 = diff_luma(wide<P>(a[1]), wide<P>(a[2]), wide<P>(a[3]));
    float l2 = diff_luma(wide<P>(b[1]), wide<P>(b[2]), wide<P>(b[3]));
    float v = x86::mul(x86::abs(x86::sub(l1, l2)), diff_gain());
    if (sizeof(P) == 4) {
        float f = x86::cap(v, 1.0f);
        o[0] = (P)1.0f;
        o[1] = o[2] = o[3] = (P)f;
    } else {
        float top = sizeof(P) == 1 ? 255.0f : 65535.0f;
        float c = x86::cap(v, top);
        P q = (P)sat64(__dadd_rn((double)c, 0.5));
        o[0] = (P)top;
        o[1] = o[2] = o[3] = q;
    }
    store4<P>(out, i, o);
}

}  // namespace

__global__ void k_debug_blend(const void* __restrict__ wp, const void* __restrict__ y, int fmt, void* __restrict__ out,
                              long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == 0) {
        uint8_t f[4], s[4];
        load4<uint8_t>(wp, i, f);
        load4<uint8_t>(y, i, s);
        lerp_px<uint8_t>(f, s, 0.5f);
        store4<uint8_t>(out, i, f);
    } else if (fmt == 1) {
        uint16_t f[4], s[4];
        load4<uint16_t>(wp, i, f);
        load4<uint16_t>(y, i, s);
        lerp_px<uint16_t>(f, s, 0.5f);
        store4<uint16_t>(out, i, f);
    } else {
        float f[4], s[4];
        load4<float>(wp, i, f);
        load4<float>(y, i, s);
        lerp_px<float>(f, s, 0.5f);
        store4<float>(out, i, f);
    }
}

__global__ void k_debug_diff(const void* __restrict__ wp, const void* __restrict__ y, int fmt, void* __restrict__ out,
                             long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == 0) diff_px<uint8_t>(wp, y, out, i);
    else if (fmt == 1) diff_px<uint16_t>(wp, y, out, i);
    else diff_px<float>(wp, y, out, i);
}

__global__ void k_debug_luma(const void* __restrict__ img, int fmt, float* __restrict__ out, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == 2) {  // debug.rs:303-310: the sums again with the rule's NaN choice when NaN
        float p[4];
        load4<float>(img, i, p);
        double tr = x86::muld(x86::widen(p[1]), 0.29), tg = x86::muld(x86::widen(p[2]), 0.59),
               tb = x86::muld(x86::widen(p[3]), 0.12);
        float v = x86::narrow(x86::addd(x86::addd(tr, tg), tb));
        if (isnan(v)) v = x86::narrow(nr::add64(nr::add64(tr, tg), tb));
        out[i] = v;
        return;
    }
    double r, g, b, s;
    if (fmt == 0) {
        uint8_t p[4];
        load4<uint8_t>(img, i, p);
        r = p[1]; g = p[2]; b = p[3]; s = 255.0;
    } else {
        uint16_t p[4];
        load4<uint16_t>(img, i, p);
        r = p[1]; g = p[2]; b = p[3]; s = 65535.0;
    }
    float v = __double2float_rn(__dadd_rn(__dadd_rn(__ddiv_rn(__dmul_rn(r, 0.29), s), __ddiv_rn(__dmul_rn(g, 0.59), s)),
                                          __ddiv_rn(__dmul_rn(b, 0.12), s)));
    out[i] = x86::cap(v, 1.0f);
}

namespace {

// debug.rs:318-346: the luma on the border, else sqrt(S / 8) of the absolute differences in row order
__device__ __forceinline__ float detail_at(const float* l, int w, int h, int x, int y) {
    float c = l[(long)y * w + x];
    if (x == 0 || y == 0 || x + 1 == w || y + 1 == h) return c;
    float s = 0.0f;
    bool first = true;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
            if (dx == 0 && dy == 0) continue;
            float d = x86::abs(x86::sub(c, l[(long)(y + dy) * w + x + dx]));
            s = first ? d : x86::add(s, d);
            first = false;
        }
    return x86::sqrt(x86::mul(s, 0.125f));
}

// debug.rs:355-378: the Sobel magnitude, border repeated, times 2 capped at 255
__device__ __forceinline__ float edge_at(const float* l, int w, int h, int x, int y) {
    auto n = [&](int dx, int dy) {
        int yy = min(max(y + dy, 0), h - 1), xx = min(max(x + dx, 0), w - 1);
        return l[(long)yy * w + xx];
    };
    using namespace x86;
    float gx = add(sub(add(sub(add(x86::neg(n(-1, -1)), n(1, -1)), mul(2.0f, n(-1, 0))), mul(2.0f, n(1, 0))), n(-1, 1)), n(1, 1));
    float gy = sub(sub(sub(add(add(mul(2.0f, n(0, -1)), n(-1, -1)), n(1, -1)), n(-1, 1)), mul(2.0f, n(0, 1))), n(1, 1));
    float m = x86::sqrt(add(mul(gy, gy), mul(gx, gx)));
    float e = narrow(muld(widen(m), 0.17677669529664));
    float sc = mul(2.0f, e);
    return x86::cap_above(sc, 255.0f);
}

__device__ __forceinline__ float overlay_value(float m, float gain) {  // debug.rs:382-391
    float v = x86::mul(gain, m);
    return x86::floor_below(x86::cap_above(v, 1.0f), 0.0f);
}

}  // namespace

__global__ void k_debug_overlay(const float* __restrict__ lw, const float* __restrict__ ly, int w, int h, int fmt,
                                int edge, void* __restrict__ out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    float mr = edge ? edge_at(lw, w, h, x, y) : detail_at(lw, w, h, x, y);
    float mg = edge ? edge_at(ly, w, h, x, y) : detail_at(ly, w, h, x, y);
    float gain = overlay_gain();
    float vr = overlay_value(mr, gain), vg = overlay_value(mg, gain);
    long i = (long)y * w + x;
    if (fmt == 0) {
        uint8_t o[4] = {255, (uint8_t)sat64(__dadd_rn(__dmul_rn((double)vr, 255.0), 0.5)), 0, 0};
        o[2] = o[3] = (uint8_t)sat64(__dadd_rn(__dmul_rn((double)vg, 255.0), 0.5));
        store4<uint8_t>(out, i, o);
    } else if (fmt == 1) {
        uint16_t o[4] = {65535, (uint16_t)sat64(__dadd_rn(__dmul_rn((double)vr, 65535.0), 0.5)), 0, 0};
        o[2] = o[3] = (uint16_t)sat64(__dadd_rn(__dmul_rn((double)vg, 65535.0), 0.5));
        store4<uint16_t>(out, i, o);
    } else {
        float o[4] = {1.0f, vr, vg, vg};
        store4<float>(out, i, o);
    }
}

}  // namespace tw
