// Strict-mode arithmetic helpers for the retime kernels (sm_100a).
//
// Every translation unit of the library is compiled with -fmad=false -prec-div=true
// -prec-sqrt=true -ftz=false: single precision adds, multiplies and divides round on their own
// exactly as the reference CPU engine's SSE code does, so the kernels can repeat its operation
// order bit for bit. These helpers give the x86 truncating conversions the reference relies on
// (cvttss2si / cvttsd2si: NaN or out of range gives the integer indefinite INT_MIN), which the
// CUDA cvt.rzi instructions do not (they saturate), and the depth store rules.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tw {

// flow/sample.rs:17-24, warp.rs:104-110: f32 -> i32 truncation, NaN / out of range -> INT_MIN
__device__ __forceinline__ int32_t cvtt32(float x) {
    if (!(x >= -2147483648.0f && x < 2147483648.0f)) return INT32_MIN;
    return __float2int_rz(x);
}
// warp.rs:113-120, image.rs:246-252: f64 -> i64 truncation
__device__ __forceinline__ int64_t cvtt64d(double x) {
    if (!(x >= -9.223372036854775808e18 && x < 9.223372036854775808e18)) return INT64_MIN;
    return __double2ll_rz(x);
}
// blend.rs:18-25: f32 -> i64 truncation
__device__ __forceinline__ int64_t cvtt64f(float x) {
    if (!(x >= -9223372036854775808.0f && x < 9223372036854775808.0f)) return INT64_MIN;
    return __float2ll_rz(x);
}
// image.rs:255-258: q(x) = trunc((f64)x + 0.5); callers keep the low byte / word
__device__ __forceinline__ int64_t qround(float x) { return cvtt64d((double)x + 0.5); }

// warp.rs:129-135: clamp(trunc(v + 0.5), 0, 255) through the -128 bias and two saturations
__device__ __forceinline__ uint8_t sat_u8(float v) {
    int32_t i = cvtt32(v + 0.5f);
    int32_t t = (int32_t)((uint32_t)i + (uint32_t)(-128));
    int32_t w = min(max(t, -32768), 32767);
    int32_t b = min(max(w, -128), 127);
    return (uint8_t)(b + 128);
}
// warp.rs:141-146
__device__ __forceinline__ uint16_t sat_u16(float v) {
    int32_t i = cvtt32(v + 0.5f);
    int32_t t = (int32_t)((uint32_t)i + (uint32_t)(-32768));
    int32_t w = min(max(t, -32768), 32767);
    return (uint16_t)(w + 32768);
}

// nanrule.rs:44-124 (the crate's default `emulator-nan` selection). Numbers are unchanged; only a
// NaN result takes the rule's payload. Used where the reference repeats an f32 kernel with the rule.
namespace nr {
__device__ __forceinline__ float quiet(float x) { return __uint_as_float(__float_as_uint(x) | 0x00400000u); }
__device__ __forceinline__ float pick(float a, float b) {
    uint32_t ba = __float_as_uint(a), bb = __float_as_uint(b);
    bool sa = (ba & 0x00400000u) == 0, sb = (bb & 0x00400000u) == 0;
    uint32_t fa = ba & 0x007fffffu, fb = bb & 0x007fffffu;
    bool a_larger = fa > fb || (fa == fb && (ba >> 31) < (bb >> 31));
    bool take_b = (sa == sb) ? !a_larger : sa;
    return quiet(take_b ? b : a);
}
__device__ __forceinline__ float fix(float r, float a, float b) {
    if (!isnan(r)) return r;
    if (isnan(a)) return isnan(b) ? pick(a, b) : quiet(a);
    if (isnan(b)) return quiet(b);
    return __uint_as_float(0xffc00000u);
}
__device__ __forceinline__ float add(float a, float b) { return fix(a + b, a, b); }
__device__ __forceinline__ float sub(float a, float b) { return fix(a - b, a, b); }
__device__ __forceinline__ float mul(float a, float b) { return fix(a * b, a, b); }
__device__ __forceinline__ float div(float a, float b) { return fix(a / b, a, b); }
// nanrule.rs:119-161: the double precision add with the rule's NaN choice
__device__ __forceinline__ double add64(double a, double b) {
    double r = __dadd_rn(a, b);
    if (!isnan(r)) return r;
    unsigned long long ba = (unsigned long long)__double_as_longlong(a), bb = (unsigned long long)__double_as_longlong(b);
    const unsigned long long Q = 0x0008000000000000ull;
    unsigned long long o;
    if (isnan(a) && isnan(b)) {
        bool sa = (ba & Q) == 0, sb = (bb & Q) == 0;
        unsigned long long fa = ba & 0x000fffffffffffffull, fb = bb & 0x000fffffffffffffull;
        bool a_larger = fa > fb || (fa == fb && (ba >> 63) < (bb >> 63));
        bool take_b = sa == sb ? !a_larger : sa;
        o = (take_b ? bb : ba) | Q;
    } else if (isnan(a)) {
        o = ba | Q;
    } else if (isnan(b)) {
        o = bb | Q;
    } else {
        o = 0xfff8000000000000ull;
    }
    return __longlong_as_double((long long)o);
}
}  // namespace nr

// The x86 SSE results of the plain single precision operations, NaNs included: a NaN operand
// propagates quieted (the first one when both are NaN), an invalid operation on numbers gives the
// default NaN 0xffc00000. The device's own NaN is canonical, so where a plain operation of the
// reference can carry a NaN into an output these give its bits; numbers are unchanged.
namespace x86 {
__device__ __forceinline__ float fix(float r, float a, float b) {
    if (!isnan(r)) return r;
    if (isnan(a)) return nr::quiet(a);
    if (isnan(b)) return nr::quiet(b);
    return __uint_as_float(0xffc00000u);
}
__device__ __forceinline__ float add(float a, float b) { return fix(a + b, a, b); }
__device__ __forceinline__ float sub(float a, float b) { return fix(a - b, a, b); }
__device__ __forceinline__ float mul(float a, float b) { return fix(a * b, a, b); }
__device__ __forceinline__ float div(float a, float b) { return fix(a / b, a, b); }
// andps / xorps: the sign bit alone, a NaN's payload kept (the device's abs and neg, which the
// compiler would make of a plain mask, may not keep it: the masks are PTX integer operations)
__device__ __forceinline__ float abs(float a) {
    uint32_t r;
    asm("and.b32 %0, %1, 0x7fffffff;" : "=r"(r) : "r"(__float_as_uint(a)));
    return __uint_as_float(r);
}
__device__ __forceinline__ float neg(float a) {
    uint32_t r;
    asm("xor.b32 %0, %1, 0x80000000;" : "=r"(r) : "r"(__float_as_uint(a)));
    return __uint_as_float(r);
}
// The branches of a clamp as a compare and a select of the sample bits in PTX: the compiler turns
// `v >= t ? t : v` on floats into a min instruction, whose NaN result is canonical, where x86's
// compare and select keep a NaN's bits.
__device__ __forceinline__ float select_bits(bool p, float a, float b) {  // p ? a : b, bit for bit
    uint32_t r;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %1, 0;\n\tselp.b32 %0, %2, %3, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(__float_as_uint(a)), "r"(__float_as_uint(b)));
    return __uint_as_float(r);
}
__device__ __forceinline__ float cap(float v, float top) { return select_bits(v >= top, top, v); }
__device__ __forceinline__ float cap_above(float v, float top) { return select_bits(v > top, top, v); }
__device__ __forceinline__ float floor_below(float v, float bottom) { return select_bits(v < bottom, bottom, v); }
// sqrtss: a NaN operand quieted, a negative number the default NaN
__device__ __forceinline__ float sqrt(float a) {
    if (isnan(a)) return nr::quiet(a);
    if (a < 0.0f) return __uint_as_float(0xffc00000u);
    return __fsqrt_rn(a);
}
// cvtss2sd / cvtsd2ss: a NaN keeps its sign and the leading bits of its payload, quieted
__device__ __forceinline__ double widen(float a) {
    if (!isnan(a)) return (double)a;
    unsigned long long b = (unsigned long long)__float_as_uint(a);
    unsigned long long o = ((b >> 31) << 63) | 0x7ff0000000000000ull | ((b & 0x007fffffull) << 29) | 0x0008000000000000ull;
    return __longlong_as_double((long long)o);
}
__device__ __forceinline__ float narrow(double a) {
    if (!isnan(a)) return __double2float_rn(a);
    unsigned long long b = (unsigned long long)__double_as_longlong(a);
    uint32_t o = (uint32_t)((b >> 63) << 31) | 0x7f800000u | (uint32_t)((b >> 29) & 0x007fffffull) | 0x00400000u;
    return __uint_as_float(o);
}
// the double operations: a NaN operand propagates quieted (the first one), an invalid operation on
// numbers gives the default NaN 0xfff8000000000000
__device__ __forceinline__ double fixd(double r, double a, double b) {
    if (!isnan(r)) return r;
    const unsigned long long Q = 0x0008000000000000ull;
    if (isnan(a)) return __longlong_as_double(__double_as_longlong(a) | (long long)Q);
    if (isnan(b)) return __longlong_as_double(__double_as_longlong(b) | (long long)Q);
    return __longlong_as_double((long long)0xfff8000000000000ull);
}
__device__ __forceinline__ double addd(double a, double b) { return fixd(__dadd_rn(a, b), a, b); }
__device__ __forceinline__ double muld(double a, double b) { return fixd(__dmul_rn(a, b), a, b); }
}  // namespace x86

// sample.rs:31-41: index and fraction of one coordinate, clamped into 0..=len-2
__device__ __forceinline__ void cell(float x, int len, int& io, float& fo) {
    int i = cvtt32(x);
    float f = x - (float)i;
    int last = len - 1;
    if (i >= last) { i = last - 1; f = 1.0f; }
    int iu = i < 0 ? 0 : i;
    int lim = len >= 2 ? len - 2 : 0;
    io = min(iu, lim);
    fo = f;
}

// sample.rs:47-64: (b - a) * f + a chains
__device__ __forceinline__ float bilinear1(const float* __restrict__ img, int w, int h, float x, float y) {
    int ix, iy;
    float fx, fy;
    cell(x, w, ix, fx);
    cell(y, h, iy, fy);
    long i = (long)iy * w + ix;
    float p00 = __ldg(img + i), p10 = __ldg(img + i + 1), p01 = __ldg(img + i + w), p11 = __ldg(img + i + w + 1);
    float top = (p10 - p00) * fx + p00;
    float bot = (p11 - p01) * fx + p01;
    return (bot - top) * fy + top;
}

// the constants and the 16 bpc wire conversion of the image boundary (image.rs:261-267,
// crates/fx-core/src/frame.rs:131-142)
__device__ __forceinline__ float inv_255() { return __uint_as_float(0x3b808081u); }            // image.rs:261
__device__ __forceinline__ float premul16_color() { return __uint_as_float(0x387fff00u); }     // image.rs:263
__device__ __forceinline__ float premul16_alpha() { return __uint_as_float(0x3fffff00u); }     // image.rs:265
__device__ __forceinline__ float unpremul16_alpha() { return __uint_as_float(0x3f000080u); }   // image.rs:267

__device__ __forceinline__ uint16_t u16_to_q15(uint16_t v) { return (uint16_t)(((uint32_t)v * 32768u + 32767u) / 65535u); }
__device__ __forceinline__ uint16_t q15_to_u16(uint16_t v) {
    uint32_t m = v < 32768 ? v : 32768;
    return (uint16_t)((m * 65535u + 16384u) / 32768u);
}

}  // namespace tw
