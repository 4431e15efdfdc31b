// The single precision powf of the plugin's C runtime (plugins/retime-engine/src/crt_powf.rs:
// 229-268), restated from its algorithm: a double precision logarithm and exponential from tables,
// narrowed once. One body for the device (the Delinearize prep, crt_powf in prep.cu) and the host
// (the Gaussian taps of the matte choke, matte.rs:366-385 and 441-470, crt_powf_host). Both only
// use IEEE basic operations in double precision, so both give the same bits. The tables come from
// gen_pow_tables.py.
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "pow_tables.h"

namespace tw {

struct PowTables {
    const unsigned long long* rcp;   // 257 reciprocals 1 / c of the table's mantissa centres
    const unsigned long long* log;   // 257 logarithms ln(2 c)
    const unsigned long long* exp2;  // 64 powers 2^(j / 64)
};

__host__ __device__ __forceinline__ double pow_dbl(unsigned long long b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
#endif
}

__host__ __device__ __forceinline__ unsigned long long pow_bits(double v) {
#ifdef __CUDA_ARCH__
    return (unsigned long long)__double_as_longlong(v);
#else
    unsigned long long b;
    memcpy(&b, &v, sizeof b);
    return b;
#endif
}

__host__ __device__ __forceinline__ float pow_f32(uint32_t b) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    memcpy(&f, &b, sizeof f);
    return f;
#endif
}

__host__ __device__ __forceinline__ uint32_t pow_u32(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t b;
    memcpy(&b, &f, sizeof b);
    return b;
#endif
}

__host__ __device__ __forceinline__ bool pow_odd_integer(float y) {
    float t = truncf(y);
    return t == y && fabsf(y) < 16777216.0f && ((long long)t & 1) != 0;
}

// The values of the double precision pow at the arguments where the runtime's code path does not
// run (C99 F.9.4.4), narrowed to float; a negative finite base with an integer exponent goes
// through the table path of its magnitude (the prep never asks for one: its base is >= 0).
__host__ __device__ __forceinline__ float pow_special(float x, float y, bool* done) {
    *done = true;
    if (y == 0.0f || x == 1.0f) return 1.0f;
    if (isnan(x)) return pow_f32(pow_u32(x) | 0x00400000u);
    if (isnan(y)) return pow_f32(pow_u32(y) | 0x00400000u);
    if (y == 1.0f) return x;
    if (x == 0.0f) {
        bool odd = pow_odd_integer(y);
        if (y > 0.0f) return odd ? x : 0.0f;
        return odd ? copysignf(INFINITY, x) : INFINITY;
    }
    if (isinf(y)) {
        float ax = fabsf(x);
        if (ax == 1.0f) return 1.0f;
        return (ax < 1.0f) == (y < 0.0f) ? INFINITY : 0.0f;
    }
    if (isinf(x)) {
        bool odd = pow_odd_integer(y);
        if (x > 0.0f) return y > 0.0f ? INFINITY : 0.0f;
        if (y > 0.0f) return odd ? -INFINITY : INFINITY;
        return odd ? -0.0f : 0.0f;
    }
    if (x < 0.0f && truncf(y) != y) return pow_f32(0xffc00000u);  // the invalid operation's NaN
    *done = false;
    return 0.0f;
}

// crt_powf.rs:229-268 for a positive finite base
__host__ __device__ __forceinline__ float pow_table_path(float x, float y, const PowTables& tb) {
    double xd = x, yd = y;
    double t = xd - 1.0;
    double l;
    if (x < 1.0625f && fabs(t) < 0.0625) {
        double sv = t / (t + 2.0);
        double st = sv * t;
        double u = sv + sv;
        double z = u * u;
        double t0 = z * pow_dbl(TW_POW_C0), t1 = z * pow_dbl(TW_POW_C1);
        double uz = u * z;
        double u0 = t0 + pow_dbl(TW_POW_A0), u1 = t1 + pow_dbl(TW_POW_A1);
        double uz3 = (z * z) * uz;
        double sum = uz * u0 + uz3 * u1;
        l = t + (sum - st);
    } else {
        unsigned long long mant = pow_bits(xd) & 0x000fffffffffffffull;
        int idx = (int)((mant >> 44) + ((mant >> 43) & 1));
        double c = pow_dbl(((unsigned long long)idx | 0x3fe00ull) << 44);
        double m = pow_dbl(mant | 0x3fe0000000000000ull);
        long long e = (long long)((pow_bits(xd) & 0x7ff0000000000000ull) >> 52) - 1023;
        double r = (c - m) * pow_dbl(tb.rcp[idx]);
        double q = r + (r * r) * (r * pow_dbl(TW_POW_THIRD) + 0.5);
        double el = (double)e * pow_dbl(TW_POW_LN2);
        l = (el + pow_dbl(tb.log[idx])) - q;
    }
    double w = yd * l;
    // the exponent range the runtime's path covers; beyond it the result over- or underflows float
    if (w > pow_dbl(TW_POW_LIM_HI)) return INFINITY;
    if (w <= pow_dbl(TW_POW_LIM_LO)) return 0.0f;
    int n = (int)rint(w * pow_dbl(TW_POW_K64));
    double r = w - (double)n * pow_dbl(TW_POW_LN2_64);
    double p = (r * r) * (r * pow_dbl(TW_POW_SIXTH) + 0.5) + r;
    double tj = pow_dbl(tb.exp2[n & 63]);
    double v = p * tj + tj;
    unsigned long long k = (unsigned long long)(unsigned int)(n >> 6);
    return (float)pow_dbl(pow_bits(v) + (k << 52));
}

__host__ __device__ __forceinline__ float crt_powf_with(float x, float y, const PowTables& tb) {
    bool done;
    float s = pow_special(x, y, &done);
    if (done) return s;
    if (x < 0.0f) {  // an integer exponent of a negative base: the sign of an odd power
        float m = pow_table_path(-x, y, tb);
        return pow_odd_integer(y) ? -m : m;
    }
    return pow_table_path(x, y, tb);
}

}  // namespace tw
