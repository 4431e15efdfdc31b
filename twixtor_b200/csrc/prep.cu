// The image prep of the optical flow (plugins/retime-engine/src/prep.rs:296-340): Delinearize with
// the plugin runtime's single precision powf (crt_powf.rs, restated from its algorithm: a double
// precision logarithm and exponential from tables, narrowed once), and the per pixel map of the
// Contrast / Edge Enhance step after its Gaussian blur. The tables come from gen_pow_tables.py.
#include "kernels.cuh"
#include "pow_tables.h"

namespace tw {

__constant__ unsigned long long c_pow_rcp[257] = TW_POW_RCP_INIT;
__constant__ unsigned long long c_pow_log[257] = TW_POW_LOG_INIT;
__constant__ unsigned long long c_pow_exp2[64] = TW_POW_EXP2_INIT;

namespace {

__device__ __forceinline__ double dbl(unsigned long long b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ unsigned long long ubits(double v) { return (unsigned long long)__double_as_longlong(v); }

__device__ __forceinline__ bool odd_integer(float y) {
    float t = truncf(y);
    return t == y && fabsf(y) < 16777216.0f && ((long long)t & 1) != 0;
}

// The values of the double precision pow at the arguments where the runtime's code path does not
// run (C99 F.9.4.4), narrowed to float; a negative finite base with an integer exponent goes
// through the table path of its magnitude (the prep never asks for one: its base is >= 0).
__device__ float pow_special(float x, float y, bool* done) {
    *done = true;
    if (y == 0.0f || x == 1.0f) return 1.0f;
    if (isnan(x)) return nr::quiet(x);
    if (isnan(y)) return nr::quiet(y);
    if (y == 1.0f) return x;
    if (x == 0.0f) {
        bool odd = odd_integer(y);
        if (y > 0.0f) return odd ? x : 0.0f;
        return odd ? copysignf(INFINITY, x) : INFINITY;
    }
    if (isinf(y)) {
        float ax = fabsf(x);
        if (ax == 1.0f) return 1.0f;
        return (ax < 1.0f) == (y < 0.0f) ? INFINITY : 0.0f;
    }
    if (isinf(x)) {
        bool odd = odd_integer(y);
        if (x > 0.0f) return y > 0.0f ? INFINITY : 0.0f;
        if (y > 0.0f) return odd ? -INFINITY : INFINITY;
        return odd ? -0.0f : 0.0f;
    }
    if (x < 0.0f && truncf(y) != y) return __uint_as_float(0xffc00000u);  // the invalid operation's NaN
    *done = false;
    return 0.0f;
}

// crt_powf.rs:229-268 for a positive finite base
__device__ float table_powf(float x, float y) {
    double xd = x, yd = y;
    double t = xd - 1.0;
    double l;
    if (x < 1.0625f && fabs(t) < 0.0625) {
        double sv = t / (t + 2.0);
        double st = sv * t;
        double u = sv + sv;
        double z = u * u;
        double t0 = z * dbl(TW_POW_C0), t1 = z * dbl(TW_POW_C1);
        double uz = u * z;
        double u0 = t0 + dbl(TW_POW_A0), u1 = t1 + dbl(TW_POW_A1);
        double uz3 = (z * z) * uz;
        double sum = uz * u0 + uz3 * u1;
        l = t + (sum - st);
    } else {
        unsigned long long mant = ubits(xd) & 0x000fffffffffffffull;
        int idx = (int)((mant >> 44) + ((mant >> 43) & 1));
        double c = dbl(((unsigned long long)idx | 0x3fe00ull) << 44);
        double m = dbl(mant | 0x3fe0000000000000ull);
        long long e = (long long)((ubits(xd) & 0x7ff0000000000000ull) >> 52) - 1023;
        double r = (c - m) * dbl(c_pow_rcp[idx]);
        double q = r + (r * r) * (r * dbl(TW_POW_THIRD) + 0.5);
        double el = (double)e * dbl(TW_POW_LN2);
        l = (el + dbl(c_pow_log[idx])) - q;
    }
    double w = yd * l;
    // the exponent range the runtime's path covers; beyond it the result over- or underflows float
    if (w > dbl(TW_POW_LIM_HI)) return INFINITY;
    if (w <= dbl(TW_POW_LIM_LO)) return 0.0f;
    int n = (int)rint(w * dbl(TW_POW_K64));
    double r = w - (double)n * dbl(TW_POW_LN2_64);
    double p = (r * r) * (r * dbl(TW_POW_SIXTH) + 0.5) + r;
    double tj = dbl(c_pow_exp2[n & 63]);
    double v = p * tj + tj;
    unsigned long long k = (unsigned long long)(unsigned int)(n >> 6);
    return (float)dbl(ubits(v) + (k << 52));
}

}  // namespace

__device__ float crt_powf(float x, float y) {
    bool done;
    float s = pow_special(x, y, &done);
    if (done) return s;
    if (x < 0.0f) {  // an integer exponent of a negative base: the sign of an odd power
        float m = table_powf(-x, y);
        return odd_integer(y) ? -m : m;
    }
    return table_powf(x, y);
}

// prep.rs:296-307 (delinearize): p = powf(max(p, 0) / 255, 1 / 2.2) * 255 (-0.0 stays -0.0)
__global__ void k_delinearize(float* __restrict__ p, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float inv = 1.0f / 2.2f;
    float v = p[i];
    if (v <= 0.0f && v != 0.0f) v = 0.0f;
    float base = v / 255.0f;
    p[i] = crt_powf(base, inv) * 255.0f;
}

// prep.rs:326-340 after the blur: the solver's one sided gradient (flow.rs:283-316) of the blurred
// plane, m = sqrt(gx^2 + gy^2), f = m <= 20 ? m * 0.05 : 1, p = (f * 255 + p) * 0.5
__global__ void k_edge_map(const float* __restrict__ src, float* __restrict__ dst, int w, int h) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)w * h) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    float c = src[i];
    float nx = 0.0f, dx = 0.0f, ny = 0.0f, dy = 0.0f;
    if (x >= 1) { nx = (c - src[i - 1]) + 0.0f; dx = 1.0f; }
    if (y >= 1) { ny = (c - src[i - w]) + 0.0f; dy = 1.0f; }
    if (x + 1 <= w - 1) { nx = nx + (src[i + 1] - c); dx = dx + 1.0f; }
    if (y + 1 <= h - 1) { ny = ny + (src[i + w] - c); dy = dy + 1.0f; }
    float gx = nx / dx, gy = ny / dy;
    float m = sqrtf(gx * gx + gy * gy);
    float f = m <= 20.0f ? m * 0.05f : 1.0f;
    dst[i] = (f * 255.0f + c) * 0.5f;
}

// the powf above over arrays, for the checks against the runtime's traced values
__global__ void k_check_powf(const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ out, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = crt_powf(x[i], y[i]);
}

}  // namespace tw
