// The natural logarithm of the forward warp's mip level, bit-identical to glibc's logf.
//
// tw_log_base(x): log(x) evaluated in double precision from IEEE basic operations only (no libm
// call, no fused multiply-add), narrowed to float: x = m * 2^e with m in [sqrt(1/2), sqrt(2)),
// log(m) = 2 atanh(s) with s = (m - 1) / (m + 1) summed as the series 2 s (1 + s^2/3 + s^4/5 + ...)
// to s^22 (|s| < 0.1716: the first omitted term is below 1e-19 relative), plus e * ln 2. The same
// source compiles for the host (gcc, -ffp-contract=off) and the device (nvcc, -fmad=false), so both
// give the same bits for every input.
//
// glibc's logf is not correctly rounded on every input; the build runs gen_logf_table.c, which
// calls glibc's logf on every positive finite float and records the inputs where it differs from
// tw_log_base (a sorted table of (input bits, glibc result bits)). The device looks the input up in
// that table and otherwise returns tw_log_base. Special inputs follow glibc: NaN -> the input
// quieted, +-0 -> -inf, +inf -> +inf, negative -> the default NaN 0xffc00000.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define TW_HD __host__ __device__ __forceinline__
#else
#define TW_HD static inline
#endif

TW_HD uint64_t tw_dbits(double d) {
    union { double d; uint64_t u; } c;
    c.d = d;
    return c.u;
}
TW_HD double tw_bitsd(uint64_t u) {
    union { double d; uint64_t u; } c;
    c.u = u;
    return c.d;
}

// x: a positive finite float (normal or subnormal), as a double (exact)
TW_HD float tw_log_base(double x) {
    uint64_t b = tw_dbits(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    double m = tw_bitsd((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e = e + 1;
    }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    double p = 1.0 / 23.0;
    p = p * z + 1.0 / 21.0;
    p = p * z + 1.0 / 19.0;
    p = p * z + 1.0 / 17.0;
    p = p * z + 1.0 / 15.0;
    p = p * z + 1.0 / 13.0;
    p = p * z + 1.0 / 11.0;
    p = p * z + 1.0 / 9.0;
    p = p * z + 1.0 / 7.0;
    p = p * z + 1.0 / 5.0;
    p = p * z + 1.0 / 3.0;
    p = p * z + 1.0;
    double lm = (2.0 * s) * p;
    double r = (double)e * 0.6931471805599453 + lm;
    return (float)r;
}
