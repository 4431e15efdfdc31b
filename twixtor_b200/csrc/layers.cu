// The layered composition with plates of the FG matte effects (layers/plates.rs, matte.rs): the
// per pixel kernels of the matte planes, the layer images, the plate OVER and the refill around
// the hole fill. The solves, warps, fills and single layer compositions are the library's own
// stages; runtime.cu (tw_compose_layers) strings them together.
//
// Matte planes hold the units of the depth (whole numbers 0..255 / 0..65535 as floats, or the float
// value itself). NaN handling follows the reference's x86 arithmetic where a NaN of a float matte
// can reach an output (the cut, in double precision there), and its NaN rule where it uses it.
#include "kernels.cuh"

#include <climits>

namespace tw {

__device__ __forceinline__ float white_of(int fmt) { return fmt == 0 ? 255.0f : fmt == 1 ? 65535.0f : 1.0f; }

// Rust's saturating float -> i64 cast (`as i64`: NaN gives 0)
__device__ __forceinline__ int64_t as_i64(float x) {
    if (isnan(x)) return 0;
    if (x >= 9223372036854775808.0f) return INT64_MAX;
    if (x < -9223372036854775808.0f) return INT64_MIN;
    return __float2ll_rz(x);
}

// matte.rs:141-188 (extract_raw) of a matte frame read straight (image.rs:142-171: the FG mattes of
// retime-fgbg, plugins/retime-fgbg/src/glue.rs:335): channel `chan` (1 R, 2 G, 3 B, else alpha) of
// the wire frame as stored, rows reversed when `flip`; 8 bpc v / 255, 16 bpc the q15 value scaled
// like from_frame's alpha, over 65535, both clamped to 0..1; float the sample times one (the x86
// product: a NaN keeps its payload, quieted).
__global__ void k_matte_extract(const void* __restrict__ wire, int fmt, int chan, int w, int h, bool flip,
                                float* __restrict__ out) {
    long n = (long)w * h;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    long si = (long)(flip ? h - 1 - y : y) * w + x;
    int c = chan == 1 ? 0 : chan == 2 ? 1 : chan == 3 ? 2 : 3;  // wire order R, G, B, A
    float v;
    if (fmt == 0) {
        v = (float)((const uint8_t*)wire)[si * 4 + c] / 255.0f;
    } else if (fmt == 1) {
        uint16_t q15 = u16_to_q15(((const uint16_t*)wire)[si * 4 + c]);
        v = (float)(uint16_t)qround((float)q15 * premul16_alpha()) / 65535.0f;
    } else {
        int plane = c == 0 ? 2 : c == 1 ? 0 : c == 2 ? 1 : 3;  // float wire planes G, B, R, A
        out[i] = x86::mul(((const float*)wire)[plane * n + si], 1.0f);
        return;
    }
    out[i] = v > 1.0f ? 1.0f : v > 0.0f ? v : 0.0f;  // matte.rs:79-87
}

// matte.rs:106-112: whether some value of a matte lies outside 0..1 (the clamp then applies to all)
__global__ void k_matte_out_of_range(const float* __restrict__ m, long n, int* __restrict__ flag) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool out = false;
    if (i < n) {
        float v = m[i];
        out = !(v >= 0.0f && v <= 1.0f);
    }
    if (__syncthreads_or(out) && threadIdx.x == 0) atomicOr(flag, 1);
}

// plates.rs:50-57: the raw matte in the units of the depth (clamped first when `*clamp`)
__global__ void k_raw_plane(const float* __restrict__ m, long n, int fmt, const int* __restrict__ clamp,
                            float* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = m[i];
    if (fmt == 2) {
        out[i] = x;
        return;
    }
    if (*clamp) x = x > 1.0f ? 1.0f : (x >= 0.0f ? x : 0.0f);  // matte.rs:94-102
    out[i] = (float)as_i64(x * white_of(fmt) + 0.5f);
}

// plates.rs:63-78, the cut of c by the matte v of a layer above, with the x86 results for NaNs: the
// double product takes v's NaN first, then c's
__device__ __forceinline__ float cut(float c, float v, float white, bool isf) {
    float x;
    if (isnan(v)) x = nr::quiet(v);
    else if (isnan(c)) x = nr::quiet(c);
    else {
        double d = (1.0 - (double)v) * (double)c;
        x = isnan(d) ? __uint_as_float(0xffc00000u) : (float)d;  // an invalid product: the default NaN
    }
    if (0.0f > x) x = 0.0f;
    else if (x > white) x = white;
    if (isf) return x86::add(x, 0.0f);
    return (float)as_i64(x + 0.5f);
}

// plates.rs:86-97 with a zero inverse matte shrink (the choke of the cut is then the clamp of
// matte.rs:350-359): layer k's composition plane; raws: nfg planes of n values, FG1 first
__global__ void k_comp_plane(const float* __restrict__ raws, const float* __restrict__ cuts, int nfg, int k, long n,
                             int fmt, float* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float white = white_of(fmt);
    bool isf = fmt == 2;
    float c = k == nfg ? white : raws[(long)k * n + i];
    float kk = 1.0f / white;
    for (int j = k - 1; j >= 0; j--) {
        float v;
        if (cuts) {
            v = cuts[(long)j * n + i];  // the choked matte of FG j (k_choke_finish)
        } else {  // no shrink: the choke is the clamp of the plane
            v = x86::mul(raws[(long)j * n + i], kk);
            if (0.0f > v) v = 0.0f;
            else if (v >= 1.0f) v = 1.0f;
        }
        c = cut(c, v, white, isf);
    }
    out[i] = c;
}

// ---- the plugin's matte choke of the cut (plates.rs:80-90 cut_matte, matte.rs:280-484 choke_pl) ------

// matte.rs:337-341 (invert_pl_value): (f32)(1.0 - (double)v), above 0.999 1.0; a NaN stays (quieted)
__device__ __forceinline__ float invert_pl(float v) {
    if (isnan(v)) return nr::quiet(v);
    float x = (float)(1.0 - (double)v);
    return x > 0.999f ? 1.0f : x;
}

// The matte FG j as the cut reads it before the shrink steps: raw * (1 / white), inverted for a grow
// (the cut enters the choke with minus the shrink, so a positive shrink grows the inverse).
__global__ void k_choke_base(const float* __restrict__ raw, long n, float kk, bool grow, float* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = x86::mul(raw[i], kk);
    out[i] = grow ? invert_pl(v) : v;
}

// matte.rs:471-484: the threshold map of a shrink step after its blur
__device__ __forceinline__ float choke_threshold(float v, float t, double den) {
    if (isnan(v)) return nr::quiet(v);
    if (t > v) return 0.0f;
    float o = (float)((double)(v - t) / den);
    return fabs((double)o - 1.0) < 1e-4 ? 1.0f : o;
}

// matte.rs:280-310 after the blurs: the step by lo (blurred into b_lo, or the base itself when lo
// shrinks nothing), the mix with the step by hi (matte.rs:326-345) when the amount is fractional,
// the inversion back after a grow, the final clamp (matte.rs:350-359)
__global__ void k_choke_finish(const float* __restrict__ base, const float* __restrict__ b_lo,
                               const float* __restrict__ b_hi, ChokeStep st, long n, float* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float m = st.lo_blur ? choke_threshold(b_lo[i], st.t_lo, st.den_lo) : base[i];
    if (st.mix) {
        float c = st.hi_blur ? choke_threshold(b_hi[i], st.t_hi, st.den_hi) : base[i];
        float x = x86::add(x86::mul(x86::sub(c, m), st.t), m);
        if (x >= 1.0f) x = 1.0f;
        else if (0.0f > x) x = 0.0f;
        m = x;
    }
    if (st.grow) m = invert_pl(m);
    if (0.0f > m) m = 0.0f;
    else if (m >= 1.0f) m = 1.0f;
    out[i] = m;
}

// a row flip of a w x h image of `px` bytes per pixel (px a multiple of 4), into another buffer
__global__ void k_flip_rows(const void* __restrict__ src, void* __restrict__ dst, int w, int h, int px) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int words = px / 4;
    long total = (long)w * h * words;
    if (i >= total) return;
    long row_words = (long)w * words;
    long y = i / row_words, r = i - y * row_words;
    ((uint32_t*)dst)[(h - 1 - y) * row_words + r] = ((const uint32_t*)src)[i];
}

// plates.rs:296-309: the solver mask of layer k, (white - (raw - comp)) / white. A mask of ones is
// the plain solve (the binary pyramid is 1 everywhere and gates nothing), so it is always built.
__global__ void k_solver_mask(const float* __restrict__ raws, int nfg, int k, const float* __restrict__ comp, long n,
                              int fmt, float* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float white = white_of(fmt);
    float r = k == nfg ? white : raws[(long)k * n + i];
    out[i] = (white - (r - comp[i])) / white;
}

// plates.rs:128-156: every channel times the plane (units)
__global__ void k_layer_times(const void* __restrict__ src, const float* __restrict__ p, void* __restrict__ out, int fmt,
                              long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float K8 = __uint_as_float(0x3b808081u), K16 = __uint_as_float(0x37800080u);  // matte.rs:921-922
    float pv = p[i];
    for (int c = 0; c < 4; c++) {
        long j = i * 4 + c;
        if (fmt == 0) ((uint8_t*)out)[j] = (uint8_t)as_i64((float)((const uint8_t*)src)[j] * (pv * K8) + 0.5f);
        else if (fmt == 1) ((uint16_t*)out)[j] = (uint16_t)as_i64((float)((const uint16_t*)src)[j] * (pv * K16) + 0.5f);
        else ((float*)out)[j] = nr::mul(pv, ((const float*)src)[j]);
    }
}

// matte.rs:923-1030: src OVER dest with the plugin's kernels
__global__ void k_over_pl(void* __restrict__ dest, const void* __restrict__ src, int fmt, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float K8 = __uint_as_float(0x3b808081u), K16 = __uint_as_float(0x37800080u);
    if (fmt == 0) {
        uint8_t* d = (uint8_t*)dest + i * 4;
        const uint8_t* s = (const uint8_t*)src + i * 4;
        uint8_t sa = s[0];
        if (sa == 0) return;
        if (sa == 255) { for (int c = 0; c < 4; c++) d[c] = s[c]; return; }
        float saf = (float)sa, f = 1.0f - saf * K8;
        uint8_t da = d[0];
        for (int c = 1; c < 4; c++) d[c] = (uint8_t)as_i64((float)d[c] * f + (float)s[c] + 0.5f);
        d[0] = (uint8_t)as_i64((float)(255 - da) * saf * K8 + (float)da + 0.5f);
    } else if (fmt == 1) {
        uint16_t* d = (uint16_t*)dest + i * 4;
        const uint16_t* s = (const uint16_t*)src + i * 4;
        uint16_t sa = s[0];
        if (sa == 0) return;
        if (sa == 65535) { for (int c = 0; c < 4; c++) d[c] = s[c]; return; }
        float saf = (float)sa, f = 1.0f - saf * K16;
        uint16_t da = d[0];
        for (int c = 1; c < 4; c++) d[c] = (uint16_t)as_i64((float)d[c] * f + (float)s[c] + 0.5f);
        d[0] = (uint16_t)as_i64((float)(65535 - (int32_t)da) * saf * K16 + (float)da + 0.5f);
    } else {
        float* d = (float*)dest + i * 4;
        const float* s = (const float*)src + i * 4;
        float sa = s[0];
        if (sa == 0.0f) return;
        if (sa == 1.0f) { for (int c = 0; c < 4; c++) d[c] = s[c]; return; }
        float f = nr::sub(1.0f, sa);
        float da = d[0];
        for (int c = 1; c < 4; c++) d[c] = nr::add(nr::add(nr::mul(f, d[c]), s[c]), 0.0f);
        d[0] = nr::add(nr::add(nr::mul(nr::sub(1.0f, da), sa), da), 0.0f);
    }
}

// plates.rs:245-256, first half: the unpremultiply of the plate (plates.rs:160-187) and its holes,
// white - alpha through the hole rule of the mask's type (holefill.rs:124-133): u8 / u16 any non
// zero value, f32 !(3.1e-5 > m) in double (a NaN alpha is a hole)
__global__ void k_refill_pre(void* __restrict__ img, int fmt, long n, uint8_t* __restrict__ holes,
                             int* __restrict__ any_hole) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool hole = false;
    if (i < n) {
        if (fmt == 0) {
            uint8_t* p = (uint8_t*)img + i * 4;
            if (p[0] != 0) {
                float s = 255.0f / (float)p[0];  // image.rs:306-320
                for (int c = 1; c < 4; c++) {
                    float v = (float)p[c] * s;
                    if (v > 255.0f) v = 255.0f;
                    p[c] = (uint8_t)qround(v);
                }
            }
            hole = (uint8_t)(0xffu - p[0]) != 0;
        } else if (fmt == 1) {
            uint16_t* p = (uint16_t*)img + i * 4;
            if (p[0] != 0) {
                float inv = 65535.0f / (float)p[0];
                for (int c = 1; c < 4; c++) {
                    float v = (float)p[c] * inv;
                    if (65535.0f < v) v = 65535.0f;
                    p[c] = (uint16_t)qround(v);
                }
            }
            hole = (uint16_t)(0xffffu - p[0]) != 0;
        } else {
            float* p = (float*)img + i * 4;
            if (!(1e-7 > (double)p[0])) {
                float inv = 1.0f / p[0];
                for (int c = 1; c < 4; c++) p[c] = nr::mul(inv, p[c]);
            }
            float m = 1.0f - p[0];
            hole = !(__longlong_as_double(0x3f0040bfe3b03e21ll) > (double)m);
        }
        holes[i] = hole ? 1 : 0;
    }
    if (__syncthreads_or(hole) && threadIdx.x == 0) atomicOr(any_hole, 1);
}

// plates.rs:245-256, second half: the alpha replaced by the plane (units; plane != null) or by the
// frame's alpha, then the premultiply of the plugin's kernel (plates.rs:191-208)
__global__ void k_refill_post(void* __restrict__ img, int fmt, long n, const float* __restrict__ plane,
                              const void* __restrict__ frame) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float K16 = __uint_as_float(0x37800080u);
    if (fmt == 0) {
        uint8_t* p = (uint8_t*)img + i * 4;
        if (plane) {
            int64_t v = as_i64(plane[i]);
            p[0] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        } else {
            p[0] = ((const uint8_t*)frame)[i * 4];
        }
        float a = (float)p[0] * __uint_as_float(0x3b808081u);  // image.rs:276-280
        for (int c = 1; c < 4; c++) p[c] = (uint8_t)qround((float)p[c] * a);
    } else if (fmt == 1) {
        uint16_t* p = (uint16_t*)img + i * 4;
        if (plane) {
            int64_t v = as_i64(plane[i]);
            p[0] = (uint16_t)(v < 0 ? 0 : v > 65535 ? 65535 : v);
        } else {
            p[0] = ((const uint16_t*)frame)[i * 4];
        }
        float f = (float)p[0] * K16;
        for (int c = 1; c < 4; c++) p[c] = (uint16_t)qround((float)p[c] * f);
    } else {
        float* p = (float*)img + i * 4;
        p[0] = plane ? plane[i] : ((const float*)frame)[i * 4];
        float r1 = p[0] * p[1], r2 = p[0] * p[2], r3 = p[0] * p[3];  // image.rs:294-303
        if (isnan(r1) || isnan(r2) || isnan(r3) || isnan(p[0])) {
            r1 = nr::mul(p[0], p[1]);
            r2 = nr::mul(p[0], p[2]);
            r3 = nr::mul(p[0], p[3]);
        }
        p[1] = r1;
        p[2] = r2;
        p[3] = r3;
    }
}

// ---- tracking points: the user displacement of a solve (points.rs:112-240) ---------------------------

// points.rs:94-101 (cvtt_f64): truncation to i32, NaN and out of range give INT_MIN
__device__ __forceinline__ int cvtt_f64_i32(double v) {
    if (isnan(v) || v >= 2147483648.0 || v <= -2147483649.0) return INT_MIN;
    return (int)v;
}

// points.rs:112-133: the pairs splatted into level 0 (w0 x h0) of an output of W x H, in point order
// (one thread: a pixel's sums follow the order of the points)
__global__ void k_user_splat(UserPairs pairs, int w0, int h0, int W, int H, float* __restrict__ du,
                             float* __restrict__ dv, float* __restrict__ uw) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (W < 2 || H < 2 || w0 == 0 || h0 == 0) return;
    float kx = (float)(w0 - 1) / (float)(W - 1), ky = (float)(h0 - 1) / (float)(H - 1);
    for (int k = 0; k < pairs.n && k < MAX_USER_PAIRS; k++) {
        float x = pairs.p[k][0] * kx, y = pairs.p[k][1] * ky;
        int ix = cvtt_f64_i32((double)x + 0.5), iy = cvtt_f64_i32((double)y + 0.5);
        if (ix < 0 || iy < 0 || ix >= w0 || iy >= h0) continue;
        long i = (long)iy * w0 + ix;
        du[i] = (pairs.p[k][2] * kx - x) + du[i];
        dv[i] = (pairs.p[k][3] * ky - y) + dv[i];
        uw[i] = uw[i] + 1.0f;
    }
}

// points.rs:134-143: the mean of the pairs on a pixel (w becomes 1), then d = -1 d everywhere
__global__ void k_user_finest(float* __restrict__ du, float* __restrict__ dv, float* __restrict__ uw, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float u = du[i], v = dv[i], w = uw[i];
    if (0.0f < w) {
        u = u / w;
        v = v / w;
        uw[i] = 1.0f;
    }
    du[i] = -1.0f * u;
    dv[i] = -1.0f * v;
}

// points.rs:103-108 (scale_xy)
__global__ void k_user_scale(float* __restrict__ du, float* __restrict__ dv, long n, float sx, float sy) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    du[i] = sx * du[i];
    dv[i] = sy * dv[i];
}

// flow/extras.rs:181-194 (apply_user): flow = d / w where w != 0
__global__ void k_apply_user(float* __restrict__ fu, float* __restrict__ fv, const float* __restrict__ du,
                             const float* __restrict__ dv, const float* __restrict__ uw, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float k = uw[i];
    if (k != 0.0f) {
        fu[i] = du[i] / k;
        fv[i] = dv[i] / k;
    }
}

}  // namespace tw
