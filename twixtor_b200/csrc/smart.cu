// Warping code 1 (Smart Blend) and the pull-push hole fill, strict mode.
//
// k_compose_smart: the two inverse warps with their coverage (warp.rs:504-561, hold off), the
// Smart Blend composite (smartblend.rs:168-262) and the holes mask (255 - max of the coverages,
// smartblend.rs:335-345), one pixel per thread. The fill (holefill.rs) then runs on "plane stacks":
// the four channels and the weight plane of a level side by side (blockIdx.z picks the plane),
// every kernel a no-op when the mask has no hole (the fill is the identity then). Float images
// run the fill's operations with the NaN rule throughout: for numbers it is the plain arithmetic
// bit for bit, and where a NaN reaches the result it gives the bits the reference's repeat with the
// rule gives.
#include "kernels.cuh"
#include "warp.cuh"

namespace tw {

// ---- Smart Blend pixel arithmetic (smartblend.rs:155-262) ------------------------------------------

template <bool RULE> struct Ar;
template <> struct Ar<false> {
    __device__ static float add(float a, float b) { return a + b; }
    __device__ static float sub(float a, float b) { return a - b; }
    __device__ static float mul(float a, float b) { return a * b; }
    __device__ static float div(float a, float b) { return a / b; }
};
template <> struct Ar<true> {
    __device__ static float add(float a, float b) { return nr::add(a, b); }
    __device__ static float sub(float a, float b) { return nr::sub(a, b); }
    __device__ static float mul(float a, float b) { return nr::mul(a, b); }
    __device__ static float div(float a, float b) { return nr::div(a, b); }
};
template <bool RULE> __device__ __forceinline__ float lerp_r(float a, float b, float f) {
    return Ar<RULE>::add(Ar<RULE>::mul(Ar<RULE>::sub(b, a), f), a);
}

template <bool R>
__device__ __forceinline__ void over_r(const float a[4], const float b[4], float white, float o[4]) {
    if (a[0] == 0.0f) { for (int c = 0; c < 4; c++) o[c] = b[c]; return; }
    if (a[0] == white) { for (int c = 0; c < 4; c++) o[c] = a[c]; return; }
    float ia = Ar<R>::sub(1.0f, Ar<R>::div(a[0], white));
    o[0] = Ar<R>::add(Ar<R>::mul(Ar<R>::sub(white, b[0]), Ar<R>::div(a[0], white)), b[0]);
#pragma unroll
    for (int c = 1; c < 4; c++) o[c] = Ar<R>::add(Ar<R>::mul(b[c], ia), a[c]);
}

// returns true for the raw store (the "result alpha is 0" fallback)
template <bool R>
__device__ __forceinline__ bool smart_px(const float p1[4], const float p2[4], float w, float white, float v[4]) {
    float c1[4], c2[4];
    over_r<R>(p1, p2, white, c1);
    over_r<R>(p2, p1, white, c2);
    float amax = p1[0] > p2[0] ? p1[0] : p2[0];
#pragma unroll
    for (int i = 0; i < 4; i++) v[i] = lerp_r<R>(c1[i], c2[i], w);
    if (v[0] == amax) return false;
    if (v[0] == 0.0f) {
        const float* s = c1[0] > c2[0] ? c1 : c2;
        for (int i = 0; i < 4; i++) v[i] = s[i];
        return true;
    }
    float alpha = v[0];
#pragma unroll
    for (int c = 1; c < 4; c++) v[c] = Ar<R>::div(Ar<R>::mul(v[c], amax), alpha);
    v[0] = amax;
    return false;
}

template <bool R>
__device__ __forceinline__ void binary_px(const float p1[4], const float p2[4], float w, float white, float v[4]) {
    float x[4], y[4];
    if (p2[0] == white) {
        float ia = Ar<R>::sub(1.0f, Ar<R>::div(p1[0], white));
        x[0] = p2[0];
        for (int c = 1; c < 4; c++) x[c] = Ar<R>::add(Ar<R>::mul(p2[c], ia), p1[c]);
    } else if (p1[0] == white) {
        for (int c = 0; c < 4; c++) x[c] = p1[c];
    } else {
        for (int c = 0; c < 4; c++) x[c] = 0.0f;
    }
    if (p1[0] == white) {
        float ia = Ar<R>::sub(1.0f, Ar<R>::div(p2[0], white));
        y[0] = p1[0];
        for (int c = 1; c < 4; c++) y[c] = Ar<R>::add(Ar<R>::mul(p1[c], ia), p2[c]);
    } else if (p2[0] == white) {
        for (int c = 0; c < 4; c++) y[c] = p2[c];
    } else {
        for (int c = 0; c < 4; c++) y[c] = 0.0f;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) v[i] = lerp_r<R>(x[i], y[i], w);
}

template <typename P> struct SPx;
template <> struct SPx<uint8_t> {
    static constexpr float WHITE = 255.0f;
    __device__ static uint8_t plain(float x) {
        float y = x + 0.5f;
        if (0.0f > y) return 0;
        if (y > 255.0f) return 255;
        return (uint8_t)cvtt64f(y);
    }
    __device__ static uint8_t raw(float x) { return (uint8_t)cvtt64f(x); }
};
template <> struct SPx<uint16_t> {
    static constexpr float WHITE = 65535.0f;
    __device__ static uint16_t plain(float x) {
        float y = x + 0.5f;
        if (0.0f > y) return 0;
        if (y > 65535.0f) return 65535;
        return (uint16_t)cvtt64f(y);
    }
    __device__ static uint16_t raw(float x) { return (uint16_t)cvtt64f(x); }
};
template <> struct SPx<float> {
    static constexpr float WHITE = 1.0f;
    __device__ static float plain(float x) { return nr::add(x, 0.0f); }
    __device__ static float raw(float x) { return x; }
};

// One Smart Blend pixel (smartblend.rs:268-298): p1 over p2 and p2 over p1 blended at w, or the
// binary alpha variant; the raw store where the blended alpha came out 0, else the plain store.
template <typename P>
__device__ __forceinline__ void smart_blend_px(const P* ta, const P* tb, float w, bool binary, P* o) {
    float p1[4], p2[4], v[4];
    for (int k = 0; k < 4; k++) {
        p1[k] = (float)ta[k];
        p2[k] = (float)tb[k];
    }
    constexpr bool R = sizeof(P) == 4;  // NaN only reaches float images
    bool raw = false;
    if (binary) binary_px<R>(p1, p2, w, SPx<P>::WHITE, v);
    else raw = smart_px<R>(p1, p2, w, SPx<P>::WHITE, v);
    for (int k = 0; k < 4; k++) o[k] = raw ? SPx<P>::raw(v[k]) : SPx<P>::plain(v[k]);
}

// One pixel of warping code 1. mode 0: Nearest (one warp: pa), 1: Blend (pa = A, pb = B, w = frac).
template <typename P>
__device__ __forceinline__ void compose_smart_px(const WarpParams& pa, const WarpParams& pb, int mode, float w,
                                                 bool binary, void* out, uint8_t* holes, int W, int H, int* any_hole,
                                                 int* bad) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    bool hole = false;
    if (x < W && y < H) {
        P ta[4], tb[4], o[4];
        bool b = false;
        uint8_t c1 = warp_pixel<P>(pa, x, y, W, H, ta, b);
        uint8_t cov = c1;
        if (mode == 0) {
            for (int k = 0; k < 4; k++) o[k] = ta[k];
        } else {
            uint8_t c2 = warp_pixel<P>(pb, x, y, W, H, tb, b);
            cov = c1 > c2 ? c1 : c2;
            smart_blend_px<P>(ta, tb, w, binary, o);
        }
        long i = (long)y * W + x;
        P* dst = (P*)out + i * 4;
        for (int k = 0; k < 4; k++) dst[k] = o[k];
        uint8_t m = (uint8_t)(0xff - cov);
        holes[i] = m;
        hole = m != 0;  // a u8 mask value is a hole iff it is not 0 (holefill.rs:124-133)
        if (b) atomicOr(bad, 1);
    }
    if (__syncthreads_or(hole) && threadIdx.x == 0) atomicOr(any_hole, 1);
}

__global__ void k_compose_smart(WarpParams pa, WarpParams pb, int fmt, int mode, float w, bool binary,
                                void* __restrict__ out, uint8_t* __restrict__ holes, int W, int H,
                                int* __restrict__ any_hole, int* __restrict__ bad) {
    if (fmt == 0) compose_smart_px<uint8_t>(pa, pb, mode, w, binary, out, holes, W, H, any_hole, bad);
    else if (fmt == 1) compose_smart_px<uint16_t>(pa, pb, mode, w, binary, out, holes, W, H, any_hole, bad);
    else compose_smart_px<float>(pa, pb, mode, w, binary, out, holes, W, H, any_hole, bad);
}

// smartblend.rs:305-315 on whole images (the stage entry point)
__global__ void k_smart_blend(const void* __restrict__ p1, const void* __restrict__ p2, int fmt, float w, bool binary,
                              void* __restrict__ out, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == 0) smart_blend_px<uint8_t>((const uint8_t*)p1 + 4 * i, (const uint8_t*)p2 + 4 * i, w, binary, (uint8_t*)out + 4 * i);
    else if (fmt == 1)
        smart_blend_px<uint16_t>((const uint16_t*)p1 + 4 * i, (const uint16_t*)p2 + 4 * i, w, binary, (uint16_t*)out + 4 * i);
    else smart_blend_px<float>((const float*)p1 + 4 * i, (const float*)p2 + 4 * i, w, binary, (float*)out + 4 * i);
}

// holefill.rs:124-133: a pixel is a hole when !(eps > m) in double (a NaN float value is a hole);
// eps is the u8 threshold for kind 1, the u16 / f32 one for kinds 2 and 3. Writes the u8 holes
// mask (1 at a hole) and sets *any_hole.
__global__ void k_mask_holes(const void* __restrict__ mask, int kind, uint8_t* __restrict__ holes, long n,
                             int* __restrict__ any_hole) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool hole = false;
    if (i < n) {
        const double u8_eps = __longlong_as_double(0x20202020202020fcll);
        const double wide_eps = __longlong_as_double(0x3f0040bfe3b03e21ll);
        double m;
        if (kind == 1) m = (double)((const uint8_t*)mask)[i];
        else if (kind == 2) m = (double)((const uint16_t*)mask)[i];
        else m = (double)((const float*)mask)[i];
        hole = !((kind == 1 ? u8_eps : wide_eps) > m);
        holes[i] = hole ? 1 : 0;
    }
    if (__syncthreads_or(hole) && threadIdx.x == 0) atomicOr(any_hole, 1);
}

// warp.rs:76-95 then the u8 hole rule (holefill.rs:126-133): the holes of a coverage image, or of the
// per byte maximum of two (Coverage::combine_max), inverted: a hole where 255 - coverage is not 0
__global__ void k_cov_holes(const uint8_t* __restrict__ c1, const uint8_t* __restrict__ c2, uint8_t* __restrict__ holes,
                            long n, int* __restrict__ any_hole) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool hole = false;
    if (i < n) {
        uint8_t c = c1[i];
        if (c2 && c2[i] > c) c = c2[i];
        hole = (uint8_t)(0xffu - c) != 0;
        holes[i] = hole ? 1 : 0;
    }
    if (__syncthreads_or(hole) && threadIdx.x == 0) atomicOr(any_hole, 1);
}

// ---- the hole fill on plane stacks (holefill.rs) ------------------------------------------------------

// holefill.rs:300-313 + :452-491: level 0 of the value planes (the four channels, holes zeroed)
// and of the weight plane (0 at a hole, else 1).
template <typename P>
__device__ __forceinline__ void fill_load_px(const void* img, const uint8_t* holes, float* stack, long n, long i) {
    const P* px = (const P*)img + i * 4;
    bool hole = holes[i] != 0;
    for (int c = 0; c < 4; c++) stack[c * n + i] = hole ? 0.0f : (float)px[c];
    stack[4 * n + i] = hole ? 0.0f : 1.0f;
}

// holefill.rs:510-517: the two components of an interleaved flow (FILL_FLOW) as value planes
__device__ __forceinline__ void fill_load_flow(const void* img, const uint8_t* holes, float* stack, long n, long i) {
    float2 v = ((const float2*)img)[i];
    bool hole = holes[i] != 0;
    stack[i] = hole ? 0.0f : v.x;
    stack[n + i] = hole ? 0.0f : v.y;
    stack[2 * n + i] = hole ? 0.0f : 1.0f;
}

__global__ void k_fill_load(const void* __restrict__ img, int fmt, const uint8_t* __restrict__ holes,
                            float* __restrict__ stack, long n, const int* __restrict__ any_hole) {
    if (!*any_hole) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == 0) fill_load_px<uint8_t>(img, holes, stack, n, i);
    else if (fmt == 1) fill_load_px<uint16_t>(img, holes, stack, n, i);
    else if (fmt == FILL_FLOW) fill_load_flow(img, holes, stack, n, i);
    else fill_load_px<float>(img, holes, stack, n, i);
}

// flow/conv.rs border element (1 channel rule) over an arithmetic set
template <bool R, bool LEFT_FIRST, int N>
__device__ __forceinline__ float border1(const float* line, long stride, int len, int i, const float* k) {
    float centre = line[(long)i * stride];
    float num = Ar<R>::mul(k[0], centre);
    float den = k[0];
#pragma unroll
    for (int j = N - 1; j >= 1; j--) {
        float kj = k[j];
#pragma unroll
        for (int side = 0; side < 2; side++) {
            bool right = (side == 0) != LEFT_FIRST;
            int t = right ? i + j : i - j;
            bool inside = t >= 0 && t < len;
            float xv = inside ? line[(long)t * stride] : 0.0f;
            float wv = inside ? kj : 0.0f;
            den = den + wv;
            num = Ar<R>::add(num, Ar<R>::mul(xv, wv));
        }
    }
    return Ar<R>::div(num, den);
}

// One element (x, y) of one pass of the 1 channel convolution of a plane s into d (conv.rs:141-190,
// :268-301).
template <bool R, int N, bool VERT, bool ABOVE_FIRST>
__device__ __forceinline__ float stack_pass_px(const float* __restrict__ s, int w, int h, int x, int y, const Taps& t) {
    float r;
    if (!VERT) {
        const float* row = s + (long)y * w;
        if (w >= 2 * N && x >= N && x < w - N) {
            r = Ar<R>::mul(row[x], t.k[0]);
#pragma unroll
            for (int j = N - 1; j >= 1; j--) r = Ar<R>::add(r, Ar<R>::mul(Ar<R>::add(row[x + j], row[x - j]), t.k[j]));
        } else {
            r = border1<R, false, N>(row, 1, w, x, t.k);
        }
    } else {
        const float* col = s + x;
        if (h >= 2 * N && y >= N && y < h - N) {
            r = Ar<R>::mul(col[(long)y * w], t.k[0]);
#pragma unroll
            for (int j = N - 1; j >= 1; j--)
                r = Ar<R>::add(r, Ar<R>::mul(Ar<R>::add(col[(long)(y + j) * w], col[(long)(y - j) * w]), t.k[j]));
        } else {
            r = border1<R, ABOVE_FIRST, N>(col, w, h, y, t.k);
        }
    }
    return r;
}

// ---- both passes of the fill's blur in one launch ---------------------------------------------------

// One element of a pass along a line held in shared memory: element t (global index in [0, len)) of
// the line at line[(t - origin) * stride]; the interior chain or the 1 channel border rule, the
// operations of stack_pass_px / border1 in their order.
template <bool R, int N, bool LEFT_FIRST>
__device__ __forceinline__ float stack_elem(const float* line, int origin, int stride, int len, int i, const Taps& t) {
    if (len >= 2 * N && i >= N && i < len - N) {
        const float* c = line + (i - origin) * stride;
        float r = Ar<R>::mul(c[0], t.k[0]);
#pragma unroll
        for (int j = N - 1; j >= 1; j--) r = Ar<R>::add(r, Ar<R>::mul(Ar<R>::add(c[j * stride], c[-j * stride]), t.k[j]));
        return r;
    }
    float num = Ar<R>::mul(t.k[0], line[(i - origin) * stride]);
    float den = t.k[0];
#pragma unroll
    for (int j = N - 1; j >= 1; j--) {
        float kj = t.k[j];
#pragma unroll
        for (int side = 0; side < 2; side++) {
            bool right = (side == 0) != LEFT_FIRST;
            int tt = right ? i + j : i - j;
            bool inside = tt >= 0 && tt < len;
            float xv = inside ? line[(tt - origin) * stride] : 0.0f;
            float wv = inside ? kj : 0.0f;
            den = den + wv;
            num = Ar<R>::add(num, Ar<R>::mul(xv, wv));
        }
    }
    return Ar<R>::div(num, den);
}

// dst = the separable blur (horizontal, then vertical) of the stack src, out of place: a 32 x 32
// output tile per block and plane (blockIdx.z), its region with the halo of N - 1 in shared memory
// (the halo's horizontal pass computed again by the neighbouring tiles).
constexpr int SB_TX = 32, SB_TY = 32, SB_MAXN = 6;  // the tile and the widest kernel (the push's r5 Gaussian)
constexpr int SB_IN = (SB_TY + 2 * SB_MAXN - 2) * (SB_TX + 2 * SB_MAXN - 1), SB_H = (SB_TY + 2 * SB_MAXN - 2) * (SB_TX + 1);

template <bool R, int N, bool ABOVE_FIRST>
__device__ __forceinline__ void stack_blur_tile(const float* __restrict__ src, float* __restrict__ dst, int w, int h,
                                                long pstride, const Taps& t, float* s_in, float* s_h) {
    constexpr int TX = SB_TX, TY = SB_TY, HL = N - 1, RW = TX + 2 * HL, RH = TY + 2 * HL, RS = RW + 1, HS = TX + 1;
    static_assert(N <= SB_MAXN && RH * RS <= SB_IN && RH * HS <= SB_H, "the shared buffers hold the widest region");
    const float* s = src + blockIdx.z * pstride;
    const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY, gx0 = X0 - HL, gy0 = Y0 - HL;
    for (int e = threadIdx.x; e < RH * RW; e += blockDim.x) {
        const int r = e / RW, c = e - r * RW, X = gx0 + c, Y = gy0 + r;
        s_in[r * RS + c] = (X >= 0 && X < w && Y >= 0 && Y < h) ? s[(long)Y * w + X] : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < RH * TX; e += blockDim.x) {
        const int r = e / TX, c = e - r * TX, X = X0 + c, Y = gy0 + r;
        if (X < w && Y >= 0 && Y < h) s_h[r * HS + c] = stack_elem<R, N, false>(s_in + r * RS, gx0, 1, w, X, t);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < TY * TX; e += blockDim.x) {
        const int r = e / TX, c = e - r * TX, X = X0 + c, Y = Y0 + r;
        if (X < w && Y < h)
            dst[blockIdx.z * pstride + (long)Y * w + X] = stack_elem<R, N, ABOVE_FIRST>(s_h + c, gy0, HS, h, Y, t);
    }
}

__global__ void __launch_bounds__(256) k_stack_blur(const float* __restrict__ src, float* __restrict__ dst, int w, int h,
                                                    long pstride, Taps t, int n, int above_first, int rule,
                                                    const int* __restrict__ any_hole) {
    if (!*any_hole) return;
    __shared__ float s_in[SB_IN];
    __shared__ float s_h[SB_H];
#define TW_SB(Rr, Nn, Aa) stack_blur_tile<Rr, Nn, Aa>(src, dst, w, h, pstride, t, s_in, s_h)
    if (rule) {
        if (n == 3) { if (above_first) TW_SB(true, 3, true); else TW_SB(true, 3, false); }
        else { if (above_first) TW_SB(true, 6, true); else TW_SB(true, 6, false); }
    } else {
        if (n == 3) { if (above_first) TW_SB(false, 3, true); else TW_SB(false, 3, false); }
        else { if (above_first) TW_SB(false, 6, true); else TW_SB(false, 6, false); }
    }
#undef TW_SB
}

// flow/sample.rs:91-112 at element (x, y) of a dw x dh plane from the sw x sh plane s (the lerps
// over the arithmetic set)
template <bool R>
__device__ __forceinline__ float stack_resample_px(const float* __restrict__ s, int sw, int sh, int dw, int dh, int x,
                                                   int y) {
    float sx = ((float)sw - 1.0f) / (float)(dw - 1);
    float sy = ((float)sh - 1.0f) / (float)(dh - 1);
    int ix, iy;
    float fx, fy;
    cell((float)x * sx, sw, ix, fx);
    cell((float)y * sy, sh, iy, fy);
    long i = (long)iy * sw + ix;
    float top = lerp_r<R>(s[i], s[i + 1], fx);
    float bot = lerp_r<R>(s[i + sw], s[i + sw + 1], fx);
    return lerp_r<R>(top, bot, fy);
}

template <bool R>
__device__ __forceinline__ void stack_resample(const float* __restrict__ src, int sw, int sh, long sstride,
                                               float* __restrict__ dst, int dw, int dh, long dstride) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    dst[blockIdx.z * dstride + (long)y * dw + x] = stack_resample_px<R>(src + blockIdx.z * sstride, sw, sh, dw, dh, x, y);
}

__global__ void k_stack_resample(const float* __restrict__ src, int sw, int sh, long sstride, float* __restrict__ dst,
                                 int dw, int dh, long dstride, int rule, const int* __restrict__ any_hole) {
    if (!*any_hole) return;
    if (rule) stack_resample<true>(src, sw, sh, sstride, dst, dw, dh, dstride);
    else stack_resample<false>(src, sw, sh, sstride, dst, dw, dh, dstride);
}

// holefill.rs:371-377: sol = weight != 0 ? value / weight : sol, for the nc channels (4 of an
// engine image, 2 of a flow); the weights are plane nc of the level's stack
__global__ void k_fill_combine(float* __restrict__ sol, const float* __restrict__ vals, long n, int nc, int rule,
                               const int* __restrict__ any_hole) {
    if (!*any_hole) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float wt = vals[nc * n + i];
    if (wt != 0.0f) {
        for (int c = 0; c < nc; c++)
            sol[c * n + i] = rule ? Ar<true>::div(vals[c * n + i], wt) : Ar<false>::div(vals[c * n + i], wt);
    }
}

// ---- the coarse levels of the fill in one block ------------------------------------------------------

long fill_coarse_floats(const int dims[][2], int k0, int top, int np, int nc) {
    long f = 0;
    for (int k = k0; k <= top; k++) f += (long)np * dims[k][0] * dims[k][1];  // the stacks
    long n0 = (long)dims[k0][0] * dims[k0][1];
    return f + 2 * np * n0 + 2 * nc * n0;  // two pass scratches, the solution and the next one
}

// holefill.rs:260-377 over the levels k0 .. top, the same elements as the stack kernels (the pull's
// blur5 and resample, the push's combine, Gaussian r5 and resample), block barriers between them.
// The pull reads level k - 1 directly (the stack kernels blur a copy, which keeps it for the push;
// here the blur writes scratch planes and the level stays as it is).
template <bool R>
__device__ void fill_coarse_body(const FillCoarseJob& J, float* fsm) {
    const int np = J.np, nc = J.nc, k0 = J.k0, top = J.top;
    const int tid = threadIdx.x, nt = blockDim.x;
    auto n_of = [&](int k) { return J.dims[k][0] * J.dims[k][1]; };
    auto stack_at = [&](int k) {
        float* p = fsm;
        for (int j = k0; j < k; j++) p += np * n_of(j);
        return p;
    };
    const int n0 = n_of(k0);
    float* T = stack_at(top + 1);
    float* U = T + np * n0;
    float* sol = U + np * n0;
    float* nxt = sol + nc * n0;
    for (int i = tid; i < np * n0; i += nt) fsm[i] = J.s_k0[i];
    __syncthreads();
    // pull: blur5 of level k - 1 (horizontal into U, vertical into T), resampled into level k
    for (int k = k0 + 1; k <= top; k++) {
        const int pw = J.dims[k - 1][0], ph = J.dims[k - 1][1], cw = J.dims[k][0], chh = J.dims[k][1];
        const int pn = pw * ph, cn = cw * chh;
        const float* P = stack_at(k - 1);
        float* C = stack_at(k);
        for (int i = tid; i < np * pn; i += nt) {
            const int pl = i / pn, e = i - pl * pn, y = e / pw, x = e - y * pw;
            U[i] = stack_pass_px<R, 3, false, false>(P + pl * pn, pw, ph, x, y, J.b5);
        }
        __syncthreads();
        for (int i = tid; i < np * pn; i += nt) {
            const int pl = i / pn, e = i - pl * pn, y = e / pw, x = e - y * pw;
            T[i] = J.above_first ? stack_pass_px<R, 3, true, true>(U + pl * pn, pw, ph, x, y, J.b5)
                                 : stack_pass_px<R, 3, true, false>(U + pl * pn, pw, ph, x, y, J.b5);
        }
        __syncthreads();
        for (int i = tid; i < np * cn; i += nt) {
            const int pl = i / cn, e = i - pl * cn, y = e / cw, x = e - y * cw;
            C[i] = stack_resample_px<R>(T + pl * pn, pw, ph, cw, chh, x, y);
        }
        __syncthreads();
    }
    // push: the solution starts at zero on the top level
    for (int i = tid; i < nc * n_of(top); i += nt) sol[i] = 0.0f;
    __syncthreads();
    for (int lv = top; lv >= k0; lv--) {
        const int lw = J.dims[lv][0], lh = J.dims[lv][1], ln = lw * lh;
        const float* V = stack_at(lv);
        for (int i = tid; i < ln; i += nt) {  // holefill.rs:371-377
            const float wt = V[nc * ln + i];
            if (wt != 0.0f)
                for (int c = 0; c < nc; c++) sol[c * ln + i] = Ar<R>::div(V[c * ln + i], wt);
        }
        __syncthreads();
        for (int i = tid; i < nc * ln; i += nt) {
            const int pl = i / ln, e = i - pl * ln, y = e / lw, x = e - y * lw;
            U[i] = stack_pass_px<R, 6, false, false>(sol + pl * ln, lw, lh, x, y, J.g5);
        }
        __syncthreads();
        for (int i = tid; i < nc * ln; i += nt) {
            const int pl = i / ln, e = i - pl * ln, y = e / lw, x = e - y * lw;
            sol[i] = J.above_first ? stack_pass_px<R, 6, true, true>(U + pl * ln, lw, lh, x, y, J.g5)
                                   : stack_pass_px<R, 6, true, false>(U + pl * ln, lw, lh, x, y, J.g5);
        }
        __syncthreads();
        const int dw = J.dims[lv - 1][0], dh = J.dims[lv - 1][1], dn = dw * dh;
        float* dst = lv > k0 ? nxt : J.out;  // level k0 - 1 is the host's to push further
        for (int i = tid; i < nc * dn; i += nt) {
            const int pl = i / dn, e = i - pl * dn, y = e / dw, x = e - y * dw;
            dst[i] = stack_resample_px<R>(sol + pl * ln, lw, lh, dw, dh, x, y);
        }
        __syncthreads();
        float* t = sol;
        sol = nxt;
        nxt = t;
    }
}

__global__ void __launch_bounds__(FILL_COARSE_THREADS) k_fill_coarse(FillCoarseJob J) {
    if (!*J.any) return;
    extern __shared__ float fsm[];
    if (J.rule) fill_coarse_body<true>(J, fsm);
    else fill_coarse_body<false>(J, fsm);
}

// holefill.rs:379-404 (+ the f32 bit copy): the filled channels back into the engine image
template <typename P>
__device__ __forceinline__ void fill_store_px(void* img, const float* sol, long n, long i) {
    P* px = (P*)img + i * 4;
    for (int c = 0; c < 4; c++) {
        float v = sol[c * n + i];
        if (sizeof(P) == 4) ((float*)px)[c] = v;
        else px[c] = SPx<P>::plain(v);
    }
}

__global__ void k_fill_store(void* __restrict__ img, int fmt, const float* __restrict__ sol, long n,
                             const int* __restrict__ any_hole) {
    if (!*any_hole) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == 0) fill_store_px<uint8_t>(img, sol, n, i);
    else if (fmt == 1) fill_store_px<uint16_t>(img, sol, n, i);
    else if (fmt == FILL_FLOW) ((float2*)img)[i] = make_float2(sol[i], sol[n + i]);
    else fill_store_px<float>(img, sol, n, i);
}

__global__ void k_stack_zero(float* __restrict__ p, long n, const int* __restrict__ any_hole) {
    if (!*any_hole) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0.0f;
}

// a hole in an image with a side of 1 pixel: the fill refuses it (holefill.rs:273-277)
__global__ void k_hole_side1(const int* __restrict__ any_hole, int* __restrict__ flag) {
    if (*any_hole) *flag = 1;
}

}  // namespace tw
