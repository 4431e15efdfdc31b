// The compositor's tails on engine images. Blur Compensation (warp/blurcomp.rs): the flow directed
// motion blur with its fused post step. The Weighted Blend filters (plugins/retime-engine/src/filters.rs): the separable
// blur of the sharpening step (radius 3, four taps, the edge formula over the taps inside the
// line), the difference mask and its clean-up, and the fused unsharp lerp + masked composite. Every
// kernel takes a gate: with a non-null gate it does nothing unless *gate is set, so a whole
// sharpening can be queued on a stream and decided on the device (the Weighted Blend without flows
// of unsound float frames).
#include "blend.cuh"
#include "warp.cuh"

namespace tw {

namespace {

__device__ __forceinline__ bool gated_off(const int* gate) { return gate && *gate == 0; }

// filters.rs:113-118
__device__ __forceinline__ int32_t store_int(float v, float max) {
    int32_t t = cvtt32(v + 0.5f);
    float f = (float)t;
    f = f > 0.0f ? f : 0.0f;
    f = f < max ? f : max;
    return cvtt32(f + 0.5f);
}

template <typename P> __device__ __forceinline__ P wb_store(float v);
template <> __device__ __forceinline__ uint8_t wb_store<uint8_t>(float v) { return (uint8_t)store_int(v, 255.0f); }
template <> __device__ __forceinline__ uint16_t wb_store<uint16_t>(float v) { return (uint16_t)store_int(v, 65535.0f); }
template <> __device__ __forceinline__ float wb_store<float>(float v) { return v; }

template <typename P> __device__ __forceinline__ void load4(const P* p, float o[4]) {
#pragma unroll
    for (int l = 0; l < 4; l++) o[l] = (float)p[l];
}

// filters.rs:171-225 (conv_pixel_with) at position i of a line of n pixels whose pixel j starts at
// line + j * stride (P samples); Rule: the NaN rule arithmetic
template <bool Rule, typename P>
__device__ __forceinline__ void conv_px(int i, int n, const WbTaps& T, const P* line, long stride, bool left_first,
                                        float out[4]) {
    auto mul = [](float a, float b) { return Rule ? nr::mul(a, b) : a * b; };
    auto add = [](float a, float b) { return Rule ? nr::add(a, b) : a + b; };
    auto dv = [](float a, float b) { return Rule ? nr::div(a, b) : a / b; };
    const float S = -1.0f;
    int count = T.count;
    int left = min(n, count);
    int mid = max(n - 2 * count, 0);
    float c[4];
    load4<P>(line + (long)i * stride, c);
    float w0 = T.w[0];
    float acc[4];
#pragma unroll
    for (int l = 0; l < 4; l++) acc[l] = mul(c[l], w0);
    if (i >= left && i < left + mid) {
        for (int k = count - 1; k >= 1; k--) {
            float r[4], lf[4];
            load4<P>(line + (long)(i + k) * stride, r);
            load4<P>(line + (long)(i - k) * stride, lf);
            float wk = T.w[k];
#pragma unroll
            for (int l = 0; l < 4; l++) acc[l] = add(acc[l], mul(add(r[l], lf[l]), wk));
        }
#pragma unroll
        for (int l = 0; l < 4; l++) out[l] = acc[l];
        return;
    }
    float wsum[4] = {w0, w0, w0, w0};
    for (int k = count - 1; k >= 1; k--) {
        float r[4] = {S, S, S, S}, lf[4] = {S, S, S, S};
        if (i + k < n) load4<P>(line + (long)(i + k) * stride, r);
        if (i >= k) load4<P>(line + (long)(i - k) * stride, lf);
        float wk = T.w[k];
#pragma unroll
        for (int l = 0; l < 4; l++) {
            float rv = left_first ? lf[l] : r[l];
            float lv = left_first ? r[l] : lf[l];
            float wr = (rv != S ? 1.0f : 0.0f) * wk;
            wsum[l] = wsum[l] + wr;
            float rt = mul(wr, rv);
            float wl = (lv != S ? 1.0f : 0.0f) * wk;
            float lt = mul(lv, wl);
            wsum[l] = wsum[l] + wl;
            acc[l] = add(add(acc[l], rt), lt);
        }
    }
#pragma unroll
    for (int l = 0; l < 4; l++) out[l] = dv(acc[l], wsum[l]);
}

// filters.rs:160-169: the plain arithmetic, again with the NaN rule where a float result is NaN
template <typename P>
__device__ __forceinline__ void conv_pixel(int i, int n, const WbTaps& T, const P* line, long stride, bool left_first,
                                           float out[4]) {
    conv_px<false, P>(i, n, T, line, stride, left_first, out);
    if (sizeof(P) == 4 && (isnan(out[0]) || isnan(out[1]) || isnan(out[2]) || isnan(out[3])))
        conv_px<true, P>(i, n, T, line, stride, left_first, out);
}

template <typename P>
__device__ __forceinline__ void blur_px(const void* src, void* dst, int w, int h, const WbTaps& T, bool cols,
                                        bool above_first) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)w * h) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    const P* s = (const P*)src;
    float v[4];
    if (!cols) conv_pixel<P>(x, w, T, s + (long)y * w * 4, 4, false, v);
    else conv_pixel<P>(y, h, T, s + (long)x * 4, (long)w * 4, above_first, v);
    P* d = (P*)dst + i * 4;
#pragma unroll
    for (int l = 0; l < 4; l++) d[l] = wb_store<P>(v[l]);
}

__device__ __forceinline__ int ring_sum(const uint8_t* t, int w, int cx, int r0, int r1, int r2) {  // filters.rs:339-345
    auto at = [&](int y, int xx) { return (int)t[(long)y * w + xx]; };
    return at(r0, cx) + at(r0, cx - 1) + at(r0, cx + 1) + at(r1, cx - 1) + at(r1, cx + 1) + at(r2, cx - 1) +
           at(r2, cx) + at(r2, cx + 1);
}

}  // namespace

// filters.rs:254-280, one pass: along the rows (cols == false) or along the columns of src
__global__ void k_wb_blur(const void* __restrict__ src, void* __restrict__ dst, int fmt, int w, int h, WbTaps T, bool cols,
                          bool above_first, const int* __restrict__ gate) {
    if (gated_off(gate)) return;
    if (fmt == 0) blur_px<uint8_t>(src, dst, w, h, T, cols, above_first);
    else if (fmt == 1) blur_px<uint16_t>(src, dst, w, h, T, cols, above_first);
    else blur_px<float>(src, dst, w, h, T, cols, above_first);
}

// filters.rs:301-334: 255 where (|dR| + |dG|) + |dB| >= limit (differences in float), else 0
__global__ void k_wb_diff_mask(const void* __restrict__ a, const void* __restrict__ b, int fmt, long n, float limit,
                               uint8_t* __restrict__ mask, const int* __restrict__ gate) {
    if (gated_off(gate)) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float d[4];
#pragma unroll
    for (int c = 1; c < 4; c++) {
        float va, vb;
        if (fmt == 0) { va = (float)((const uint8_t*)a)[i * 4 + c]; vb = (float)((const uint8_t*)b)[i * 4 + c]; }
        else if (fmt == 1) { va = (float)((const uint16_t*)a)[i * 4 + c]; vb = (float)((const uint16_t*)b)[i * 4 + c]; }
        else { va = ((const float*)a)[i * 4 + c]; vb = ((const float*)b)[i * 4 + c]; }
        d[c] = fabsf(va - vb);
    }
    float sum = (d[1] + d[2]) + d[3];
    mask[i] = sum >= limit ? 0xff : 0;
}

// filters.rs:360-375 (mask_prune) from the snapshot src into dst; needs w >= 3 and h >= 5
__global__ void k_mask_prune(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int w, int h, int limit,
                             const int* __restrict__ gate) {
    if (gated_off(gate)) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)w * h) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    uint8_t v = src[i];
    if (v != 0 && x >= 1 && x <= w - 2 && y >= 2 && y <= h - 3 && ring_sum(src, w, x, y - 2, y, y + 2) < limit) v = 0;
    dst[i] = v;
}

// filters.rs:406-418 (mask_dilate_rows); needs h >= 3
__global__ void k_mask_dilate(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int w, int h,
                              const int* __restrict__ gate) {
    if (gated_off(gate)) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)w * h) return;
    int y = (int)(i / w);
    uint8_t v = src[i];
    if (y >= 1 && y <= h - 2 && (src[i - w] == 255 || src[i + w] == 255)) v = 255;
    dst[i] = v;
}

// filters.rs:387-400 (mask_fill) followed by :425-496 (mask_replicate_border), for w >= 3 and
// h >= 3: there the border copy is the fill's result at the coordinate clamped to the inner
// rectangle 1..w-2 x 1..h-2
__global__ void k_mask_fill_border(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int w, int h, int limit,
                                   int value, const int* __restrict__ gate) {
    if (gated_off(gate)) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)w * h) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    int cx = min(max(x, 1), w - 2), cy = min(max(y, 1), h - 2);
    uint8_t v = src[(long)cy * w + cx];
    if (v == 0 && limit < ring_sum(src, w, cx, cy - 1, cy, cy + 1)) v = (uint8_t)value;
    dst[i] = v;
}

// filters.rs:507-520 for frames with a side below 3, by one thread: the dilate (h >= 3) and four
// replicate border passes (the prune and the fills need both sides >= 3), with the reference's
// float rectangle tests; scratch holds w * h bytes
__global__ void k_mask_clean_small(uint8_t* __restrict__ m, uint8_t* __restrict__ scratch, int w, int h,
                                   const int* __restrict__ gate) {
    if (gated_off(gate) || threadIdx.x != 0 || blockIdx.x != 0) return;
    long n = (long)w * h;
    if (h >= 3) {
        for (long i = 0; i < n; i++) scratch[i] = m[i];
        for (int y = 1; y < h - 1; y++)
            for (int x = 0; x < w; x++)
                if (scratch[(long)(y - 1) * w + x] == 255 || scratch[(long)(y + 1) * w + x] == 255) m[(long)y * w + x] = 255;
    }
    float p2 = 1.0f, p3 = 1.0f, p4 = (float)(w - 2), p5 = (float)(h - 2);
    long iv14 = (long)(int)p5;
    float fy0 = p3, fy1 = p5;
    if (p5 < p3) { fy0 = p5; fy1 = p3; }
    float fx0 = p2, fx1 = p4;
    if (p4 < p2) { fx0 = p4; fx1 = p2; }
    auto idx = [&](long x, long y) -> long { return (x >= 0 && x < w && y >= 0 && y < h) ? y * w + x : -1; };
    auto outside = [&](long x, long y) {
        float xf = (float)x, yf = (float)y;
        return yf < fy0 || fy1 < yf || fx1 < xf || xf < fx0;
    };
    for (int pass = 0; pass < 4; pass++) {
        for (long y = 0; (float)y < fy0; y++)
            for (long x = 0; x < w; x++)
                if (outside(x, y)) {
                    long d = idx(x, y), s = idx(x, (long)(int)p3);
                    if (d >= 0 && s >= 0) m[d] = m[s];
                }
        for (long y = (long)(int)fy1; y < h; y++)
            for (long x = 0; x < w; x++)
                if (outside(x, y)) {
                    long d = idx(x, y), s = idx(x, iv14);
                    if (d >= 0 && s >= 0) m[d] = m[s];
                }
        for (long y = 0; y < h; y++) {
            for (long x = 0; (float)x < fx0; x++) {
                long d = idx(x, y), s = idx((long)(int)p2, y);
                if (d >= 0 && s >= 0) m[d] = m[s];
            }
            long first = (long)(int)fx1, c4 = (long)(int)p4;
            for (long j = 0; first + j < w; j++) {
                long d = idx(c4 + j, y), s = idx(c4, y);
                if (d >= 0 && s >= 0) m[d] = m[s];
            }
        }
    }
}

// filters.rs:649-657, steps 3 to 5 on one pixel: sharp = lerp(blurred, frame, c) (with lerp's
// w == 1 / w == 0 early outs), then the composite of sharp into frame with the inverted mask
// (filters.rs:543-612: 255 - mask is the weight of the frame)
template <typename P>
__device__ __forceinline__ void finish_px(P* frame, const P* blurred, uint8_t mask, float c) {
    P f[4], s[4];
#pragma unroll
    for (int k = 0; k < 4; k++) { f[k] = blurred[k]; s[k] = frame[k]; }
    if (c == 0.0f) {
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = s[k];
    } else if (c != 1.0f) {
        lerp_px<P>(f, s, c);
    }
    uint8_t m = (uint8_t)(255 - mask);
    if (m == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) frame[k] = f[k];
        return;
    }
    float fl = (float)m / 255.0f;
    float g = (float)(1.0 - (double)fl);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (sizeof(P) == 4) {
            float sv = (float)f[k], dvv = (float)s[k];
            float plain = (g * sv + fl * dvv) + 0.0f;
            frame[k] = (P)(isnan(plain) ? nr::add(nr::add(nr::mul(g, sv), nr::mul(fl, dvv)), 0.0f) : plain);
        } else {
            frame[k] = (P)cvtt64f(((float)f[k] * g + (float)s[k] * fl) + 0.5f);
        }
    }
}

__global__ void k_wb_finish(void* __restrict__ frame, const void* __restrict__ blurred, const uint8_t* __restrict__ mask,
                            int fmt, long n, float c, const int* __restrict__ gate) {
    if (gated_off(gate)) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == 0) finish_px<uint8_t>((uint8_t*)frame + i * 4, (const uint8_t*)blurred + i * 4, mask[i], c);
    else if (fmt == 1) finish_px<uint16_t>((uint16_t*)frame + i * 4, (const uint16_t*)blurred + i * 4, mask[i], c);
    else finish_px<float>((float*)frame + i * 4, (const float*)blurred + i * 4, mask[i], c);
}

// a copy of n 16-byte units (one float pixel each) when the gate is set, bits unchanged
__global__ void k_copy_gated(const uint4* __restrict__ src, uint4* __restrict__ dst, long n, const int* __restrict__ gate) {
    if (gated_off(gate)) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

// blend.rs:298-300 (sound_float): sets *flag when some sample is NaN or of magnitude above 1e30
__global__ void k_f32_unsound(const float* __restrict__ a, long n, int* __restrict__ flag) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = i < n && !(fabsf(a[i]) <= 1.0e30f);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// blend.rs:276-296 (weighted_blend_noflow) of float frames, one pixel: with *unsound the blend of
// the sharpened copies a1 / b1 (weighted_blend_noflow_reference), else of a + 0.0 and b + 0.0
// (mode: blend's branch, as k_compose_blend takes it), into the engine image out
__global__ void k_wb_noflow_f32(const float* __restrict__ a, const float* __restrict__ b, const float* __restrict__ a1,
                                const float* __restrict__ b1, const int* __restrict__ unsound, float w, float wl, int mode,
                                float* __restrict__ out, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool ref = *unsound != 0;
    float pa[4], pb[4], o[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        pa[k] = ref ? a1[i * 4 + k] : a[i * 4 + k] + 0.0f;
        pb[k] = ref ? b1[i * 4 + k] : b[i * 4 + k] + 0.0f;
    }
    blend_px<float>(pa, pb, w, wl, mode, o);
#pragma unroll
    for (int k = 0; k < 4; k++) out[i * 4 + k] = o[k];
}

// ---- Blur Compensation (warp/blurcomp.rs) ---------------------------------------------------------

namespace {

constexpr int TAP_LIMIT = 1 << 16;

template <typename P> __device__ __forceinline__ P store_blur(float v);
template <> __device__ __forceinline__ uint8_t store_blur<uint8_t>(float v) {  // warp.rs:272-274
    float f = fmaxf((float)cvtt32(v + 0.5f), 0.0f);
    return (uint8_t)fminf(f, 255.0f);
}
template <> __device__ __forceinline__ uint16_t store_blur<uint16_t>(float v) {
    float f = fmaxf((float)cvtt32(v + 0.5f), 0.0f);
    return (uint16_t)fminf(f, 65535.0f);
}
template <> __device__ __forceinline__ float store_blur<float>(float v) { return v; }

// the sum of the taps: x86 arithmetic for float samples (a NaN keeps the payload of the first NaN
// operand), exact integers for the others
template <typename P> __device__ __forceinline__ float acc_add(float a, float b) {
    return sizeof(P) == 4 ? x86::add(a, b) : a + b;
}
template <typename P> __device__ __forceinline__ float acc_mul(float a, float b) {
    return sizeof(P) == 4 ? x86::mul(a, b) : a * b;
}

template <typename P>
__device__ __forceinline__ void motion_blur_px(const MotionBlur& B, long i, int x, int y) {
    const P* src = (const P*)B.src;
    float xf = (float)x, yf = (float)y;
    float du, dv;
    flow_bilerp(B.flow, xf * B.rx, yf * B.ry, du, dv);
    float vx = du * B.kx, vy = dv * B.ky;
    float d2 = vy * vy + vx * vx;
    const float TINY = __uint_as_float(0x358637bdu);
    P o[4];
    if (B.bilinear && TINY > d2) {  // blurcomp.rs:373-378: the source pixel
#pragma unroll
        for (int c = 0; c < 4; c++) o[c] = src[i * 4 + c];
    } else {
        float dist = sqrtf(d2);
        float cx = B.shifted ? vx * B.k + xf : xf, cy = B.shifted ? vy * B.k + yf : yf;
        if (!B.bilinear) { cx = cx + 0.5f; cy = cy + 0.5f; }
        int n = cvtt32(dist + 1.0f);
        float sx, sy;
        if (n < 2) { n = 2; sx = vx; sy = vy; }
        else { float dd = (float)(n - 1); sx = vx / dd; sy = vy / dd; }
        if (n > TAP_LIMIT) {
            atomicOr(B.bad, 2);
#pragma unroll
            for (int c = 0; c < 4; c++) o[c] = (P)0;
        } else {
            float sum[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            int cnt = 0;
            float wf = (float)B.w, hf = (float)B.h;
            int w1 = B.w - 1, h1 = B.h - 1;
            for (int pass = 0; pass < 2; pass++) {  // n forward taps from the centre, n - 1 backward
                float qx = pass == 0 ? cx : cx - sx, qy = pass == 0 ? cy : cy - sy;
                float stx = pass == 0 ? sx : -sx, sty = pass == 0 ? sy : -sy;
                int count = pass == 0 ? n : n - 1;
                for (int j = 0; j < count; j++) {
                    if (B.bilinear) {  // blurcomp.rs:398-455
                        if (isnan(qx) || isnan(qy)) {
                            atomicOr(B.bad, 2);
                        } else if (0.0f <= qx && qx < wf && 0.0f <= qy && qy < hf) {
                            cnt++;
                            float t[4];
                            bilerp4<P>(src, B.w, w1, h1, qx, qy, t);
#pragma unroll
                            for (int c = 0; c < 4; c++) sum[c] = acc_add<P>(sum[c], t[c]);
                        }
                    } else {  // blurcomp.rs:459-559: a backward tap always counts
                        int ix = cvtt32(qx), iy = cvtt32(qy);
                        bool in = ix >= 0 && ix < B.w && iy >= 0 && iy < B.h;
                        if (in) {
                            const P* s = src + ((long)iy * B.w + ix) * 4;
#pragma unroll
                            for (int c = 0; c < 4; c++) sum[c] = acc_add<P>(sum[c], Pix<P>::f(s[c]));
                        }
                        if (in || pass == 1) cnt++;
                    }
                    qx += stx;
                    qy += sty;
                }
            }
            float inv = 1.0f / (float)cnt;
#pragma unroll
            for (int c = 0; c < 4; c++) o[c] = store_blur<P>(acc_mul<P>(inv, sum[c]));
        }
    }
    if (B.post == 1) {  // blurcomp.rs:134-149: colour cleared where alpha is exactly zero
        if (Pix<P>::f(o[0]) == 0.0f) o[1] = o[2] = o[3] = (P)0;
    } else if (B.post == 2 && B.lerp_w != 1.0f) {  // lerp(blurred, image, amount), blend.rs:144-179
        P s[4];
#pragma unroll
        for (int c = 0; c < 4; c++) s[c] = src[i * 4 + c];
        if (B.lerp_w == 0.0f) {
#pragma unroll
            for (int c = 0; c < 4; c++) o[c] = s[c];
        } else {
            lerp_px<P>(o, s, B.lerp_w);
        }
    }
    P* d = (P*)B.dst + i * 4;
#pragma unroll
    for (int c = 0; c < 4; c++) d[c] = o[c];
}

}  // namespace

// warp/blurcomp.rs:176-559 (motion_blur, is360 off) of B.src into B.dst with the post step of
// compensate (blurcomp.rs:105-130): 1 the clear of a positive amount, 2 the lerp of a negative one
__global__ void k_motion_blur(MotionBlur B) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)B.w * B.h) return;
    int y = (int)(i / B.w), x = (int)(i - (long)y * B.w);
    if (B.fmt == 0) motion_blur_px<uint8_t>(B, i, x, y);
    else if (B.fmt == 1) motion_blur_px<uint16_t>(B, i, x, y);
    else motion_blur_px<float>(B, i, x, y);
}

}  // namespace tw
