// The forward warp (forward.rs:229-373): a displaced triangle mesh rasterised into a running mean.
//
// The reference renders the 2 (w-1)(h-1) triangles one after the other in cell order and folds
// every covered pixel into a per-pixel running mean with a saturating u8 counter. The fold is not
// associative, so a pixel's result depends on the order of its hits; but a triangle covers a pixel
// at most once, so that order is simply the ascending triangle index. The device therefore:
//
//   1. k_fw_vertices: the displaced vertex grid and the per vertex mip level (one thread a vertex);
//   2. k_fw_count: every triangle scan converted by its own thread (the reference's scan
//      converter, arithmetic for arithmetic), counting the hits of every pixel (atomicAdd);
//   3. an exclusive scan of the counts gives every pixel a segment of the hit list;
//   4. k_fw_emit: the same scan conversion again, each hit written into its pixel's
//      segment as (triangle index, colour): the textured variant samples the mip pyramid there,
//      the Gouraud variant carries the interpolated vertex colours;
//   5. k_fw_resolve: per pixel, the segment sorted by triangle index (registers for short lists,
//      a shared-memory bitonic sort per CTA for long ones, a global merge for huge ones), then the
//      running mean in that order, the conversion to the depth and the coverage byte.
//
// Results equal the sequential render bit for bit. Payload arithmetic repeats the reference's
// single precision steps with its NaN handling: the x86 results (NaN operands propagated quieted,
// the default NaN for invalid operations) where the reference runs plain arithmetic, the NaN rule
// (nanrule.rs) where it switches to the rule.
#include "kernels.cuh"
#include "twlog.h"
#include "warp.cuh"

namespace tw {

// ---- arithmetic of the payload: x86 (plain) or the NaN rule, chosen per triangle ---------------------
struct Ar {
    bool rule;
    __device__ float add(float a, float b) const { return rule ? nr::add(a, b) : x86::add(a, b); }
    __device__ float sub(float a, float b) const { return rule ? nr::sub(a, b) : x86::sub(a, b); }
    __device__ float mul(float a, float b) const { return rule ? nr::mul(a, b) : x86::mul(a, b); }
};

// ---- glibc's logf (twlog.h): the base evaluation and the table of inputs where glibc differs --------
__device__ __forceinline__ float logf_glibc(float x, const uint2* __restrict__ tab, int ntab) {
    uint32_t b = __float_as_uint(x);
    if (isnan(x)) return nr::quiet(x);
    if ((b & 0x7fffffffu) == 0) return __uint_as_float(0xff800000u);
    if (b >> 31) return __uint_as_float(0xffc00000u);
    if (b == 0x7f800000u) return x;
    int lo = 0, hi = ntab;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(&tab[mid].x) < b) lo = mid + 1;
        else hi = mid;
    }
    if (lo < ntab && __ldg(&tab[lo].x) == b) return __uint_as_float(__ldg(&tab[lo].y));
    return tw_log_base((double)x);
}

__global__ void k_logf_glibc(const float* __restrict__ x, float* __restrict__ out, long n, const uint2* __restrict__ tab,
                             int ntab) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = logf_glibc(x[i], tab, ntab);
}

// ---- early out (forward.rs:214-222): some |component| above 0.0001 compared as doubles -----------------
__global__ void k_fw_flow_nonzero(const float* __restrict__ flow, long n, int* __restrict__ flag) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    bool big = false;
    if (i < n) {
        float v = flow[i];
        float a = v < 0.0f ? -v : v;
        big = 0.0001 < (double)a;
    }
    if (__syncthreads_or(big) && threadIdx.x == 0) atomicOr(flag, 1);
}

// ---- the mesh (forward/mesh.rs) -------------------------------------------------------------------
__device__ __forceinline__ void flow_at(const float* __restrict__ f, int fw, int fh, float x, float y, float& fx,
                                        float& fy) {  // flow/sample.rs:69-86 (bilinear2)
    int ix, iy;
    float ax, ay;
    cell(x, fw, ix, ax);
    cell(y, fh, iy, ay);
    long i = ((long)iy * fw + ix) * 2;
    long r = (long)fw * 2;
    float o[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        float p00 = __ldg(f + i + c), p10 = __ldg(f + i + 2 + c), p01 = __ldg(f + i + r + c), p11 = __ldg(f + i + r + 2 + c);
        float top = (p10 - p00) * ax + p00;
        float bot = (p11 - p01) * ax + p01;
        o[c] = (bot - top) * ay + top;
    }
    fx = o[0];
    fy = o[1];
}

// mesh.rs:32-46 (positions with the tie breaking epsilon) and :63-91 (the mip level)
__global__ void k_fw_vertices(const float* __restrict__ flow, int fw, int fh, FwGrid g, float* __restrict__ vx,
                              float* __restrict__ vy, float* __restrict__ vd, float inv_ln2,
                              const uint2* __restrict__ tab, int ntab) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)g.w * g.h) return;
    int r = (int)(i / g.w), c = (int)(i - (long)r * g.w);
    float cf = (float)c, rf = (float)r;
    float fx, fy;
    flow_at(flow, fw, fh, cf * g.rx, rf * g.ry, fx, fy);
    float x = fx * g.sx + cf, y = fy * g.sy + rf;
    if (!vd) {
        if (r != 0 && c >= 1) {
            x = (float)((double)x + 0.0001);
            y = (float)((double)y + 0.0001);
        }
        vx[i] = x;
        vy[i] = y;
        return;
    }
    float xc = x, yc = y;
    if (r != 0 && c >= 1) {
        x = (float)((double)x + 0.0001);
        y = (float)((double)y + 0.0001);
    }
    vx[i] = x;
    vy[i] = y;
    int up = r - 1 < 0 ? 1 : r - 1;
    int down = g.h - 1 < r + 1 ? g.h - 2 : r + 1;
    int left = c - 1 < 0 ? 1 : c - 1;
    int right = g.w - 1 < c + 1 ? g.w - 2 : c + 1;
    auto len = [&](int ci, int ri) {
        float nx, ny;
        flow_at(flow, fw, fh, (float)ci * g.rx, (float)ri * g.ry, nx, ny);
        float dx = (nx * g.sx + (float)ci) - xc;
        float dy = (ny * g.sy + (float)ri) - yc;
        return sqrtf(dy * dy + dx * dx);
    };
    float ru = len(right, up), lu = len(left, up), ld = len(left, down), rd = len(right, down);
    float u = len(c, up), dn = len(c, down), l = len(left, r), rr = len(right, r);
    float diag = ((ru + lu) + ld) + rd;
    double t = (double)diag * 0.7071067811865476;
    t += (double)u;
    t += (double)dn;
    t += (double)l;
    t += (double)rr;
    float m = (float)((double)(float)t * 0.125);
    vd[i] = -(logf_glibc(m, tab, ntab) * inv_ln2) + 0.0f;
}

// ---- the mip pyramid of the textured variant (forward/pyramid.rs) --------------------------------------
template <typename P> struct FwS;
template <> struct FwS<uint8_t> {
    static constexpr bool F = false;
    __device__ static uint8_t store(float v) {  // pyramid.rs:130-137
        int32_t t = cvtt32(v + 0.5f);
        float f = (float)t;
        f = f > 0.0f ? f : 0.0f;
        f = f < 255.0f ? f : 255.0f;
        return (uint8_t)cvtt32(f + 0.5f);
    }
};
template <> struct FwS<uint16_t> {
    static constexpr bool F = false;
    __device__ static uint16_t store(float v) {
        int32_t t = cvtt32(v + 0.5f);
        float f = (float)t;
        f = f > 0.0f ? f : 0.0f;
        f = f < 65535.0f ? f : 65535.0f;
        return (uint16_t)cvtt32(f + 0.5f);
    }
};
template <> struct FwS<float> {
    static constexpr bool F = true;
    __device__ static float store(float v) { return v; }
};

// pyramid.rs:175-213 over one line of n samples (stride `st` pixels), 4 channels
template <typename P>
__device__ __forceinline__ void conv4(const P* __restrict__ line, long st, int i, int n, float out[4]) {
    const float k[3] = {0.375f, 0.25f, 0.0625f};
    auto get = [&](int j, float o[4]) {
        const P* p = line + (long)j * st * 4;
#pragma unroll
        for (int c = 0; c < 4; c++) o[c] = (float)p[c];
    };
    // x86 arithmetic for float samples (a NaN sample keeps its bits), plain for the integer depths
    auto add = [](float a, float b) { return FwS<P>::F ? x86::add(a, b) : a + b; };
    auto mul = [](float a, float b) { return FwS<P>::F ? x86::mul(a, b) : a * b; };
    auto dvd = [](float a, float b) { return FwS<P>::F ? x86::div(a, b) : a / b; };
    int left = n < 3 ? n : 3;
    int mid = n > 6 ? n - 6 : 0;
    float c[4], acc[4];
    get(i, c);
#pragma unroll
    for (int q = 0; q < 4; q++) acc[q] = mul(c[q], k[0]);
    if (i >= left && i < left + mid) {
#pragma unroll
        for (int j = 2; j >= 1; j--) {
            float r[4], l[4];
            get(i + j, r);
            get(i - j, l);
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] = add(acc[q], mul(add(r[q], l[q]), k[j]));
        }
#pragma unroll
        for (int q = 0; q < 4; q++) out[q] = acc[q];
        return;
    }
    const float s = -1.0f;
    float ws[4] = {k[0], k[0], k[0], k[0]};
#pragma unroll
    for (int j = 2; j >= 1; j--) {
        float r[4] = {s, s, s, s}, l[4] = {s, s, s, s};
        if (i + j < n) get(i + j, r);
        if (i >= j) get(i - j, l);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float wr = (r[q] != s ? 1.0f : 0.0f) * k[j];
            ws[q] = ws[q] + wr;
            float rt = mul(wr, r[q]);
            float wl = (l[q] != s ? 1.0f : 0.0f) * k[j];
            float lt = mul(l[q], wl);
            ws[q] = ws[q] + wl;
            acc[q] = add(add(acc[q], rt), lt);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) out[q] = dvd(acc[q], ws[q]);
}

template <typename P>
__device__ __forceinline__ void fwp_blur_px(const void* in, void* out, int w, int h, int vertical, int x, int y) {
    float v[4];
    if (!vertical) conv4<P>((const P*)in + (long)y * w * 4, 1, x, w, v);
    else conv4<P>((const P*)in + (long)x * 4, w, y, h, v);
    P* o = (P*)out + ((long)y * w + x) * 4;
#pragma unroll
    for (int q = 0; q < 4; q++) o[q] = FwS<P>::store(v[q]);
}

// pyramid.rs:215-241: one pass of the blur (rows, or columns of the stored rows)
__global__ void k_fwp_blur(const void* __restrict__ in, void* __restrict__ out, int w, int h, int vertical, int fmt) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    if (fmt == 0) fwp_blur_px<uint8_t>(in, out, w, h, vertical, x, y);
    else if (fmt == 1) fwp_blur_px<uint16_t>(in, out, w, h, vertical, x, y);
    else fwp_blur_px<float>(in, out, w, h, vertical, x, y);
}

template <typename P>
__device__ __forceinline__ void fwp_resample_px(const void* src, int sw, int sh, void* dst, int dw, int dh, int x, int y) {
    float sx = ((float)sw - 1.0f) / (float)(dw - 1);
    float sy = ((float)sh - 1.0f) / (float)(dh - 1);
    float v[4];
    bilerp4<P>((const P*)src, sw, sw - 1, sh - 1, (float)x * sx, (float)y * sy, v);
    P* o = (P*)dst + ((long)y * dw + x) * 4;
#pragma unroll
    for (int q = 0; q < 4; q++) o[q] = Pix<P>::store(v[q]);
}

// pyramid.rs:258-280: the corner aligned resample of a blurred level to the next size
__global__ void k_fwp_resample(const void* __restrict__ src, int sw, int sh, void* __restrict__ dst, int dw, int dh,
                               int fmt) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    if (fmt == 0) fwp_resample_px<uint8_t>(src, sw, sh, dst, dw, dh, x, y);
    else if (fmt == 1) fwp_resample_px<uint16_t>(src, sw, sh, dst, dw, dh, x, y);
    else fwp_resample_px<float>(src, sw, sh, dst, dw, dh, x, y);
}

// pyramid.rs:98-108: one bilinear tap at (w1 * u, h1 * v). A coordinate that leaves the image
// (the reference indexes out of its slice there) reads nothing and raises the bad flag.
template <typename P>
__device__ __forceinline__ void fw_tap(const void* img, int w, int h, float u, float v, float o[4], int* bad) {
    int w1 = w - 1, h1 = h - 1;
    float x = (float)w1 * u, y = (float)h1 * v;
    int ix = cvtt32(x), iy = cvtt32(y);
    if (ix >= w1) ix = w1 - 1;
    if (iy >= h1) iy = h1 - 1;
    if (ix < 0 || iy < 0) {
        atomicOr(bad, 1);
#pragma unroll
        for (int q = 0; q < 4; q++) o[q] = 0.0f;
        return;
    }
    bilerp4<P>((const P*)img, w, w1, h1, x, y, o);
}

// pyramid.rs:72-95 (the hit: forward.rs:134-145)
template <typename P>
__device__ __forceinline__ void fw_sample(const FwLevels& L, float u, float v, float d, float o[4], int* bad) {
    if (0.0f < d) {
        if (d < (float)(L.count - 1)) {
            int i = cvtt32(d);
            float frac = d - (float)i;
            float a[4], b[4];
            fw_tap<P>(L.p[i], L.w[i], L.h[i], u, v, a, bad);
            fw_tap<P>(L.p[i + 1], L.w[i + 1], L.h[i + 1], u, v, b, bad);
#pragma unroll
            for (int q = 0; q < 4; q++) o[q] = x86::add(x86::mul(x86::sub(b[q], a[q]), frac), a[q]);
            return;
        }
        fw_tap<P>(L.p[L.count - 1], L.w[L.count - 1], L.h[L.count - 1], u, v, o, bad);
        return;
    }
    fw_tap<P>(L.p[0], L.w[0], L.h[0], u, v, o, bad);
}

// ---- the scan converter (forward/raster.rs) ------------------------------------------------------------
struct Vt {
    float x, y, p[4];  // position and payload: (u, v, d, -) textured, (c0, c1, c2, c3) Gouraud
};
struct Edge {
    float ay, by, x, dx, p[4], dp[4];
};

// raster.rs:61-86; channels 0..2 run the arithmetic `a`, channel 3 the arithmetic `b`
__device__ __forceinline__ void edge_init(const Vt& a, const Vt& b, float y, Edge e[2], int& count, Ar aa, Ar ab) {
    if (a.y <= y && y < b.y) {
        const bool second = count != 0;
        count += 1;
        Edge s;
        float dx = b.x - a.x;
        float inv = 1.0f / (b.y - a.y);
        float t = ((y - 1.0f) - a.y) * inv;
        s.ay = a.y;
        s.by = b.y;
        s.x = dx * t + a.x;
        s.dx = dx * inv;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            Ar A = q < 3 ? aa : ab;
            float dq = A.sub(b.p[q], a.p[q]);
            s.p[q] = A.add(A.mul(dq, t), a.p[q]);
            s.dp[q] = A.mul(dq, inv);
        }
        // a constant index on both sides: the two edges stay in registers (a runtime index would
        // put them in local memory)
        if (second) e[1] = s;
        else e[0] = s;
    }
}

// one closed span from x0 to x1 with the payload lerped from l to r (raster.rs:116-153, :252-299)
template <typename Sink>
__device__ __forceinline__ void run(int x0, int x1, float lx, float wid, const float* lp, const float* rp, int yi,
                                    bool check, int w1, int h1, Ar aa, Ar ab, Sink& sink) {
    float inv = 1.0f / wid;
    float t = ((float)x0 - lx) * inv;
    float p[4], dp[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        Ar A = q < 3 ? aa : ab;
        dp[q] = A.sub(rp[q], lp[q]);
        p[q] = A.add(A.mul(dp[q], t), lp[q]);
    }
    int x = x0;
    if (x0 != x1) {
        while (x < x1) {
            if (check && (x < 0 || x > w1 || yi < 0 || yi > h1)) sink.outside();
            else sink.hit(x, yi, p);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                Ar A = q < 3 ? aa : ab;
                p[q] = A.add(p[q], A.mul(dp[q], inv));
            }
            x += 1;
        }
    }
    if (check && (x < 0 || x > w1 || yi < 0 || yi > h1)) sink.outside();
    else sink.hit(x, yi, p);
}

__device__ __forceinline__ void sort3(const Vt* v, Vt* o) {  // raster.rs:90-113
    float y0 = v[0].y, y1 = v[1].y, y2 = v[2].y;
    int a, b, c;
    if (y1 < y0) {
        if (y2 < y0) {
            if (y2 < y1) { a = 2; b = 1; c = 0; }
            else { a = 1; b = 2; c = 0; }
        } else { a = 1; b = 0; c = 2; }
    } else if (y2 < y1) {
        if (y0 < y2) { a = 0; b = 2; c = 1; }
        else { a = 2; b = 0; c = 1; }
    } else { a = 0; b = 1; c = 2; }
    // copies by constant indices (v[a] with a runtime a would put the vertices in local memory)
    auto pick = [&](int k, Vt& d) {
        d.x = k == 0 ? v[0].x : k == 1 ? v[1].x : v[2].x;
        d.y = k == 0 ? v[0].y : k == 1 ? v[1].y : v[2].y;
#pragma unroll
        for (int q = 0; q < 4; q++) d.p[q] = k == 0 ? v[0].p[q] : k == 1 ? v[1].p[q] : v[2].p[q];
    };
    pick(a, o[0]);
    pick(b, o[1]);
    pick(c, o[2]);
}

// raster.rs:171-300
template <typename Sink>
__device__ __forceinline__ void triangle(const Vt* t, int w1, int h1, Ar aa, Ar ab, Sink& sink) {
    float w1f = (float)w1, h1f = (float)h1;
    bool ok = (0.0f <= t[0].x || 0.0f <= t[1].x || 0.0f <= t[2].x) && (0.0f <= t[0].y || 0.0f <= t[1].y || 0.0f <= t[2].y) &&
              (t[0].x <= w1f || t[1].x <= w1f || t[2].x <= w1f) && (t[0].y <= h1f || t[1].y <= h1f || t[2].y <= h1f);
    if (!ok) return;
    Vt vs[3];
    sort3(t, vs);
    float y = ceilf(vs[0].y);
    float y_end = floorf(vs[2].y);
    if (y < 0.0f) y = 0.0f;
    if (h1f < y_end) y_end = h1f;
    if (y <= y_end) {
        int vi = 0, count = 0;
        Edge e[2] = {};
        for (;;) {  // at most h rows: y advances by 1 from >= 0 to <= h1
            if (vi < 3) {
                for (;;) {
                    if (y < (vi == 0 ? vs[0].y : vi == 1 ? vs[1].y : vs[2].y)) break;
                    if (count == 1) {
                        if (e[0].ay <= y && e[0].by <= y) count = 0;
                    } else if (count == 2) {
                        if (y < e[1].ay || y < e[1].by) {
                            if (!(y < e[0].ay || y < e[0].by)) {
                                e[0] = e[1];
                                count = 1;
                            }
                        } else if (e[0].ay <= y && e[0].by <= y) {
                            count = 0;
                        } else {
                            count = 1;
                        }
                    }
                    // the edges from vertex vi to the next two (vi, vi + 1), (vi, vi + 2) mod 3, with
                    // constant indices per case
                    if (vi == 0) {
                        edge_init(vs[0], vs[1], y, e, count, aa, ab);
                        edge_init(vs[0], vs[2], y, e, count, aa, ab);
                    } else if (vi == 1) {
                        edge_init(vs[1], vs[2], y, e, count, aa, ab);
                        edge_init(vs[1], vs[0], y, e, count, aa, ab);
                    } else {
                        edge_init(vs[2], vs[0], y, e, count, aa, ab);
                        edge_init(vs[2], vs[1], y, e, count, aa, ab);
                    }
                    vi += 1;
                    if (vi >= 3) break;
                }
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                e[k].x += e[k].dx;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    Ar A = q < 3 ? aa : ab;
                    e[k].p[q] = A.add(e[k].p[q], e[k].dp[q]);
                }
            }
            if (count == 2) {
                const bool sw = e[1].x < e[0].x;  // the left edge is e[1]
                const float lx = sw ? e[1].x : e[0].x, rx = sw ? e[0].x : e[1].x;
                float lp[4], rp[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    lp[q] = sw ? e[1].p[q] : e[0].p[q];
                    rp[q] = sw ? e[0].p[q] : e[1].p[q];
                }
                int x0 = max(cvtt32(ceilf(lx)), 0);
                int x1 = min(cvtt32(floorf(rx)), w1);
                float wid = rx - lx;
                if (x0 <= x1 && (double)wid > 1e-08) run(x0, x1, lx, wid, lp, rp, cvtt32(y), false, w1, h1, aa, ab, sink);
            }
            y += 1.0f;
            if (!(y <= y_end)) break;
        }
    }
    const Vt& mid = vs[1];
    const Vt& bot = vs[2];
    if (mid.y == h1f && mid.y == bot.y) {
        const bool bl = bot.x <= mid.x;  // the left vertex is bot
        const float lx = bl ? bot.x : mid.x, rx = bl ? mid.x : bot.x;
        float lp[4], rp[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            lp[q] = bl ? bot.p[q] : mid.p[q];
            rp[q] = bl ? mid.p[q] : bot.p[q];
        }
        float yy = bl ? bot.y : mid.y;
        float yt = (float)cvtt32(yy);
        if (0.0f <= yt && yt <= h1f && !((double)(yy - yt) > 0.01)) {
            int x0 = max(cvtt32(ceilf(lx)), 0);
            int x1 = min(cvtt32(floorf(rx)), w1);
            float wid = rx - lx;
            if ((double)wid > 1e-05) run(x0, x1, lx, wid, lp, rp, cvtt32(yt), true, w1, h1, aa, ab, sink);
        }
    }
}

// ---- the two raster passes ------------------------------------------------------------------------------
struct CountSink {
    uint32_t* cnt;
    int w;
    int* out_flag;
    __device__ void hit(int x, int y, const float*) { atomicAdd(&cnt[(long)y * w + x], 1u); }
    __device__ void outside() { atomicOr(out_flag, 1); }
};

template <typename P>
struct EmitSink {
    const FwRaster& R;
    uint32_t tri;
    __device__ void hit(int x, int y, const float* p) {
        long px = (long)y * R.w + x;
        uint32_t k = atomicAdd(&R.fill[px], 1u);
        if (k >= R.cnt[px]) {  // the count pass saw fewer hits: never expected, never written
            atomicOr(R.bad, 2);
            return;
        }
        uint32_t slot = R.off[px] + k;
        R.keys[slot] = tri;
        float c[4];
        if (R.pyramid) {
            if (0.0f < p[2]) fw_sample<P>(R.levels, p[0], p[1], p[2], c, R.bad);
            else fw_tap<P>(R.levels.p[0], R.levels.w[0], R.levels.h[0], p[0], p[1], c, R.bad);
        } else {
#pragma unroll
            for (int q = 0; q < 4; q++) c[q] = p[q];
        }
        R.cols[slot] = make_float4(c[0], c[1], c[2], c[3]);
    }
    __device__ void outside() { atomicOr(R.outside, 1); }
};

// The Gouraud variant's sink: the hit's interpolated colours; its pointers copied out of the kernel
// parameters (a reference to them, which the textured sink's mip level table needs, makes every
// thread copy the whole parameter block to local memory)
struct EmitSinkG {
    uint32_t* fill;
    const uint32_t* cnt;
    const uint32_t* off;
    uint32_t* keys;
    float4* cols;
    int* bad;
    int* out_flag;
    int w;
    uint32_t tri;
    __device__ void hit(int x, int y, const float* p) {
        long px = (long)y * w + x;
        uint32_t k = atomicAdd(&fill[px], 1u);
        if (k >= cnt[px]) {  // the count pass saw fewer hits: never expected, never written
            atomicOr(bad, 2);
            return;
        }
        uint32_t slot = off[px] + k;
        keys[slot] = tri;
        cols[slot] = make_float4(p[0], p[1], p[2], p[3]);
    }
    __device__ void outside() { atomicOr(out_flag, 1); }
};

template <typename P>
__device__ __forceinline__ void load_vertex(const FwRaster& R, int r, int c, Vt& v) {
    long i = (long)r * R.w + c;
    v.x = R.vx[i];
    v.y = R.vy[i];
    if (R.pyramid) {
        v.p[0] = (float)c / (float)(R.w - 1);
        v.p[1] = (float)r / (float)(R.h - 1);
        v.p[2] = R.vd ? R.vd[i] : 0.0f;
        v.p[3] = 0.0f;
    } else {
        const P* s = (const P*)R.levels.p[0] + i * 4;
#pragma unroll
        for (int q = 0; q < 4; q++) v.p[q] = (float)s[q];
    }
}

// MODE 0: the count pass; 1: the emit of the Gouraud variant; 2: the emit of the textured variant
template <typename P, int MODE>
__device__ __forceinline__ void raster_one(const FwRaster& R) {
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long cells = (long)(R.w - 1) * (R.h - 1);
    if (t >= 2 * cells) return;
    long cell = t >> 1;
    int r = (int)(cell / (R.w - 1)), c = (int)(cell - (long)r * (R.w - 1));
    Vt v[3];
    if ((t & 1) == 0) {  // T1 = (v[r][c], v[r][c+1], v[r+1][c])
        load_vertex<P>(R, r, c, v[0]);
        load_vertex<P>(R, r, c + 1, v[1]);
        load_vertex<P>(R, r + 1, c, v[2]);
    } else {  // T2 = (v[r+1][c+1], v[r][c+1], v[r+1][c])
        load_vertex<P>(R, r + 1, c + 1, v[0]);
        load_vertex<P>(R, r, c + 1, v[1]);
        load_vertex<P>(R, r + 1, c, v[2]);
    }
    // raster.rs:158-166: the rule when a payload of the triangle is NaN (per scan: the Gouraud
    // variant's two scans, colours 0..2 and colour 3, choose on their own)
    bool na = false, nb = false;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        na = na || isnan(v[k].p[0]) || isnan(v[k].p[1]) || isnan(v[k].p[2]);
        nb = nb || isnan(v[k].p[3]);
    }
    Ar aa{na}, ab{nb};
    if (MODE == 2) {
        EmitSink<P> s{R, (uint32_t)t};
        triangle(v, R.w - 1, R.h - 1, aa, ab, s);
    } else if (MODE == 1) {
        EmitSinkG s{R.fill, R.cnt, R.off, R.keys, R.cols, R.bad, R.outside, R.w, (uint32_t)t};
        triangle(v, R.w - 1, R.h - 1, aa, ab, s);
    } else {
        CountSink s{R.cnt, R.w, R.outside};
        triangle(v, R.w - 1, R.h - 1, aa, ab, s);
    }
}

__global__ void __launch_bounds__(128) k_fw_count(FwRaster R) {
    if (R.fmt == 0) raster_one<uint8_t, 0>(R);
    else if (R.fmt == 1) raster_one<uint16_t, 0>(R);
    else raster_one<float, 0>(R);
}

// the emit of the Gouraud variant (R.pyramid false)
__global__ void __launch_bounds__(128, 6) k_fw_emit(FwRaster R) {
    if (R.fmt == 0) raster_one<uint8_t, 1>(R);
    else if (R.fmt == 1) raster_one<uint16_t, 1>(R);
    else raster_one<float, 1>(R);
}

// the emit of the textured variant (R.pyramid true)
__global__ void __launch_bounds__(128, 4) k_fw_emit_tex(FwRaster R) {
    if (R.fmt == 0) raster_one<uint8_t, 2>(R);
    else if (R.fmt == 1) raster_one<uint16_t, 2>(R);
    else raster_one<float, 2>(R);
}

// ---- the exclusive scan of the per pixel counts ---------------------------------------------------------
constexpr int SCAN_T = 256, SCAN_PER = 8, SCAN_BLOCK = SCAN_T * SCAN_PER;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    total = s_warp[(blockDim.x >> 5) - 1];
    uint32_t before = wid > 0 ? s_warp[wid - 1] : 0;
    return before + x - v;
}

// per block: the exclusive scan of SCAN_BLOCK counts and the block's sum; also the largest count
__global__ void __launch_bounds__(SCAN_T) k_scan_block(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       long n, uint32_t* __restrict__ sums, uint32_t* __restrict__ maxc) {
    __shared__ uint32_t s_warp[32];
    long base = (long)blockIdx.x * SCAN_BLOCK + (long)threadIdx.x * SCAN_PER;
    uint32_t v[SCAN_PER], loc = 0, mx = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        v[k] = base + k < n ? in[base + k] : 0u;
        loc += v[k];
        mx = max(mx, v[k]);
    }
    uint32_t total;
    uint32_t pre = block_excl_scan(loc, s_warp, total);
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(maxc, mx);
}

// one block: the exclusive scan of the block sums in place; totals[0] = the sum (64 bit)
__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t* __restrict__ sums, int nb,
                                                    unsigned long long* __restrict__ total) {
    __shared__ uint32_t s_warp[32];
    unsigned long long carry = 0;
    for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
        int i = b0 + threadIdx.x;
        uint32_t v = i < nb ? sums[i] : 0u;
        uint32_t tot;
        uint32_t pre = block_excl_scan(v, s_warp, tot);
        if (i < nb) sums[i] = (uint32_t)(carry + pre);
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, long n, const uint32_t* __restrict__ sums) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / SCAN_BLOCK];
}

// ---- resolve: the running mean of every pixel in triangle order (forward.rs:103-128, :192-210) --------
__device__ __forceinline__ void fold(float a[4], uint32_t& n, const float c[4]) {
    if (n == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) a[k] = x86::add(c[k], 0.0f);
        n = 1;
    } else if (n == 255) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float plain = (a[k] * 255.0f + c[k]) * 0.00390625f + 0.0f;
            a[k] = isnan(plain) ? nr::add(nr::mul(nr::add(nr::mul(a[k], 255.0f), c[k]), 0.00390625f), 0.0f) : plain;
        }
    } else {
        float nf = (float)n;
        float r = (float)(1.0 / ((double)nf + 1.0));
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float plain = (nf * a[k] + c[k]) * r + 0.0f;
            a[k] = isnan(plain) ? nr::add(nr::mul(nr::add(nr::mul(nf, a[k]), c[k]), r), 0.0f) : plain;
        }
        n = n + 1;
    }
}

template <typename P>
__device__ __forceinline__ void store_px(void* out, uint8_t* cov, long p, const float a[4], uint32_t n) {
    P* o = (P*)out + p * 4;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (sizeof(P) == 4) ((float*)o)[k] = x86::add(a[k], 0.0f);
        else o[k] = (P)cvtt64f(a[k] + 0.5f);
    }
    if (cov) cov[p] = n != 0 ? 0xff : 0;
}

constexpr int FW_SHORT = 16;

template <typename P>
__device__ __forceinline__ void resolve_px(const FwRaster& R, long p) {
    uint32_t n = R.cnt[p];
    if (n > FW_SHORT) {
        uint32_t q = atomicAdd(R.nlong, 1u);
        R.longq[q] = (uint32_t)p;
        return;
    }
    uint32_t k[FW_SHORT];
    uint8_t ix[FW_SHORT];
    uint32_t o = R.off[p];
    for (uint32_t j = 0; j < n; j++) {  // insertion sort by triangle index
        uint32_t key = R.keys[o + j];
        int m = (int)j - 1;
        while (m >= 0 && k[m] > key) {
            k[m + 1] = k[m];
            ix[m + 1] = ix[m];
            m--;
        }
        k[m + 1] = key;
        ix[m + 1] = (uint8_t)j;
    }
    float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    uint32_t cn = 0;
    for (uint32_t j = 0; j < n; j++) {
        float4 c4 = R.cols[o + ix[j]];
        float c[4] = {c4.x, c4.y, c4.z, c4.w};
        fold(a, cn, c);
    }
    store_px<P>(R.out, R.cov, p, a, cn);
}

__global__ void k_fw_resolve(FwRaster R) {
    long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long)R.w * R.h) return;
    if (R.fmt == 0) resolve_px<uint8_t>(R, p);
    else if (R.fmt == 1) resolve_px<uint16_t>(R, p);
    else resolve_px<float>(R, p);
}

// Long lists: one CTA per pixel of the queue. Up to FW_SMEM entries: (key, index) pairs sorted by
// a bitonic sort in shared memory; longer lists: sorted runs of FW_SMEM merged pairwise in global
// scratch (R.scratch, two halves of R.total pairs). Then one thread folds in order.
constexpr int FW_SMEM = 4096;

__device__ void bitonic_smem(uint2* s, int np2) {
    for (int k = 2; k <= np2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < np2; i += blockDim.x) {
                int l = i ^ j;
                if (l > i) {
                    bool up = (i & k) == 0;
                    uint2 a = s[i], b = s[l];
                    if ((a.x > b.x) == up) {
                        s[i] = b;
                        s[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

template <typename P>
__device__ void resolve_long(const FwRaster& R, uint32_t p, uint2* s) {
    uint32_t n = R.cnt[p], o = R.off[p];
    const uint2* order;
    if (n <= (uint32_t)FW_SMEM) {
        int np2 = 1;
        while (np2 < (int)n) np2 <<= 1;
        for (int i = threadIdx.x; i < np2; i += blockDim.x)
            s[i] = i < (int)n ? make_uint2(R.keys[o + i], (uint32_t)i) : make_uint2(0xffffffffu, 0u);
        __syncthreads();
        bitonic_smem(s, np2);
        order = s;
    } else {
        // sorted runs of FW_SMEM into scratch half A, then pairwise merges between the halves
        uint2* A = R.scratch + o;
        uint2* B = R.scratch + R.total + o;
        for (uint32_t r0 = 0; r0 < n; r0 += FW_SMEM) {
            uint32_t len = min((uint32_t)FW_SMEM, n - r0);
            for (int i = threadIdx.x; i < FW_SMEM; i += blockDim.x)
                s[i] = i < (int)len ? make_uint2(R.keys[o + r0 + i], r0 + (uint32_t)i) : make_uint2(0xffffffffu, 0u);
            __syncthreads();
            bitonic_smem(s, FW_SMEM);
            for (int i = threadIdx.x; i < (int)len; i += blockDim.x) A[r0 + i] = s[i];
            __syncthreads();
        }
        uint2 *src = A, *dst = B;
        for (uint32_t run = FW_SMEM; run < n; run <<= 1) {
            // one thread per pair of runs
            uint32_t pairs = (n + 2 * run - 1) / (2 * run);
            for (uint32_t q = threadIdx.x; q < pairs; q += blockDim.x) {
                uint32_t a0 = q * 2 * run, a1 = min(a0 + run, n), b1 = min(a0 + 2 * run, n);
                uint32_t i = a0, j = a1, k = a0;
                while (i < a1 && j < b1) dst[k++] = src[i].x <= src[j].x ? src[i++] : src[j++];
                while (i < a1) dst[k++] = src[i++];
                while (j < b1) dst[k++] = src[j++];
            }
            __syncthreads();
            uint2* t = src;
            src = dst;
            dst = t;
        }
        order = src;
    }
    if (threadIdx.x == 0) {
        float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        uint32_t cn = 0;
        for (uint32_t j = 0; j < n; j++) {
            float4 c4 = R.cols[o + order[j].y];
            float c[4] = {c4.x, c4.y, c4.z, c4.w};
            fold(a, cn, c);
        }
        store_px<P>(R.out, R.cov, p, a, cn);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(512) k_fw_resolve_long(FwRaster R) {
    extern __shared__ uint2 s_pairs[];
    uint32_t nq = *R.nlong;
    for (uint32_t q = blockIdx.x; q < nq; q += gridDim.x) {
        uint32_t p = R.longq[q];
        if (R.fmt == 0) resolve_long<uint8_t>(R, p, s_pairs);
        else if (R.fmt == 1) resolve_long<uint16_t>(R, p, s_pairs);
        else resolve_long<float>(R, p, s_pairs);
    }
}

}  // namespace tw
