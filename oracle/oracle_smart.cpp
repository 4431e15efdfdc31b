// CPU oracle: Smart Blend composites and the pull-push hole fill (warping code 1). TEST
// INFRASTRUCTURE ONLY. Restates plugins/retime-engine/src/smartblend.rs and holefill.rs; every
// single precision step in the reference's order, the NaN rule repeat where the reference repeats.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "oracle_core.h"
#include "oracle_smart.h"
#include "oracle_filters.h"

namespace orc {

// The two arithmetic sets of nanrule.rs:183-231: the processor's own and the NaN rule.
struct Plain {
    static float add(float a, float b) { return a + b; }
    static float sub(float a, float b) { return a - b; }
    static float mul(float a, float b) { return a * b; }
    static float div(float a, float b) { return a / b; }
};
struct Rule {
    static float add(float a, float b) { return nr::add(a, b); }
    static float sub(float a, float b) { return nr::sub(a, b); }
    static float mul(float a, float b) { return nr::mul(a, b); }
    static float div(float a, float b) { return nr::div(a, b); }
};
template <class A> static inline float lerp_g(float a, float b, float f) { return A::add(A::mul(A::sub(b, a), f), a); }

static inline bool any_nan4(const float v[4]) {
    return std::isnan(v[0]) || std::isnan(v[1]) || std::isnan(v[2]) || std::isnan(v[3]);
}

// =============================================================================================
// Smart Blend (smartblend.rs:155-262)

template <class A>
static void over_with(const float a[4], const float b[4], float white, float o[4]) {  // smartblend.rs:168-178
    if (a[0] == 0.0f) { std::memcpy(o, b, 16); return; }
    if (a[0] == white) { std::memcpy(o, a, 16); return; }
    float ia = A::sub(1.0f, A::div(a[0], white));
    float alpha = A::add(A::mul(A::sub(white, b[0]), A::div(a[0], white)), b[0]);
    o[0] = alpha;
    for (int c = 1; c < 4; c++) o[c] = A::add(A::mul(b[c], ia), a[c]);
}

template <class A>
static bool smart_pixel_with(const float p1[4], const float p2[4], float w, float white, float v[4]) {  // :191-215
    float c1[4], c2[4];
    over_with<A>(p1, p2, white, c1);
    over_with<A>(p2, p1, white, c2);
    float amax = p1[0] > p2[0] ? p1[0] : p2[0];
    for (int i = 0; i < 4; i++) v[i] = lerp_g<A>(c1[i], c2[i], w);
    if (v[0] == amax) return false;
    if (v[0] == 0.0f) {
        std::memcpy(v, c1[0] > c2[0] ? c1 : c2, 16);
        return true;
    }
    float alpha = v[0];
    for (int c = 1; c < 4; c++) v[c] = A::div(A::mul(v[c], amax), alpha);
    v[0] = amax;
    return false;
}

static bool smart_pixel(const float p1[4], const float p2[4], float w, float white, float v[4]) {
    bool raw = smart_pixel_with<Plain>(p1, p2, w, white, v);
    if (any_nan4(v)) raw = smart_pixel_with<Rule>(p1, p2, w, white, v);
    return raw;
}

template <class A>
static bool binary_pixel_with(const float p1[4], const float p2[4], float w, float white, float v[4]) {  // :228-249
    float x[4], y[4];
    if (p2[0] == white) {
        float ia = A::sub(1.0f, A::div(p1[0], white));
        x[0] = p2[0];
        for (int c = 1; c < 4; c++) x[c] = A::add(A::mul(p2[c], ia), p1[c]);
    } else if (p1[0] == white) {
        std::memcpy(x, p1, 16);
    } else {
        for (int c = 0; c < 4; c++) x[c] = 0.0f;
    }
    if (p1[0] == white) {
        float ia = A::sub(1.0f, A::div(p2[0], white));
        y[0] = p1[0];
        for (int c = 1; c < 4; c++) y[c] = A::add(A::mul(p1[c], ia), p2[c]);
    } else if (p2[0] == white) {
        std::memcpy(y, p2, 16);
    } else {
        for (int c = 0; c < 4; c++) y[c] = 0.0f;
    }
    for (int i = 0; i < 4; i++) v[i] = lerp_g<A>(x[i], y[i], w);
    return false;
}

static bool binary_pixel(const float p1[4], const float p2[4], float w, float white, float v[4]) {
    bool raw = binary_pixel_with<Plain>(p1, p2, w, white, v);
    if (any_nan4(v)) raw = binary_pixel_with<Rule>(p1, p2, w, white, v);
    return raw;
}

// smartblend.rs:86-147: the depth stores
template <typename T> static T store_plain_int(float x, float white) {
    float y = x + 0.5f;
    if (0.0f > y) return 0;
    if (y > white) return (T)white;
    return (T)cvtt64f(y);
}

void smart_blend(Image& out, const Image& p1, const Image& p2, float w, bool binary) {  // :268-298
    out = Image(p1.w, p1.h, p1.fmt);
    long n = (long)p1.w * p1.h;
    for (long i = 0; i < n; i++) {
        float a[4], b[4], v[4];
        float white = p1.fmt == U8 ? 255.0f : p1.fmt == U16 ? 65535.0f : 1.0f;
        for (int c = 0; c < 4; c++) {
            if (p1.fmt == U8) { a[c] = (float)p1.u8[i * 4 + c]; b[c] = (float)p2.u8[i * 4 + c]; }
            else if (p1.fmt == U16) { a[c] = (float)p1.u16[i * 4 + c]; b[c] = (float)p2.u16[i * 4 + c]; }
            else { a[c] = p1.f32[i * 4 + c]; b[c] = p2.f32[i * 4 + c]; }
        }
        bool raw = binary ? binary_pixel(a, b, w, white, v) : smart_pixel(a, b, w, white, v);
        for (int c = 0; c < 4; c++) {
            if (p1.fmt == U8) out.u8[i * 4 + c] = raw ? (uint8_t)cvtt64f(v[c]) : store_plain_int<uint8_t>(v[c], 255.0f);
            else if (p1.fmt == U16) out.u16[i * 4 + c] = raw ? (uint16_t)cvtt64f(v[c]) : store_plain_int<uint16_t>(v[c], 65535.0f);
            else out.f32[i * 4 + c] = raw ? v[c] : v[c] + 0.0f;
        }
    }
}

// =============================================================================================
// Hole fill (holefill.rs)

// holefill.rs:140-171
FillGeometry fill_geometry(int w, int h) {
    long a = w, b = h;
    int count = 1;
    for (;;) {
        a /= 2;
        b /= 2;
        if (a < 2) a = 2;
        if (b < 2) b = 2;
        count += 1;
        if (!(a > 1 && b > 1 && (a != 2 || b != 2))) break;
    }
    FillGeometry g;
    int cw = w, ch = h;
    for (int k = 0; k <= count; k++) {
        g.dims.push_back({cw, ch});
        cw = std::max(cw / 2, 2);
        ch = std::max(ch / 2, 2);
    }
    g.top = count - 1;
    return g;
}

// flow/conv.rs, the 1 channel passes over an arithmetic set (conv.rs:101-190, :268-301)
template <class A, bool LEFT_FIRST>
static float border1(const float* line, long stride, int len, int i, const float* k, int n) {
    float centre = line[(long)i * stride];
    float num = A::mul(k[0], centre);
    float den = k[0];
    for (int j = n - 1; j >= 1; j--) {
        float kj = k[j];
        for (int side = 0; side < 2; side++) {
            bool right = (side == 0) != LEFT_FIRST;
            int t = right ? i + j : i - j;
            bool inside = t >= 0 && t < len;
            float xv = inside ? line[(long)t * stride] : 0.0f;
            float wv = inside ? kj : 0.0f;
            den += wv;
            num = A::add(num, A::mul(xv, wv));
        }
    }
    return A::div(num, den);
}

template <class A>
static void convolve1(float* data, int w, int h, const float* k, int n, bool above_first) {
    if ((long)w * h == 0 || n == 0) return;
    std::vector<float> tmp((size_t)w * h);
    for (int y = 0; y < h; y++) {
        const float* x = data + (long)y * w;
        float* o = tmp.data() + (long)y * w;
        int head = std::min(n, w), interior = std::max(w - 2 * n, 0);
        for (int i = 0; i < w; i++) {
            if (i >= head && i < head + interior) {
                float s = A::mul(x[i], k[0]);
                for (int j = n - 1; j >= 1; j--) s = A::add(s, A::mul(A::add(x[i + j], x[i - j]), k[j]));
                o[i] = s;
            } else {
                o[i] = border1<A, false>(x, 1, w, i, k, n);
            }
        }
    }
    int head = std::min(n, h), interior = std::max(h - 2 * n, 0);
    for (int y = 0; y < h; y++) {
        for (int xc = 0; xc < w; xc++) {
            float r;
            if (y >= head && y < head + interior) {
                r = A::mul(tmp[(long)y * w + xc], k[0]);
                for (int j = n - 1; j >= 1; j--)
                    r = A::add(r, A::mul(A::add(tmp[(long)(y + j) * w + xc], tmp[(long)(y - j) * w + xc]), k[j]));
            } else if (above_first) {
                r = border1<A, true>(tmp.data() + xc, w, h, y, k, n);
            } else {
                r = border1<A, false>(tmp.data() + xc, w, h, y, k, n);
            }
            data[(long)y * w + xc] = r;
        }
    }
}

// flow/sample.rs:91-112 over an arithmetic set
template <class A>
static std::vector<float> resample1_g(const std::vector<float>& src, int sw, int sh, int dw, int dh) {
    std::vector<float> dst((size_t)dw * dh, 0.0f);
    float sx = ((float)sw - 1.0f) / (float)(dw - 1);
    float sy = ((float)sh - 1.0f) / (float)(dh - 1);
    for (int y = 0; y < dh; y++) {
        float fyv = (float)y * sy;
        for (int x = 0; x < dw; x++) {
            float fxv = (float)x * sx;
            auto cellf = [](float v, int len, int& io, float& fo) {
                int i = cvtt32(v);
                float f = v - (float)i;
                int last = len - 1;
                if (i >= last) { i = last - 1; f = 1.0f; }
                int iu = i < 0 ? 0 : i;
                io = std::min(iu, len >= 2 ? len - 2 : 0);
                fo = f;
            };
            int ix, iy;
            float fx, fy;
            cellf(fxv, sw, ix, fx);
            cellf(fyv, sh, iy, fy);
            long i = (long)iy * sw + ix;
            float top = lerp_g<A>(src[i], src[i + 1], fx);
            float bot = lerp_g<A>(src[i + sw], src[i + sw + 1], fx);
            dst[(size_t)y * dw + x] = lerp_g<A>(top, bot, fy);
        }
    }
    return dst;
}

static const float BIN5[3] = {0.375f, 0.25f, 0.0625f};

// The wrap-around (360) passes of the fill (holefill.rs:174-236, conv.rs:518-536, sample.rs:
// 204-227) over an arithmetic set: the circular horizontal pass (tap indices modulo the width, no
// renormalisation), the column walk of the equirectangular frame (reflect at the edge row, half a
// turn across), and the period keeping resample (steps sw / dw, sh / dh, the sphere sampler)
template <class A>
static void convolve1_wrap(float* data, int w, int h, const float* k, int n) {
    if (w == 0 || h == 0 || n == 0) return;
    std::vector<float> tmp((size_t)w * h);
    for (int y = 0; y < h; y++) {
        const float* x = data + (long)y * w;
        for (int i = 0; i < w; i++) {
            float sum = A::mul(x[i], k[0]);
            for (int j = n - 1; j >= 1; j--) {
                int r = (i + j) % w;
                int l = ((i - j) % w + w) % w;
                sum = A::add(sum, A::mul(A::add(x[r], x[l]), k[j]));
            }
            tmp[(size_t)y * w + i] = sum;
        }
    }
    int half = w / 2, pad = n - 1;
    std::vector<float> g((size_t)h + 2 * pad);
    for (int x = 0; x < w; x++) {
        auto walk = [&](int start, int dir, int m_out, float* dst_rev, bool reverse) {
            int c = x, r = start, d = dir;
            for (int m = 0; m < m_out; m++) {
                r += d;
                if (r < 0) { r = 0; d = -d; c = (half + c) % w; }
                else if (r >= h) { r = h - 1; d = -d; c = (half + c) % w; }
                float v = tmp[(size_t)r * w + c];
                if (reverse) dst_rev[m_out - 1 - m] = v;
                else dst_rev[m] = v;
            }
        };
        walk(0, -1, pad, g.data(), true);
        for (int r = 0; r < h; r++) g[pad + r] = tmp[(size_t)r * w + x];
        walk(h - 1, 1, pad, g.data() + pad + h, false);
        for (int y = 0; y < h; y++) {
            int e = pad + y;
            float sum = A::mul(g[e], k[0]);
            for (int j = n - 1; j >= 1; j--) sum = A::add(sum, A::mul(A::add(g[e + j], g[e - j]), k[j]));
            data[(size_t)y * w + x] = sum;
        }
    }
}

template <class A>
static std::vector<float> resample1_wrap(const std::vector<float>& src, int sw, int sh, int dw, int dh) {
    std::vector<float> dst((size_t)dw * dh, 0.0f);
    if (dw == 0 || dh == 0) return dst;
    float sx = (float)sw / (float)dw, sy = (float)sh / (float)dh;
    int w1 = sw - 1, h1 = sh - 1;
    for (int y = 0; y < dh; y++) {
        float yf = (float)y * sy;
        for (int x = 0; x < dw; x++) {
            float xf = (float)x * sx;
            int tx = cvtt32(xf), ty = cvtt32(yf);
            int ix = std::min(std::max(tx, 0), w1), iy = std::min(std::max(ty, 0), h1);
            float fx = xf - (float)tx, fy = yf - (float)ty;
            int x1 = ix + 1 > w1 ? 0 : ix + 1;
            int xc = ix, xd = x1, yc = iy + 1;
            if (iy + 1 > h1) {
                int half = sw / 2;
                xc = (half + ix) % sw;
                xd = (half + x1) % sw;
                yc = h1;
            }
            float p00 = src[(size_t)iy * sw + ix], p10 = src[(size_t)iy * sw + x1];
            float p01 = src[(size_t)yc * sw + xc], p11 = src[(size_t)yc * sw + xd];
            float top = lerp_g<A>(p00, p10, fx);
            float bot = lerp_g<A>(p01, p11, fx);
            dst[(size_t)y * dw + x] = lerp_g<A>(top, bot, fy);
        }
    }
    return dst;
}

template <class A>
static void fill_conv(float* data, int w, int h, const float* k, int n, bool above_first, bool wrap) {
    if (wrap) convolve1_wrap<A>(data, w, h, k, n);
    else convolve1<A>(data, w, h, k, n, above_first);
}
template <class A>
static std::vector<float> fill_resample(const std::vector<float>& src, int sw, int sh, int dw, int dh, bool wrap) {
    return wrap ? resample1_wrap<A>(src, sw, sh, dw, dh) : resample1_g<A>(src, sw, sh, dw, dh);
}

template <class A>
static std::vector<float> fill_solve(const FillGeometry& geo, const std::vector<bool>& hole,
                                     const std::vector<std::vector<float>>& wts, const std::vector<float>& plane,
                                     bool above_first, const std::vector<float>& g5, bool wrap) {
    std::vector<std::vector<float>> vals;
    std::vector<float> v0 = plane;
    for (size_t i = 0; i < v0.size(); i++)
        if (hole[i]) v0[i] = 0.0f;
    vals.push_back(v0);
    for (int k = 1; k <= geo.top; k++) {  // pull (holefill.rs:315-323)
        int pw = geo.dims[k - 1].first, ph = geo.dims[k - 1].second;
        int cw = geo.dims[k].first, ch = geo.dims[k].second;
        std::vector<float> tmp = vals[k - 1];
        fill_conv<A>(tmp.data(), pw, ph, BIN5, 3, above_first, wrap);
        vals.push_back(fill_resample<A>(tmp, pw, ph, cw, ch, wrap));
    }
    int tw = geo.dims[geo.top].first, th = geo.dims[geo.top].second;
    std::vector<float> sol((size_t)tw * th, 0.0f);
    for (int level = geo.top; level >= 0; level--) {  // push (holefill.rs:324-337)
        int lw = geo.dims[level].first, lh = geo.dims[level].second;
        auto combine = [&](std::vector<float>& s, const std::vector<float>& v, const std::vector<float>& wt) {
            for (size_t i = 0; i < s.size(); i++)
                if (wt[i] != 0.0f) s[i] = A::div(v[i], wt[i]);
        };
        combine(sol, vals[level], wts[level]);
        fill_conv<A>(sol.data(), lw, lh, g5.data(), (int)g5.size(), above_first, wrap);
        if (level == 0) {
            combine(sol, vals[0], wts[0]);
        } else {
            int nw = geo.dims[level - 1].first, nh = geo.dims[level - 1].second;
            sol = fill_resample<A>(sol, lw, lh, nw, nh, wrap);
        }
    }
    return sol;
}

// holefill.rs:238-345 (Filler): the hole flags and the weight pyramid of a mask, shared by every
// channel; fill() solves one plane with the processor's arithmetic and again with the NaN rule
// when that result holds a NaN (holefill.rs:303-309).
struct PlaneFiller {
    FillGeometry geo;
    std::vector<bool> hole;
    std::vector<std::vector<float>> wts;
    std::vector<float> g5;
    bool above_first = false;
    bool wrap = false;
    void fill(std::vector<float>& plane) const {
        std::vector<float> sol = fill_solve<Plain>(geo, hole, wts, plane, above_first, g5, wrap);
        bool has_nan = false;
        for (float v : sol) has_nan = has_nan || std::isnan(v);
        if (has_nan) sol = fill_solve<Rule>(geo, hole, wts, plane, above_first, g5, wrap);
        plane.swap(sol);
    }
};

// holefill.rs:251-298 (Filler::new): 0 with *none set when the mask has no hole, 2 for a hole in an
// image with a side of 1; a pixel is a hole when !(eps > m) (holefill.rs:124-133), mask_kind 1 u8,
// 2 u16, 3 f32
static int make_filler(int w, int h, const void* mask, int mask_kind, bool above_first, PlaneFiller* f, bool* none,
                       std::string* err, bool wrap) {
    long n = (long)w * h;
    const double U8_EPS = [] { uint64_t b = 0x20202020202020fcull; double d; std::memcpy(&d, &b, 8); return d; }();
    const double WIDE_EPS = [] { uint64_t b = 0x3f0040bfe3b03e21ull; double d; std::memcpy(&d, &b, 8); return d; }();
    f->hole.assign((size_t)n, false);
    bool any = false;
    for (long i = 0; i < n; i++) {
        double m;
        if (mask_kind == 1) m = ((const uint8_t*)mask)[i];
        else if (mask_kind == 2) m = ((const uint16_t*)mask)[i];
        else m = ((const float*)mask)[i];
        double eps = mask_kind == 1 ? U8_EPS : WIDE_EPS;
        f->hole[i] = !(eps > m);
        any = any || f->hole[i];
    }
    *none = !any;
    if (!any) return 0;
    if (w < 2 || h < 2) { *err = "hole fill of an image with a side of 1"; return 2; }
    f->geo = fill_geometry(w, h);
    f->above_first = above_first;
    f->wrap = wrap;
    f->g5 = gaussian_kernel(5.0f);
    std::vector<float> w0((size_t)n);
    for (long i = 0; i < n; i++) w0[i] = f->hole[i] ? 0.0f : 1.0f;
    f->wts.push_back(w0);
    for (int k = 1; k <= f->geo.top; k++) {
        int pw = f->geo.dims[k - 1].first, ph = f->geo.dims[k - 1].second;
        int cw = f->geo.dims[k].first, ch = f->geo.dims[k].second;
        std::vector<float> tmp = f->wts[k - 1];
        fill_conv<Plain>(tmp.data(), pw, ph, BIN5, 3, above_first, wrap);
        f->wts.push_back(fill_resample<Plain>(tmp, pw, ph, cw, ch, wrap));
    }
    return 0;
}

// holefill.rs:452-491 (fill_holes_masked_with, plain passes): mask_kind 1 u8, 2 u16, 3 f32
int fill_holes(Image& img, const void* mask, int mask_kind, bool above_first, std::string* err, bool wrap) {
    int w = img.w, h = img.h;
    long n = (long)w * h;
    PlaneFiller f;
    bool none = false;
    int rc = make_filler(w, h, mask, mask_kind, above_first, &f, &none, err, wrap);
    if (rc || none) return rc;
    std::vector<float> plane((size_t)n);
    for (int c = 0; c < 4; c++) {
        plane.resize((size_t)n);
        for (long i = 0; i < n; i++)
            plane[i] = img.fmt == U8 ? (float)img.u8[i * 4 + c] : img.fmt == U16 ? (float)img.u16[i * 4 + c] : img.f32[i * 4 + c];
        f.fill(plane);
        for (long i = 0; i < n; i++) {
            if (img.fmt == U8) img.u8[i * 4 + c] = store_plain_int<uint8_t>(plane[i], 255.0f);
            else if (img.fmt == U16) img.u16[i * 4 + c] = store_plain_int<uint16_t>(plane[i], 65535.0f);
            else img.f32[i * 4 + c] = plane[i];
        }
    }
    return 0;
}

// holefill.rs:497-518 (fill_flow_holes_with, is360 off): both components of a flow filled as
// planes with the mask of the flow's size
int fill_flow_holes(FlowField& flow, const void* mask, int mask_kind, bool above_first, std::string* err, bool wrap) {
    long n = (long)flow.w * flow.h;
    PlaneFiller f;
    bool none = false;
    int rc = make_filler(flow.w, flow.h, mask, mask_kind, above_first, &f, &none, err, wrap);
    if (rc || none) return rc;
    std::vector<float> plane((size_t)n);
    for (int c = 0; c < 2; c++) {
        plane.resize((size_t)n);
        for (long i = 0; i < n; i++) plane[i] = flow.d[i * 2 + c];
        f.fill(plane);
        for (long i = 0; i < n; i++) flow.d[i * 2 + c] = plane[i];
    }
    return 0;
}

// smartblend.rs:350-393 (nearest_smart, blend_smart); smart_finish_with :335-345
int compose_smart(const ComposeSettings& cs, const Selection& sel, const Image& a, const Image& b, const FlowField* f_ab,
                  const FlowField* f_ba, bool taps_above_first, Image* out, std::string* err) {
    float wa = sel.wa;
    WarpOpts o;
    o.hold = false;
    o.is360 = sel.interp != 2 && cs.wrap_360;  // the weighted variant keeps the flag off (smartblend.rs:408)
    if (sel.interp == 0) {
        bool use_ab = nearest_uses_f_ab(wa, 1);
        const FlowField* flow = use_ab ? f_ab : f_ba;
        if (!flow) { *err = "missing flow"; return 1; }
        *out = Image(a.w, a.h, a.fmt);
        Coverage cov;
        int rc = !(0.5f > wa) ? inv_warp(*out, a, *flow, 1.0f - wa, o, &cov, err) : inv_warp(*out, b, *flow, wa, o, &cov, err);
        if (rc) return rc;
        for (auto& v : cov.d) v = 0xff - v;
        return fill_holes(*out, cov.d.data(), 1, taps_above_first, err, cs.wrap_360);
    }
    if (sel.interp == 1) {
        if (!f_ab || !f_ba) { *err = "missing flow"; return 1; }
        float frac = 1.0f - wa;
        Image ta(a.w, a.h, a.fmt), tb(b.w, b.h, b.fmt);
        Coverage c1, c2;
        int rc = inv_warp(ta, a, *f_ba, frac, o, &c1, err);
        if (rc) return rc;
        rc = inv_warp(tb, b, *f_ab, wa, o, &c2, err);
        if (rc) return rc;
        smart_blend(*out, ta, tb, frac, cs.video_360);
        for (size_t i = 0; i < c1.d.size(); i++) c1.d[i] = 0xff - std::max(c1.d[i], c2.d[i]);
        return fill_holes(*out, c1.d.data(), 1, taps_above_first, err, cs.wrap_360);
    }
    if (sel.interp == 2) {  // smartblend.rs:400-420 (weighted_blend_smart) and :427-456 (weighted_tail)
        if (!f_ab || !f_ba) { *err = "missing flow"; return 1; }
        float frac = 1.0f - wa;
        Image ta(a.w, a.h, a.fmt), tb(b.w, b.h, b.fmt);
        Coverage c1, c2;
        int rc = inv_warp(ta, a, *f_ba, frac, o, &c1, err);
        if (rc) return rc;
        rc = inv_warp(tb, b, *f_ab, wa, o, &c2, err);
        if (rc) return rc;
        return weighted_tail(*out, ta, a, tb, b, wa, &c1, &c2, taps_above_first, err);
    }
    *err = "bad interpolation mode";
    return 1;
}

int weighted_tail(Image& out, Image& ta, const Image& a, Image& tb, const Image& b, float wa, Coverage* c1,
                  const Coverage* c2, bool taps_above_first, std::string* err) {
    float frac = 1.0f - wa;
    sharpen_step(ta, a, frac, taps_above_first);
    sharpen_step(tb, b, wa, taps_above_first);
    out = Image(a.w, a.h, a.fmt);
    if (!c1) {
        blend(out, ta, tb, frac);
        return 0;
    }
    smart_blend(out, ta, tb, frac, false);  // always the plain Smart Blend kernel, the fill without wrap
    for (size_t i = 0; i < c1->d.size(); i++) c1->d[i] = 0xff - std::max(c1->d[i], c2->d[i]);
    return fill_holes(out, c1->d.data(), 1, taps_above_first, err);
}

}  // namespace orc
