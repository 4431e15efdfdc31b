// CPU oracle of the forward warp. TEST INFRASTRUCTURE ONLY (see oracle_core.h).
//
// Restates plugins/retime-engine/src/forward.rs (the mesh render and the running mean),
// forward/mesh.rs (vertex positions, mip levels), forward/raster.rs (the scan converter) and
// forward/pyramid.rs (the mip pyramid and its sampler). The render is sequential in cell order
// like the reference's, so the running mean of every pixel folds its hits in the same order.
#include "oracle_forward.h"
#include "oracle_smart.h"

#include <algorithm>
#include <cmath>

#ifdef _OPENMP
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

namespace orc {

// ---- arithmetic sets of the payload (nanrule.rs: Plain is the x86 arithmetic, Rule the NaN rule)
struct APlain {
    static float add(float a, float b) { return a + b; }
    static float sub(float a, float b) { return a - b; }
    static float mul(float a, float b) { return a * b; }
};
struct ARule {
    static float add(float a, float b) { return nr::add(a, b); }
    static float sub(float a, float b) { return nr::sub(a, b); }
    static float mul(float a, float b) { return nr::mul(a, b); }
};

// ---- the mip pyramid (forward/pyramid.rs) -------------------------------------------------------

int fw_level_count(int w, int h) {  // pyramid.rs:20-36
    int n = 1;
    int a = std::max(w, 2), b = std::max(h, 2);
    for (;;) {
        a /= 2;
        if (a < 2) break;
        b /= 2;
        if (b < 2) break;
        n++;
    }
    return n;
}

static const float BLUR5_TAPS[3] = {0.375f, 0.25f, 0.0625f};  // pyramid.rs:116

static int32_t store_int(float v, float max) {  // pyramid.rs:130-137
    int32_t t = cvtt32(v + 0.5f);
    float f = (float)t;
    f = f > 0.0f ? f : 0.0f;
    f = f < max ? f : max;
    return cvtt32(f + 0.5f);
}

static float load_s(const Image& img, size_t i) {
    return img.fmt == U8 ? (float)img.u8[i] : img.fmt == U16 ? (float)img.u16[i] : img.f32[i];
}
static void store_s(Image& img, size_t i, float v) {  // pyramid.rs:139-165 (Sample::store)
    if (img.fmt == U8) img.u8[i] = (uint8_t)store_int(v, 255.0f);
    else if (img.fmt == U16) img.u16[i] = (uint16_t)store_int(v, 65535.0f);
    else img.f32[i] = v;
}

// pyramid.rs:175-213: one output pixel of the 1D filter; `get(j)` loads element j of the line.
template <typename Get>
static void conv_pixel(int i, int n, const Get& get, float out[4]) {
    const int count = 3;
    int left = std::min(n, count);
    int mid = n > 2 * count ? n - 2 * count : 0;
    float c[4];
    get(i, c);
    float w0 = BLUR5_TAPS[0];
    float acc[4];
    for (int k = 0; k < 4; k++) acc[k] = c[k] * w0;
    if (i >= left && i < left + mid) {
        for (int k = count - 1; k >= 1; k--) {
            float r[4], l[4];
            get(i + k, r);
            get(i - k, l);
            float wk = BLUR5_TAPS[k];
            for (int lane = 0; lane < 4; lane++) acc[lane] = acc[lane] + (r[lane] + l[lane]) * wk;
        }
        for (int k = 0; k < 4; k++) out[k] = acc[k];
        return;
    }
    const float s = -1.0f;  // the sentinel of a tap outside the line
    float wsum[4] = {w0, w0, w0, w0};
    for (int k = count - 1; k >= 1; k--) {
        float r[4] = {s, s, s, s}, l[4] = {s, s, s, s};
        if (i + k < n) get(i + k, r);
        if (i >= k) get(i - k, l);
        float wk = BLUR5_TAPS[k];
        for (int lane = 0; lane < 4; lane++) {
            float wr = (r[lane] != s ? 1.0f : 0.0f) * wk;
            wsum[lane] = wsum[lane] + wr;
            float rt = wr * r[lane];
            float wl = (l[lane] != s ? 1.0f : 0.0f) * wk;
            float lt = l[lane] * wl;
            wsum[lane] = wsum[lane] + wl;
            acc[lane] = (acc[lane] + rt) + lt;
        }
    }
    for (int lane = 0; lane < 4; lane++) out[lane] = acc[lane] / wsum[lane];
}

static void fw_blur5(Image& img) {  // pyramid.rs:215-241: rows, stored, then columns of the stored rows
    int w = img.w, h = img.h;
    OMP_FOR
    for (int y = 0; y < h; y++) {
        std::vector<float> line((size_t)w * 4);
        for (int x = 0; x < w * 4; x++) line[x] = load_s(img, ((size_t)y * w) * 4 + x);
        for (int x = 0; x < w; x++) {
            float v[4];
            conv_pixel(x, w, [&](int j, float o[4]) { for (int k = 0; k < 4; k++) o[k] = line[(size_t)j * 4 + k]; }, v);
            for (int k = 0; k < 4; k++) store_s(img, ((size_t)y * w + x) * 4 + k, v[k]);
        }
    }
    Image snap = img;
    OMP_FOR
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            float v[4];
            conv_pixel(y, h, [&](int j, float o[4]) { for (int k = 0; k < 4; k++) o[k] = load_s(snap, ((size_t)j * w + x) * 4 + k); }, v);
            for (int k = 0; k < 4; k++) store_s(img, ((size_t)y * w + x) * 4 + k, v[k]);
        }
    }
}

static void fw_resample(Image& dst, const Image& src) {  // pyramid.rs:258-280
    float sx = ((float)src.w - 1.0f) / (float)(dst.w - 1);
    float sy = ((float)src.h - 1.0f) / (float)(dst.h - 1);
    OMP_FOR
    for (int y = 0; y < dst.h; y++) {
        float fy = (float)y * sy;
        for (int x = 0; x < dst.w; x++) {
            float v[4];
            bilerp4_image(src, (float)x * sx, fy, v);
            size_t i = ((size_t)y * dst.w + x) * 4;
            for (int k = 0; k < 4; k++) {
                if (dst.fmt == U8) dst.u8[i + k] = sat_u8(v[k]);
                else if (dst.fmt == U16) dst.u16[i + k] = sat_u16(v[k]);
                else dst.f32[i + k] = v[k];
            }
        }
    }
}

struct FwPyramid {  // pyramid.rs:39-70
    std::vector<Image> levels;  // levels 1..count-1
    int count = 1;
    void build(const Image& src) {
        count = fw_level_count(src.w, src.h);
        int cw = std::max(src.w, 2), ch = std::max(src.h, 2);
        for (int i = 1; i < count; i++) {
            Image tmp = i == 1 ? src : levels[i - 2];
            fw_blur5(tmp);
            cw = std::max(cw / 2, 2);
            ch = std::max(ch / 2, 2);
            Image lvl(cw, ch, src.fmt);
            fw_resample(lvl, tmp);
            levels.push_back(std::move(lvl));
        }
    }
};

// A texture coordinate whose cell leaves the level: the reference indexes outside its slice there
// (a panic); here it is recorded and reads zeros, and the warp reports an error.
static bool g_tap_bad = false;

static void tap(const Image& img, float u, float v, float out[4]) {  // pyramid.rs:98-108
    int w1 = img.w - 1, h1 = img.h - 1;
    float x = (float)w1 * u, y = (float)h1 * v;
    int ix = cvtt32(x), iy = cvtt32(y);
    if (ix >= w1) ix = w1 - 1;
    if (iy >= h1) iy = h1 - 1;
    if (ix < 0 || iy < 0) {
        g_tap_bad = true;
        for (int k = 0; k < 4; k++) out[k] = 0.0f;
        return;
    }
    bilerp4_image(img, x, y, out);
}

static void sample(const FwPyramid& p, const Image& src, float u, float v, float d, float out[4]) {  // :72-95
    auto level = [&](int i) -> const Image& { return i == 0 ? src : p.levels[i - 1]; };
    if (0.0f < d) {
        if (d < (float)(p.count - 1)) {
            int i = cvtt32(d);
            float frac = d - (float)i;
            float a[4], b[4];
            tap(level(i), u, v, a);
            tap(level(i + 1), u, v, b);
            for (int k = 0; k < 4; k++) out[k] = (b[k] - a[k]) * frac + a[k];
            return;
        }
        tap(level(p.count - 1), u, v, out);
        return;
    }
    tap(src, u, v, out);
}

// ---- the mesh (forward/mesh.rs) ------------------------------------------------------------------

struct Grid {
    int w, h;
    float rx, ry, sx, sy;
    Grid(int w_, int h_, const FlowField& f, float amount) : w(w_), h(h_) {
        rx = (float)(f.w - 1) / (float)(w - 1);
        ry = (float)(f.h - 1) / (float)(h - 1);
        sx = amount / rx;
        sy = amount / ry;
    }
};

void fw_positions(int w, int h, const FlowField& flow, float amount, std::vector<float>* xy) {  // mesh.rs:32-46
    Grid g(w, h, flow, amount);
    xy->assign((size_t)w * h * 2, 0.0f);
    OMP_FOR
    for (int r = 0; r < h; r++) {
        float fy_pos = (float)r * g.ry;
        float rf = (float)r;
        for (int c = 0; c < w; c++) {
            float cf = (float)c;
            float f[2];
            bilinear2(flow.d.data(), flow.w, flow.h, cf * g.rx, fy_pos, f);
            float x = f[0] * g.sx + cf, y = f[1] * g.sy + rf;
            if (r != 0 && c >= 1) {
                x = (float)((double)x + 0.0001);
                y = (float)((double)y + 0.0001);
            }
            (*xy)[((size_t)r * w + c) * 2] = x;
            (*xy)[((size_t)r * w + c) * 2 + 1] = y;
        }
    }
}

float fw_mip_level(int w, int h, const FlowField& flow, float amount, int c, int r) {  // mesh.rs:63-91
    Grid g(w, h, flow, amount);
    int up = r - 1 < 0 ? 1 : r - 1;
    int down = h - 1 < r + 1 ? h - 2 : r + 1;
    int left = c - 1 < 0 ? 1 : c - 1;
    int right = w - 1 < c + 1 ? w - 2 : c + 1;
    float f[2];
    bilinear2(flow.d.data(), flow.w, flow.h, (float)c * g.rx, (float)r * g.ry, f);
    float xc = f[0] * g.sx + (float)c;
    float yc = f[1] * g.sy + (float)r;
    auto len = [&](int ci, int ri) {
        float n[2];
        bilinear2(flow.d.data(), flow.w, flow.h, (float)ci * g.rx, (float)ri * g.ry, n);
        float dx = (n[0] * g.sx + (float)ci) - xc;
        float dy = (n[1] * g.sy + (float)ri) - yc;
        return std::sqrt(dy * dy + dx * dx);
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
    float inv_ln2 = 1.0f / logf(2.0f);
    return -(logf(m) * inv_ln2) + 0.0f;
}

// ---- the scan converter (forward/raster.rs) ------------------------------------------------------

struct Edge {
    float ay = 0, by = 0, x = 0, u = 0, v = 0, d = 0, dx = 0, du = 0, dv = 0, dd = 0;
};

template <typename A>
static void edge_init(const FwVtx& a, const FwVtx& b, float y, Edge e[2], int* count) {  // raster.rs:61-86
    if (a.y <= y && y < b.y) {
        int slot = *count != 0 ? 1 : 0;
        *count += 1;
        float dx = b.x - a.x;
        float du = A::sub(b.u, a.u), dv = A::sub(b.v, a.v), dd = A::sub(b.d, a.d);
        float inv = 1.0f / (b.y - a.y);
        float t = ((y - 1.0f) - a.y) * inv;
        Edge& s = e[slot];
        s.ay = a.y;
        s.by = b.y;
        s.x = dx * t + a.x;
        s.u = A::add(A::mul(du, t), a.u);
        s.v = A::add(A::mul(dv, t), a.v);
        s.d = A::add(A::mul(dd, t), a.d);
        s.dx = dx * inv;
        s.du = A::mul(du, inv);
        s.dv = A::mul(dv, inv);
        s.dd = A::mul(dd, inv);
    }
}

static void sort_by_y(const FwVtx v[3], FwVtx o[3]) {  // raster.rs:90-113
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
    o[0] = v[a];
    o[1] = v[b];
    o[2] = v[c];
}

template <typename A>
static void emit_run(int x0, int x1, float lx, float wid, const float lu[3], const float ru[3], int yi, bool check,
                     int w1, int h1, FwHits* sink) {
    // one span from x0 to x1 (closed) with the payload lerped from the left to the right edge
    auto emit = [&](int x, float u, float v, float d) {
        if (check && (x < 0 || x > w1 || yi < 0 || yi > h1)) sink->outside = true;
        else sink->hits.push_back(FwHit{x, yi, u, v, d});
    };
    float inv = 1.0f / wid;
    if (x0 == x1) {
        float t = ((float)x0 - lx) * inv;
        emit(x0, A::add(A::mul(A::sub(ru[0], lu[0]), t), lu[0]), A::add(A::mul(A::sub(ru[1], lu[1]), t), lu[1]),
             A::add(A::mul(A::sub(ru[2], lu[2]), t), lu[2]));
        return;
    }
    float du = A::sub(ru[0], lu[0]), dv = A::sub(ru[1], lu[1]), dd = A::sub(ru[2], lu[2]);
    float t = ((float)x0 - lx) * inv;
    float u = A::add(A::mul(du, t), lu[0]);
    float v = A::add(A::mul(dv, t), lu[1]);
    float d = A::add(A::mul(dd, t), lu[2]);
    int x = x0;
    while (x < x1) {
        emit(x, u, v, d);
        u = A::add(u, A::mul(du, inv));
        v = A::add(v, A::mul(dv, inv));
        d = A::add(d, A::mul(dd, inv));
        x += 1;
    }
    emit(x, u, v, d);
}

template <typename A>
static void span(const Edge& l, const Edge& r, float y, int w1, FwHits* sink) {  // raster.rs:116-153
    int x0 = std::max(cvtt32(std::ceil(l.x)), 0);
    int x1 = std::min(cvtt32(std::floor(r.x)), w1);
    float wid = r.x - l.x;
    if (x0 > x1) return;
    if (!((double)wid > 1e-08)) return;
    int yi = cvtt32(y);
    float lu[3] = {l.u, l.v, l.d}, ru[3] = {r.u, r.v, r.d};
    // the single pixel span computes t with (1 / wid) like the run does
    emit_run<A>(x0, x1, l.x, wid, lu, ru, yi, false, w1, 0, sink);
}

template <typename A>
static void triangle_with(const FwVtx t[3], int w1, int h1, FwHits* sink) {  // raster.rs:171-300
    float w1f = (float)w1, h1f = (float)h1;
    bool ok = (0.0f <= t[0].x || 0.0f <= t[1].x || 0.0f <= t[2].x) && (0.0f <= t[0].y || 0.0f <= t[1].y || 0.0f <= t[2].y) &&
              (t[0].x <= w1f || t[1].x <= w1f || t[2].x <= w1f) && (t[0].y <= h1f || t[1].y <= h1f || t[2].y <= h1f);
    if (!ok) return;
    FwVtx vs[3];
    sort_by_y(t, vs);
    float y = std::ceil(vs[0].y);
    float y_end = std::floor(vs[2].y);
    if (y < 0.0f) y = 0.0f;
    if (h1f < y_end) y_end = h1f;
    if (y <= y_end) {
        int vi = 0, count = 0;
        Edge e[2];
        for (;;) {
            if (vi < 3) {
                for (;;) {
                    if (y < vs[vi].y) break;
                    if (count != 0) {
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
                    }
                    if (vi == 0) {
                        edge_init<A>(vs[0], vs[1], y, e, &count);
                        edge_init<A>(vs[0], vs[2], y, e, &count);
                    } else if (vi == 1) {
                        edge_init<A>(vs[1], vs[2], y, e, &count);
                        edge_init<A>(vs[1], vs[0], y, e, &count);
                    } else {
                        edge_init<A>(vs[2], vs[0], y, e, &count);
                        edge_init<A>(vs[2], vs[1], y, e, &count);
                    }
                    vi += 1;
                    if (vi >= 3) break;
                }
            }
            for (int k = 0; k < 2; k++) {
                e[k].x += e[k].dx;
                e[k].u = A::add(e[k].u, e[k].du);
                e[k].v = A::add(e[k].v, e[k].dv);
                e[k].d = A::add(e[k].d, e[k].dd);
            }
            if (count == 2) {
                if (e[1].x < e[0].x) span<A>(e[1], e[0], y, w1, sink);
                else span<A>(e[0], e[1], y, w1, sink);
            }
            y += 1.0f;
            if (!(y <= y_end)) break;
        }
    }
    // the degenerate pass: both lower vertices exactly on the last row
    const FwVtx& mid = vs[1];
    const FwVtx& bot = vs[2];
    if (mid.y == h1f && mid.y == bot.y) {
        const FwVtx& l = bot.x <= mid.x ? bot : mid;
        const FwVtx& r = bot.x <= mid.x ? mid : bot;
        float yy = l.y;
        float yt = (float)cvtt32(yy);
        if (0.0f <= yt && yt <= h1f && !((double)(yy - yt) > 0.01)) {
            int x0 = std::max(cvtt32(std::ceil(l.x)), 0);
            int x1 = std::min(cvtt32(std::floor(r.x)), w1);
            float wid = r.x - l.x;
            if ((double)wid > 1e-05) {
                float lu[3] = {l.u, l.v, l.d}, ru[3] = {r.u, r.v, r.d};
                emit_run<A>(x0, x1, l.x, wid, lu, ru, cvtt32(yt), true, w1, h1, sink);
            }
        }
    }
}

void fw_triangle(const FwVtx tri[3], int w1, int h1, FwHits* sink) {  // raster.rs:158-166
    bool nan = false;
    for (int i = 0; i < 3; i++) nan = nan || std::isnan(tri[i].u) || std::isnan(tri[i].v) || std::isnan(tri[i].d);
    if (nan) triangle_with<ARule>(tri, w1, h1, sink);
    else triangle_with<APlain>(tri, w1, h1, sink);
}

// ---- the render (forward.rs) ----------------------------------------------------------------------

static void fold(float* acc, uint8_t* cnt, size_t i, const float c[4]) {  // forward.rs:103-128
    uint8_t n = cnt[i];
    float* a = acc + i * 4;
    if (n == 0) {
        for (int k = 0; k < 4; k++) a[k] = c[k] + 0.0f;
        cnt[i] = 1;
    } else if (n == 0xff) {
        for (int k = 0; k < 4; k++) {
            float plain = (a[k] * 255.0f + c[k]) * 0.00390625f + 0.0f;
            a[k] = std::isnan(plain) ? nr::add(nr::mul(nr::add(nr::mul(a[k], 255.0f), c[k]), 0.00390625f), 0.0f) : plain;
        }
    } else {
        float nf = (float)n;
        float r = (float)(1.0 / ((double)nf + 1.0));
        for (int k = 0; k < 4; k++) {
            float plain = (nf * a[k] + c[k]) * r + 0.0f;
            a[k] = std::isnan(plain) ? nr::add(nr::mul(nr::add(nr::mul(nf, a[k]), c[k]), r), 0.0f) : plain;
        }
        cnt[i] = n + 1;
    }
}

static void convert(Image& out, const std::vector<float>& acc) {  // forward.rs:192-210
    size_t n = out.samples();
    for (size_t i = 0; i < n; i++) {
        if (out.fmt == F32) out.f32[i] = acc[i] + 0.0f;
        else if (out.fmt == U8) out.u8[i] = (uint8_t)cvtt64f(acc[i] + 0.5f);
        else out.u16[i] = (uint16_t)cvtt64f(acc[i] + 0.5f);
    }
}

static bool flow_is_zero(const FlowField& f) {  // forward.rs:214-222
    for (float v : f.d) {
        float a = v < 0.0f ? -v : v;
        if (0.0001 < (double)a) return false;
    }
    return true;
}

static void texel(const Image& src, int c, int r, float t[4]) {  // forward.rs:178-186
    size_t i = ((size_t)r * src.w + c) * 4;
    for (int k = 0; k < 4; k++) t[k] = load_s(src, i + k);
}

int forward_warp(Image& out, const Image& src, const FlowField& flow, float amount, bool pyramid, Coverage* cov,
                 std::string* err) {  // forward.rs:229-320
    if (out.w != src.w || out.h != src.h || out.fmt != src.fmt) { *err = "forward warp: shape mismatch"; return 1; }
    if (src.w < 2 || src.h < 2 || flow.w < 2 || flow.h < 2) { *err = "forward warp needs at least 2x2"; return 1; }
    int w = src.w, h = src.h;
    float a = 0.0f > amount ? -amount : amount;
    if (1e-05 > (double)a || flow_is_zero(flow)) {
        copy_image(out, src);
        if (cov) { cov->w = w; cov->h = h; cov->d.assign((size_t)w * h, 0xff); }
        return 0;
    }
    std::vector<float> pos;
    fw_positions(w, h, flow, amount, &pos);
    g_tap_bad = false;
    std::vector<float> acc((size_t)w * h * 4, 0.0f);
    std::vector<uint8_t> cnt((size_t)w * h, 0);
    int w1 = w - 1, h1 = h - 1;
    bool outside = false;
    if (pyramid) {
        int levels = fw_level_count(w, h);
        std::vector<float> mips;
        if (levels > 1) {
            mips.assign((size_t)w * h, 0.0f);
            OMP_FOR
            for (int r = 0; r < h; r++)
                for (int c = 0; c < w; c++) mips[(size_t)r * w + c] = fw_mip_level(w, h, flow, amount, c, r);
        }
        FwPyramid pyr;
        bool built = false;
        auto vtx = [&](int r, int c) {
            size_t i = (size_t)r * w + c;
            return FwVtx{pos[i * 2], pos[i * 2 + 1], (float)c / (float)w1, (float)r / (float)h1, mips.empty() ? 0.0f : mips[i]};
        };
        FwHits hits;
        for (int r = 0; r < h - 1; r++) {
            for (int c = 0; c < w - 1; c++) {
                FwVtx t1[3] = {vtx(r, c), vtx(r, c + 1), vtx(r + 1, c)};
                FwVtx t2[3] = {vtx(r + 1, c + 1), vtx(r, c + 1), vtx(r + 1, c)};
                for (const FwVtx* t : {t1, t2}) {
                    hits.hits.clear();
                    fw_triangle(t, w1, h1, &hits);
                    for (const FwHit& hh : hits.hits) {
                        float col[4];
                        if (0.0f < hh.d) {
                            if (!built) { pyr.build(src); built = true; }
                            sample(pyr, src, hh.u, hh.v, hh.d, col);
                        } else {
                            tap(src, hh.u, hh.v, col);
                        }
                        fold(acc.data(), cnt.data(), (size_t)hh.y * w + hh.x, col);
                    }
                }
                outside = outside || hits.outside;
            }
        }
        outside = outside || hits.outside;
    } else {
        auto vtx3 = [&](int r, int c) {
            size_t i = (size_t)r * w + c;
            float t[4];
            texel(src, c, r, t);
            return FwVtx{pos[i * 2], pos[i * 2 + 1], t[0], t[1], t[2]};
        };
        auto vtx1 = [&](int r, int c) {
            size_t i = (size_t)r * w + c;
            float t[4];
            texel(src, c, r, t);
            return FwVtx{pos[i * 2], pos[i * 2 + 1], t[3], 0.0f, 0.0f};
        };
        for (int r = 0; r < h - 1; r++) {
            for (int c = 0; c < w - 1; c++) {
                const int tri[2][3][2] = {{{r, c}, {r, c + 1}, {r + 1, c}}, {{r + 1, c + 1}, {r, c + 1}, {r + 1, c}}};
                for (int k = 0; k < 2; k++) {
                    FwVtx ta[3], tb[3];
                    for (int j = 0; j < 3; j++) {
                        ta[j] = vtx3(tri[k][j][0], tri[k][j][1]);
                        tb[j] = vtx1(tri[k][j][0], tri[k][j][1]);
                    }
                    FwHits ha, hb;
                    fw_triangle(ta, w1, h1, &ha);
                    fw_triangle(tb, w1, h1, &hb);
                    outside = outside || ha.outside || hb.outside;
                    size_t m = std::min(ha.hits.size(), hb.hits.size());
                    for (size_t j = 0; j < m; j++) {
                        const FwHit& x = ha.hits[j];
                        float col[4] = {x.u, x.v, x.d, hb.hits[j].u};
                        fold(acc.data(), cnt.data(), (size_t)x.y * w + x.x, col);
                    }
                }
            }
        }
    }
    if (outside) {
        *err = "forward warp: the degenerate last row pass of the rasteriser would write outside the image";
        return 2;
    }
    if (g_tap_bad) {
        *err = "forward warp: a texture coordinate outside the image";
        return 2;
    }
    convert(out, acc);
    if (cov) {
        cov->w = w;
        cov->h = h;
        cov->d.resize((size_t)w * h);
        for (size_t i = 0; i < cov->d.size(); i++) cov->d[i] = cnt[i] != 0 ? 0xff : 0;
    }
    return 0;
}

// ---- the compositions of the forward warp codes (compose/vector.rs:117-147, forward.rs:384-496) ----
// The forward warps are the textured variant unless cs.gouraud (the stage set of retime-fgbg,
// plugins/retime-fgbg/src/glue.rs:142-143, wraps every forward warp as the Gouraud variant).

int compose_forward(const ComposeSettings& cs, const Selection& sel, const Image& a, const Image& b,
                    const FlowField* f_ab, const FlowField* f_ba, Image* out, std::string* err) {
    float wa = sel.wa;
    bool fill = cs.warp_mode == 2;
    *out = Image(a.w, a.h, a.fmt);
    if (sel.interp == 0) {
        // the pushed frame uses its own flow: F_AB for wa >= 0.5 (nearest_uses_f_ab with code 2 / 3)
        const FlowField* flow = nearest_uses_f_ab(wa, cs.warp_mode) ? f_ab : f_ba;
        if (!flow) { *err = "missing flow"; return 1; }
        Coverage cov;
        bool take_a = !(0.5f > wa);  // a NaN weight takes A
        int rc = take_a ? forward_warp(*out, a, *flow, 1.0f - wa, !cs.gouraud, fill ? &cov : nullptr, err)
                        : forward_warp(*out, b, *flow, wa, !cs.gouraud, fill ? &cov : nullptr, err);
        if (rc || !fill) return rc;
        for (auto& v : cov.d) v = 0xff - v;  // warp.rs:76-80
        return fill_holes(*out, cov.d.data(), 1, cs.taps_above_first, err, cs.wrap_360);
    }
    if (sel.interp == 1) {
        if (!f_ab || !f_ba) { *err = "missing flow"; return 1; }
        float frac = 1.0f - wa;
        Image ta(a.w, a.h, a.fmt), tb(b.w, b.h, b.fmt);
        Coverage c1, c2;
        int rc = forward_warp(ta, a, *f_ab, frac, !cs.gouraud, fill ? &c1 : nullptr, err);
        if (rc) return rc;
        rc = forward_warp(tb, b, *f_ba, wa, !cs.gouraud, fill ? &c2 : nullptr, err);
        if (rc) return rc;
        if (!fill) {  // smartblend.rs:458-477 without coverage: the plain blend
            blend(*out, ta, tb, frac);
            return 0;
        }
        smart_blend(*out, ta, tb, frac, cs.video_360);  // smart_composite, then smart_finish_with
        for (size_t i = 0; i < c1.d.size(); i++) c1.d[i] = 0xff - std::max(c1.d[i], c2.d[i]);
        return fill_holes(*out, c1.d.data(), 1, cs.taps_above_first, err, cs.wrap_360);
    }
    if (sel.interp == 2) {  // forward.rs:498-572 (weighted_forward, weighted_forward_fill)
        if (!f_ab || !f_ba) { *err = "missing flow"; return 1; }
        float frac = 1.0f - wa;
        Image ta(a.w, a.h, a.fmt), tb(b.w, b.h, b.fmt);
        Coverage c1, c2;
        int rc = forward_warp(ta, a, *f_ab, frac, !cs.gouraud, fill ? &c1 : nullptr, err);
        if (rc) return rc;
        rc = forward_warp(tb, b, *f_ba, wa, !cs.gouraud, fill ? &c2 : nullptr, err);
        if (rc) return rc;
        return weighted_tail(*out, ta, a, tb, b, wa, fill ? &c1 : nullptr, fill ? &c2 : nullptr, cs.taps_above_first, err);
    }
    *err = "bad interpolation mode";
    return 1;
}

}  // namespace orc
