// Test infrastructure: the CPU oracle's restatement of the compositor's tails, the Weighted Blend
// filters (plugins/retime-engine/src/filters.rs) and Blur Compensation (warp/blurcomp.rs). Plain
// single-threaded C++, compiled without FP contraction; each function names the reference lines it
// follows.
#include "oracle_filters.h"
#include <algorithm>
#include <cmath>

namespace orc {

// filters.rs:75-93: w[i] = powf(2, -(i*i / t^2)), t = radius / 3, divided by 2 * sum - w[0]
std::vector<float> wb_blur_taps(float radius) {
    float t = radius / 3.0f;
    float t2 = t * t;
    int count = std::max((int)radius, 0) + 1;
    std::vector<float> w;
    float sum = 0.0f;
    for (int i = 0; i < count; i++) {
        float fi = (float)i;
        float x = fi * fi;
        x = x / t2;
        x = -x;
        float p = powf(2.0f, x);
        w.push_back(p);
        sum += p;
    }
    float denom = sum * 2.0f - w[0];
    for (auto& p : w) p /= denom;
    return w;
}

namespace {

// filters.rs:113-118: trunc(v + 0.5), clamped to 0..max as a float, truncated again
int32_t store_int(float v, float max) {
    int32_t t = cvtt32(v + 0.5f);
    float f = (float)t;
    f = f > 0.0f ? f : 0.0f;
    f = f < max ? f : max;
    return cvtt32(f + 0.5f);
}

// filters.rs:171-225 (conv_pixel_with): one output pixel of the 1D line filter, four lanes;
// Rule: the NaN rule arithmetic
template <bool Rule>
void conv_pixel_with(int i, int n, const std::vector<float>& taps, const float* const* line, bool left_first, float out[4]) {
    auto mul = [](float a, float b) { return Rule ? nr::mul(a, b) : a * b; };
    auto add = [](float a, float b) { return Rule ? nr::add(a, b) : a + b; };
    auto dv = [](float a, float b) { return Rule ? nr::div(a, b) : a / b; };
    const float S = -1.0f;
    int count = (int)taps.size();
    int left = std::min(n, count);
    int mid = std::max(n - 2 * count, 0);
    const float* c = line[i];
    float w0 = taps[0];
    float acc[4];
    for (int l = 0; l < 4; l++) acc[l] = mul(c[l], w0);
    if (i >= left && i < left + mid) {
        for (int k = count - 1; k >= 1; k--) {
            const float* r = line[i + k];
            const float* lf = line[i - k];
            float wk = taps[k];
            for (int l = 0; l < 4; l++) acc[l] = add(acc[l], mul(add(r[l], lf[l]), wk));
        }
        for (int l = 0; l < 4; l++) out[l] = acc[l];
        return;
    }
    static const float sent[4] = {S, S, S, S};
    float wsum[4] = {w0, w0, w0, w0};
    for (int k = count - 1; k >= 1; k--) {
        const float* r = i + k < n ? line[i + k] : sent;
        const float* lf = i >= k ? line[i - k] : sent;
        if (left_first) std::swap(r, lf);
        float wk = taps[k];
        for (int l = 0; l < 4; l++) {
            float wr = (r[l] != S ? 1.0f : 0.0f) * wk;
            wsum[l] = wsum[l] + wr;
            float rt = mul(wr, r[l]);
            float wl = (lf[l] != S ? 1.0f : 0.0f) * wk;
            float lt = mul(lf[l], wl);
            wsum[l] = wsum[l] + wl;
            acc[l] = add(add(acc[l], rt), lt);
        }
    }
    for (int l = 0; l < 4; l++) out[l] = dv(acc[l], wsum[l]);
}

// filters.rs:160-169 (conv_pixel): the plain arithmetic, repeated with the NaN rule for a float
// result holding a NaN
void conv_pixel(int i, int n, const std::vector<float>& taps, const float* const* line, bool left_first, bool is_float,
                float out[4]) {
    conv_pixel_with<false>(i, n, taps, line, left_first, out);
    if (is_float && (std::isnan(out[0]) || std::isnan(out[1]) || std::isnan(out[2]) || std::isnan(out[3])))
        conv_pixel_with<true>(i, n, taps, line, left_first, out);
}

template <typename T>
void blur_plane(T* data, int w, int h, const std::vector<float>& taps, bool above_first, bool is_float, float max) {
    if (w == 0 || h == 0) return;
    auto store = [&](float v) -> T {
        if (is_float) return (T)v;
        return (T)store_int(v, max);
    };
    size_t rl = (size_t)w * 4;
    // pass 1, the rows (filters.rs:232-241)
    std::vector<float> buf((size_t)std::max(w, h) * 4);
    std::vector<const float*> line((size_t)std::max(w, h));
    for (int y = 0; y < h; y++) {
        T* row = data + y * rl;
        for (int x = 0; x < w; x++) {
            for (int l = 0; l < 4; l++) buf[(size_t)x * 4 + l] = (float)row[x * 4 + l];
            line[x] = &buf[(size_t)x * 4];
        }
        for (int x = 0; x < w; x++) {
            float v[4];
            conv_pixel(x, w, taps, line.data(), false, is_float, v);
            for (int l = 0; l < 4; l++) row[x * 4 + l] = store(v[l]);
        }
    }
    // pass 2, the columns of the result of pass 1 (filters.rs:242-252)
    std::vector<T> snap(data, data + rl * h);
    for (int x = 0; x < w; x++) {
        for (int y = 0; y < h; y++) {
            for (int l = 0; l < 4; l++) buf[(size_t)y * 4 + l] = (float)snap[y * rl + x * 4 + l];
            line[y] = &buf[(size_t)y * 4];
        }
        for (int y = 0; y < h; y++) {
            float v[4];
            conv_pixel(y, h, taps, line.data(), above_first, is_float, v);
            for (int l = 0; l < 4; l++) data[y * rl + x * 4 + l] = store(v[l]);
        }
    }
}

int ring_sum(const Mask& t, int x, int r0, int r1, int r2) {  // filters.rs:339-345
    auto at = [&](int y, int dx) { return (int)t.d[(size_t)y * t.w + x + dx]; };
    return at(r0, 1) + at(r0, 0) + at(r0, 2) + at(r1, 0) + at(r1, 2) + at(r2, 0) + at(r2, 1) + at(r2, 2);
}

float white(Fmt f) { return f == U8 ? 255.0f : f == U16 ? 65535.0f : 1.0f; }

}  // namespace

void wb_blur(Image& img, float radius, bool above_first) {  // filters.rs:269-280
    if (0.0 > (double)radius) return;
    std::vector<float> taps = wb_blur_taps(radius);
    if (img.fmt == U8) blur_plane(img.u8.data(), img.w, img.h, taps, above_first, false, 255.0f);
    else if (img.fmt == U16) blur_plane(img.u16.data(), img.w, img.h, taps, above_first, false, 65535.0f);
    else blur_plane(img.f32.data(), img.w, img.h, taps, above_first, true, 0.0f);
}

float wb_mask_limit(Fmt fmt, float threshold) { return threshold * white(fmt) * threshold * threshold * 3.0f; }

Mask difference_mask(const Image& a, const Image& b, float threshold) {
    Mask m(a.w, a.h);
    float limit = wb_mask_limit(a.fmt, threshold);
    size_t n = (size_t)a.w * a.h;
    for (size_t i = 0; i < n; i++) {
        auto d = [&](int c) -> float {
            float va, vb;
            if (a.fmt == U8) { va = (float)a.u8[i * 4 + c]; vb = (float)b.u8[i * 4 + c]; }
            else if (a.fmt == U16) { va = (float)a.u16[i * 4 + c]; vb = (float)b.u16[i * 4 + c]; }
            else { va = a.f32[i * 4 + c]; vb = b.f32[i * 4 + c]; }
            return std::fabs(va - vb);
        };
        float sum = (d(1) + d(2)) + d(3);
        m.d[i] = sum >= limit ? 0xff : 0;
    }
    return m;
}

void mask_prune(Mask& m, int limit) {
    int w = m.w, h = m.h;
    if (h < 5 || w < 3) return;
    Mask t = m;
    for (int y0 = 0; y0 < h - 4; y0++)
        for (int x = 0; x < w - 2; x++) {
            int sum = ring_sum(t, x, y0, y0 + 2, y0 + 4);
            size_t dst = (size_t)(y0 + 2) * w + x + 1;
            if (sum < limit && m.d[dst] != 0) m.d[dst] = 0;
        }
}

void mask_fill(Mask& m, int limit, uint8_t value) {
    int w = m.w, h = m.h;
    if (h < 3 || w < 3) return;
    Mask t = m;
    for (int y0 = 0; y0 < h - 2; y0++)
        for (int x = 0; x < w - 2; x++) {
            int sum = ring_sum(t, x, y0, y0 + 1, y0 + 2);
            size_t dst = (size_t)(y0 + 1) * w + x + 1;
            if (limit < sum && m.d[dst] == 0) m.d[dst] = value;
        }
}

void mask_dilate_rows(Mask& m) {
    int w = m.w, h = m.h;
    if (h < 3) return;
    Mask t = m;
    for (int y = 1; y < h - 1; y++)
        for (int x = 0; x < w; x++)
            if (t.d[(size_t)(y - 1) * w + x] == 255 || t.d[(size_t)(y + 1) * w + x] == 255) m.d[(size_t)y * w + x] = 255;
}

void mask_replicate_border(Mask& m) {  // the rectangle tests in float, as the reference makes them
    int64_t w = m.w, h = m.h;
    if (w == 0 || h == 0) return;
    float p2 = 1.0f, p3 = 1.0f, p4 = (float)(w - 2), p5 = (float)(h - 2);
    int64_t iv14 = (int64_t)(int32_t)p5;
    float fy0 = p3, fy1 = p5;
    if (p5 < p3) { fy0 = p5; fy1 = p3; }
    float fx0 = p2, fx1 = p4;
    if (p4 < p2) { fx0 = p4; fx1 = p2; }
    auto idx = [&](int64_t x, int64_t y) -> int64_t { return (x >= 0 && x < w && y >= 0 && y < h) ? y * w + x : -1; };
    auto outside = [&](int64_t x, int64_t y) {
        float xf = (float)x, yf = (float)y;
        return yf < fy0 || fy1 < yf || fx1 < xf || xf < fx0;
    };
    for (int64_t y = 0; (float)y < fy0; y++)
        for (int64_t x = 0; x < w; x++)
            if (outside(x, y)) {
                int64_t d = idx(x, y), s = idx(x, (int64_t)(int32_t)p3);
                if (d >= 0 && s >= 0) m.d[d] = m.d[s];
            }
    for (int64_t y = (int64_t)(int32_t)fy1; y < h; y++)
        for (int64_t x = 0; x < w; x++)
            if (outside(x, y)) {
                int64_t d = idx(x, y), s = idx(x, iv14);
                if (d >= 0 && s >= 0) m.d[d] = m.d[s];
            }
    for (int64_t y = 0; y < h; y++) {
        for (int64_t x = 0; (float)x < fx0; x++) {
            int64_t d = idx(x, y), s = idx((int64_t)(int32_t)p2, y);
            if (d >= 0 && s >= 0) m.d[d] = m.d[s];
        }
        int64_t first = (int64_t)(int32_t)fx1;
        int64_t c4 = (int64_t)(int32_t)p4;
        for (int64_t j = 0; first + j < w; j++) {
            int64_t d = idx(c4 + j, y), s = idx(c4, y);
            if (d >= 0 && s >= 0) m.d[d] = m.d[s];
        }
    }
}

void clean_mask(Mask& m) {
    for (int pass = 0; pass < 2; pass++) mask_prune(m, 254 + 255 * pass);
    mask_dilate_rows(m);
    for (int i = 0; i < 2; i++) {
        mask_fill(m, 254, 255);
        mask_replicate_border(m);
    }
    int limit = 254, value = 128;
    for (int i = 0; i < 2; i++) {
        mask_fill(m, limit, (uint8_t)value);
        mask_replicate_border(m);
        limit = (int)((double)limit * 0.5 + 0.5);
        value = (int)((double)value * 0.5 + 0.5);
    }
}

Mask change_mask(const Image& warped, const Image& original) {
    Mask m = difference_mask(warped, original, 0.4f);
    clean_mask(m);
    return m;
}

void composite_masked(Image& dest, const Image& src, const Mask& m) {
    size_t n = (size_t)dest.w * dest.h;
    for (size_t i = 0; i < n; i++) {
        uint8_t mv = m.d[i];
        float f = (float)mv / 255.0f;
        float g = (float)(1.0 - (double)f);  // filters.rs:608-612
        for (int c = 0; c < 4; c++) {
            size_t j = i * 4 + c;
            if (dest.fmt == U8) {
                dest.u8[j] = mv == 0 ? src.u8[j] : (uint8_t)cvtt64f(((float)src.u8[j] * g + (float)dest.u8[j] * f) + 0.5f);
            } else if (dest.fmt == U16) {
                dest.u16[j] = mv == 0 ? src.u16[j]
                                      : (uint16_t)cvtt64f(((float)src.u16[j] * g + (float)dest.u16[j] * f) + 0.5f);
            } else if (mv == 0) {
                dest.f32[j] = src.f32[j];
            } else {
                float plain = (g * src.f32[j] + f * dest.f32[j]) + 0.0f;
                dest.f32[j] = std::isnan(plain) ? nr::add(nr::add(nr::mul(g, src.f32[j]), nr::mul(f, dest.f32[j])), 0.0f) : plain;
            }
        }
    }
}

float sharpen_weight(float t) {
    double x = 1.0 - std::fabs(0.5 - (double)t) * 2.0;
    float neg = -(float)x;
    return (float)((double)neg * 0.5);
}

void sharpen_step(Image& frame, const Image& original, float t, bool above_first) {
    Mask mask = change_mask(frame, original);
    Image sharp = frame;
    wb_blur(sharp, 3.0f, above_first);
    Image base = frame;
    lerp(sharp, base, sharpen_weight(t));
    for (auto& v : mask.d) v = 255 - v;
    composite_masked(frame, sharp, mask);
}

// ---- Blur Compensation (warp/blurcomp.rs) --------------------------------------------------------------

namespace {

const int TAP_LIMIT = 1 << 16;

float store_blur_int(float v, float white) {  // warp.rs:272-274 / :292-294
    float f = (float)cvtt32(v + 0.5f);
    f = std::max(f, (float)0.0f);
    return std::min(f, white);
}

}  // namespace

// blurcomp.rs:282-322 (Blur::wrap_x): x into [0, W) by the loops of the 360 inverse warp, false past
// their bound or when the result is outside (NaN, infinite)
static bool wrap_x(float qx, float wf, float* out) {
    float x = qx;
    unsigned guard = 0;
    while (x < 0.0f) { x += wf; if (++guard > (unsigned)TAP_LIMIT) return false; }
    while (wf <= x) { x -= wf; if (++guard > (unsigned)TAP_LIMIT) return false; }
    *out = x;
    return x >= 0.0f && x < wf;
}

// blurcomp.rs:248-280 (sphere_tap): y into [0, H) counting the periods; after an odd count x moves half
// a turn and a y other than 0 becomes H - y; false past the loops' bound or outside the frame
static bool sphere_tap(float x, float qy, float wf, float hf, float* ox, float* oy) {
    float y = qy;
    unsigned steps = 0;
    while (y < 0.0f) { y += hf; if (++steps > (unsigned)TAP_LIMIT) return false; }
    while (hf <= y) { y -= hf; if (++steps > (unsigned)TAP_LIMIT) return false; }
    if (steps % 2 == 1) {
        x = wf * 0.5f + x;
        if (!(x < wf)) x -= wf;
        if (y != 0.0f) y = hf - y;
    }
    *ox = x;
    *oy = y;
    return x >= 0.0f && x < wf && y >= 0.0f && y < hf;
}

int motion_blur(Image& dest, const Image& src, const FlowField& flow, float amount, bool hiq, float shutter,
                std::string* err, bool is360) {
    if (dest.w != src.w || dest.h != src.h || dest.fmt != src.fmt) { *err = "motion blur: shapes"; return 1; }
    if (src.w < 2 || src.h < 2 || flow.w < 2 || flow.h < 2) { *err = "motion blur needs at least 2x2"; return 1; }
    int w = src.w, h = src.h;
    int w1i = w - 1, h1i = h - 1;
    float rx = (float)(flow.w - 1) / (float)w1i;
    float ry = (float)(flow.h - 1) / (float)h1i;
    float kx = (0.5f / rx) * amount;
    float ky = (0.5f / ry) * amount;
    bool shifted = shutter != 0.5f;
    float k = shutter * 2.0f - 1.0f;
    float wf = (float)w, hf = (float)h;
    const float TINY = bits_f(0x358637bdu);
    bool bad = false;
    auto sample = [&](size_t i, int c) -> float {
        return src.fmt == U8 ? (float)src.u8[i * 4 + c] : src.fmt == U16 ? (float)src.u16[i * 4 + c] : src.f32[i * 4 + c];
    };
    auto store = [&](size_t i, int c, float v) {
        if (dest.fmt == U8) dest.u8[i * 4 + c] = (uint8_t)store_blur_int(v, 255.0f);
        else if (dest.fmt == U16) dest.u16[i * 4 + c] = (uint16_t)store_blur_int(v, 65535.0f);
        else dest.f32[i * 4 + c] = v;
    };
    for (int y = 0; y < h; y++) {
        float yf = (float)y, fy = yf * ry;
        for (int x = 0; x < w; x++) {
            size_t i = (size_t)y * w + x;
            float xf = (float)x;
            float d[2];
            warp_flow_bilerp(flow, xf * rx, fy, d);
            float vx = d[0] * kx, vy = d[1] * ky;
            float d2 = vy * vy + vx * vx;
            if (hiq && TINY > d2) {  // the source pixel, copied
                if (dest.fmt == U8) for (int c = 0; c < 4; c++) dest.u8[i * 4 + c] = src.u8[i * 4 + c];
                else if (dest.fmt == U16) for (int c = 0; c < 4; c++) dest.u16[i * 4 + c] = src.u16[i * 4 + c];
                else for (int c = 0; c < 4; c++) dest.f32[i * 4 + c] = src.f32[i * 4 + c];
                continue;
            }
            float dist = std::sqrt(d2);
            float cx = shifted ? vx * k + xf : xf, cy = shifted ? vy * k + yf : yf;
            if (!hiq) { cx = cx + 0.5f; cy = cy + 0.5f; }
            int n = cvtt32(dist + 1.0f);
            float sx, sy;
            if (n < 2) { n = 2; sx = vx; sy = vy; }
            else { float dd = (float)(n - 1); sx = vx / dd; sy = vy / dd; }
            if (n > TAP_LIMIT) {
                bad = true;
                for (int c = 0; c < 4; c++) store(i, c, 0.0f);
                continue;
            }
            float sum[4] = {0, 0, 0, 0};
            int cnt = 0;
            if (hiq) {  // blurcomp.rs:398-455
                auto tap = [&](float qx, float qy) {
                    if (std::isnan(qx) || std::isnan(qy)) { bad = true; return; }
                    if (is360) {  // blurcomp.rs:425-434: every tap counts, on the sphere, the 360 sampler
                        float wx, sx2, sy2;
                        if (!wrap_x(qx, wf, &wx) || !sphere_tap(wx, qy, wf, hf, &sx2, &sy2)) { bad = true; return; }
                        cnt++;
                        float t[4];
                        bilerp360_image(src, sx2, sy2, t);
                        for (int c = 0; c < 4; c++) sum[c] += t[c];
                    } else if (0.0f <= qx && qx < wf && 0.0f <= qy && qy < hf) {
                        cnt++;
                        float t[4];
                        bilerp4_image(src, qx, qy, t);
                        for (int c = 0; c < 4; c++) sum[c] += t[c];
                    }
                };
                float qx = cx, qy = cy;
                for (int j = 0; j < n; j++) { tap(qx, qy); qx += sx; qy += sy; }
                float nsx = -sx, nsy = -sy;
                qx = cx - sx; qy = cy - sy;
                for (int j = 1; j < n; j++) { tap(qx, qy); qx += nsx; qy += nsy; }
            } else {  // blurcomp.rs:459-559: the backward taps always count
                int wi = w, hi = (int)hf;
                float qx = cx, qy = cy;
                // blurcomp.rs:496-512 with is360: a tap whose row is inside reads the column of its wrapped x
                auto column = [&](float q, int* ix) {
                    float wx;
                    if (!wrap_x(q, wf, &wx)) { bad = true; return false; }
                    *ix = cvtt32(wx);
                    return true;
                };
                for (int j = 0; j < n; j++) {
                    int ix = cvtt32(qx), iy = cvtt32(qy);
                    if (is360) {
                        if (iy >= 0 && iy < hi && column(qx, &ix)) {
                            cnt++;
                            for (int c = 0; c < 4; c++) sum[c] += sample((size_t)iy * w + ix, c);
                        }
                    } else if (ix >= 0 && ix < wi && iy >= 0 && iy < hi) {
                        cnt++;
                        for (int c = 0; c < 4; c++) sum[c] += sample((size_t)iy * w + ix, c);
                    }
                    qx += sx; qy += sy;
                }
                float nsx = -sx, nsy = -sy;
                qx = cx - sx; qy = cy - sy;
                for (int j = 1; j < n; j++) {
                    int ix = cvtt32(qx), iy = cvtt32(qy);
                    if (is360) {
                        if (iy >= 0 && iy < hi && column(qx, &ix))
                            for (int c = 0; c < 4; c++) sum[c] += sample((size_t)iy * w + ix, c);
                    } else if (ix >= 0 && ix < wi && iy >= 0 && iy < hi) {
                        for (int c = 0; c < 4; c++) sum[c] += sample((size_t)iy * w + ix, c);
                    }
                    cnt++;
                    qx += nsx; qy += nsy;
                }
            }
            float inv = 1.0f / (float)cnt;
            for (int c = 0; c < 4; c++) store(i, c, inv * sum[c]);
        }
    }
    if (bad) { *err = "motion blur: a tap coordinate is NaN or a vector needs more than 65536 taps"; return 2; }
    return 0;
}

int blur_compensation(Image& img, const FlowField& flow, float s0, float s1, float blur, bool hiq, std::string* err,
                      bool is360) {
    float a = std::fabs(s0 - s1);  // blurcomp.rs:42-48 (blur_amount)
    if (!((double)a > 1e-6) || !((double)blur > 0.005)) return 0;
    float amount = (a - 1.0f) * blur;
    if (20.0f < amount) amount = 20.0f;  // blurcomp.rs:105-128 (compensate)
    else if (amount < -10.0f) amount = -10.0f;
    if ((double)std::fabs(amount) < 1e-6) return 0;
    Image tmp(img.w, img.h, img.fmt);
    if (0.0f < amount) {
        int rc = motion_blur(tmp, img, flow, amount, hiq, 0.5f, err, is360);
        if (rc) return rc;
        size_t n = (size_t)img.w * img.h;  // blurcomp.rs:134-149 (clear_rgb_where_transparent)
        for (size_t i = 0; i < n; i++) {
            bool clear = tmp.fmt == U8 ? tmp.u8[i * 4] == 0 : tmp.fmt == U16 ? tmp.u16[i * 4] == 0 : tmp.f32[i * 4] == 0.0f;
            if (!clear) continue;
            for (int c = 1; c < 4; c++) {
                if (tmp.fmt == U8) tmp.u8[i * 4 + c] = 0;
                else if (tmp.fmt == U16) tmp.u16[i * 4 + c] = 0;
                else tmp.f32[i * 4 + c] = 0.0f;
            }
        }
    } else {
        int rc = motion_blur(tmp, img, flow, 0.5f, hiq, 0.5f, err, is360);
        if (rc) return rc;
        lerp(tmp, img, amount);
    }
    copy_image(img, tmp);
    return 0;
}

}  // namespace orc
