// CPU oracle, core functions. TEST INFRASTRUCTURE ONLY (see oracle_core.h). Each function cites
// the reference file:line (crate plugins/retime-engine/src/) whose arithmetic it restates.
#include "oracle_core.h"
#include "oracle_smart.h"
#include "oracle_forward.h"
#include "oracle_filters.h"
#include "pow_tables.h"
#include <cstring>

#include <algorithm>
#include <cstdio>

#ifdef _OPENMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

namespace orc {

// =============================================================================================
// image boundary

static const float INV_255 = bits_f(0x3b808081u);            // image.rs:261
static const float PREMUL_16_COLOR = bits_f(0x387fff00u);    // image.rs:263
static const float PREMUL_16_ALPHA = bits_f(0x3fffff00u);    // image.rs:265
static const float UNPREMUL_16_ALPHA = bits_f(0x3f000080u);  // image.rs:267

static inline uint16_t u16_to_q15(uint16_t v) { return (uint16_t)(((uint32_t)v * 32768u + 32767u) / 65535u); }
static inline uint16_t q15_to_u16(uint16_t v) {
    uint32_t m = v < 32768 ? v : 32768;
    return (uint16_t)((m * 65535u + 16384u) / 32768u);
}

// image.rs:276-280
void premultiply_u8(const uint8_t p[4], uint8_t o[4]) {
    float a = (float)p[0] * INV_255;
    o[0] = p[0];
    for (int c = 1; c < 4; c++) o[c] = (uint8_t)q((float)p[c] * a);
}
// image.rs:283-291
static inline void premultiply_u16(const uint16_t p[4], uint16_t o[4]) {
    float a = (float)p[0] * PREMUL_16_COLOR;
    o[0] = (uint16_t)q((float)p[0] * PREMUL_16_ALPHA);
    for (int c = 1; c < 4; c++) o[c] = (uint16_t)q((float)p[c] * a);
}
// image.rs:294-303
void premultiply_f32(const float p[4], float o[4]) {
    float r[4] = {p[0], p[0] * p[1], p[0] * p[2], p[0] * p[3]};
    if (std::isnan(r[1]) || std::isnan(r[2]) || std::isnan(r[3]) || std::isnan(r[0])) {
        r[1] = nr::mul(p[0], p[1]);
        r[2] = nr::mul(p[0], p[2]);
        r[3] = nr::mul(p[0], p[3]);
    }
    for (int c = 0; c < 4; c++) o[c] = r[c];
}
// image.rs:306-320
void unpremultiply_u8(const uint8_t p[4], uint8_t o[4]) {
    if (p[0] == 0) { for (int c = 0; c < 4; c++) o[c] = p[c]; return; }
    float s = 255.0f / (float)p[0];
    o[0] = p[0];
    for (int c = 1; c < 4; c++) {
        float v = (float)p[c] * s;
        if (v > 255.0f) v = 255.0f;
        o[c] = (uint8_t)q(v);
    }
}
// image.rs:325-332
static inline void unpremultiply_u16(const uint16_t p[4], uint16_t o[4]) {
    if (p[0] == 0) { for (int c = 0; c < 4; c++) o[c] = p[c]; return; }
    float a = (float)p[0];
    float s = 32768.0f / a;
    o[0] = (uint16_t)q(a * UNPREMUL_16_ALPHA);
    for (int c = 1; c < 4; c++) o[c] = (uint16_t)q((float)p[c] * s);
}
// image.rs:339-351
static inline void unpremultiply_f32(const float p[4], float o[4]) {
    if ((double)p[0] < 1e-12) { for (int c = 0; c < 4; c++) o[c] = 0.0f; return; }
    float inv = 1.0f / p[0];
    float r[4] = {p[0], p[1] * inv, p[2] * inv, p[3] * inv};
    if (std::isnan(r[0]) || std::isnan(r[1]) || std::isnan(r[2]) || std::isnan(r[3])) {
        r[1] = nr::mul(p[1], inv);
        r[2] = nr::mul(p[2], inv);
        r[3] = nr::mul(p[3], inv);
    }
    for (int c = 0; c < 4; c++) o[c] = r[c];
}

// image.rs:142-171 (from_frame_straight): the channels as stored, in the engine order A, R, G, B; 16
// bpc every channel to 0..32768 and then scaled like the alpha of from_frame
Image from_frame_straight(const void* wire, int w, int h, Fmt fmt) {
    Image img(w, h, fmt);
    size_t n = (size_t)w * h;
    if (fmt == U8) {
        const uint8_t* px = (const uint8_t*)wire;
        for (size_t i = 0; i < n; i++) {
            uint8_t* o = &img.u8[i * 4];
            o[0] = px[i * 4 + 3]; o[1] = px[i * 4 + 0]; o[2] = px[i * 4 + 1]; o[3] = px[i * 4 + 2];
        }
    } else if (fmt == U16) {
        const uint16_t* px = (const uint16_t*)wire;
        static const int order[4] = {3, 0, 1, 2};
        for (size_t i = 0; i < n; i++)
            for (int c = 0; c < 4; c++)
                img.u16[i * 4 + c] = (uint16_t)q((float)u16_to_q15(px[i * 4 + order[c]]) * PREMUL_16_ALPHA);
    } else {
        const float* pl = (const float*)wire;  // planes G, B, R, A
        for (size_t i = 0; i < n; i++) {
            float* o = &img.f32[i * 4];
            o[0] = pl[3 * n + i]; o[1] = pl[2 * n + i]; o[2] = pl[0 * n + i]; o[3] = pl[1 * n + i];
        }
    }
    return img;
}

Image from_frame(const void* wire, int w, int h, Fmt fmt) {
    Image img(w, h, fmt);
    size_t n = (size_t)w * h;
    if (fmt == U8) {
        const uint8_t* px = (const uint8_t*)wire;
        OMP_FOR
        for (long i = 0; i < (long)n; i++) {
            uint8_t p[4] = {px[i * 4 + 3], px[i * 4 + 0], px[i * 4 + 1], px[i * 4 + 2]};
            premultiply_u8(p, &img.u8[i * 4]);
        }
    } else if (fmt == U16) {
        const uint16_t* px = (const uint16_t*)wire;  // little endian host
        OMP_FOR
        for (long i = 0; i < (long)n; i++) {
            uint16_t p[4] = {u16_to_q15(px[i * 4 + 3]), u16_to_q15(px[i * 4 + 0]), u16_to_q15(px[i * 4 + 1]),
                             u16_to_q15(px[i * 4 + 2])};
            premultiply_u16(p, &img.u16[i * 4]);
        }
    } else {
        const float* pl = (const float*)wire;  // planes G, B, R, A
        OMP_FOR
        for (long i = 0; i < (long)n; i++) {
            float p[4] = {pl[3 * n + i], pl[2 * n + i], pl[0 * n + i], pl[1 * n + i]};
            premultiply_f32(p, &img.f32[i * 4]);
        }
    }
    return img;
}

void to_frame(const Image& img, void* wire) {
    size_t n = (size_t)img.w * img.h;
    if (img.fmt == U8) {
        uint8_t* out = (uint8_t*)wire;
        OMP_FOR
        for (long i = 0; i < (long)n; i++) {
            uint8_t o[4];
            unpremultiply_u8(&img.u8[i * 4], o);
            out[i * 4 + 0] = o[1]; out[i * 4 + 1] = o[2]; out[i * 4 + 2] = o[3]; out[i * 4 + 3] = o[0];
        }
    } else if (img.fmt == U16) {
        uint16_t* out = (uint16_t*)wire;
        OMP_FOR
        for (long i = 0; i < (long)n; i++) {
            uint16_t o[4];
            unpremultiply_u16(&img.u16[i * 4], o);
            out[i * 4 + 0] = q15_to_u16(o[1]); out[i * 4 + 1] = q15_to_u16(o[2]);
            out[i * 4 + 2] = q15_to_u16(o[3]); out[i * 4 + 3] = q15_to_u16(o[0]);
        }
    } else {
        float* pl = (float*)wire;
        OMP_FOR
        for (long i = 0; i < (long)n; i++) {
            float o[4];
            unpremultiply_f32(&img.f32[i * 4], o);
            // pixel [r, g, b, a] -> planes in the channel order 1, 2, 0, 3 = G, B, R, A
            pl[0 * n + i] = o[2]; pl[1 * n + i] = o[3]; pl[2 * n + i] = o[1]; pl[3 * n + i] = o[0];
        }
    }
}

Image rows_reversed(const Image& img) {
    Image out(img.w, img.h, img.fmt);
    size_t es = img.fmt == U8 ? 1 : img.fmt == U16 ? 2 : 4;
    size_t row = (size_t)img.w * 4 * es;
    const uint8_t* s = (const uint8_t*)img.data();
    uint8_t* o = (uint8_t*)out.data();
    for (int y = 0; y < img.h; y++) std::memcpy(o + (size_t)y * row, s + (size_t)(img.h - 1 - y) * row, row);
    return out;
}

// =============================================================================================
// geometry (prep.rs:63-146, flow.rs:129-197)

void flow_resolution(int qv, bool hiq, int w, int h, int* r_out, int* w0, int* h0) {
    int r = (qv <= 2) ? 3 : (qv == 3) ? 2 : (qv == 4) ? 1 : 0;
    if (!hiq) r = (r == 0) ? 1 : (r == 1) ? 2 : (r == 2) ? 3 : r;
    while (r > 0 && ((w >> r) < 2 || (h >> r) < 2)) r -= 1;
    int ww = w, hh = h;
    for (int i = 0; i < r; i++) { ww /= 2; hh /= 2; }
    *r_out = r; *w0 = ww; *h0 = hh;
}

int level_count(int w0, int h0, int min_size) {
    int levels = 1, w = w0, h = h0;
    for (;;) {
        w /= 2;
        if (w < min_size) break;
        h /= 2;
        if (h < min_size) break;
        if (w > 2 && h > 2 && !(w == 2 && h == 2)) levels += 1;
        else break;
    }
    return levels;
}

bool geometry(const FlowSettings& s, int w, int h, Geometry* g, std::string* err) {
    if (s.quality == 0 || s.quality > 5) { *err = "flow quality outside 1..=5"; return false; }
    if (!(s.sensitivity >= 0.0f) || !std::isfinite(s.sensitivity)) { *err = "bad sensitivity"; return false; }
    flow_resolution(s.quality, s.hiq, w, h, &g->reduction, &g->w, &g->h);
    if (g->w < 2 || g->h < 2) { *err = "working size below 2x2"; return false; }
    g->levels = level_count(g->w, g->h, 2);
    g->sizes.clear();
    int lw = g->w, lh = g->h;
    for (int i = 0; i < g->levels; i++) {
        g->sizes.push_back({lw, lh});
        lw = std::max(lw / 2, 2);
        lh = std::max(lh / 2, 2);
    }
    return true;
}

// flow.rs:179-197
void start_level(float sensitivity, int levels, int* start, float* damp) {
    float p = (float)std::pow((double)sensitivity, 2.0);
    float l1 = (float)std::log((double)p);
    float l2 = (float)std::log(2.0);
    float lv = (float)levels;
    float x = l1 / l2 + lv;
    if (0.0f <= x || std::isnan(x)) {
        if (x < lv || std::isnan(x)) {
            float f = std::floor(x);
            int s = cvtt32(f);
            int su = s < 0 ? 0 : s;
            *start = std::min(su, levels - 1);
            *damp = x - (float)su;
        } else {
            *start = levels - 1;
            *damp = 1.0f;
        }
    } else {
        *start = 0;
        *damp = 0.0f;
    }
}

// =============================================================================================
// separable convolution (flow/conv.rs)

std::vector<float> gaussian_kernel(float r) {  // conv.rs:64-86
    int ri = std::isnan(r) ? 0 : (r >= 2147483648.0f ? INT32_MAX : (r < -2147483648.0f ? INT32_MIN : (int)r));
    long nn = (long)ri + 1;
    int n = nn < 0 ? 0 : (int)nn;
    float s3 = r / 3.0f;
    float d = s3 * s3;
    std::vector<float> k;
    float sum = 0.0f;
    for (int i = 0; i < n; i++) {
        float fi = (float)i;
        float t = fi * fi;
        float e = -(t / d);
        float v = (float)std::pow(2.0, (double)e);
        k.push_back(v);
        sum += v;
    }
    if (n == 0) return k;
    float den = sum * 2.0f - k[0];
    for (auto& v : k) v /= den;
    return k;
}

// conv.rs:101-137, border element; element t of the line at line[t * stride]
template <int C, bool LEFT_FIRST>
static inline float border_value(const float* line, long stride, int len, int i, const float* k, int n) {
    float centre = (i >= 0 && i < len) ? line[(long)i * stride] : 0.0f;
    float num = k[0] * centre;
    float den = k[0];
    for (int j = n - 1; j >= 1; j--) {
        float kj = k[j];
        for (int side = 0; side < 2; side++) {
            bool right = (side == 0) != LEFT_FIRST;
            int t = right ? i + j : i - j;
            bool inside = t >= 0 && t < len;
            float xv, w;
            if (C == 1) {
                if (inside) { xv = line[(long)t * stride]; w = kj; }
                else { xv = 0.0f; w = 0.0f; }
            } else {
                float v = inside ? line[(long)t * stride] : -1.0f;
                float mask = (v != -1.0f) ? 1.0f : 0.0f;
                xv = v;
                w = mask * kj;
            }
            den = den + w;
            num = num + xv * w;
        }
    }
    return num / den;
}

// conv.rs:141-190: one row of the horizontal pass
template <int C>
static void hrow(const float* x, float* out, int len, const float* k, int n) {
    int head = std::min(n, len);
    int interior = std::max(len - 2 * n, 0);
    for (int c = 0; c < C; c++) {
        for (int i = 0; i < head; i++) out[i * C + c] = border_value<C, false>(x + c, C, len, i, k, n);
        for (int i = head + interior; i < len; i++) out[i * C + c] = border_value<C, false>(x + c, C, len, i, k, n);
    }
    if (interior > 0) {
        int a = head * C, b = (head + interior) * C;
        float k0 = k[0];
        for (int t = a; t < b; t++) out[t] = x[t] * k0;
        for (int j = n - 1; j >= 1; j--) {
            int off = j * C;
            float kj = k[j];
            for (int t = a; t < b; t++) out[t] = out[t] + (x[t + off] + x[t - off]) * kj;
        }
    }
}

// conv.rs:268-301 (vrow_ordered); ABOVE_FIRST is the solver's order
template <int C, bool ABOVE_FIRST>
static void vrow_ordered(const float* src, float* out, int y, int w, int h, const float* k, int n) {
    long row = (long)w * C;
    int head = std::min(n, h);
    int interior = std::max(h - 2 * n, 0);
    if (y >= head && y < head + interior) {
        float k0 = k[0];
        const float* s0 = src + (long)y * row;
        for (long t = 0; t < row; t++) out[t] = s0[t] * k0;
        for (int j = n - 1; j >= 1; j--) {
            const float* below = src + (long)(y + j) * row;
            const float* above = src + (long)(y - j) * row;
            float kj = k[j];
            for (long t = 0; t < row; t++) out[t] = out[t] + (below[t] + above[t]) * kj;
        }
    } else {
        for (int xc = 0; xc < w; xc++)
            for (int c = 0; c < C; c++)
                out[xc * C + c] = border_value<C, ABOVE_FIRST>(src + (long)xc * C + c, row, h, y, k, n);
    }
}

template <int C, bool ABOVE_FIRST>
static void convolve_c(float* data, int w, int h, const float* k, int n) {
    if ((long)w * h == 0 || n == 0) return;
    std::vector<float> tmp((size_t)w * h * C);
    long row = (long)w * C;
    OMP_FOR
    for (int y = 0; y < h; y++) hrow<C>(data + y * row, tmp.data() + y * row, w, k, n);
    OMP_FOR
    for (int y = 0; y < h; y++) vrow_ordered<C, ABOVE_FIRST>(tmp.data(), data + y * row, y, w, h, k, n);
}

// conv.rs:598-615 (convolve_above_first) and conv.rs:306-318 (convolve, tap below first)
void convolve(float* data, int w, int h, int c, const float* k, int n, bool above_first) {
    if (above_first) {
        if (c == 1) convolve_c<1, true>(data, w, h, k, n);
        else if (c == 2) convolve_c<2, true>(data, w, h, k, n);
        else convolve_c<3, true>(data, w, h, k, n);
    } else {
        if (c == 1) convolve_c<1, false>(data, w, h, k, n);
        else if (c == 2) convolve_c<2, false>(data, w, h, k, n);
        else convolve_c<3, false>(data, w, h, k, n);
    }
}

void blur_gaussian(float* data, int w, int h, int c, float r, bool above_first) {  // conv.rs:618-624
    if ((double)r < 0.001) return;
    std::vector<float> k = gaussian_kernel(r);
    convolve(data, w, h, c, k.data(), (int)k.size(), above_first);
}

static const float BINOMIAL5[3] = {0.375f, 0.25f, 0.0625f};  // conv.rs:48
void blur5(float* data, int w, int h, bool above_first) { convolve(data, w, h, 1, BINOMIAL5, 3, above_first); }

// =============================================================================================
// samplers (flow/sample.rs)

static inline void cell(float x, int len, int* io, float* fo) {  // sample.rs:31-41
    int i = cvtt32(x);
    float f = x - (float)i;
    int last = len - 1;
    if (i >= last) { i = last - 1; f = 1.0f; }
    int iu = i < 0 ? 0 : i;
    int lim = len >= 2 ? len - 2 : 0;
    *io = std::min(iu, lim);
    *fo = f;
}

float bilinear1(const float* img, int w, int h, float x, float y) {  // sample.rs:47-64
    int ix, iy; float fx, fy;
    cell(x, w, &ix, &fx);
    cell(y, h, &iy, &fy);
    long i = (long)iy * w + ix;
    float p00 = img[i], p10 = img[i + 1], p01 = img[i + w], p11 = img[i + w + 1];
    float top = (p10 - p00) * fx + p00;
    float bot = (p11 - p01) * fx + p01;
    return (bot - top) * fy + top;
}

void bilinear2(const float* img, int w, int h, float x, float y, float out[2]) {  // sample.rs:69-86
    int ix, iy; float fx, fy;
    cell(x, w, &ix, &fx);
    cell(y, h, &iy, &fy);
    long i = ((long)iy * w + ix) * 2;
    long r = (long)w * 2;
    for (int c = 0; c < 2; c++) {
        float p00 = img[i + c], p10 = img[i + 2 + c], p01 = img[i + r + c], p11 = img[i + r + 2 + c];
        float top = (p10 - p00) * fx + p00;
        float bot = (p11 - p01) * fx + p01;
        out[c] = (bot - top) * fy + top;
    }
}

Plane resample1(const Plane& src, int dw, int dh) {  // sample.rs:91-112
    Plane dst(dw, dh);
    float sx = ((float)src.w - 1.0f) / (float)(dw - 1);
    float sy = ((float)src.h - 1.0f) / (float)(dh - 1);
    if (dw == 0 || dh == 0) return dst;
    OMP_FOR
    for (int y = 0; y < dh; y++) {
        float fy = (float)y * sy;
        for (int x = 0; x < dw; x++) dst.d[(size_t)y * dw + x] = bilinear1(src.d.data(), src.w, src.h, (float)x * sx, fy);
    }
    return dst;
}

// =============================================================================================
// prep (prep.rs:168-259) and the pyramid (flow.rs:242-275)

Plane luma(const Image& img, bool track_alpha, bool video_range) {
    Plane out(img.w, img.h);
    const float W30F = 0.3f, W59F = 0.59f, W11F = 0.11f;
    const double W30D = 0.3, W59D = 0.59, W11D = 0.11;
    long n = (long)img.w * img.h;
    if (img.fmt == U8) {
        OMP_FOR
        for (long i = 0; i < n; i++) {
            const uint8_t* px = &img.u8[i * 4];
            float a = (float)px[0], r = (float)px[1], g = (float)px[2], b = (float)px[3];
            float v;
            if (video_range) v = ((r - 16.0f) * 255.0f) / 219.0f;
            else {
                float sum = (r * W30F + g * W59F) + b * W11F;
                v = track_alpha ? (float)((double)sum + (double)a * W30D) : sum;
            }
            out.d[i] = v;
        }
    } else if (img.fmt == U16) {
        OMP_FOR
        for (long i = 0; i < n; i++) {
            const uint16_t* px = &img.u16[i * 4];
            double a = px[0], r = px[1], g = px[2], b = px[3];
            float v;
            if (video_range) v = (((float)px[1] / 257.0f - 16.0f) * 255.0f) / 219.0f;
            else {
                double sum = (g * W59D + r * W30D) + b * W11D;
                if (track_alpha) sum += a * W30D;
                v = (float)(sum / 257.0);
            }
            out.d[i] = v;
        }
    } else {
        OMP_FOR
        for (long i = 0; i < n; i++) {
            const float* px = &img.f32[i * 4];
            double a = px[0], r = px[1], g = px[2], b = px[3];
            float v;
            if (video_range) v = ((px[1] * 255.0f - 16.0f) * 255.0f) / 219.0f;
            else {
                double sum = (g * W59D + r * W30D) + b * W11D;
                if (track_alpha) sum += a * W30D;
                v = (float)(sum * 255.0);
            }
            out.d[i] = v;
        }
    }
    return out;
}

// crt_powf.rs:229-268: the plugin runtime's single precision powf for a positive finite base (a
// logarithm and an exponential in double precision from tables, narrowed once), the rounded double
// precision pow elsewhere. The tables are the closed forms of the generator beside the library's
// sources (1/c, ln 2c, 2^(j/64)).
float crt_powf(float x, float y) {
    static const uint64_t RCP[257] = TW_POW_RCP_INIT;
    static const uint64_t LOG[257] = TW_POW_LOG_INIT;
    static const uint64_t EXP2[64] = TW_POW_EXP2_INIT;
    auto d = [](uint64_t b) { double v; std::memcpy(&v, &b, 8); return v; };
    auto u = [](double v) { uint64_t b; std::memcpy(&b, &v, 8); return b; };
    if (!(x > 0.0f) || !std::isfinite(x) || !std::isfinite(y) || y == 0.0f || y == 1.0f)
        return (float)std::pow((double)x, (double)y);
    double xd = x, yd = y;
    double t = xd - 1.0;
    double l;
    if (x < 1.0625f && std::fabs(t) < 0.0625) {
        double sv = t / (t + 2.0);
        double st = sv * t;
        double uu = sv + sv;
        double z = uu * uu;
        double t0 = z * d(TW_POW_C0), t1 = z * d(TW_POW_C1);
        double uz = uu * z;
        double u0 = t0 + d(TW_POW_A0), u1 = t1 + d(TW_POW_A1);
        double uz3 = (z * z) * uz;
        double sum = uz * u0 + uz3 * u1;
        l = t + (sum - st);
    } else {
        uint64_t mant = u(xd) & 0x000fffffffffffffull;
        size_t idx = (size_t)((mant >> 44) + ((mant >> 43) & 1));
        double c = d(((uint64_t)idx | 0x3fe00ull) << 44);
        double m = d(mant | 0x3fe0000000000000ull);
        int64_t e = (int64_t)((u(xd) & 0x7ff0000000000000ull) >> 52) - 1023;
        double r = (c - m) * d(RCP[idx]);
        double q = r + (r * r) * (r * d(TW_POW_THIRD) + 0.5);
        double el = (double)e * d(TW_POW_LN2);
        l = (el + d(LOG[idx])) - q;
    }
    double w = yd * l;
    if (w > d(TW_POW_LIM_HI) || w <= d(TW_POW_LIM_LO)) return (float)std::pow(xd, yd);
    int32_t n = (int32_t)std::nearbyint(w * d(TW_POW_K64));
    double r = w - (double)n * d(TW_POW_LN2_64);
    double p = (r * r) * (r * d(TW_POW_SIXTH) + 0.5) + r;
    double tj = d(EXP2[n & 63]);
    double v = p * tj + tj;
    uint64_t k = (uint64_t)(uint32_t)(n >> 6);
    return (float)d(u(v) + (k << 52));
}

// prep.rs:296-307 (delinearize): p = powf(max(p, 0) / 255, 1 / 2.2) * 255; -0.0 stays
void delinearize(Plane& p) {
    const float inv = 1.0f / 2.2f;
    for (auto& v : p.d) {
        if (v <= 0.0f && v != 0.0f) v = 0.0f;
        float base = v / 255.0f;
        v = crt_powf(base, inv) * 255.0f;
    }
}

// prep.rs:326-340 (edge_enhance): the Gaussian of radius 2.0, the solver's gradient, then per pixel
// m = sqrt(gx^2 + gy^2), f = m <= 20 ? m * 0.05 : 1, p = (f * 255 + p) * 0.5
void edge_enhance(Plane& p, bool above_first) {
    blur_gaussian(p.d.data(), p.w, p.h, 1, 2.0f, above_first);
    std::vector<float> g = calc_grad(p.d.data(), p.w, p.h);
    for (size_t i = 0; i < p.d.size(); i++) {
        float gx = g[i * 2], gy = g[i * 2 + 1];
        float m = std::sqrt(gx * gx + gy * gy);
        float f = m <= 20.0f ? m * 0.05f : 1.0f;
        p.d[i] = (f * 255.0f + p.d[i]) * 0.5f;
    }
}

std::vector<float> calc_grad_wrap(const float* img, int w, int h);
void blur_gaussian_wrap(float* data, int w, int h, int c, float r);

// prep.rs:377-398 (edge_enhance_with, wrap): the 360 Gaussian of radius 2.0 and the 360 gradient,
// then the plain per pixel step
static void edge_enhance_wrap(Plane& p) {
    blur_gaussian_wrap(p.d.data(), p.w, p.h, 1, 2.0f);
    std::vector<float> g = calc_grad_wrap(p.d.data(), p.w, p.h);
    for (size_t i = 0; i < p.d.size(); i++) {
        float gx = g[i * 2], gy = g[i * 2 + 1];
        float m = std::sqrt(gx * gx + gy * gy);
        float f = m <= 20.0f ? m * 0.05f : 1.0f;
        p.d[i] = (f * 255.0f + p.d[i]) * 0.5f;
    }
}

// conv.rs:192-244 (hrow_wrapx): every sample s = x[i] k0, then s = s + (x[(i+j) mod w] + x[(i-j) mod w]) k[j]
// for j = n-1 down to 1 (the interior run is the same chain without a wrap); c interleaved channels
static void hpass_wrapx(const float* src, float* dst, int w, int h, int c, const float* k, int n) {
    OMP_FOR
    for (int y = 0; y < h; y++) {
        const float* x = src + (long)y * w * c;
        for (int i = 0; i < w; i++) {
            for (int ch = 0; ch < c; ch++) {
                float sum = x[(long)i * c + ch] * k[0];
                for (int j = n - 1; j >= 1; j--) {
                    int r = (i + j) % w;
                    int l = ((i - j) % w + w) % w;
                    sum = sum + (x[(long)r * c + ch] + x[(long)l * c + ch]) * k[j];
                }
                dst[((long)y * w + i) * c + ch] = sum;
            }
        }
    }
}

// conv.rs:326-400 (vpass_sphere): each column padded by n - 1 elements at both ends with the
// equirectangular walk (reflect at the edge row, move half a turn in x), then the plain chain
static void vpass_sphere(const float* src, float* dst, int w, int h, int c, const float* k, int n) {
    int half = w / 2, pad = n - 1;
    OMP_FOR
    for (int x = 0; x < w; x++) {
        auto walk = [&](int start, int dir, int steps, std::vector<std::pair<int, int>>& out) {
            int cc = x, r = start, d = dir;
            for (int m = 0; m < steps; m++) {
                r += d;
                if (r < 0) { r = 0; d = -d; cc = (half + cc) % w; }
                else if (r >= h) { r = h - 1; d = -d; cc = (half + cc) % w; }
                out.push_back({cc, r});
            }
        };
        std::vector<std::pair<int, int>> up, down;
        walk(0, -1, pad, up);
        walk(h - 1, 1, pad, down);
        std::vector<float> g((size_t)h + 2 * pad);
        for (int ch = 0; ch < c; ch++) {
            auto at = [&](int cc, int r) { return src[((long)r * w + cc) * c + ch]; };
            for (int m = 0; m < pad; m++) g[pad - 1 - m] = at(up[m].first, up[m].second);
            for (int r = 0; r < h; r++) g[pad + r] = at(x, r);
            for (int m = 0; m < pad; m++) g[pad + h + m] = at(down[m].first, down[m].second);
            for (int y = 0; y < h; y++) {
                int e = pad + y;
                float sum = g[e] * k[0];
                for (int j = n - 1; j >= 1; j--) sum = sum + (g[e + j] + g[e - j]) * k[j];
                dst[((long)y * w + x) * c + ch] = sum;
            }
        }
    }
}

// conv.rs:646-660 (convolve_wrapx_above_first): the circular horizontal pass, then the column walk
// over the poles
void convolve_wrapx_sphere(float* data, int w, int h, const float* k, int n, int c) {
    if (w == 0 || h == 0 || n == 0) return;
    std::vector<float> tmp((size_t)w * h * c);
    hpass_wrapx(data, tmp.data(), w, h, c, k, n);
    vpass_sphere(tmp.data(), data, w, h, c, k, n);
}

// conv.rs:662-668 (blur_gaussian_wrapx_above_first)
void blur_gaussian_wrap(float* data, int w, int h, int c, float r) {
    if ((double)r < 0.001) return;
    std::vector<float> k = gaussian_kernel(r);
    convolve_wrapx_sphere(data, w, h, k.data(), (int)k.size(), c);
}

// sample.rs:255-286 (bilinear1_sphere)
static float bilinear1_sphere(const float* img, int w, int h, float x, float y) {
    int w1 = w - 1, h1 = h - 1;
    int tx = cvtt32(x), ty = cvtt32(y);
    int ix = std::min(std::max(tx, 0), w1), iy = std::min(std::max(ty, 0), h1);
    float fx = x - (float)tx, fy = y - (float)ty;
    int x1 = ix + 1 > w1 ? 0 : ix + 1;
    int xc = ix, xd = x1, yc = iy + 1;
    if (iy + 1 > h1) {
        int half = w / 2;
        xc = (half + ix) % w;
        xd = (half + x1) % w;
        yc = h1;
    }
    float p00 = img[(long)iy * w + ix], p10 = img[(long)iy * w + x1];
    float p01 = img[(long)yc * w + xc], p11 = img[(long)yc * w + xd];
    float top = (p10 - p00) * fx + p00;
    float bot = (p11 - p01) * fx + p01;
    return (bot - top) * fy + top;
}

Plane resample1_wrapx(const Plane& src, int dw, int dh) {
    Plane d;
    d.w = dw;
    d.h = dh;
    d.d.assign((size_t)dw * dh, 0.0f);
    if (dw == 0 || dh == 0) return d;
    float sx = (float)src.w / (float)dw, sy = (float)src.h / (float)dh;
    OMP_FOR
    for (int y = 0; y < dh; y++) {
        float fy = (float)y * sy;
        for (int x = 0; x < dw; x++) d.d[(long)y * dw + x] = bilinear1_sphere(src.d.data(), src.w, src.h, (float)x * sx, fy);
    }
    return d;
}

// prep.rs:261-299 with wrap: blur5_wrapx_above_first (conv.rs:662) and resample1_wrapx
static void blur5_wrap(Plane& p) { convolve_wrapx_sphere(p.d.data(), p.w, p.h, BINOMIAL5, 3); }

Plane reduce(Plane t, int r, bool above_first) {  // prep.rs:252-259
    for (int i = 0; i < r; i++) {
        blur5(t.d.data(), t.w, t.h, above_first);
        int nw = t.w / 2, nh = t.h / 2;
        t = resample1(t, nw, nh);
    }
    return t;
}

bool build_pyramid(const Image& img, const FlowSettings& s, Pyramid* out, std::string* err) {
    if (!geometry(s, img.w, img.h, &out->geo, err)) return false;
    if (s.video_range_luma && s.track_alpha) { *err = "video range luma with track alpha"; return false; }
    Plane orig = luma(img, s.track_alpha, s.video_range_luma);
    if (s.wrap) {  // prep.rs:288-299 (reduce_with)
        for (int r = 0; r < out->geo.reduction; r++) {
            blur5_wrap(orig);
            orig = resample1_wrapx(orig, orig.w / 2, orig.h / 2);
        }
    } else {
        orig = reduce(std::move(orig), out->geo.reduction, s.taps_above_first);
    }
    if (s.prep_delinearize) delinearize(orig);  // flow.rs:248-253: Delinearize, then Contrast/Edge
    if (s.prep_contrast_edge) {
        if (s.wrap) edge_enhance_wrap(orig);
        else edge_enhance(orig, s.taps_above_first);
    }
    int n = out->geo.levels;
    out->levels.clear();
    for (int i = 0; i < n; i++) {
        Plane tmp = orig;
        if (s.wrap) blur5_wrap(tmp);
        else blur5(tmp.d.data(), tmp.w, tmp.h, s.taps_above_first);
        Plane next;
        bool has_next = i + 1 < n;
        if (has_next) {
            int nw = out->geo.sizes[i + 1].first, nh = out->geo.sizes[i + 1].second;
            next = s.wrap ? resample1_wrapx(tmp, nw, nh) : resample1(tmp, nw, nh);
        }
        Plane band = orig;
        for (size_t k = 0; k < band.d.size(); k++) band.d[k] = band.d[k] - tmp.d[k];
        out->levels.push_back(std::move(band));
        if (!has_next) break;
        orig = std::move(next);
    }
    return true;
}

// =============================================================================================
// solver kernels (flow.rs:277-442)

std::vector<float> calc_grad(const float* img, int w, int h) {  // flow.rs:283-316
    std::vector<float> g((size_t)w * h * 2, 0.0f);
    if (w == 0 || h == 0) return g;
    OMP_FOR
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            float c = img[(long)y * w + x];
            float nx = 0.0f, dx = 0.0f, ny = 0.0f, dy = 0.0f;
            if (x >= 1) { nx = (c - img[(long)y * w + x - 1]) + 0.0f; dx = 1.0f; }
            if (y >= 1) { ny = (c - img[(long)(y - 1) * w + x]) + 0.0f; dy = 1.0f; }
            if (x + 1 <= w - 1) { nx = nx + (img[(long)y * w + x + 1] - c); dx = dx + 1.0f; }
            if (y + 1 <= h - 1) { ny = ny + (img[(long)(y + 1) * w + x] - c); dy = dy + 1.0f; }
            g[((long)y * w + x) * 2] = nx / dx;
            g[((long)y * w + x) * 2 + 1] = ny / dy;
        }
    }
    return g;
}

std::vector<float> calc_a(const std::vector<float>& grad, int w, int h) {  // flow.rs:319-328
    std::vector<float> a((size_t)w * h * 3);
    long n = (long)w * h;
    OMP_FOR
    for (long i = 0; i < n; i++) {
        float gx = grad[i * 2], gy = grad[i * 2 + 1];
        a[i * 3] = gx * gx;
        a[i * 3 + 1] = gx * gy;
        a[i * 3 + 2] = gy * gy;
    }
    return a;
}

std::vector<float> calc_b(const float* i1, const float* i0, const float* grad, const float* flow, int w,
                          int h) {  // flow.rs:334-357
    std::vector<float> b((size_t)w * h * 2, 0.0f);
    float fw = (float)w, fh = (float)h;
    OMP_FOR
    for (int y = 0; y < h; y++) {
        float fy = (float)y;
        for (int x = 0; x < w; x++) {
            float fx = (float)x;
            long i = (long)y * w + x;
            float sx = fx - flow[i * 2];
            float sy = fy - flow[i * 2 + 1];
            if (sx < 0.0f || fw - 1.0f < sx || sy < 0.0f || fh - 1.0f < sy) {
                b[i * 2] = 0.0f;
                b[i * 2 + 1] = 0.0f;
            } else {
                float s = bilinear1(i0, w, h, sx, sy);
                float r = s - i1[i];
                b[i * 2] = r * grad[i * 2];
                b[i * 2 + 1] = r * grad[i * 2 + 1];
            }
        }
    }
    return b;
}

void new_disp(float* flow, const float* a, const float* b, size_t npx) {  // flow.rs:361-371
    OMP_FOR
    for (long i = 0; i < (long)npx; i++) {
        float aa = a[i * 3], ab = a[i * 3 + 1], ad = a[i * 3 + 2];
        float bx = b[i * 2], by = b[i * 2 + 1];
        float t = ab * ab - ad * aa;
        if (std::fabs(t) > 40.0f) {
            flow[i * 2] = (ab * by - ad * bx) / t + flow[i * 2];
            flow[i * 2 + 1] = (ab * bx - aa * by) / t + flow[i * 2 + 1];
        }
    }
}

std::vector<float> upsample_flow(const float* src, int sw, int sh, int dw, int dh) {  // flow.rs:376-391
    float sx = ((float)dw - 1.0f) / (float)(sw - 1);
    float sy = ((float)dh - 1.0f) / (float)(sh - 1);
    float rx = (float)(1.0 / (double)sx);
    float ry = (float)(1.0 / (double)sy);
    std::vector<float> dst((size_t)dw * dh * 2, 0.0f);
    OMP_FOR
    for (int y = 0; y < dh; y++) {
        float fy = (float)y * ry;
        for (int x = 0; x < dw; x++) {
            float v[2];
            bilinear2(src, sw, sh, (float)x * rx, fy, v);
            dst[((long)y * dw + x) * 2] = v[0] * sx;
            dst[((long)y * dw + x) * 2 + 1] = v[1] * sy;
        }
    }
    return dst;
}

void scale_values(float* d, size_t n, float f) {  // flow.rs:422-427
    if (f == 1.0f) return;
    for (size_t i = 0; i < n; i++) d[i] = f * d[i];
}

bool all_flow_out_of_range(const float* flow, int w, int h) {  // flow.rs:430-442
    float fw = (float)(w - 1), fh = (float)(h - 1);
    for (int y = 0; y < h; y++) {
        float fy = (float)y;
        for (int x = 0; x < w; x++) {
            float px = (float)x + flow[((long)y * w + x) * 2];
            float py = fy + flow[((long)y * w + x) * 2 + 1];
            if (0.0f <= px && px <= fw && 0.0f <= py && py <= fh) return false;
        }
    }
    return true;
}

// flow.rs:474-523 (Block::cost)
float block_cost(const float* a, const float* b, int w, int h, const float p[9], float x2, float y2, bool* some) {
    (void)a;
    float wm2 = (float)(w - 2), hm2 = (float)(h - 2);
    *some = false;
    if (x2 > wm2 || y2 > hm2) return 0.0f;
    int ix, iy; float fx, fy;
    if (x2 == wm2) { ix = cvtt32(wm2 - 1.0f); fx = 1.0f; }
    else { ix = cvtt32(x2); fx = x2 - (float)ix; }
    if (y2 == hm2) { iy = cvtt32(hm2 - 1.0f); fy = 1.0f; }
    else { iy = cvtt32(y2); fy = y2 - (float)iy; }
    if (ix < 1 || iy < 1) return 0.0f;
    float w11 = fy * fx;
    float w10 = fx - w11;
    float w01 = fy - w11;
    float w00 = ((1.0f - fx) - fy) + w11;
    const float* base = b + (long)(iy - 1) * w + ix - 1;
    float sq[9];
    int n = 0;
    for (int bb = 0; bb < 3; bb++) {
        for (int aa = 0; aa < 3; aa++) {
            const float* t = base + (long)bb * w + aa;
            float qv = ((w00 * t[0] + w10 * t[1]) + w01 * t[w]) + w11 * t[w + 1];
            float d = p[n] - qv;
            sq[n] = d * d;
            n++;
        }
    }
    float s = sq[0] + sq[1];
    for (int k = 2; k < 8; k++) s = s + sq[k];
    *some = true;
    return sq[8] + s;
}

// flow.rs:529-546 (Block::step); returns true when the neighbour replaces the vector
static inline bool bm_step(const float* a, const float* b, int w, int h, int x, int y, const float cur[2],
                           const float nb[2]) {
    float tx = (float)x - cur[0];
    float ty = (float)y - cur[1];
    float w1 = (float)(w - 1), h1 = (float)(h - 1);
    if (0.0f <= tx && tx <= w1 && 0.0f <= ty && ty <= h1) {
        float p[9];
        const float* pa = a + (long)(y - 1) * w + x - 1;
        p[0] = pa[0]; p[1] = pa[1]; p[2] = pa[2];
        p[3] = pa[w]; p[4] = pa[w + 1]; p[5] = pa[w + 2];
        p[6] = pa[2 * w]; p[7] = pa[2 * w + 1]; p[8] = pa[2 * w + 2];
        bool s0, s1;
        float c0 = block_cost(a, b, w, h, p, tx, ty, &s0);
        if (s0) {
            float c1 = block_cost(a, b, w, h, p, (float)x - nb[0], (float)y - nb[1], &s1);
            if (s1 && c1 < c0) return true;
        }
    }
    return false;
}

void block_match(const float* a, const float* b, float* flow, int w, int h) {  // flow.rs:551-622
    block_match_gated(a, b, flow, w, h, nullptr);
}

// flow.rs:1225-1245 without wrap: a pixel whose gate value is below 0.95 keeps its vector
void block_match_gated(const float* a, const float* b, float* flow, int w, int h, const float* gate) {
    if (w < 3 || h < 3) return;
    auto bm_step = [&](const float* A, const float* B, int W, int H, int x, int y, const float* cur, float* nb) {
        if (gate && gate[(long)y * W + x] < 0.95f) return false;
        return ::orc::bm_step(A, B, W, H, x, y, cur, nb);
    };
    OMP_FOR
    for (int y = 1; y <= h - 2; y++) {
        float* row = flow + (long)y * w * 2;
        for (int x = 1; x <= w - 2; x++) {
            float cur[2] = {row[x * 2], row[x * 2 + 1]};
            float nb[2] = {row[(x - 1) * 2], row[(x - 1) * 2 + 1]};
            if (bm_step(a, b, w, h, x, y, cur, nb)) { row[x * 2] = nb[0]; row[x * 2 + 1] = nb[1]; }
        }
    }
    OMP_FOR
    for (int y = 1; y <= h - 2; y++) {
        float* row = flow + (long)y * w * 2;
        for (int x = w - 2; x >= 1; x--) {
            float cur[2] = {row[x * 2], row[x * 2 + 1]};
            float nb[2] = {row[(x + 1) * 2], row[(x + 1) * 2 + 1]};
            if (bm_step(a, b, w, h, x, y, cur, nb)) { row[x * 2] = nb[0]; row[x * 2 + 1] = nb[1]; }
        }
    }
    // the column sweeps run in place on the field; the reference transposes for contiguity only
    OMP_FOR
    for (int x = 1; x <= w - 2; x++) {
        for (int y = 1; y <= h - 2; y++) {
            float* c = flow + ((long)y * w + x) * 2;
            float* p = flow + ((long)(y - 1) * w + x) * 2;
            float cur[2] = {c[0], c[1]};
            float nb[2] = {p[0], p[1]};
            if (bm_step(a, b, w, h, x, y, cur, nb)) { c[0] = nb[0]; c[1] = nb[1]; }
        }
    }
    OMP_FOR
    for (int x = 1; x <= w - 2; x++) {
        for (int y = h - 2; y >= 1; y--) {
            float* c = flow + ((long)y * w + x) * 2;
            float* p = flow + ((long)(y + 1) * w + x) * 2;
            float cur[2] = {c[0], c[1]};
            float nb[2] = {p[0], p[1]};
            if (bm_step(a, b, w, h, x, y, cur, nb)) { c[0] = nb[0]; c[1] = nb[1]; }
        }
    }
}

// flow.rs:743-761 (wrap off): the gradient is zero where the level mask is below 0.95 at the pixel
// or at one of its four neighbours that exist
void mask_gradient(float* grad, const float* mask, int w, int h) {
    OMP_FOR
    for (int y = 0; y < h; y++) {
        auto off = [&](int xx, int yy) { return mask[(long)yy * w + xx] < 0.95f; };
        for (int x = 0; x < w; x++) {
            bool out = off(x, y) || (y >= 1 && off(x, y - 1)) || (y + 1 < h && off(x, y + 1)) || (x >= 1 && off(x - 1, y)) ||
                       (x + 1 < w && off(x + 1, y));
            if (out) { grad[((long)y * w + x) * 2] = 0.0f; grad[((long)y * w + x) * 2 + 1] = 0.0f; }
        }
    }
}

// flow.rs:777-845 (wrap off): calc_b with the warped mask of Y at least 0.999 at the target
std::vector<float> calc_b_masked(const float* i1, const float* i0, const float* grad, const float* flow, int w, int h,
                                 const float* mask_y) {
    std::vector<float> b((size_t)w * h * 2, 0.0f);
    float fw = (float)w, fh = (float)h;
    OMP_FOR
    for (int y = 0; y < h; y++) {
        float fy = (float)y;
        for (int x = 0; x < w; x++) {
            float fx = (float)x;
            long i = (long)y * w + x;
            float sx = fx - flow[i * 2], sy = fy - flow[i * 2 + 1];
            bool inside = !(sx < 0.0f || fw - 1.0f < sx || sy < 0.0f || fh - 1.0f < sy);
            bool pass = inside && (!mask_y || bilinear1(mask_y, w, h, sx, sy) >= 0.999f);
            if (pass) {
                float r = bilinear1(i0, w, h, sx, sy) - i1[i];
                b[i * 2] = r * grad[i * 2];
                b[i * 2 + 1] = r * grad[i * 2 + 1];
            }
        }
    }
    return b;
}

// ---- the wrap-around (360) solve (flow.rs:625-1246 with flow/extras.rs:286-430) ----------------

// flow.rs:661-690 (sphere_target): x into [0, fw) and y into [0, fh) one period at a time; an odd
// count of vertical periods moves x half a turn and mirrors y (unless it is 0). Non-finite
// positions are returned as they are. The loops are bounded: a finite position past 2^25 periods
// would not move (x + fw == x there) and is returned as it is, where the reference's loop would
// not end.
static inline void sphere_target(float& x, float& y, float fw, float fh) {
    if (!(std::isfinite(x) && std::isfinite(y)) || !(fw > 0.0f && fh > 0.0f)) return;
    const long cap = 1L << 25;
    float x0 = x, y0 = y;
    long m = 0;
    while (x < 0.0f && m < cap) { x = x + fw; m++; }
    while (fw <= x && m < cap) { x = x - fw; m++; }
    unsigned n = 0;
    while (y < 0.0f && m < cap) { y = y + fh; n++; m++; }
    while (fh <= y && m < cap) { y = y - fh; n++; m++; }
    if (m >= cap) { x = x0; y = y0; return; }
    if (n % 2 == 1) {
        x = fw * 0.5f + x;
        if (fw <= x) x = x - fw;
        if (y != 0.0f) y = fh - y;
    }
}

// sample.rs:231-252 (bilinear2_sphere): bilinear1_sphere on (dx, dy) pairs
static void bilinear2_sphere(const float* img, int w, int h, float x, float y, float out[2]) {
    int w1 = w - 1, h1 = h - 1;
    int tx = cvtt32(x), ty = cvtt32(y);
    int ix = std::min(std::max(tx, 0), w1), iy = std::min(std::max(ty, 0), h1);
    float fx = x - (float)tx, fy = y - (float)ty;
    int x1 = ix + 1 > w1 ? 0 : ix + 1;
    int xc = ix, xd = x1, yc = iy + 1;
    if (iy + 1 > h1) {
        int half = w / 2;
        xc = (half + ix) % w;
        xd = (half + x1) % w;
        yc = h1;
    }
    for (int c = 0; c < 2; c++) {
        float p00 = img[((long)iy * w + ix) * 2 + c], p10 = img[((long)iy * w + x1) * 2 + c];
        float p01 = img[((long)yc * w + xc) * 2 + c], p11 = img[((long)yc * w + xd) * 2 + c];
        float top = (p10 - p00) * fx + p00;
        float bot = (p11 - p01) * fx + p01;
        out[c] = (bot - top) * fy + top;
    }
}

// flow.rs:716-741 (calc_grad_wrap): central differences times 0.5, the columns modulo the width;
// above row 0 and below row h - 1 the same edge row half a turn away
std::vector<float> calc_grad_wrap(const float* img, int w, int h) {
    std::vector<float> g((size_t)w * h * 2, 0.0f);
    if (w == 0 || h == 0) return g;
    OMP_FOR
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            float c = img[(long)y * w + x];
            float left = img[(long)y * w + (x + w - 1) % w];
            float right = img[(long)y * w + (x + 1) % w];
            int pole = (w / 2 + x) % w;
            float up = y >= 1 ? img[(long)(y - 1) * w + x] : img[pole];
            float down = y + 1 <= h - 1 ? img[(long)(y + 1) * w + x] : img[(long)(h - 1) * w + pole];
            g[((long)y * w + x) * 2] = ((c - left) + (right - c)) * 0.5f;
            g[((long)y * w + x) * 2 + 1] = ((c - up) + (down - c)) * 0.5f;
        }
    }
    return g;
}

// flow.rs:743-761 with wrap: the left and right neighbours of the mask test modulo the width
static void mask_gradient_wrap(float* grad, const float* mask, int w, int h) {
    OMP_FOR
    for (int y = 0; y < h; y++) {
        auto off = [&](int xx, int yy) { return mask[(long)yy * w + xx] < 0.95f; };
        for (int x = 0; x < w; x++) {
            bool out = off(x, y) || (y >= 1 && off(x, y - 1)) || (y + 1 < h && off(x, y + 1)) || off((x + w - 1) % w, y) ||
                       off((x + 1) % w, y);
            if (out) { grad[((long)y * w + x) * 2] = 0.0f; grad[((long)y * w + x) * 2 + 1] = 0.0f; }
        }
    }
}

// flow.rs:777-822 (calc_b_with, wrap): a flow of a whole width or height or more gives B = 0; else
// the target (x - u, y - v) goes onto the sphere and is sampled with the 360 sampler (the warped
// mask of Y, when given, at least 0.999 there)
static std::vector<float> calc_b_wrap(const float* i1, const float* i0, const float* grad, const float* flow, int w, int h,
                                      const float* mask_y) {
    std::vector<float> b((size_t)w * h * 2, 0.0f);
    float fw = (float)w, fh = (float)h;
    OMP_FOR
    for (int y = 0; y < h; y++) {
        float fy = (float)y;
        for (int x = 0; x < w; x++) {
            long i = (long)y * w + x;
            float u = flow[i * 2], v = flow[i * 2 + 1];
            if (fw <= std::fabs(u) || fh <= std::fabs(v)) continue;
            float sx = (float)x - u, sy = fy - v;
            sphere_target(sx, sy, fw, fh);
            if (mask_y && !(bilinear1_sphere(mask_y, w, h, sx, sy) >= 0.999f)) continue;
            float r = bilinear1_sphere(i0, w, h, sx, sy) - i1[i];
            b[i * 2] = r * grad[i * 2];
            b[i * 2 + 1] = r * grad[i * 2 + 1];
        }
    }
    return b;
}

// flow.rs:862-884 (Block::patch_sphere): the 3x3 patch of A, each column modulo the width, each
// row brought into [0, 2h) and past the last row mirrored onto the column half a turn away
static void patch_sphere(const float* a, int w, int h, int x, int y, float p[9]) {
    int n = 0;
    for (int dy = -1; dy <= 1; dy++) {
        for (int dx = -1; dx <= 1; dx++) {
            int c = ((x + dx) % w + w) % w;
            int r = ((y + dy) % (2 * h) + 2 * h) % (2 * h);
            if (r > h - 1) {
                c += w / 2;
                if (c >= w) c -= w;
                r = 2 * h - r - 1;
            }
            p[n++] = a[(long)r * w + c];
        }
    }
}

// flow.rs:891-911 (Block::cost_sphere): the target on the sphere, the nine positions around it each
// on the sphere again, sampled with the 360 sampler; d8^2 + ((d0^2 + d1^2) + ... + d7^2)
static float cost_sphere(const float* b, int w, int h, const float p[9], float tx, float ty) {
    float fw = (float)w, fh = (float)h;
    sphere_target(tx, ty, fw, fh);
    float xs[3] = {tx - 1.0f, tx, tx + 1.0f}, ys[3] = {ty - 1.0f, ty, ty + 1.0f};
    float sq[9];
    int n = 0;
    for (int j = 0; j < 3; j++) {
        for (int i = 0; i < 3; i++) {
            float sx = xs[i], sy = ys[j];
            sphere_target(sx, sy, fw, fh);
            float d = p[n] - bilinear1_sphere(b, w, h, sx, sy);
            sq[n++] = d * d;
        }
    }
    float s = sq[0];
    for (int k = 1; k < 8; k++) s = s + sq[k];
    return sq[8] + s;
}

// flow.rs:916-925 (Block::step_sphere): no range check, the neighbour wins on a smaller cost
static inline bool bm_step_sphere(const float* a, const float* b, int w, int h, int x, int y, const float cur[2],
                                  const float nb[2]) {
    float p[9];
    patch_sphere(a, w, h, x, y, p);
    float c0 = cost_sphere(b, w, h, p, (float)x - cur[0], (float)y - cur[1]);
    float c1 = cost_sphere(b, w, h, p, (float)x - nb[0], (float)y - nb[1]);
    return c1 < c0;
}

// flow.rs:1087-1145 (sweeps_sphere) through flow.rs:1225-1245 (block_match_with, wrap): the two row
// sweeps over every row and every column in place (the left neighbour modulo the width with the
// columns increasing, then the right one with the columns decreasing) with the 360 step, then the
// two column sweeps of the plain block matching; a pixel whose gate value is below 0.95 keeps its
// vector
void block_match_sphere(const float* a, const float* b, float* flow, int w, int h, const float* gate) {
    if (w < 3 || h < 3) return;
    auto gated = [&](int x, int y) { return gate && gate[(long)y * w + x] < 0.95f; };
    for (int right = 0; right < 2; right++) {
        OMP_FOR
        for (int y = 0; y < h; y++) {
            float* row = flow + (long)y * w * 2;
            for (int m = 0; m < w; m++) {
                int x = right ? w - 1 - m : m;
                int nx = right ? (x + 1) % w : (x + w - 1) % w;
                float cur[2] = {row[x * 2], row[x * 2 + 1]};
                float nb[2] = {row[nx * 2], row[nx * 2 + 1]};
                if (!gated(x, y) && bm_step_sphere(a, b, w, h, x, y, cur, nb)) { row[x * 2] = nb[0]; row[x * 2 + 1] = nb[1]; }
            }
        }
    }
    for (int below = 0; below < 2; below++) {
        OMP_FOR
        for (int x = 1; x <= w - 2; x++) {
            for (int m = 1; m <= h - 2; m++) {
                int y = below ? h - 1 - m : m;
                float* c = flow + ((long)y * w + x) * 2;
                float* q = flow + ((long)(below ? y + 1 : y - 1) * w + x) * 2;
                float cur[2] = {c[0], c[1]};
                float nb[2] = {q[0], q[1]};
                if (!gated(x, y) && bm_step(a, b, w, h, x, y, cur, nb)) { c[0] = nb[0]; c[1] = nb[1]; }
            }
        }
    }
}

// flow.rs:401-420 (upsample_flow_wrapx): the scales dw / sw and dh / sh, the steps their double
// reciprocals narrowed, the 2 channel 360 sampler
std::vector<float> upsample_flow_wrapx(const float* src, int sw, int sh, int dw, int dh) {
    float sx = (float)dw / (float)sw, sy = (float)dh / (float)sh;
    float rx = (float)(1.0 / (double)sx), ry = (float)(1.0 / (double)sy);
    std::vector<float> dst((size_t)dw * dh * 2, 0.0f);
    OMP_FOR
    for (int y = 0; y < dh; y++) {
        float fy = (float)y * ry;
        for (int x = 0; x < dw; x++) {
            float v[2];
            bilinear2_sphere(src, sw, sh, (float)x * rx, fy, v);
            dst[((long)y * dw + x) * 2] = v[0] * sx;
            dst[((long)y * dw + x) * 2 + 1] = v[1] * sy;
        }
    }
    return dst;
}

static void binarize(Plane& p) {  // flow/extras.rs:64-72 (a NaN gives 0)
    for (auto& v : p.d) v = v >= 0.95f ? 1.0f : 0.0f;
}

// flow/extras.rs:76-123: the binary mask pyramid of a matte (values 0..1, the output size)
bool mask_pyramid(const float* matte, int w, int h, const FlowSettings& s, std::vector<Plane>* levels, std::string* err) {
    Geometry g;
    if (!geometry(s, w, h, &g, err)) return false;
    Plane cur(w, h);
    std::memcpy(cur.d.data(), matte, sizeof(float) * (size_t)w * h);
    binarize(cur);
    auto step = [&](const Plane& p, int nw, int nh) {  // flow/extras.rs:76-85 (mask_step; wrap: the 360 passes)
        Plane t = p;
        if (s.wrap) blur5_wrap(t);
        else blur5(t.d.data(), t.w, t.h, s.taps_above_first);
        Plane r = s.wrap ? resample1_wrapx(t, nw, nh) : resample1(t, nw, nh);
        binarize(r);
        return r;
    };
    for (int i = 0; i < g.reduction; i++) cur = step(cur, cur.w / 2, cur.h / 2);
    levels->clear();
    for (int i = 0; i < g.levels; i++) {
        Plane next;
        bool has_next = i + 1 < g.levels;
        if (has_next) next = step(cur, g.sizes[i + 1].first, g.sizes[i + 1].second);
        levels->push_back(std::move(cur));
        if (!has_next) break;
        cur = std::move(next);
    }
    return true;
}

// flow.rs:1258-1307
FlowField solve_pyramids(const Pyramid& x, const Pyramid& y, const FlowSettings& s) {
    return solve_pyramids_masked(x, y, s, nullptr, nullptr, false);
}

// flow/extras.rs:244-430 without user displacement and wrap: the plain driver with the gradient
// masked by X's level mask, the B step gated by Y's warped level mask, and (gate) the block
// matching sweeps gated by X's mask. With no masks it is the plain driver.
// points.rs:94-101 (cvtt_f64): truncation of a double to i32, NaN and out of range give INT_MIN
static int32_t cvtt_f64_i32(double v) {
    if (std::isnan(v) || v >= 2147483648.0 || v <= -2147483649.0) return INT32_MIN;
    return (int32_t)v;
}

std::vector<UserLevel> user_displacement(const std::vector<std::array<float, 4>>& pairs, const Geometry& geo, int W,
                                         int H) {
    std::vector<UserLevel> levels;
    for (int l = 0; l < geo.levels; l++) {
        int wl = geo.sizes[l].first, hl = geo.sizes[l].second;
        UserLevel lv;
        lv.d.assign((size_t)wl * hl * 2, 0.0f);
        lv.w.assign((size_t)wl * hl, 0.0f);
        if (l == 0) {  // points.rs:112-144 (finest_level)
            if (W >= 2 && H >= 2 && wl > 0 && hl > 0) {
                float kx = (float)(wl - 1) / (float)(W - 1), ky = (float)(hl - 1) / (float)(H - 1);
                for (const auto& pr : pairs) {
                    float x = pr[0] * kx, y = pr[1] * ky;
                    int ix = cvtt_f64_i32((double)x + 0.5), iy = cvtt_f64_i32((double)y + 0.5);
                    if (ix < 0 || iy < 0 || ix >= wl || iy >= hl) continue;
                    size_t i = (size_t)iy * wl + ix;
                    lv.d[2 * i] = (pr[2] * kx - x) + lv.d[2 * i];
                    lv.d[2 * i + 1] = (pr[3] * ky - y) + lv.d[2 * i + 1];
                    lv.w[i] = lv.w[i] + 1.0f;
                }
                for (size_t i = 0; i < lv.w.size(); i++)
                    if (0.0f < lv.w[i]) {
                        lv.d[2 * i] = lv.d[2 * i] / lv.w[i];
                        lv.d[2 * i + 1] = lv.d[2 * i + 1] / lv.w[i];
                        lv.w[i] = 1.0f;
                    }
            }
            for (float& v : lv.d) v = -1.0f * v;  // points.rs:103-108 (scale_xy by -1)
        } else {  // points.rs:147-171 (coarser_level)
            const UserLevel& pv = levels[l - 1];
            int pw = geo.sizes[l - 1].first, ph = geo.sizes[l - 1].second;
            std::vector<float> t = pv.d;
            convolve(t.data(), pw, ph, 2, BINOMIAL5, 3, true);
            Plane c0, c1, u;
            c0.w = c1.w = u.w = pw;
            c0.h = c1.h = u.h = ph;
            c0.d.resize((size_t)pw * ph);
            c1.d.resize((size_t)pw * ph);
            for (size_t i = 0; i < c0.d.size(); i++) { c0.d[i] = t[2 * i]; c1.d[i] = t[2 * i + 1]; }
            u.d = pv.w;
            convolve(u.d.data(), pw, ph, 1, BINOMIAL5, 3, true);
            Plane rx = resample1(c0, wl, hl), ry = resample1(c1, wl, hl), rw = resample1(u, wl, hl);
            float sx = (float)(wl - 1) / (float)(pw - 1), sy = (float)(hl - 1) / (float)(ph - 1);
            for (size_t i = 0; i < rx.d.size(); i++) {
                lv.d[2 * i] = sx * rx.d[i];
                lv.d[2 * i + 1] = sy * ry.d[i];
            }
            lv.w = rw.d;
        }
        levels.push_back(std::move(lv));
    }
    return levels;
}

// flow/extras.rs:181-194 (apply_user): flow = d / w where w != 0
static void apply_user(std::vector<float>& flow, const UserLevel& u) {
    for (size_t i = 0; i < u.w.size(); i++) {
        float k = u.w[i];
        if (k != 0.0f) {
            flow[2 * i] = u.d[2 * i] / k;
            flow[2 * i + 1] = u.d[2 * i + 1] / k;
        }
    }
}

FlowField solve_pyramids_masked(const Pyramid& x, const Pyramid& y, const FlowSettings& s, const std::vector<Plane>* mx,
                                const std::vector<Plane>* my, bool gate, const std::vector<UserLevel>* user) {
    const Geometry& geo = x.geo;
    int levels = geo.levels;
    int start; float damp;
    start_level(s.sensitivity, levels, &start, &damp);
    int sw0 = geo.sizes[start].first, sh0 = geo.sizes[start].second;
    std::vector<float> flow((size_t)sw0 * sh0 * 2, 0.0f);
    bool check = true;
    for (int l = start; l >= 0; l--) {
        int w = geo.sizes[l].first, h = geo.sizes[l].second;
        const float* img_a = x.levels[l].d.data();
        const float* img_b = y.levels[l].d.data();
        const float* mask_x = mx ? (*mx)[l].d.data() : nullptr;
        const float* mask_y = my ? (*my)[l].d.data() : nullptr;
        const float* g8 = gate ? mask_x : nullptr;
        // flow/extras.rs:198-215 (solve_extended's hooks): the user displacement after the start or
        // the upsample, after the finest level's block matching and at the end of every level
        const UserLevel* u = user ? &(*user)[l] : nullptr;
        if (u) apply_user(flow, *u);
        // flow/extras.rs:337-380 (level_step_gated): with wrap the periodic gradient, the circular
        // Gaussians, the 360 B step and the 360 block matching
        const bool wrap = s.wrap;
        auto blur = [&](std::vector<float>& d, int c, float r) {
            if (wrap) blur_gaussian_wrap(d.data(), w, h, c, r);
            else blur_gaussian(d.data(), w, h, c, r, s.taps_above_first);
        };
        auto refine = [&]() {
            if (wrap) block_match_sphere(img_a, img_b, flow.data(), w, h, g8);
            else block_match_gated(img_a, img_b, flow.data(), w, h, g8);
        };
        std::vector<float> grad = wrap ? calc_grad_wrap(img_a, w, h) : calc_grad(img_a, w, h);
        if (mask_x) {
            if (wrap) mask_gradient_wrap(grad.data(), mask_x, w, h);
            else mask_gradient(grad.data(), mask_x, w, h);
        }
        std::vector<float> a = calc_a(grad, w, h);
        blur(a, 3, 7.0f);
        for (int it = 0; it < 3; it++) {
            std::vector<float> b = wrap     ? calc_b_wrap(img_a, img_b, grad.data(), flow.data(), w, h, mask_y)
                                   : mask_y ? calc_b_masked(img_a, img_b, grad.data(), flow.data(), w, h, mask_y)
                                            : calc_b(img_a, img_b, grad.data(), flow.data(), w, h);
            blur(b, 2, 7.0f);
            new_disp(flow.data(), a.data(), b.data(), (size_t)w * h);
            blur(flow, 2, 5.0f);
            if (it == 1 && l == 0) {
                if (!s.skip_refine) refine();
                if (u) apply_user(flow, *u);
            }
        }
        if (l != 0 && !s.skip_refine) refine();
        if (u) apply_user(flow, *u);
        if (check) {
            if (all_flow_out_of_range(flow.data(), w, h)) std::fill(flow.begin(), flow.end(), 0.0f);
            else check = false;
        }
        if (l == start && std::fabs((double)damp - 1.0) >= 1e-6) scale_values(flow.data(), flow.size(), damp);
        if (l > 0) {
            int nw = geo.sizes[l - 1].first, nh = geo.sizes[l - 1].second;
            flow = wrap ? upsample_flow_wrapx(flow.data(), w, h, nw, nh) : upsample_flow(flow.data(), w, h, nw, nh);
        }
    }
    scale_values(flow.data(), flow.size(), -1.0f);
    FlowField out;
    out.w = geo.w;
    out.h = geo.h;
    out.d = std::move(flow);
    return out;
}

bool solve(const Image& x, const Image& y, const FlowSettings& s, FlowField* out, std::string* err) {
    if (x.w != y.w || x.h != y.h || x.fmt != y.fmt) { *err = "incompatible inputs"; return false; }
    Pyramid px, py;
    if (!build_pyramid(x, s, &px, err) || !build_pyramid(y, s, &py, err)) return false;
    *out = solve_pyramids(px, py, s);
    return true;
}

bool solve_pair(const Image& a, const Image& b, const FlowSettings& s, FlowField* f_ab, FlowField* f_ba,
                std::string* err) {  // flow.rs:1347-1353
    if (a.w != b.w || a.h != b.h || a.fmt != b.fmt) { *err = "incompatible inputs"; return false; }
    Pyramid pa, pb;
    if (!build_pyramid(a, s, &pa, err) || !build_pyramid(b, s, &pb, err)) return false;
    *f_ba = solve_pyramids(pb, pa, s);
    *f_ab = solve_pyramids(pa, pb, s);
    return true;
}

// =============================================================================================
// inverse warp (warp.rs)

uint8_t sat_u8(float v) {  // warp.rs:129-135
    int32_t i = cvtt32(v + 0.5f);
    int32_t t = (int32_t)((uint32_t)i + (uint32_t)(-128));
    int32_t wv = std::min(std::max(t, -32768), 32767);
    int32_t bv = std::min(std::max(wv, -128), 127);
    return (uint8_t)(bv + 128);
}
uint16_t sat_u16(float v) {  // warp.rs:141-146
    int32_t i = cvtt32(v + 0.5f);
    int32_t t = (int32_t)((uint32_t)i + (uint32_t)(-32768));
    int32_t wv = std::min(std::max(t, -32768), 32767);
    return (uint16_t)(wv + 32768);
}
static inline uint8_t scale_u8(uint8_t b, float f) {  // warp.rs:152-155
    float v = (float)b * f;
    return (uint8_t)cvtt64d((double)v + 0.5);
}
static inline uint16_t scale_u16(uint16_t b, float f) {  // warp.rs:159-162
    float v = (float)b * f;
    return (uint16_t)cvtt64d((double)v + 0.5);
}

bool clip_to_rect(float x, float y, float* ix, float* iy, float w1, float h1) {  // warp.rs:178-215
    for (int it = 0; it < 4096; it++) {
        if (*ix < 0.0f) {
            float dy = y - *iy, dxs = x - *ix, num = x - 0.0f;
            *ix = 0.0f;
            *iy = y - (num / dxs) * dy;
            continue;
        }
        if (*ix > w1) {
            float dy = y - *iy, dxs = x - *ix, num = x - w1;
            *ix = w1;
            *iy = y - (num / dxs) * dy;
            continue;
        }
        if (*iy < 0.0f) {
            float dyy = y - *iy, num = y - 0.0f, dx = x - *ix;
            *ix = x - (num / dyy) * dx;
            *iy = 0.0f;
            continue;
        }
        if (*iy > h1) {
            float dyy = y - *iy, num = y - h1, dx = x - *ix;
            *ix = x - (num / dyy) * dx;
            *iy = h1;
            continue;
        }
        return true;
    }
    return false;
}

template <typename P> struct PixT;
template <> struct PixT<uint8_t> {
    static float f(uint8_t v) { return (float)v; }
    static uint8_t store(float v) { return sat_u8(v); }
    static uint8_t faded(float v, float f) { return scale_u8(sat_u8(v), f); }
};
template <> struct PixT<uint16_t> {
    static float f(uint16_t v) { return (float)v; }
    static uint16_t store(float v) { return sat_u16(v); }
    static uint16_t faded(float v, float f) { return scale_u16(sat_u16(v), f); }
};
template <> struct PixT<float> {
    static float f(float v) { return v; }
    static float store(float v) { return v; }
    static float faded(float v, float f) { return v * f; }
};

// warp.rs:290-360 (bilerp4 + mix4 with the NaN rule repeat)
template <typename P>
static inline void bilerp4(const P* src, int w, int w1, int h1, float x, float y, float out[4]) {
    int ix = cvtt32(x), iy = cvtt32(y);
    float fx = x - (float)ix, fy = y - (float)iy;
    if (ix >= w1) { ix = w1 - 1; fx = 1.0f; }
    if (iy >= h1) { iy = h1 - 1; fy = 1.0f; }
    long i00 = ((long)iy * w + ix) * 4;
    long i01 = i00 + (long)w * 4;
    bool any = false;
    for (int k = 0; k < 4; k++) {
        float p00 = PixT<P>::f(src[i00 + k]), p10 = PixT<P>::f(src[i00 + 4 + k]);
        float p01 = PixT<P>::f(src[i01 + k]), p11 = PixT<P>::f(src[i01 + 4 + k]);
        float top = p00 + (p10 - p00) * fx;
        float bot = p01 + (p11 - p01) * fx;
        out[k] = top + (bot - top) * fy;
        any = any || std::isnan(out[k]);
    }
    if (any) {
        for (int k = 0; k < 4; k++) {
            float p00 = PixT<P>::f(src[i00 + k]), p10 = PixT<P>::f(src[i00 + 4 + k]);
            float p01 = PixT<P>::f(src[i01 + k]), p11 = PixT<P>::f(src[i01 + 4 + k]);
            float top = nr::add(p00, nr::mul(nr::sub(p10, p00), fx));
            float bot = nr::add(p01, nr::mul(nr::sub(p11, p01), fx));
            out[k] = nr::add(top, nr::mul(nr::sub(bot, top), fy));
        }
    }
}

// warp.rs:339-352 (mix4): the three lerps of four taps, repeated with the NaN rule when NaN
template <typename P>
static inline void mix4(const P* a, const P* b, const P* c, const P* d, float fx, float fy, float out[4]) {
    bool any = false;
    for (int k = 0; k < 4; k++) {
        float p00 = PixT<P>::f(a[k]), p10 = PixT<P>::f(b[k]), p01 = PixT<P>::f(c[k]), p11 = PixT<P>::f(d[k]);
        float top = p00 + (p10 - p00) * fx;
        float bot = p01 + (p11 - p01) * fx;
        out[k] = top + (bot - top) * fy;
        any = any || std::isnan(out[k]);
    }
    if (any) {
        for (int k = 0; k < 4; k++) {
            float p00 = PixT<P>::f(a[k]), p10 = PixT<P>::f(b[k]), p01 = PixT<P>::f(c[k]), p11 = PixT<P>::f(d[k]);
            float top = nr::add(p00, nr::mul(nr::sub(p10, p00), fx));
            float bot = nr::add(p01, nr::mul(nr::sub(p11, p01), fx));
            out[k] = nr::add(top, nr::mul(nr::sub(bot, top), fy));
        }
    }
}

// warp.rs:362-396 (bilerp360): the right neighbour of the last column is column 0; below the last
// row the taps come from the last row shifted by half the width
template <typename P>
static inline void bilerp360(const P* src, int w, int w1, int h1, float x, float y, float out[4]) {
    int ix = cvtt32(x), iy = cvtt32(y);
    float fx = x - (float)ix, fy = y - (float)iy;
    int x1 = ix + 1 > w1 ? 0 : ix + 1;
    int xc, xd, yc;
    if (iy + 1 > h1) {
        int half = w / 2;
        xc = (half + ix) % w;
        xd = (half + x1) % w;
        yc = h1;
    } else {
        xc = ix;
        xd = x1;
        yc = iy + 1;
    }
    int ya = std::min(iy, h1);
    xc = std::max(xc, 0);
    xd = std::max(xd, 0);
    auto at = [&](int xx, int yy) { return src + ((long)yy * w + xx) * 4; };
    mix4(at(ix, ya), at(x1, ya), at(xc, yc), at(xd, yc), fx, fy, out);
}

// warp.rs:563-621 (pixel_360): the point wrapped into the image by whole turns, an odd number of
// vertical wraps reflected over the pole (half a turn across, H - iy), then the 360 sampler; false
// when the wrap loops would not end or the point is NaN
template <typename P>
static inline bool pixel_360(const P* src, int width, int w1i, int h1i, float wf, float hf, float ix, float iy, P* px) {
    const uint32_t WRAP_LIMIT = 1u << 16;
    uint32_t guard = 0, n = 0;
    while (ix < 0.0f) { ix += wf; if (++guard > WRAP_LIMIT) break; }
    while (wf <= ix) { ix -= wf; if (++guard > WRAP_LIMIT) break; }
    while (iy < 0.0f) { iy += hf; n++; if (++guard > WRAP_LIMIT) break; }
    while (hf <= iy) { iy -= hf; n++; if (++guard > WRAP_LIMIT) break; }
    if (guard > WRAP_LIMIT || !(ix >= 0.0f && ix < wf) || std::isnan(iy)) {
        for (int k = 0; k < 4; k++) px[k] = P(0);
        return false;
    }
    if (n & 1) {
        ix = wf * 0.5f + ix;
        if (ix >= wf) ix -= wf;
        if (iy != 0.0f) iy = hf - iy;
    }
    float s[4];
    bilerp360(src, width, w1i, h1i, ix, iy, s);
    for (int k = 0; k < 4; k++) px[k] = PixT<P>::store(s[k]);
    return true;
}

// warp.rs:415-442 (Flow::bilerp)
static inline void flow_bilerp(const float* d, int fw, int fw1, int fh1, float x, float y, float out[2]) {
    int ix = cvtt32(x), iy = cvtt32(y);
    float fx = x - (float)ix, fy = y - (float)iy;
    if (ix >= fw1) { ix = fw1 - 1; fx = 1.0f; }
    if (iy >= fh1) { iy = fh1 - 1; fy = 1.0f; }
    long i00 = ((long)iy * fw + ix) * 2;
    long i01 = i00 + (long)fw * 2;
    for (int k = 0; k < 2; k++) {
        float p00 = d[i00 + k], p10 = d[i00 + 2 + k], p01 = d[i01 + k], p11 = d[i01 + 2 + k];
        float top = (p10 - p00) * fx + p00;
        float bot = (p11 - p01) * fx + p01;
        out[k] = (bot - top) * fy + top;
    }
}

template <typename P>
static bool warp_run(P* out, uint8_t* cov, const P* src, const FlowField& flow, float amount, WarpOpts o, int width,
                     int height) {  // warp.rs:446-651
    int w1i = width - 1, h1i = height - 1;
    float rx = (float)(flow.w - 1) / (float)w1i;
    float ry = (float)(flow.h - 1) / (float)h1i;
    float sx = amount / rx, sy = amount / ry;
    float wf = (float)width, hf = (float)height, w1 = (float)w1i, h1 = (float)h1i;
    int fw1 = flow.w - 1, fh1 = flow.h - 1;
    bool bad = false;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(|| : bad)
#endif
    for (int y = 0; y < height; y++) {
        float yf = (float)y;
        float fy = yf * ry;
        for (int x = 0; x < width; x++) {
            float xf = (float)x;
            float dd[2];
            flow_bilerp(flow.d.data(), flow.w, fw1, fh1, xf * rx, fy, dd);
            float ix = dd[0] * sx + xf;
            float iy = dd[1] * sy + yf;
            P* px = out + ((long)y * width + x) * 4;
            if (o.is360) {
                if (!pixel_360(src, width, w1i, h1i, wf, hf, ix, iy, px)) bad = true;
            } else if (o.hold) {
                if (!clip_to_rect(xf, yf, &ix, &iy, w1, h1) || std::isnan(ix) || std::isnan(iy)) {
                    bad = true;
                    for (int k = 0; k < 4; k++) px[k] = P(0);
                    continue;
                }
                float s[4];
                bilerp4(src, width, w1i, h1i, ix, iy, s);
                for (int k = 0; k < 4; k++) px[k] = PixT<P>::store(s[k]);
            } else {
                uint8_t c;
                if (!(ix > -1.0f && ix < wf && iy > -1.0f && iy < hf)) {
                    for (int k = 0; k < 4; k++) px[k] = P(0);
                    c = 0;
                } else if (ix >= 0.0f && ix <= w1 && iy >= 0.0f && iy <= h1) {
                    float s[4];
                    bilerp4(src, width, w1i, h1i, ix, iy, s);
                    for (int k = 0; k < 4; k++) px[k] = PixT<P>::store(s[k]);
                    c = 255;
                } else {
                    float f = ix < 0.0f ? ix + 1.0f : (ix <= w1 ? 1.0f : wf - ix);
                    if (iy < 0.0f) f *= iy + 1.0f;
                    else if (iy > h1) f *= hf - iy;
                    if (!clip_to_rect(xf, yf, &ix, &iy, w1, h1) || std::isnan(ix) || std::isnan(iy)) {
                        bad = true;
                        for (int k = 0; k < 4; k++) px[k] = P(0);
                        c = 0;
                    } else {
                        float s[4];
                        bilerp4(src, width, w1i, h1i, ix, iy, s);
                        for (int k = 0; k < 4; k++) px[k] = PixT<P>::faded(s[k], f);
                        float cc = f * 255.0f + 0.5f;
                        c = cc <= 255.0f ? (uint8_t)cvtt64d((double)cc) : 255;
                    }
                }
                if (cov) cov[(long)y * width + x] = c;
            }
        }
    }
    return !bad;
}

int inv_warp(Image& out, const Image& src, const FlowField& flow, float amount, WarpOpts o, Coverage* cov,
             std::string* err) {  // warp.rs:693-786
    if (out.w != src.w || out.h != src.h || out.fmt != src.fmt) { *err = "inverse warp: shape mismatch"; return 1; }
    if (out.w < 2 || out.h < 2 || flow.w < 2 || flow.h < 2) { *err = "inverse warp: below 2x2"; return 1; }
    if (cov) { cov->w = out.w; cov->h = out.h; cov->d.assign((size_t)out.w * out.h, 0xff); }
    int width = out.w, height = out.h;
    float a = amount < 0.0f ? -amount : amount;
    bool copy_only = 0.005 > (double)a;
    if (!copy_only) {
        float r = (float)(flow.w - 1) / (float)(width - 1);
        float qq = (float)((double)amount / (double)r);
        if (qq < 0.0f) qq = -qq;
        copy_only = 0.0001 > (double)qq;
    }
    if (copy_only) { copy_image(out, src); return 0; }
    if (o.mode != 1) { *err = "inverse warp: mip map sampling"; return 2; }
    uint8_t* c = cov ? cov->d.data() : nullptr;
    bool ok;
    if (out.fmt == U8) ok = warp_run<uint8_t>(out.u8.data(), c, src.u8.data(), flow, amount, o, width, height);
    else if (out.fmt == U16) ok = warp_run<uint16_t>(out.u16.data(), c, src.u16.data(), flow, amount, o, width, height);
    else ok = warp_run<float>(out.f32.data(), c, src.f32.data(), flow, amount, o, width, height);
    if (!ok) { *err = "inverse warp: a sample coordinate is NaN or never converges"; return 2; }
    return 0;
}

// =============================================================================================
// blend (blend.rs)

void warp_flow_bilerp(const FlowField& f, float x, float y, float out[2]) {
    flow_bilerp(f.d.data(), f.w, f.w - 1, f.h - 1, x, y, out);
}

void bilerp4_image(const Image& img, float x, float y, float out[4]) {
    int w1 = img.w - 1, h1 = img.h - 1;
    if (img.fmt == U8) bilerp4(img.u8.data(), img.w, w1, h1, x, y, out);
    else if (img.fmt == U16) bilerp4(img.u16.data(), img.w, w1, h1, x, y, out);
    else bilerp4(img.f32.data(), img.w, w1, h1, x, y, out);
}

void bilerp360_image(const Image& img, float x, float y, float out[4]) {
    int w1 = img.w - 1, h1 = img.h - 1;
    if (img.fmt == U8) bilerp360(img.u8.data(), img.w, w1, h1, x, y, out);
    else if (img.fmt == U16) bilerp360(img.u16.data(), img.w, w1, h1, x, y, out);
    else bilerp360(img.f32.data(), img.w, w1, h1, x, y, out);
}

void copy_image(Image& out, const Image& src) {  // blend.rs:117-125
    std::memcpy(out.data(), src.data(), src.bytes());
}

template <typename T>
static inline void lerp_pixel_int(T* f, const T* s, float w, float scale) {  // blend.rs:214-249
    auto diff = [&](int i) { return (float)((int32_t)f[i] - (int32_t)s[i]); };
    auto sf = [&](int i) { return (float)(int32_t)s[i]; };
    auto store = [](float v) { return (T)cvtt64f(v); };
    float a = diff(0) * w + sf(0);
    float n = a / scale;
    if (!(n > 0.0f)) { T z = store(0.0f); for (int i = 0; i < 4; i++) f[i] = z; return; }
    float r = diff(1) * w + sf(1), g = diff(2) * w + sf(2), b = diff(3) * w + sf(3);
    if (n > 1.0f) { r = r / n; g = g / n; b = b / n; a = scale; }
    auto clamp = [&](float c) { return c > a ? a : (0.0f > c ? 0.0f : c); };
    r = clamp(r); g = clamp(g); b = clamp(b);
    f[1] = store(r + 0.5f);
    f[2] = store(g + 0.5f);
    f[3] = store(b + 0.5f);
    f[0] = store(a + 0.5f);
}

static inline void lerp_pixel_f32(float* f, const float* s, float w) {  // blend.rs:182-211
    bool rule = false;
    for (int i = 0; i < 4; i++) rule = rule || std::isnan(f[i]) || std::isnan(s[i]);
    if (!rule) {
        float a = (f[0] - s[0]) * w + s[0];
        if (!(a > 0.0f)) { for (int i = 0; i < 4; i++) f[i] = 0.0f; return; }
        float r = (f[1] - s[1]) * w + s[1], g = (f[2] - s[2]) * w + s[2], b = (f[3] - s[3]) * w + s[3];
        if (a > 1.0f) { r = r / a; g = g / a; b = b / a; a = 1.0f; }
        f[1] = r + 0.0f; f[2] = g + 0.0f; f[3] = b + 0.0f; f[0] = a + 0.0f;
    } else {
        auto L = [](float a, float b, float w) { return nr::add(nr::mul(nr::sub(b, a), w), a); };
        float a = L(s[0], f[0], w);
        if (!(a > 0.0f)) { for (int i = 0; i < 4; i++) f[i] = 0.0f; return; }
        float r = L(s[1], f[1], w), g = L(s[2], f[2], w), b = L(s[3], f[3], w);
        if (a > 1.0f) { r = nr::div(r, a); g = nr::div(g, a); b = nr::div(b, a); a = 1.0f; }
        f[1] = nr::add(r, 0.0f); f[2] = nr::add(g, 0.0f); f[3] = nr::add(b, 0.0f); f[0] = nr::add(a, 0.0f);
    }
}

void lerp(Image& first, const Image& second, float w) {  // blend.rs:144-179
    if (w == 1.0f) return;
    if (w == 0.0f) { copy_image(first, second); return; }
    long n = (long)first.w * first.h;
    if (first.fmt == U8) {
        OMP_FOR
        for (long i = 0; i < n; i++) lerp_pixel_int<uint8_t>(&first.u8[i * 4], &second.u8[i * 4], w, 255.0f);
    } else if (first.fmt == U16) {
        OMP_FOR
        for (long i = 0; i < n; i++) lerp_pixel_int<uint16_t>(&first.u16[i * 4], &second.u16[i * 4], w, 65535.0f);
    } else {
        OMP_FOR
        for (long i = 0; i < n; i++) lerp_pixel_f32(&first.f32[i * 4], &second.f32[i * 4], w);
    }
}

void blend(Image& out, const Image& a, const Image& b, float w) {  // blend.rs:55-114
    const double SNAP = 0.005;
    if (SNAP > (double)std::fabs(w)) { copy_image(out, a); return; }
    if (SNAP > std::fabs((double)w - 1.0)) { copy_image(out, b); return; }
    if (w < 0.0f || w > 1.0f) {
        copy_image(out, a);
        lerp(out, b, (float)(1.0 - (double)w));
        return;
    }
    long n = (long)out.w * out.h * 4;
    if (out.fmt == U8) {
        OMP_FOR
        for (long i = 0; i < n; i++) {
            float af = (float)a.u8[i], bf = (float)b.u8[i];
            out.u8[i] = (uint8_t)cvtt64f((bf - af) * w + af + 0.5f);
        }
    } else if (out.fmt == U16) {
        OMP_FOR
        for (long i = 0; i < n; i++) {
            float af = (float)a.u16[i], bf = (float)b.u16[i];
            out.u16[i] = (uint16_t)cvtt64f((bf - af) * w + af + 0.5f);
        }
    } else {
        long row = (long)out.w * 4;
        OMP_FOR
        for (int y = 0; y < out.h; y++) {
            bool any = false;
            for (long i = y * row; i < (y + 1) * row; i++) {
                out.f32[i] = (b.f32[i] - a.f32[i]) * w + a.f32[i] + 0.0f;
                any = any || std::isnan(out.f32[i]);
            }
            if (any)
                for (long i = y * row; i < (y + 1) * row; i++)
                    out.f32[i] = nr::add(nr::add(nr::mul(nr::sub(b.f32[i], a.f32[i]), w), a.f32[i]), 0.0f);
        }
    }
}

// =============================================================================================
// composition (compose/vector.rs:209-284, compose.rs:218-231)

bool nearest_uses_f_ab(float wa, int code) {  // compose/vector.rs:61-64
    unsigned c = (unsigned)code;
    return (wa < 0.5f && c < 2) || (0.5f <= wa && c > 1);
}

static int compose_body(const ComposeSettings& cs, const Selection& sel, const Image& a, const Image& b,
                        const FlowField* f_ab, const FlowField* f_ba, Image* out, std::string* err) {
    if (cs.warp_mode == 1) return compose_smart(cs, sel, a, b, f_ab, f_ba, cs.taps_above_first, out, err);
    if (cs.warp_mode == 2 || cs.warp_mode == 3) return compose_forward(cs, sel, a, b, f_ab, f_ba, out, err);
    if (cs.warp_mode != 0) { *err = "compose: warping code not 0 to 3"; return 1; }
    float wa = sel.wa;
    float frac = 1.0f - wa;
    WarpOpts o;
    o.is360 = cs.wrap_360;  // compose/vector.rs:214 (every interpolation mode of code 0)
    *out = Image(a.w, a.h, a.fmt);
    if (sel.interp == 0) {
        const FlowField* flow = nearest_uses_f_ab(wa, cs.warp_mode) ? f_ab : f_ba;
        if (!flow) { *err = "missing flow"; return 1; }
        if (0.5f <= wa) return inv_warp(*out, a, *flow, frac, o, nullptr, err);
        return inv_warp(*out, b, *flow, wa, o, nullptr, err);
    }
    if (sel.interp == 1 || sel.interp == 2) {
        if (!f_ab || !f_ba) { *err = "missing flow"; return 1; }
        Image ta(a.w, a.h, a.fmt), tb(b.w, b.h, b.fmt);
        int rc = inv_warp(ta, a, *f_ba, frac, o, nullptr, err);
        if (rc) return rc;
        rc = inv_warp(tb, b, *f_ab, wa, o, nullptr, err);
        if (rc) return rc;
        if (sel.interp == 2) {  // compose/vector.rs:264-269: the sharpening of each warped frame
            sharpen_step(ta, a, frac, cs.taps_above_first);
            sharpen_step(tb, b, wa, cs.taps_above_first);
        }
        blend(*out, ta, tb, frac);
        return 0;
    }
    *err = "bad interpolation mode";
    return 1;
}

int compose_vectors(const ComposeSettings& cs, const Selection& sel, const Image& a, const Image& b,
                    const FlowField* f_ab, const FlowField* f_ba, Image* out, std::string* err) {
    int rc = compose_body(cs, sel, a, b, f_ab, f_ba, out, err);
    if (rc) return rc;
    // compose/vector.rs:276-281: the Blur Compensation tail with F_AB, else the single flow
    const FlowField* flow = f_ab ? f_ab : f_ba;
    if (!flow) return 0;
    return blur_compensation(*out, *flow, sel.s0, sel.s1, cs.blur, cs.quality_high, err, cs.wrap_360);
}

int interpolate(const Selection& sel, const Image& a, const Image& b, Image* out, std::string* err) {
    *out = Image(a.w, a.h, a.fmt);
    if (sel.interp == 0) { copy_image(*out, sel.wa >= 0.5f ? a : b); return 0; }
    if (sel.interp == 1) { blend(*out, a, b, (float)(1.0 - (double)sel.wa)); return 0; }
    if (sel.interp == 2) {
        // blend.rs:281-302: Weighted Blend without flows equals the plain Blend with weight 1 - wa
        // for 8 and 16 bpc, and for float data whose samples are finite and at most 1e30
        if (a.fmt == F32) {
            bool sound = true;
            for (float v : a.f32) sound = sound && std::fabs(v) <= 1.0e30f;
            for (float v : b.f32) sound = sound && std::fabs(v) <= 1.0e30f;
            if (!sound) {  // blend.rs:316-324 (weighted_blend_noflow_reference): every filter, engine taps
                float t = 1.0f - sel.wa;
                Image a1 = a, b1 = b;
                sharpen_step(a1, a, t, false);
                sharpen_step(b1, b, sel.wa, false);
                blend(*out, a1, b1, t);
                return 0;
            }
            Image a1 = a, b1 = b;
            for (auto& v : a1.f32) v = v + 0.0f;
            for (auto& v : b1.f32) v = v + 0.0f;
            blend(*out, a1, b1, 1.0f - sel.wa);
            return 0;
        }
        blend(*out, a, b, 1.0f - sel.wa);
        return 0;
    }
    *err = "bad interpolation mode";
    return 1;
}

}  // namespace orc
