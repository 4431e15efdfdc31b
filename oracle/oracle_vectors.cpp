// CPU oracle of the vector encoder and the single layer Create Vectors pass. TEST
// INFRASTRUCTURE ONLY (see oracle_core.h).
#include "oracle_vectors.h"

#include <algorithm>
#include <cmath>

#include "oracle_forward.h"
#include "oracle_smart.h"

namespace orc {

static inline void clamp_unit(float* v) {  // vectors.rs:133-140: a NaN falls through
    if (*v > 1.0f) *v = 1.0f;
    else if (-1.0f > *v) *v = -1.0f;
}

int encode_vectors(Image& dst, const FlowField& flow, float scale, std::string* err) {  // vectors.rs:57-130
    if (dst.w < 2 || dst.h < 2 || flow.w < 2 || flow.h < 2) {
        *err = "vector encode needs images and a flow of at least 2x2";
        return 1;
    }
    float dw1 = (float)(dst.w - 1), dh1 = (float)(dst.h - 1);
    float fw1 = (float)(flow.w - 1), fh1 = (float)(flow.h - 1);
    float sx = fw1 / dw1, sy = fh1 / dh1;
    float kx = (dw1 / fw1) / scale, ky = (dh1 / fh1) / scale;
    for (int y = 0; y < dst.h; y++) {
        for (int x = 0; x < dst.w; x++) {
            float uv[2];
            warp_flow_bilerp(flow, (float)x * sx, (float)y * sy, uv);
            float a = uv[0] * kx, b = uv[1] * ky;
            size_t i = ((size_t)y * dst.w + x) * 4;
            if (dst.fmt == F32) {
                dst.f32[i] = 1.0f;
                dst.f32[i + 1] = (a + 1.0f) * 0.5f;
                dst.f32[i + 2] = (b + 1.0f) * 0.5f;
                dst.f32[i + 3] = 0.0f;
                continue;
            }
            clamp_unit(&a);
            clamp_unit(&b);
            a = a + 1.0f;
            b = b + 1.0f;
            if (dst.fmt == U8) {
                dst.u8[i] = 0xff;
                dst.u8[i + 1] = (uint8_t)cvtt64d((double)a * 127.0 + 0.5);
                dst.u8[i + 2] = (uint8_t)cvtt64d((double)b * 127.0 + 0.5);
                dst.u8[i + 3] = 0;
            } else {
                dst.u16[i] = 0xffff;
                dst.u16[i + 1] = (uint16_t)cvtt64d((double)a * 32767.0 + 0.5);
                dst.u16[i + 2] = (uint16_t)cvtt64d((double)b * 32767.0 + 0.5);
                dst.u16[i + 3] = 0;
            }
        }
    }
    return 0;
}

Image zero_vectors_image(int w, int h, Fmt fmt) {  // vectors.rs:148-156
    Image img(w, h, fmt);
    for (size_t i = 0; i < (size_t)w * h; i++) {
        if (fmt == U8) { img.u8[i * 4] = 0xff; img.u8[i * 4 + 1] = 127; img.u8[i * 4 + 2] = 127; img.u8[i * 4 + 3] = 0; }
        else if (fmt == U16) { img.u16[i * 4] = 0xffff; img.u16[i * 4 + 1] = 32767; img.u16[i * 4 + 2] = 32767; img.u16[i * 4 + 3] = 0; }
        else { img.f32[i * 4] = 1.0f; img.f32[i * 4 + 1] = 0.5f; img.f32[i * 4 + 2] = 0.5f; img.f32[i * 4 + 3] = 0.0f; }
    }
    return img;
}

int create_vectors(const Image& x, const Image& y, const CreateVectorsSettings& s, Image* out, std::string* err) {
    if (!(x.w >= 2 && x.h >= 2)) {  // prep::searchable (prep.rs:100-102)
        *out = zero_vectors_image(x.w, x.h, x.fmt);
        return 0;
    }
    FlowSettings fs;  // create_vectors.rs:121-135
    fs.quality = s.quality;
    fs.hiq = s.hiq;
    fs.sensitivity = s.sensitivity;
    fs.track_alpha = s.track_rgb_a;
    fs.video_range_luma = false;
    fs.skip_refine = false;
    fs.taps_above_first = s.taps_above_first;
    fs.prep_contrast_edge = s.prep_contrast_edge;
    fs.prep_delinearize = s.prep_delinearize;
    FlowField flow;
    if (!solve(x, y, fs, &flow, err)) return 1;
    *out = Image(x.w, x.h, x.fmt);
    return encode_vectors(*out, flow, s.max_displace, err);
}

}  // namespace orc

// ---- Vectors In: the vector layer's flow and the flow inversion ---------------------------------

namespace orc {

// vectors.rs:525-528: ((c * 2) / den - 1) * scale in double precision, narrowed once
static inline float dec_int(double c, double den, double scale) { return (float)(((c * 2.0) / den - 1.0) * scale); }

FlowField decode_vectors(const Image& vec, float max_displace) {  // vectors.rs:474-522
    FlowField flow(vec.w, vec.h);
    double md = (double)max_displace;
    size_t n = (size_t)vec.w * vec.h;
    for (size_t i = 0; i < n; i++) {
        float* o = &flow.d[i * 2];
        if (vec.fmt == U8) {
            const uint8_t* p = &vec.u8[i * 4];
            if (p[0] == 0) { o[0] = 0.0f; o[1] = 0.0f; }
            else { o[0] = dec_int((double)p[1], 254.0, md); o[1] = dec_int((double)p[2], 254.0, md); }
        } else if (vec.fmt == U16) {
            const uint16_t* p = &vec.u16[i * 4];
            if (p[0] == 0) { o[0] = 0.0f; o[1] = 0.0f; }
            else { o[0] = dec_int((double)p[1], 65534.0, md); o[1] = dec_int((double)p[2], 65534.0, md); }
        } else {
            const float* p = &vec.f32[i * 4];
            if (p[0] == 0.0f) { o[0] = 0.0f; o[1] = 0.0f; }
            else {
                o[0] = (p[1] * 2.0f - 1.0f) * max_displace;
                o[1] = (p[2] * 2.0f - 1.0f) * max_displace;
            }
        }
    }
    return flow;
}

// vectors.rs:555-561: the inverted alpha as a mask of the image's sample type (kind 1 u8, 2 u16,
// 3 f32), as raw bytes
void vector_hole_mask(const Image& vec, std::vector<uint8_t>* bytes, int* kind) {
    size_t n = (size_t)vec.w * vec.h;
    if (vec.fmt == U8) {
        *kind = 1;
        bytes->resize(n);
        for (size_t i = 0; i < n; i++) (*bytes)[i] = (uint8_t)(0xffu - vec.u8[i * 4]);
    } else if (vec.fmt == U16) {
        *kind = 2;
        bytes->resize(n * 2);
        uint16_t* m = (uint16_t*)bytes->data();
        for (size_t i = 0; i < n; i++) m[i] = (uint16_t)(0xffffu - vec.u16[i * 4]);
    } else {
        *kind = 3;
        bytes->resize(n * sizeof(float));
        float* m = (float*)bytes->data();
        for (size_t i = 0; i < n; i++) m[i] = 1.0f - vec.f32[i * 4];
    }
}

void apply_vec_scale(FlowField& flow, float sx, float sy) {  // vectors.rs:573-578
    for (size_t i = 0; i + 1 < flow.d.size(); i += 2) {
        flow.d[i] = sx * flow.d[i];
        flow.d[i + 1] = sy * flow.d[i + 1];
    }
}

// compose/vector.rs:335-345 (flow_from_vector_image_with): decode, the flow hole fill of the
// inverted alpha (is360 off), Vec Scale
int flow_from_vector_image(const Image& vec, float max_displace, float sx, float sy, bool above_first, FlowField* out,
                           std::string* err) {
    *out = decode_vectors(vec, max_displace);
    std::vector<uint8_t> mask;
    int kind = 1;
    vector_hole_mask(vec, &mask, &kind);
    int rc = fill_flow_holes(*out, mask.data(), kind, above_first, err);
    if (rc) return rc;
    apply_vec_scale(*out, sx, sy);
    return 0;
}

// compose/vector.rs:370-397 (invert_flow_on): T = (-1, -fx, -fy, -1) pushed along the flow itself
// at amount 1 with coverage (textured, or the Gouraud variant when !pyramid), the coverage
// inverted, channels 1 and 2 of the pushed image as the flow, the holes filled (u8 mask)
int invert_flow(const FlowField& flow, bool pyramid, bool above_first, FlowField* out, std::string* err) {
    int w = flow.w, h = flow.h;
    Image t(w, h, F32), pushed(w, h, F32);
    size_t n = (size_t)w * h;
    for (size_t i = 0; i < n; i++) {
        t.f32[i * 4] = -1.0f * 1.0f;
        t.f32[i * 4 + 1] = -1.0f * flow.d[i * 2];
        t.f32[i * 4 + 2] = -1.0f * flow.d[i * 2 + 1];
        t.f32[i * 4 + 3] = -1.0f * 1.0f;
    }
    Coverage cov;
    int rc = forward_warp(pushed, t, flow, 1.0f, pyramid, &cov, err);
    if (rc) return rc;
    for (auto& b : cov.d) b = (uint8_t)(0xffu - b);
    *out = FlowField(w, h);
    for (size_t i = 0; i < n; i++) {
        out->d[i * 2] = pushed.f32[i * 4 + 1];
        out->d[i * 2 + 1] = pushed.f32[i * 4 + 2];
    }
    return fill_flow_holes(*out, cov.d.data(), 1, above_first, err);
}

// Rust's saturating `f32 as i64`: NaN 0, the ends of the range at the ends
static inline int64_t sat_i64(float v) {
    if (std::isnan(v)) return 0;
    if ((double)v >= 9223372036854775807.0) return INT64_MAX;
    if ((double)v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

// plugins/vectors-in/src/vectorin.rs:125-155 (matte_step): the alpha capped by the matte in the
// units of the depth; a NaN matte keeps the alpha
void matte_step(Image& img, const std::vector<float>& m) {
    size_t n = (size_t)img.w * img.h;
    for (size_t i = 0; i < n; i++) {
        float v = m[i];
        if (img.fmt == U8) {
            int64_t c = sat_i64(v * 255.0f + 0.5f);
            uint8_t cc = (uint8_t)std::min<int64_t>(std::max<int64_t>(c, 0), 255);
            if (cc < img.u8[i * 4]) img.u8[i * 4] = cc;
        } else if (img.fmt == U16) {
            int64_t c = sat_i64(v * 65535.0f + 0.5f);
            uint16_t cc = (uint16_t)std::min<int64_t>(std::max<int64_t>(c, 0), 65535);
            if (cc < img.u16[i * 4]) img.u16[i * 4] = cc;
        } else if (v < img.f32[i * 4]) {
            img.f32[i * 4] = v;
        }
    }
}

}  // namespace orc

// ---- the Debug views of Create Vectors (debug.rs) ---------------------------------------------

#include "oracle_layers.h"

namespace orc {

namespace {

inline int64_t sat64(double v) {  // Rust's saturating `f64 as i64`
    if (std::isnan(v)) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

const float VIEW_AMOUNT = 0.6f;  // debug.rs:70-78
float diff_gain() {
    float amount = (float)(1.0 - (double)VIEW_AMOUNT);
    return (float)(1.0 / (double)std::fabs(amount));
}
float overlay_gain() {  // debug.rs:83-90
    float amount = 0.001 > (double)VIEW_AMOUNT ? 0.001f : VIEW_AMOUNT;
    float half = (float)((double)amount * 0.5);
    float rest = (float)(1.0 - (double)half);
    return (float)(1.0 / (double)rest);
}

float diff_luma(double r, double g, double b) { return (float)(((r * 0.29) + (g * 0.59)) + (b * 0.12)); }

// debug.rs:285-310: the luma of the Detail and Edge views
std::vector<float> debug_luma(const Image& img) {
    size_t n = (size_t)img.w * img.h;
    std::vector<float> out(n);
    for (size_t i = 0; i < n; i++) {
        if (img.fmt == F32) {
            const float* p = &img.f32[i * 4];
            double tr = (double)p[1] * 0.29, tg = (double)p[2] * 0.59, tb = (double)p[3] * 0.12;
            float v = (float)((tr + tg) + tb);
            if (std::isnan(v)) v = (float)nr::add64(nr::add64(tr, tg), tb);
            out[i] = v;
        } else {
            double s = img.fmt == U8 ? 255.0 : 65535.0;
            double r = img.fmt == U8 ? img.u8[i * 4 + 1] : img.u16[i * 4 + 1];
            double g = img.fmt == U8 ? img.u8[i * 4 + 2] : img.u16[i * 4 + 2];
            double b = img.fmt == U8 ? img.u8[i * 4 + 3] : img.u16[i * 4 + 3];
            float v = (float)((((r * 0.29) / s + (g * 0.59) / s)) + (b * 0.12) / s);
            out[i] = v >= 1.0f ? 1.0f : v;
        }
    }
    return out;
}

// debug.rs:318-346: the luma on the border, sqrt(S / 8) inside
std::vector<float> detail(const std::vector<float>& l, int w, int h) {
    std::vector<float> out((size_t)w * h);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            float c = l[(size_t)y * w + x];
            if (x == 0 || y == 0 || x + 1 == w || y + 1 == h) { out[(size_t)y * w + x] = c; continue; }
            bool first = true;
            float s = 0.0f;
            for (int yy = y - 1; yy <= y + 1; yy++)
                for (int xx = x - 1; xx <= x + 1; xx++) {
                    if (yy == y && xx == x) continue;
                    float d = std::fabs(c - l[(size_t)yy * w + xx]);
                    s = first ? d : s + d;
                    first = false;
                }
            out[(size_t)y * w + x] = std::sqrt(s * 0.125f);
        }
    return out;
}

// debug.rs:355-378: the Sobel magnitude, border repeated, times 2 capped at 255
std::vector<float> edge(const std::vector<float>& l, int w, int h) {
    std::vector<float> out((size_t)w * h);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            auto n = [&](int dx, int dy) {
                int yy = std::min(std::max(y + dy, 0), h - 1), xx = std::min(std::max(x + dx, 0), w - 1);
                return l[(size_t)yy * w + xx];
            };
            float gx = ((((-n(-1, -1) + n(1, -1)) - 2.0f * n(-1, 0)) + 2.0f * n(1, 0)) - n(-1, 1)) + n(1, 1);
            float gy = ((((2.0f * n(0, -1) + n(-1, -1)) + n(1, -1)) - n(-1, 1)) - 2.0f * n(0, 1)) - n(1, 1);
            float e = (float)((double)std::sqrt(gy * gy + gx * gx) * 0.17677669529664);
            float sc = 2.0f * e;
            out[(size_t)y * w + x] = sc > 255.0f ? 255.0f : sc;
        }
    return out;
}

float overlay_value(float m, float gain) {  // debug.rs:382-391
    float v = gain * m;
    if (v > 1.0f) return 1.0f;
    if (v < 0.0f) return 0.0f;
    return v;
}

// debug.rs:399-434: red the measure r, green and blue the measure g, alpha white
void overlay(Image& out, const std::vector<float>& r, const std::vector<float>& g) {
    float gain = overlay_gain();
    size_t n = (size_t)out.w * out.h;
    for (size_t i = 0; i < n; i++) {
        float vr = overlay_value(r[i], gain), vg = overlay_value(g[i], gain);
        if (out.fmt == U8) {
            uint8_t* p = &out.u8[i * 4];
            p[0] = 255;
            p[1] = (uint8_t)sat64((double)vr * 255.0 + 0.5);
            p[2] = (uint8_t)sat64((double)vg * 255.0 + 0.5);
            p[3] = p[2];
        } else if (out.fmt == U16) {
            uint16_t* p = &out.u16[i * 4];
            p[0] = 65535;
            p[1] = (uint16_t)sat64((double)vr * 65535.0 + 0.5);
            p[2] = (uint16_t)sat64((double)vg * 65535.0 + 0.5);
            p[3] = p[2];
        } else {
            float* p = &out.f32[i * 4];
            p[0] = 1.0f;
            p[1] = vr;
            p[2] = vg;
            p[3] = vg;
        }
    }
}

// debug.rs:437-476: the grey Diff, alpha white
void diff(Image& out, const Image& a, const Image& b) {
    float gain = diff_gain();
    size_t n = (size_t)out.w * out.h;
    for (size_t i = 0; i < n; i++) {
        auto luma = [&](const Image& im) {
            if (im.fmt == U8) return diff_luma(im.u8[i * 4 + 1], im.u8[i * 4 + 2], im.u8[i * 4 + 3]);
            if (im.fmt == U16) return diff_luma(im.u16[i * 4 + 1], im.u16[i * 4 + 2], im.u16[i * 4 + 3]);
            return diff_luma(im.f32[i * 4 + 1], im.f32[i * 4 + 2], im.f32[i * 4 + 3]);
        };
        float v = std::fabs(luma(a) - luma(b)) * gain;
        if (out.fmt == F32) {
            float o = v >= 1.0f ? 1.0f : v;
            float* p = &out.f32[i * 4];
            p[0] = 1.0f;
            p[1] = p[2] = p[3] = o;
        } else {
            float top = out.fmt == U8 ? 255.0f : 65535.0f;
            float c = v >= top ? top : v;
            int64_t q = sat64((double)c + 0.5);
            if (out.fmt == U8) {
                uint8_t* p = &out.u8[i * 4];
                p[0] = 255;
                p[1] = p[2] = p[3] = (uint8_t)q;
            } else {
                uint16_t* p = &out.u16[i * 4];
                p[0] = 65535;
                p[1] = p[2] = p[3] = (uint16_t)q;
            }
        }
    }
}

}  // namespace

// the primitives of the views, for the tests
std::vector<float> debug_luma_plane(const Image& img) { return debug_luma(img); }
std::vector<float> debug_detail(const std::vector<float>& l, int w, int h) { return detail(l, w, h); }
std::vector<float> debug_edge(const std::vector<float>& l, int w, int h) { return edge(l, w, h); }
void debug_overlay(Image& out, const std::vector<float>& r, const std::vector<float>& g) { overlay(out, r, g); }

// debug.rs:155-171 (views_of)
Image debug_views_of(const Image& wp, const Image& y, int code) {
    Image out(wp.w, wp.h, wp.fmt);
    if (code == 0) {
        copy_image(out, wp);
        lerp(out, y, 0.5f);
    } else if (code == 1) {
        diff(out, wp, y);
    } else if (code == 2) {
        overlay(out, detail(debug_luma(wp), wp.w, wp.h), detail(debug_luma(y), y.w, y.h));
    } else {
        overlay(out, edge(debug_luma(wp), wp.w, wp.h), edge(debug_luma(y), y.w, y.h));
    }
    return out;
}

// debug.rs:104-152 (debug_view_on): the forward warp of x by the flow at amount 1 (the Gouraud
// variant with gouraud, else the textured one), then W' = (y OVER transparent) with W OVER it, then
// the view; sides of 1: the zero vector image
int debug_view(const Image& x, const Image& y, const FlowField& flow, int code, bool gouraud, Image* out,
               std::string* err) {
    if (!(x.w >= 2 && x.h >= 2)) {
        *out = zero_vectors_image(x.w, x.h, x.fmt);
        return 0;
    }
    Image warped(x.w, x.h, x.fmt);
    int rc = forward_warp(warped, x, flow, 1.0f, !gouraud, nullptr, err);
    if (rc) return rc;
    if (code == 4) {
        *out = warped;
        return 0;
    }
    Image wp(y.w, y.h, y.fmt);
    over_pl(wp, y);
    over_pl(wp, warped);
    *out = debug_views_of(wp, y, code);
    return 0;
}

}  // namespace orc
