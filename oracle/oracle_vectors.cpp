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
