// CPU oracle of the vector encoder and the single layer Create Vectors pass. TEST
// INFRASTRUCTURE ONLY (see oracle_core.h).
#include "oracle_vectors.h"

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
