// CPU oracle of the retime hot path: a C++ restatement of the reference's CPU engine
// (baairon/twixtor, crate plugins/retime-engine). TEST INFRASTRUCTURE ONLY: the parity tests,
// the smoke check and the CPU baseline leg of the benchmark call it as the checker. The product
// (libtwixtor_b200.so) never links or calls it.
//
// Every function cites the reference file:line it restates (paths inside the reference crate
// `plugins/retime-engine/src/`). Arithmetic is single precision in the order the reference writes,
// no FMA contraction (built with -ffp-contract=off), the stated double precision steps, and x86
// truncation semantics (NaN / out of range -> INT_MIN) for every float-to-int conversion.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <array>
#include <vector>
#include <string>

namespace orc {

// ---------------------------------------------------------------------------------------------
// conversions (flow/sample.rs:17-24, warp.rs:104-122, blend.rs:18-25, image.rs:246-258)

inline int32_t cvtt32(float x) {
    if (std::isnan(x) || x >= 2147483648.0f || x < -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
inline int64_t cvtt64d(double x) {
    if (std::isnan(x) || x >= 9.223372036854775808e18 || x < -9.223372036854775808e18) return INT64_MIN;
    return (int64_t)x;
}
inline int64_t cvtt64f(float x) {
    const float two63 = 9223372036854775808.0f;
    if (std::isnan(x) || x >= two63 || x < -two63) return INT64_MIN;
    return (int64_t)x;
}
// image.rs:255-258: q(x) = trunc((x as f64) + 0.5)
inline int64_t q(float x) { return cvtt64d((double)x + 0.5); }

inline float bits_f(uint32_t b) { float f; std::memcpy(&f, &b, 4); return f; }
inline uint32_t f_bits(float f) { uint32_t b; std::memcpy(&b, &f, 4); return b; }

// ---------------------------------------------------------------------------------------------
// NaN rule, emulator variant (nanrule.rs:44-124; the crate's default feature `emulator-nan`)
namespace nr {
inline float quiet(float x) { return bits_f(f_bits(x) | 0x00400000u); }
inline float pick(float a, float b) {
    uint32_t ba = f_bits(a), bb = f_bits(b);
    bool sa = (ba & 0x00400000u) == 0, sb = (bb & 0x00400000u) == 0;
    uint32_t fa = ba & 0x007fffffu, fb = bb & 0x007fffffu;
    bool a_larger = fa > fb || (fa == fb && (ba >> 31) < (bb >> 31));
    bool take_b;
    if (sa == sb) take_b = !a_larger; else take_b = sa;  // (S, Q) -> Q = b; (Q, S) -> a
    return quiet(take_b ? b : a);
}
inline float fix(float r, float a, float b) {
    if (!std::isnan(r)) return r;
    if (std::isnan(a)) return std::isnan(b) ? pick(a, b) : quiet(a);
    if (std::isnan(b)) return quiet(b);
    return bits_f(0xffc00000u);
}
inline float add(float a, float b) { return fix(a + b, a, b); }
inline float sub(float a, float b) { return fix(a - b, a, b); }
inline float mul(float a, float b) { return fix(a * b, a, b); }
inline float div(float a, float b) { return fix(a / b, a, b); }
// nanrule.rs:119-161: the double precision add with the rule's NaN choice
inline double add64(double a, double b) {
    double r = a + b;
    if (!std::isnan(r)) return r;
    uint64_t ba, bb;
    std::memcpy(&ba, &a, 8);
    std::memcpy(&bb, &b, 8);
    const uint64_t Q = 0x0008000000000000ull;
    uint64_t o;
    if (std::isnan(a) && std::isnan(b)) {
        bool sa = (ba & Q) == 0, sb = (bb & Q) == 0;
        uint64_t fa = ba & 0x000fffffffffffffull, fb = bb & 0x000fffffffffffffull;
        bool a_larger = fa > fb || (fa == fb && (ba >> 63) < (bb >> 63));
        bool take_b = sa == sb ? !a_larger : sa;
        o = (take_b ? bb : ba) | Q;
    } else if (std::isnan(a)) {
        o = ba | Q;
    } else if (std::isnan(b)) {
        o = bb | Q;
    } else {
        o = 0xfff8000000000000ull;
    }
    double d;
    std::memcpy(&d, &o, 8);
    return d;
}
}  // namespace nr

// ---------------------------------------------------------------------------------------------
// engine images (image.rs:17-96): interleaved A,R,G,B, premultiplied, top row first

enum Fmt : int { U8 = 0, U16 = 1, F32 = 2 };

struct Image {
    int w = 0, h = 0;
    Fmt fmt = U8;
    std::vector<uint8_t> u8;
    std::vector<uint16_t> u16;
    std::vector<float> f32;
    Image() {}
    Image(int w_, int h_, Fmt f) : w(w_), h(h_), fmt(f) {
        size_t n = (size_t)w * h * 4;
        if (f == U8) u8.assign(n, 0);
        else if (f == U16) u16.assign(n, 0);
        else f32.assign(n, 0.0f);
    }
    size_t samples() const { return (size_t)w * h * 4; }
    void* data() { return fmt == U8 ? (void*)u8.data() : fmt == U16 ? (void*)u16.data() : (void*)f32.data(); }
    const void* data() const { return fmt == U8 ? (const void*)u8.data() : fmt == U16 ? (const void*)u16.data() : (const void*)f32.data(); }
    size_t bytes() const { return samples() * (fmt == U8 ? 1 : fmt == U16 ? 2 : 4); }
};

struct Plane {  // prep.rs:31-44
    int w = 0, h = 0;
    std::vector<float> d;
    Plane() {}
    Plane(int w_, int h_) : w(w_), h(h_), d((size_t)w_ * h_, 0.0f) {}
};

struct FlowField {  // flow.rs:37-76
    int w = 0, h = 0;
    std::vector<float> d;  // (dx, dy) interleaved
    FlowField() {}
    FlowField(int w_, int h_) : w(w_), h(h_), d((size_t)w_ * h_ * 2, 0.0f) {}
};

struct Coverage {  // warp.rs:57-97
    int w = 0, h = 0;
    std::vector<uint8_t> d;
};

// wire frames (crates/fx-core/src/frame.rs:79-141): u8 RGBA interleaved, u16 LE RGBA interleaved,
// f32 planar in the plane order G, B, R, A.
// image.rs:276-320: the per pixel premultiply / unpremultiply of the boundary
void premultiply_u8(const uint8_t p[4], uint8_t o[4]);
void premultiply_f32(const float p[4], float o[4]);
void unpremultiply_u8(const uint8_t p[4], uint8_t o[4]);
Image from_frame(const void* wire, int w, int h, Fmt fmt);                  // image.rs:178-206
Image from_frame_straight(const void* wire, int w, int h, Fmt fmt);         // image.rs:142-171
void to_frame(const Image& img, void* wire);                                 // image.rs:213-245
Image rows_reversed(const Image& img);                                       // image.rs:96-114

// ---------------------------------------------------------------------------------------------
// flow settings and geometry (flow.rs:83-197, prep.rs:63-146)

struct FlowSettings {
    int quality = 4;
    bool hiq = true;
    float sensitivity = 0.7f;
    bool prep_contrast_edge = false;
    bool prep_delinearize = false;
    bool track_alpha = false;
    bool video_range_luma = false;
    bool skip_refine = false;
    // Vertical border-row tap order of every separable filter of the solve: true is the tap
    // above first (flow/conv.rs:598-615, the reference's current order); false is the tap below
    // first, the order of the reference revision whose outputs the parity grid
    // parity/retime-flow/results/base.grid.tsv records.
    bool taps_above_first = true;
    // The wrap-around (360) mode of the pyramid's filters (flow.rs:236-275 with prep.rs:261-299):
    // the circular horizontal pass, the equirectangular vertical pass and resample.
    bool wrap = false;
};

struct Geometry {
    int reduction = 0, w = 0, h = 0, levels = 0;
    std::vector<std::pair<int, int>> sizes;
};

void flow_resolution(int q, bool hiq, int w, int h, int* r, int* w0, int* h0);
int level_count(int w0, int h0, int min_size);
bool geometry(const FlowSettings& s, int w, int h, Geometry* g, std::string* err);
void start_level(float sensitivity, int levels, int* start, float* damp);

// ---------------------------------------------------------------------------------------------
// filters (flow/conv.rs) and samplers (flow/sample.rs)

std::vector<float> gaussian_kernel(float r);
void convolve(float* data, int w, int h, int c, const float* k, int n, bool above_first);
void blur_gaussian(float* data, int w, int h, int c, float r, bool above_first);
void blur5(float* data, int w, int h, bool above_first);
float bilinear1(const float* img, int w, int h, float x, float y);
void bilinear2(const float* img, int w, int h, float x, float y, float out[2]);
Plane resample1(const Plane& src, int dw, int dh);
// conv.rs:643-660 (convolve_wrapx_above_first, c interleaved channels): hpass_wrapx then vpass_sphere
void convolve_wrapx_sphere(float* data, int w, int h, const float* k, int n, int c = 1);
// conv.rs:662-668 (blur_gaussian_wrapx_above_first): radii below 0.001 do nothing
void blur_gaussian_wrap(float* data, int w, int h, int c, float r);
// sample.rs:205-230 (resample1_wrapx): bilinear1_sphere at (x sw / dw, y sh / dh)
Plane resample1_wrapx(const Plane& src, int dw, int dh);

// ---------------------------------------------------------------------------------------------
// prep and pyramid (prep.rs, flow.rs:199-275)

Plane luma(const Image& img, bool track_alpha, bool video_range);
Plane reduce(Plane t, int r, bool above_first);
struct Pyramid {
    Geometry geo;
    std::vector<Plane> levels;  // band pass images, finest first
};
bool build_pyramid(const Image& img, const FlowSettings& s, Pyramid* out, std::string* err);

// ---------------------------------------------------------------------------------------------
// solver (flow.rs:277-1353)

std::vector<float> calc_grad(const float* img, int w, int h);
void edge_enhance(Plane& p, bool above_first);  // prep.rs:326-340
void delinearize(Plane& p);                      // prep.rs:296-307
float crt_powf(float x, float y);                // crt_powf.rs:229-268
std::vector<float> calc_a(const std::vector<float>& grad, int w, int h);
std::vector<float> calc_b(const float* i1, const float* i0, const float* grad, const float* flow, int w, int h);
void new_disp(float* flow, const float* a, const float* b, size_t npx);
std::vector<float> upsample_flow(const float* src, int sw, int sh, int dw, int dh);
void scale_values(float* d, size_t n, float f);
bool all_flow_out_of_range(const float* flow, int w, int h);
float block_cost(const float* a, const float* b, int w, int h, const float p[9], float x2, float y2, bool* some);
void block_match(const float* a, const float* b, float* flow, int w, int h);
void block_match_gated(const float* a, const float* b, float* flow, int w, int h, const float* gate);
void mask_gradient(float* grad, const float* mask, int w, int h);
std::vector<float> calc_b_masked(const float* i1, const float* i0, const float* grad, const float* flow, int w, int h,
                                 const float* mask_y);
bool mask_pyramid(const float* matte, int w, int h, const FlowSettings& s, std::vector<Plane>* levels, std::string* err);
FlowField solve_pyramids(const Pyramid& x, const Pyramid& y, const FlowSettings& s);
// flow/extras.rs:151-158 (UserLevel): the user displacement of one level, d interleaved (dx, dy)
// and the weight w, in the solver's internal sign
struct UserLevel {
    std::vector<float> d, w;
};
// points.rs:201-240 (user_displacement_with, no wrap): pairs (from x, from y, to x, to y) in output
// pixels of W x H, one level per level of geo, finest first
std::vector<UserLevel> user_displacement(const std::vector<std::array<float, 4>>& pairs, const Geometry& geo, int W,
                                         int H);
FlowField solve_pyramids_masked(const Pyramid& x, const Pyramid& y, const FlowSettings& s, const std::vector<Plane>* mx,
                                const std::vector<Plane>* my, bool gate,
                                const std::vector<UserLevel>* user = nullptr);
bool solve(const Image& x, const Image& y, const FlowSettings& s, FlowField* out, std::string* err);
bool solve_pair(const Image& a, const Image& b, const FlowSettings& s, FlowField* f_ab, FlowField* f_ba,
                std::string* err);

// ---------------------------------------------------------------------------------------------
// inverse warp (warp.rs), blend (blend.rs)

struct WarpOpts {
    bool hold = true;
    bool is360 = false;
    int mode = 1;
};
uint8_t sat_u8(float v);
uint16_t sat_u16(float v);
bool clip_to_rect(float x, float y, float* ix, float* iy, float w1, float h1);
// returns 0 ok, 1 mismatch, 2 unsupported; cov may be null
int inv_warp(Image& out, const Image& src, const FlowField& flow, float amount, WarpOpts o, Coverage* cov,
             std::string* err);
void copy_image(Image& out, const Image& src);
// warp.rs:415-442 Flow::bilerp (the warps' two channel flow sampler)
void warp_flow_bilerp(const FlowField& f, float x, float y, float out[2]);
// warp.rs:308-331 bilerp4 (with mix4's NaN rule repeat) over an image, w1 = w - 1, h1 = h - 1
void bilerp4_image(const Image& img, float x, float y, float out[4]);
// warp.rs:362-396 (bilerp360) on an engine image
void bilerp360_image(const Image& img, float x, float y, float out[4]);
void blend(Image& out, const Image& a, const Image& b, float w);
void lerp(Image& first, const Image& second, float w);

// ---------------------------------------------------------------------------------------------
// composition (compose/vector.rs, compose.rs) and the time model (timeline.rs)

struct Selection {  // timeline.rs:391-414
    float s0 = 0, s1 = 0;
    int a = 0, b = 1;
    float wa = 1.0f;
    bool exact = true;
    int vectors_quality = 4;
    int interp = 1;
};

struct ComposeSettings {
    int warp_mode = 0;        // 0 inverse, 1 Smart Blend (inverse + coverage), 2/3 forward
    bool video_360 = false;   // binary alpha Smart Blend / video range luma
    // the engine's wrap-around (360) flag (compose/vector.rs:1-13): the inverse warps of code 0, the
    // warps and fills of Smart Blend (codes 1 and 2), the Blur Compensation tail
    bool wrap_360 = false;
    bool quality_high = true;
    float blur = 0.0f;        // blur compensation slider
    bool taps_above_first = true;  // Stages::vertical_taps() of the hole fill (stages.rs:66-70)
    bool gouraud = false;     // forward warps of codes 2/3 as the Gouraud variant (stages::GouraudForward)
};

bool nearest_uses_f_ab(float wa, int code);
// compose_vectors for warping code 0 (and 1 once Smart Blend is present); flows may be null where
// the interpolation mode does not read them.
int compose_vectors(const ComposeSettings& cs, const Selection& sel, const Image& a, const Image& b,
                    const FlowField* f_ab, const FlowField* f_ba, Image* out, std::string* err);
int interpolate(const Selection& sel, const Image& a, const Image& b, Image* out, std::string* err);

}  // namespace orc
