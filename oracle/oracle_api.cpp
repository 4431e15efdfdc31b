// CPU oracle: the time model of the `retime` effect and the extern "C" surface the tests, the
// smoke check and the CPU baseline leg of the benchmark load through ctypes. TEST
// INFRASTRUCTURE ONLY; the product library never links it.
//
// Time model restated from plugins/retime-engine/src/timeline.rs (Rates :106-131,
// frame_positions :136-142, RemapTimeMap::src_pos :266-331, frame_time :336-344, select :451-469,
// exact_position :429-439), the parameter reads of frontend.rs:184-244 and the frame loop of
// crates/fx-cli/src/temporal.rs:183-250 (current_time = n * time_step, missing frames blank:
// host.rs:338-352).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "oracle_core.h"
#include "oracle_smart.h"
#include "oracle_forward.h"
#include "oracle_vectors.h"
#include "oracle_layers.h"
#include "oracle_filters.h"

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

namespace {

thread_local std::string g_err;

int fail(int rc, const std::string& e) {
    g_err = e;
    return rc;
}

struct Key {
    long long time;
    double value;
    bool ease;
    bool hold;
};

// crates/fx-core/src/curves.rs:282-310, :348-375 and :537-544: a float curve (constant when no
// key), keys sorted by time, a held key keeps its value up to the next
struct Curve {
    double constant = 0.0;
    std::vector<Key> keys;
    // keys at frames (ticks: frame * lts rounded half away from zero, time.rs:117-119); flags bit 0
    // ease, bit 1 hold
    void set(int n, const double* frames, const double* values, const int* flags, int lts) {
        keys.clear();
        for (int i = 0; i < n; i++) {
            long long t = (long long)std::llround(frames[i] * (double)lts);
            int f = flags ? flags[i] : 0;
            keys.push_back({t, values[i], (f & 1) != 0, (f & 2) != 0});
        }
        std::stable_sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) { return a.time < b.time; });
    }
    double at(long long time) const {
        if (keys.empty()) return constant;
        size_t last = keys.size() - 1;
        if (time <= keys[0].time) return keys[0].value;
        if (time >= keys[last].time) return keys[last].value;
        size_t i = 0;
        while (i + 1 < keys.size() && keys[i + 1].time <= time) i++;
        const Key &a = keys[i], &b = keys[i + 1];
        if (a.hold) return a.value;
        double u = (double)(time - a.time) / (double)(b.time - a.time);
        double f;
        if (!a.ease && !b.ease) f = u;
        else if (a.ease && b.ease) f = u * u * (3.0 - 2.0 * u);
        else if (a.ease) f = u * u * (2.0 - u);
        else f = u * (1.0 + u * (1.0 - u));
        return a.value + (b.value - a.value) * f;
    }
};

// crates/fx-core/src/fixed.rs:8-10
int32_t float_to_fixed(double f) {
    double v = f * 65536.0 + (f < 0.0 ? -0.5 : 0.5);
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0) return INT32_MAX;
    if (v <= -2147483648.0) return INT32_MIN;
    return (int32_t)v;
}
// frontend.rs:131-133
float fixed_reader(int32_t fixed, float scale) { return (float)((double)fixed * (1.0 / 65536.0)) * scale; }

int32_t cvtt_i32_d(double x) {  // timeline.rs:43-49
    if (x > -2147483649.0 && x < 2147483648.0) return (int32_t)x;
    return INT32_MIN;
}
int32_t cvtt_i32_f(float x) {  // timeline.rs:52-58
    if (x > -2147483904.0f && x < 2147483648.0f) return (int32_t)x;
    return INT32_MIN;
}

struct TimeMap {
    double frame_time_k = 0.05;  // FRAME_TIME_K (timeline.rs:25)
    bool plain_frame_time = false;  // plugins 03 and 04: trunc(dur * k + 0.5) at every rate
    Curve speed;
    int remap_mode = 1;  // Time Remap Mode: 1 Speed, 2 Frame Number
    Curve frame_num;
    double in_fps = 30.0, out_fps = 30.0;
    float dur = 100.0f;
    int lts = 100;
    int base = 0;
    // timeline.rs:266-331 (Src Time Offset 0)
    float src_pos(float t) {
        float lts_f = (float)lts;
        if (remap_mode == 2) {  // Frame Number: the curve at trunc((lts * t) + K), times in / out
            base = 0;
            int time = cvtt_i32_d((double)(lts_f * t) + 0.05);
            float v = (float)frame_num.at(time);
            return (float)((in_fps / out_fps) * (double)v);
        }
        float out = 0.0f;
        int time0 = cvtt_i32_d((double)(lts_f * t) + 0.05);
        (void)time0;
        base = 0;  // -trunc(0 * 2^-16)
        int n2 = cvtt_i32_f(t * 2.0f);
        float k = 1.0f;
        while ((float)n2 >= k) {
            int time = cvtt_i32_d((double)((lts_f * k) / 2.0f) + 0.05);
            float sp = (float)((double)float_to_fixed(speed.at(time)) / 6553600.0);
            out = (sp / 2.0f) + out;
            k += 1.0f;
        }
        float tt = t * 2.0f;
        float rem = tt - (k + -1.0f);
        if ((double)rem > 0.0001) {
            int time = cvtt_i32_d((double)((tt * lts_f) / 2.0f) + 0.05);
            float sp = (float)((double)float_to_fixed(speed.at(time)) / 6553600.0);
            out = ((rem * sp) / 2.0f) + out;
        }
        return (float)((in_fps / out_fps) * (double)out);
    }
    // timeline.rs:347-354 (marker): Src: Mark Segments at trunc(((f - base) * dur) + 0.5), the popup's
    // 1..5 as 0..4, anything else 0
    Curve marks;
    int marker(float f) const {
        float d = f - (float)base;
        int time = cvtt_i32_d((double)(d * dur) + 0.5);
        long long v = (long long)marks.at(time);
        return v >= 1 && v <= 5 ? (int)v - 1 : 0;
    }
    int frame_time(float f) const {  // timeline.rs:336-344
        float d = f - (float)base;
        if (plain_frame_time || std::fabs(in_fps - out_fps) < frame_time_k)
            return cvtt_i32_d((double)d * (double)dur + 0.5);
        return cvtt_i32_d((double)(d * dur) + (double)dur * frame_time_k);
    }
};

bool exact_position(float s0, float s1, float blur) {  // timeline.rs:429-439
    bool exact = true;
    float frac = s0 - std::floor(s0);
    if ((double)std::fabs(frac) > 0.005 && (double)std::fabs((float)((double)frac - 1.0)) > 0.005) exact = false;
    if ((double)std::fabs(s0 - s1) > 1e-6 && (double)blur > 0.005) exact = false;
    return exact;
}

}  // namespace

extern "C" {

// Parameters of one `retime` render, as the effect reads them (plugins/retime/src/lib.rs:59-99).
// Popups carry their raw 1-based values. The speed curve is constant (`nkeys == 0`) or keyed at
// frame numbers with an optional ease flag per key.
struct or_retime_params {
    int fps_num, fps_den;      // --fps
    int quality_high;          // --quality (1 high, 0 draft)
    double speed_percent;      // constant Speed %
    int nkeys;                 // keyed Speed % (0: constant)
    const double* key_frames;  // frame numbers of the keys
    const double* key_values;
    const int* key_ease;       // per key: bit 0 ease, bit 1 hold
    int vectors;               // popup 1..5 (5 Best)
    int frame_interp;          // popup 1..3 (2 Blend)
    int smart_blend;
    double sensitivity;        // slider, percent
    double blur_compensation;  // slider
    // The two orders the reference changed after its parity grid was recorded (docs/parity.md,
    // "The rewrite" table): 1, 1 is the reference's current code (plugins/retime/src/glue.rs:39-40,
    // flow/conv.rs:598-615); 0, 0 reproduces parity/retime-flow/results/base.grid.tsv.
    int rows_reversed;         // motion path on bottom-up rows
    int taps_above_first;      // vertical border rows of the solver's filters
    int video_360;             // "360 Video": video range luma, binary alpha Smart Blend
    int prep;                  // Image Prep popup: 1 None, 2 Contrast/Edge Enhance, 3 Delinearize; 4 both stages
                               // (retime-fgbg's Contrast/Edge, plugins/retime-fgbg/src/glue.rs:153-154)
    int track_rgb_a;           // retime-fgbg's Track RGB+A (alpha in the luma; the layered pyramids' 360 filters)
    // the rest of the time model (timeline.rs:106-131, :266-344): Time Remap Mode (0 or 1 Speed,
    // 2 Frame Number) with Frame Num constant or keyed, and "In FPS is Out FPS" off (own_input_rate:
    // the input rate Input: Frame Rate, the output rate the composition's)
    int remap_mode;
    double frame_num;
    int nfn_keys;
    const double* fn_key_frames;
    const double* fn_key_values;
    const int* fn_key_ease;    // per key: bit 0 ease, bit 1 hold
    int own_input_rate;
    double input_frame_rate;
    // the bias of the frame time between unequal rates (timeline.rs:25, :336-344): 0 reads as 0.05,
    // the reference's current value; 0.1 is the revision the parity grids record
    double frame_time_bias;
    // retime-fgbg's frame time: trunc(dur * k + 0.5) at every rate (timeline.rs:204-210)
    int frame_time_plain;
    // retime-fgbg's "360 Video": the engine's wrap-around flag (plugins/retime-fgbg/src/glue.rs:146-151),
    // the wrap solve, the 360 warps, fills and Blur Compensation
    int wrap_360;
    // Input: Fields (plugins/retime/src/lib.rs:70; 1 None, 2 Upper Field First, 3 Lower Field First):
    // any field order doubles the source rate (timeline.rs:123-125)
    int input_fields;
    // Src: Mark Segments (1 Cut A, 2 Cut B, 3 Cut C, 4 No MV Use Nearest, 5 No MV Frame Blend), a
    // constant or keys (a popup holds its value from one key to the next)
    int mark_segs;
    int nmark_keys;
    const double* mark_key_frames;
    const double* mark_key_values;
};

// timeline.rs:69-76: a rate within 2e-5 (an f32 difference) of 29.97, 59.94 or 23.976 becomes it
static double snap_rate(double rate) {
    for (double t : {29.97, 59.94, 23.976})
        if ((double)std::fabs((float)(rate - t)) < 2e-5) rate = t;
    return rate;
}

// The time map of the `retime` effect for its parameters (timeline.rs:106-131, the curves of
// frontend.rs:184-244). Returns the ticks per frame.
static int retime_map(const or_retime_params* p, TimeMap* map) {
    bool integer = p->fps_den == 1;
    int time_step = integer ? 100 : p->fps_den;
    double in = 30.0, out = 30.0;  // In FPS is Out FPS (default on): both rates 30 (timeline.rs:117-120)
    if (p->own_input_rate) {
        in = (double)((float)p->input_frame_rate * 1.0f);
        out = (double)p->fps_num / (double)p->fps_den;
    }
    map->lts = time_step;
    if (p->frame_time_bias > 0.0) map->frame_time_k = p->frame_time_bias;
    map->plain_frame_time = p->frame_time_plain != 0;
    map->in_fps = snap_rate(in);
    map->out_fps = snap_rate(out);
    if (p->input_fields == 2 || p->input_fields == 3) map->in_fps *= 2.0;
    map->dur = (float)(((double)time_step * map->out_fps) / map->in_fps);
    map->speed.constant = p->speed_percent;
    map->speed.set(p->nkeys, p->key_frames, p->key_values, p->key_ease, time_step);
    map->remap_mode = p->remap_mode == 2 ? 2 : 1;
    map->frame_num.constant = p->frame_num;
    map->frame_num.set(p->nfn_keys, p->fn_key_frames, p->fn_key_values, p->fn_key_ease, time_step);
    map->marks.constant = p->mark_segs > 0 ? p->mark_segs : 1;
    std::vector<int> hold(p->nmark_keys > 0 ? p->nmark_keys : 0, 2);
    map->marks.set(p->nmark_keys, p->mark_key_frames, p->mark_key_values, hold.data(), time_step);
    return time_step;
}

// The clip frame a position shows: host.rs:155-159 (frame_time) and the frame of that tick
static long long clip_frame(const TimeMap& map, int pos) {
    int time = map.frame_time((float)pos);
    return time >= 0 ? time / map.lts : -(((long long)-time + map.lts - 1) / map.lts);
}

const char* or_last_error(void) { return g_err.c_str(); }

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// ---- single functions, for the parity tests ---------------------------------------------------

int or_from_frame(const void* wire, int w, int h, int fmt, void* engine) {
    Image img = from_frame(wire, w, h, (Fmt)fmt);
    std::memcpy(engine, img.data(), img.bytes());
    return 0;
}

int or_to_frame(const void* engine, int w, int h, int fmt, void* wire) {
    Image img(w, h, (Fmt)fmt);
    std::memcpy(img.data(), engine, img.bytes());
    to_frame(img, wire);
    return 0;
}

int or_gaussian_kernel(float r, float* out, int cap) {
    std::vector<float> k = gaussian_kernel(r);
    int n = (int)k.size();
    for (int i = 0; i < n && i < cap; i++) out[i] = k[i];
    return n;
}

void or_start_level(float sensitivity, int levels, int* start, float* damp) { start_level(sensitivity, levels, start, damp); }

float or_block_cost(const float* b, int w, int h, const float* p9, float x2, float y2, int* some) {
    bool s;
    float c = block_cost(nullptr, b, w, h, p9, x2, y2, &s);
    *some = s ? 1 : 0;
    return c;
}

void or_convolve(float* data, int w, int h, int c, const float* k, int n, int above_first) {
    convolve(data, w, h, c, k, n, above_first != 0);
}
void or_calc_grad(const float* img, int w, int h, float* g) {
    auto v = calc_grad(img, w, h);
    std::memcpy(g, v.data(), v.size() * sizeof(float));
}
void or_new_disp(float* flow, const float* a, const float* b, long npx) { new_disp(flow, a, b, (size_t)npx); }
void or_upsample_flow(const float* src, int sw, int sh, int dw, int dh, float* dst) {
    auto v = upsample_flow(src, sw, sh, dw, dh);
    std::memcpy(dst, v.data(), v.size() * sizeof(float));
}
void or_block_match(const float* a, const float* b, float* flow, int w, int h) { block_match(a, b, flow, w, h); }
int or_all_out_of_range(const float* flow, int w, int h) { return all_flow_out_of_range(flow, w, h) ? 1 : 0; }

// Flow geometry: returns the level count and writes (w, h) per level into sizes (2 * cap ints).
int or_geometry(int quality, int hiq, int w, int h, int* reduction, int* sizes, int cap) {
    FlowSettings s;
    s.quality = quality;
    s.hiq = hiq != 0;
    Geometry g;
    std::string e;
    if (!geometry(s, w, h, &g, &e)) return fail(-1, e);
    *reduction = g.reduction;
    for (int i = 0; i < g.levels && i < cap; i++) { sizes[2 * i] = g.sizes[i].first; sizes[2 * i + 1] = g.sizes[i].second; }
    return g.levels;
}

// The band pass levels of one engine image, concatenated finest first.
int or_build_pyramid(const void* engine, int w, int h, int fmt, int quality, int hiq, float sensitivity, int above_first,
                     int prep, int wrap, int track_alpha, float* levels_out) {
    Image img(w, h, (Fmt)fmt);
    std::memcpy(img.data(), engine, img.bytes());
    FlowSettings s;
    s.wrap = wrap != 0;
    s.track_alpha = track_alpha != 0;
    s.prep_contrast_edge = prep == 2;
    s.prep_delinearize = prep == 3;
    s.taps_above_first = above_first != 0;
    s.quality = quality;
    s.hiq = hiq != 0;
    s.sensitivity = sensitivity;
    Pyramid p;
    std::string e;
    if (!build_pyramid(img, s, &p, &e)) return fail(-1, e);
    size_t off = 0;
    for (auto& l : p.levels) { std::memcpy(levels_out + off, l.d.data(), l.d.size() * sizeof(float)); off += l.d.size(); }
    return p.geo.levels;
}

// flow::solve_pair on two engine images; f_ab and f_ba receive the working size fields.
int or_solve_pair(const void* a_eng, const void* b_eng, int w, int h, int fmt, int quality, int hiq, float sensitivity,
                  int skip_refine, int above_first, float* f_ab, float* f_ba) {
    Image a(w, h, (Fmt)fmt), b(w, h, (Fmt)fmt);
    std::memcpy(a.data(), a_eng, a.bytes());
    std::memcpy(b.data(), b_eng, b.bytes());
    FlowSettings s;
    s.quality = quality;
    s.hiq = hiq != 0;
    s.sensitivity = sensitivity;
    s.skip_refine = skip_refine != 0;
    s.taps_above_first = above_first != 0;
    FlowField fab, fba;
    std::string e;
    if (!solve_pair(a, b, s, &fab, &fba, &e)) return fail(-1, e);
    std::memcpy(f_ab, fab.d.data(), fab.d.size() * sizeof(float));
    std::memcpy(f_ba, fba.d.data(), fba.d.size() * sizeof(float));
    return 0;
}

// flow::solve (flow.rs:1328-1332) X -> Y with the image prep (0 none, 2 Contrast/Edge Enhance,
// 3 Delinearize, as FlowSettings reads it): `out` receives the working size field.
int or_solve(const void* x_eng, const void* y_eng, int w, int h, int fmt, int quality, int hiq, float sensitivity,
             int skip_refine, int above_first, int prep, float* out) {
    Image x(w, h, (Fmt)fmt), y(w, h, (Fmt)fmt);
    std::memcpy(x.data(), x_eng, x.bytes());
    std::memcpy(y.data(), y_eng, y.bytes());
    FlowSettings s;
    s.quality = quality;
    s.hiq = hiq != 0;
    s.sensitivity = sensitivity;
    s.skip_refine = skip_refine != 0;
    s.taps_above_first = above_first != 0;
    s.prep_contrast_edge = prep == 2;
    s.prep_delinearize = prep == 3;
    FlowField f;
    std::string e;
    if (!solve(x, y, s, &f, &e)) return fail(-1, e);
    std::memcpy(out, f.d.data(), f.d.size() * sizeof(float));
    return 0;
}

// flow::extras::solve_pyramids_with (flow/extras.rs:244-265) for the test of the device entry that
// takes the caller's pyramids: the band pyramids of X and Y, the mask pyramids of two mattes (both
// null: none; ungated, as the effects build them) and the user displacement of the point pairs
// (from x, from y, to x, to y, npts of them; 0: none) built here and returned beside the flow
// (user_d: the levels' (dx, dy) interleaved, user_w: their weights, levels concatenated).
int or_solve_pyramids_with(const void* x_eng, const void* y_eng, int w, int h, int fmt, int quality, int hiq,
                           float sensitivity, int above_first, const float* matte_x, const float* matte_y,
                           const float* pts, int npts, float* x_levels, float* y_levels, float* mask_x, float* mask_y,
                           float* user_d, float* user_w, float* out) {
    Image x(w, h, (Fmt)fmt), y(w, h, (Fmt)fmt);
    std::memcpy(x.data(), x_eng, x.bytes());
    std::memcpy(y.data(), y_eng, y.bytes());
    FlowSettings s;
    s.quality = quality;
    s.hiq = hiq != 0;
    s.sensitivity = sensitivity;
    s.taps_above_first = above_first != 0;
    Pyramid px, py;
    std::string e;
    if (!build_pyramid(x, s, &px, &e) || !build_pyramid(y, s, &py, &e)) return fail(-1, e);
    size_t off = 0;
    for (size_t l = 0; l < px.levels.size(); l++) {
        std::memcpy(x_levels + off, px.levels[l].d.data(), px.levels[l].d.size() * sizeof(float));
        std::memcpy(y_levels + off, py.levels[l].d.data(), py.levels[l].d.size() * sizeof(float));
        off += px.levels[l].d.size();
    }
    std::vector<Plane> mx, my;
    if (matte_x) {
        if (!mask_pyramid(matte_x, w, h, s, &mx, &e) || !mask_pyramid(matte_y, w, h, s, &my, &e)) return fail(-1, e);
        size_t o = 0;
        for (size_t l = 0; l < mx.size(); l++) {
            std::memcpy(mask_x + o, mx[l].d.data(), mx[l].d.size() * sizeof(float));
            std::memcpy(mask_y + o, my[l].d.data(), my[l].d.size() * sizeof(float));
            o += mx[l].d.size();
        }
    }
    std::vector<UserLevel> u;
    if (npts > 0) {
        std::vector<std::array<float, 4>> pairs;
        for (int i = 0; i < npts; i++) pairs.push_back({pts[4 * i], pts[4 * i + 1], pts[4 * i + 2], pts[4 * i + 3]});
        u = user_displacement(pairs, px.geo, w, h);
        size_t od = 0, ow = 0;
        for (auto& lv : u) {
            std::memcpy(user_d + od, lv.d.data(), lv.d.size() * sizeof(float));
            std::memcpy(user_w + ow, lv.w.data(), lv.w.size() * sizeof(float));
            od += lv.d.size();
            ow += lv.w.size();
        }
    }
    FlowField f = solve_pyramids_masked(px, py, s, matte_x ? &mx : nullptr, matte_x ? &my : nullptr, false,
                                        npts > 0 ? &u : nullptr);
    std::memcpy(out, f.d.data(), f.d.size() * sizeof(float));
    return 0;
}

// warp::inv_warp / inv_warp_coverage on engine images (hold, mode 1, no 360). cov may be null.
int or_inv_warp(void* out_eng, const void* src_eng, int w, int h, int fmt, const float* flow, int fw, int fh, float amount,
                int hold, uint8_t* cov) {
    Image src(w, h, (Fmt)fmt), out(w, h, (Fmt)fmt);
    std::memcpy(src.data(), src_eng, src.bytes());
    std::memcpy(out.data(), out_eng, out.bytes());
    FlowField f(fw, fh);
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    WarpOpts o;
    o.hold = (hold & 1) != 0;  // bit 0 hold, bit 1 is360 (warp.rs:29-50)
    o.is360 = (hold & 2) != 0;
    Coverage c;
    std::string e;
    int rc = inv_warp(out, src, f, amount, o, cov ? &c : nullptr, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    if (cov) std::memcpy(cov, c.d.data(), c.d.size());
    return 0;
}

int or_blend(void* out_eng, const void* a_eng, const void* b_eng, int w, int h, int fmt, float wt) {
    Image a(w, h, (Fmt)fmt), b(w, h, (Fmt)fmt), out(w, h, (Fmt)fmt);
    std::memcpy(a.data(), a_eng, a.bytes());
    std::memcpy(b.data(), b_eng, b.bytes());
    blend(out, a, b, wt);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// compose::compose_vectors (warping code 0) on engine images with given flows.
int or_compose_vectors(const void* a_eng, const void* b_eng, int w, int h, int fmt, const float* f_ab, const float* f_ba,
                       int fw, int fh, float wa, int interp, void* out_eng) {
    Image a(w, h, (Fmt)fmt), b(w, h, (Fmt)fmt), out;
    std::memcpy(a.data(), a_eng, a.bytes());
    std::memcpy(b.data(), b_eng, b.bytes());
    FlowField fab(fw, fh), fba(fw, fh);
    if (f_ab) std::memcpy(fab.d.data(), f_ab, fab.d.size() * sizeof(float));
    if (f_ba) std::memcpy(fba.d.data(), f_ba, fba.d.size() * sizeof(float));
    ComposeSettings cs;
    Selection sel;
    sel.wa = wa;
    sel.interp = interp;
    std::string e;
    int rc = compose_vectors(cs, sel, a, b, f_ab ? &fab : nullptr, f_ba ? &fba : nullptr, &out, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// smartblend.rs:268-298 on engine images (binary != 0: the binary alpha variant)
int or_smart_blend(void* out_eng, const void* p1_eng, const void* p2_eng, int w, int h, int fmt, float wt, int binary) {
    Image p1(w, h, (Fmt)fmt), p2(w, h, (Fmt)fmt), out;
    std::memcpy(p1.data(), p1_eng, p1.bytes());
    std::memcpy(p2.data(), p2_eng, p2.bytes());
    smart_blend(out, p1, p2, wt, binary != 0);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// holefill.rs:452-491 in place on an engine image; mask_kind 1 u8, 2 u16, 3 f32
int or_fill_holes(void* eng, int w, int h, int fmt, const void* mask, int mask_kind, int above_first) {
    Image img(w, h, (Fmt)fmt);
    std::memcpy(img.data(), eng, img.bytes());
    std::string e;
    int rc = fill_holes(img, mask, mask_kind, above_first != 0, &e);
    if (rc) return fail(rc, e);
    std::memcpy(eng, img.data(), img.bytes());
    return 0;
}

// forward.rs:229-320 (pyramid != 0: textured) / :327-373 (Gouraud); cov may be null
int or_forward_warp(void* out_eng, const void* src_eng, int w, int h, int fmt, const float* flow, int fw, int fh,
                    float amount, int pyramid, uint8_t* cov) {
    Image src(w, h, (Fmt)fmt), out(w, h, (Fmt)fmt);
    std::memcpy(src.data(), src_eng, src.bytes());
    FlowField f(fw, fh);
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    Coverage c;
    std::string e;
    int rc = forward_warp(out, src, f, amount, pyramid != 0, cov ? &c : nullptr, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    if (cov) std::memcpy(cov, c.d.data(), c.d.size());
    return 0;
}

// forward/mesh.rs:63-91 and forward/pyramid.rs:20-36
float or_fw_mip_level(int w, int h, const float* flow, int fw, int fh, float amount, int c, int r) {
    FlowField f(fw, fh);
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    return fw_mip_level(w, h, f, amount, c, r);
}
int or_fw_level_count(int w, int h) { return fw_level_count(w, h); }

// forward/raster.rs:158-300 on one triangle (5 floats x, y, u, v, d per vertex); writes up to cap
// hits (x, y, u, v, d as floats) and returns their count, or -1 when the degenerate pass would
// write outside the image
int or_fw_triangle(const float* v, int w1, int h1, float* hits, int cap) {
    FwVtx t[3];
    for (int i = 0; i < 3; i++) t[i] = FwVtx{v[i * 5], v[i * 5 + 1], v[i * 5 + 2], v[i * 5 + 3], v[i * 5 + 4]};
    FwHits s;
    fw_triangle(t, w1, h1, &s);
    int n = 0;
    for (const FwHit& hh : s.hits) {
        if (n < cap) {
            float* o = hits + (size_t)n * 5;
            o[0] = (float)hh.x; o[1] = (float)hh.y; o[2] = hh.u; o[3] = hh.v; o[4] = hh.d;
        }
        n++;
    }
    return s.outside ? -1 : n;
}

// glibc's logf over an array (the mip level's libm call), for the device's logf check
void or_logf(const float* x, float* out, long n) {
    for (long i = 0; i < n; i++) out[i] = logf(x[i]);
}

// compose::compose_vectors with a warping code (0 inverse, 1 Smart Blend) and the binary alpha flag
int or_compose_vectors2(const void* a_eng, const void* b_eng, int w, int h, int fmt, const float* f_ab, const float* f_ba,
                        int fw, int fh, float wa, int interp, int warp_mode, int video_360, int taps_above_first,
                        int gouraud, void* out_eng) {
    Image a(w, h, (Fmt)fmt), b(w, h, (Fmt)fmt), out;
    std::memcpy(a.data(), a_eng, a.bytes());
    std::memcpy(b.data(), b_eng, b.bytes());
    FlowField fab(fw, fh), fba(fw, fh);
    if (f_ab) std::memcpy(fab.d.data(), f_ab, fab.d.size() * sizeof(float));
    if (f_ba) std::memcpy(fba.d.data(), f_ba, fba.d.size() * sizeof(float));
    ComposeSettings cs;
    cs.warp_mode = warp_mode;
    cs.video_360 = video_360 != 0;
    cs.taps_above_first = taps_above_first != 0;
    cs.gouraud = gouraud != 0;
    Selection sel;
    sel.wa = wa;
    sel.interp = interp;
    std::string e;
    int rc = compose_vectors(cs, sel, a, b, f_ab ? &fab : nullptr, f_ba ? &fba : nullptr, &out, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// warp/blurcomp.rs:176-559 (motion_blur, is360 off) on engine images
int or_motion_blur(void* out_eng, const void* src_eng, int w, int h, int fmt, const float* flow, int fw, int fh,
                   float amount, int hiq, float shutter) {
    Image src(w, h, (Fmt)fmt), out(w, h, (Fmt)fmt);
    std::memcpy(src.data(), src_eng, src.bytes());
    FlowField f(fw, fh);
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    std::string e;
    int rc = motion_blur(out, src, f, amount, hiq != 0, shutter, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// crt_powf.rs:229-268 over arrays (the Delinearize powf)
void or_crt_powf(const float* x, const float* y, float* out, int n) {
    for (int i = 0; i < n; i++) out[i] = crt_powf(x[i], y[i]);
}

// compose_vectors with the whole selection and compose settings (the Blur Compensation tail reads
// s0, s1, the slider and the render quality)
int or_compose_vectors3(const void* a_eng, const void* b_eng, int w, int h, int fmt, const float* f_ab, const float* f_ba,
                        int fw, int fh, float s0, float s1, float wa, int interp, int warp_mode, int video_360,
                        int taps_above_first, int gouraud, float blur, int quality_high, void* out_eng) {
    Image a(w, h, (Fmt)fmt), b(w, h, (Fmt)fmt), out;
    std::memcpy(a.data(), a_eng, a.bytes());
    std::memcpy(b.data(), b_eng, b.bytes());
    FlowField fab(fw, fh), fba(fw, fh);
    if (f_ab) std::memcpy(fab.d.data(), f_ab, fab.d.size() * sizeof(float));
    if (f_ba) std::memcpy(fba.d.data(), f_ba, fba.d.size() * sizeof(float));
    ComposeSettings cs;
    cs.warp_mode = warp_mode;
    cs.video_360 = video_360 != 0;
    cs.taps_above_first = taps_above_first != 0;
    cs.gouraud = gouraud != 0;
    cs.blur = blur;
    cs.quality_high = quality_high != 0;
    Selection sel;
    sel.s0 = s0;
    sel.s1 = s1;
    sel.wa = wa;
    sel.interp = interp;
    std::string e;
    int rc = compose_vectors(cs, sel, a, b, f_ab ? &fab : nullptr, f_ba ? &fba : nullptr, &out, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// ---- the whole effect ---------------------------------------------------------------------------

// One output frame's selection (timeline.rs:451-469) for output frame index n of a clip.
int or_select(const or_retime_params* p, int n, int w, int h, float* s0, float* s1, int* a, float* wa, int* exact,
              int* vq, int* interp) {
    TimeMap map;
    int time_step = retime_map(p, &map);
    int cur = n * time_step;
    float t0 = (float)cur / (float)time_step;
    float t1 = ((float)time_step + (float)cur) / (float)time_step;
    *s0 = map.src_pos(t0);
    *s1 = map.src_pos(t1);
    float blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
    *a = cvtt_i32_f(*s0);
    float frac = *s0 - (float)*a;
    *wa = 1.0f - frac;
    *exact = exact_position(*s0, *s1, blur) ? 1 : 0;
    int vqr = p->vectors - 1;
    *vq = (w >= 2 && h >= 2) ? vqr : 0;  // prep.rs:111-117
    *interp = p->frame_interp - 1;
    // timeline.rs:418-441 (marker_override, the core's g = trunc(s0 + 1.0)): markers that differ
    // give (No Vectors, Nearest), then "No MV, Use Nearest" (0, Nearest) and "No MV, Frame Blend"
    // (0, Blend)
    int g = cvtt_i32_d((double)*s0 + 1.0);
    int ma = map.marker((float)*a), mb = map.marker((float)g);
    if (ma != mb) { *vq = 0; *interp = 0; }
    if (ma == 3) { *vq = 0; *interp = 0; }
    if (ma == 4) { *vq = 0; *interp = 1; }
    return 0;
}

// The clip frames output frame n's positions a and a + 1 show (host.rs:155-159)
int or_clip_frames(const or_retime_params* p, int n, int w, int h, int* clip_a, int* clip_b) {
    float s0, s1, wa;
    int a, exact, vq, interp;
    or_select(p, n, w, h, &s0, &s1, &a, &wa, &exact, &vq, &interp);
    TimeMap map;
    retime_map(p, &map);
    *clip_a = (int)clip_frame(map, a);
    *clip_b = (int)clip_frame(map, a + 1);
    return 0;
}

// Renders output frame n of the `retime` effect over a raw clip of `nframes` wire frames into
// `out` (one wire frame). Returns 0, or a nonzero status with or_last_error() naming what is not
// restated.
// One output frame of the plain vector path; `gouraud`: the forward warps of codes 2/3 as the
// Gouraud variant (the stage set of retime-fgbg, plugins/retime-fgbg/src/glue.rs:142-143).
// `frames` holds the clip frames [first, first + count) of a clip of nframes frames (the whole clip:
// first 0, count nframes); a frame the selection needs outside that window is an error (-2).
static int retime_one(const void* frames, int nframes, int w, int h, int fmt, const or_retime_params* p, int n, void* out,
                      bool gouraud, const std::vector<std::array<float, 4>>* pts = nullptr, int first = 0, int count = -1) {
    if (count < 0) count = nframes;
    Fmt f = (Fmt)fmt;
    size_t es = f == U8 ? 1 : f == U16 ? 2 : 4;
    size_t frame_bytes = (size_t)w * h * 4 * es;
    bool integer = p->fps_den == 1;
    int time_step = integer ? 100 : p->fps_den;
    float sensitivity = fixed_reader(float_to_fixed(p->sensitivity), 1.0f) / 100.0f;
    float s0, s1, wa;
    int a, exact, vq, interp;
    or_select(p, n, w, h, &s0, &s1, &a, &wa, &exact, &vq, &interp);
    bool outside_window = false;
    TimeMap map;
    retime_map(p, &map);
    auto fetch = [&](int pos) -> Image {
        long long idx = clip_frame(map, pos);  // main_frame(position): frame_time, then the clip frame of that tick
        if (idx < 0 || idx >= nframes) return Image(w, h, f);
        if (idx < first || idx >= (long long)first + count) { outside_window = true; return Image(w, h, f); }
        return from_frame((const uint8_t*)frames + (size_t)(idx - first) * frame_bytes, w, h, f);
    };
    Image A = fetch(a), B = fetch(a + 1), result;
    if (outside_window) return fail(2, "output frame needs a source frame outside the window it was given");
    Selection sel;
    sel.s0 = s0; sel.s1 = s1; sel.a = a; sel.b = a + 1; sel.wa = wa; sel.exact = exact != 0;
    sel.vectors_quality = vq; sel.interp = interp;
    std::string e;
    if (vq != 0 && !exact) {
        if (interp < 0 || interp > 2) return fail(1, "bad interpolation mode");
        // plugin 01 runs the motion path on bottom-up rows (plugins/retime/src/glue.rs:39-40,
        // compose/vector.rs:303-314)
        Image ar = p->rows_reversed ? rows_reversed(A) : A, br = p->rows_reversed ? rows_reversed(B) : B;
        FlowSettings fs;
        fs.quality = vq;
        fs.hiq = p->quality_high != 0;
        fs.sensitivity = sensitivity;
        fs.taps_above_first = p->taps_above_first != 0;
        fs.video_range_luma = p->video_360 != 0;  // compose/vector.rs:72-82 (flow_settings)
        fs.track_alpha = p->track_rgb_a != 0;     // plugins/retime-fgbg/src/glue.rs:34-38
        fs.wrap = p->wrap_360 != 0;
        fs.prep_contrast_edge = p->prep == 2 || p->prep == 4;  // frontend.rs:224-225; 4: both stages, retime-fgbg's
        fs.prep_delinearize = p->prep == 3 || p->prep == 4;    // Contrast/Edge (plugins/retime-fgbg/src/glue.rs:153-154)
        FlowField fab, fba;
        bool have_ab = false, have_ba = false;
        if (pts && !pts->empty()) {
            // layers.rs:310-336 (single_layer_with_points): the solves take the points' user
            // displacement (points on the motion path's rows: y -> (H - 1) - y)
            std::vector<std::array<float, 4>> fwd, bwd;
            float last_row = (float)h - 1.0f;
            for (const auto& q : *pts) {
                float ay = p->rows_reversed ? last_row - q[1] : q[1], by = p->rows_reversed ? last_row - q[3] : q[3];
                fwd.push_back({q[0], ay, q[2], by});
                bwd.push_back({q[2], by, q[0], ay});
            }
            Pyramid pa, pb;
            if (!build_pyramid(ar, fs, &pa, &e) || !build_pyramid(br, fs, &pb, &e)) return fail(1, e);
            std::vector<UserLevel> uab = user_displacement(fwd, pa.geo, w, h), uba = user_displacement(bwd, pa.geo, w, h);
            bool one = interp == 0, ab = nearest_uses_f_ab(wa, p->smart_blend);
            if (!one || ab) { fab = solve_pyramids_masked(pa, pb, fs, nullptr, nullptr, false, &uab); have_ab = true; }
            if (!one || !ab) { fba = solve_pyramids_masked(pb, pa, fs, nullptr, nullptr, false, &uba); have_ba = true; }
        } else if (interp == 0) {
            if (nearest_uses_f_ab(wa, p->smart_blend)) {
                if (!solve(ar, br, fs, &fab, &e)) return fail(1, e);
                have_ab = true;
            } else {
                if (!solve(br, ar, fs, &fba, &e)) return fail(1, e);
                have_ba = true;
            }
        } else {
            if (!solve_pair(ar, br, fs, &fab, &fba, &e)) return fail(1, e);
            have_ab = have_ba = true;
        }
        ComposeSettings cs;
        cs.quality_high = fs.hiq;
        cs.blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
        cs.warp_mode = p->smart_blend;  // plugins/retime frontend: warp_mode = i32::from(smart_blend); 2, 3 the Warping popup of plugin 03
        cs.video_360 = p->video_360 != 0;
        cs.wrap_360 = p->wrap_360 != 0;
        cs.taps_above_first = p->taps_above_first != 0;
        cs.gouraud = gouraud;
        Image o;
        int rc = compose_vectors(cs, sel, ar, br, have_ab ? &fab : nullptr, have_ba ? &fba : nullptr, &o, &e);
        if (rc) return fail(rc, e);
        result = p->rows_reversed ? rows_reversed(o) : o;
    } else {
        int rc = interpolate(sel, A, B, &result, &e);
        if (rc) return fail(rc, e);
    }
    to_frame(result, out);
    return 0;
}

int or_retime_one(const void* frames, int nframes, int w, int h, int fmt, const or_retime_params* p, int n, void* out) {
    return retime_one(frames, nframes, w, h, fmt, p, n, out, false);
}

// Output frame n of a clip of nframes frames from the window of clip frames [first, first + count)
// alone (the frames one rank of a sharded render holds); -2 when the frame needs one outside it.
int or_retime_window(const void* frames, int first, int count, int nframes, int w, int h, int fmt,
                     const or_retime_params* p, int n, void* out) {
    return retime_one(frames, nframes, w, h, fmt, p, n, out, false, nullptr, first, count);
}

// ---- retime-fgbg with FG matte layers (plugins/retime-fgbg/src/glue.rs, compose.rs:149-170,
// layers.rs:530-567) --------------------------------------------------------------------------------

// matte.rs:141-188 (extract_raw): the channel (1 R, 2 G, 3 B, else alpha) of an engine image as a
// matte; 8 and 16 bpc v / white then clamped to 0..1, float the sample itself
static std::vector<float> extract_raw(const Image& img, int chan) {
    int c = chan == 1 ? 1 : chan == 2 ? 2 : chan == 3 ? 3 : 0;
    size_t n = (size_t)img.w * img.h;
    std::vector<float> m(n);
    for (size_t i = 0; i < n; i++) {
        float v;
        if (img.fmt == U8) v = (float)img.u8[i * 4 + c] / 255.0f;
        else if (img.fmt == U16) v = (float)img.u16[i * 4 + c] / 65535.0f;
        else { m[i] = img.f32[i * 4 + c] * 1.0f; continue; }
        m[i] = v > 1.0f ? 1.0f : v > 0.0f ? v : 0.0f;  // matte.rs:79-87 (clamp01)
    }
    return m;
}

static std::vector<float> flip_matte(const std::vector<float>& m, int w, int h) {
    std::vector<float> o(m.size());
    for (int y = 0; y < h; y++) std::memcpy(&o[(size_t)y * w], &m[(size_t)(h - 1 - y) * w], sizeof(float) * w);
    return o;
}

// Output frame n of retime-fgbg with `nfg` FG matte clips (wire frames back to back, the size and
// format of the footage): fg_chan / fg_sens per layer (popup 1..4, sensitivity 0..100). The
// selection is the retime time map of p (plugin 03's without the source time offset: the same at
// equal rates); p->smart_blend carries the warping code (0 to 3); fg_shrink the inverse matte shrink of
// every layer (16.16 reader); display the Display popup (1, 3 to 6). No tracking points.
int or_retime_fgbg_one(const void* frames, int nframes, const void* const* matte_clips, int nfg, const int* fg_chan,
                       const double* fg_sens, const double* fg_shrink, int display, const float* pts, const int* npts,
                       int w, int h, int fmt, const or_retime_params* p, int n, void* out) {
    // the tracking points of every layer at this frame (x, y at A, x, y at B; host rows), Main_BG last
    std::vector<std::vector<std::array<float, 4>>> points(nfg + 1);
    for (int k = 0, o = 0; pts && npts && k <= nfg; k++)
        for (int i = 0; i < npts[k]; i++, o++) points[k].push_back({pts[4 * o], pts[4 * o + 1], pts[4 * o + 2], pts[4 * o + 3]});
    // compose.rs:155-161: without FG layers the plain vector path (with points the single layer one),
    // with the stage set of the effect (the Gouraud forward warps)
    if (nfg == 0) return retime_one(frames, nframes, w, h, fmt, p, n, out, true, &points[0]);
    Fmt f = (Fmt)fmt;
    size_t es = f == U8 ? 1 : f == U16 ? 2 : 4;
    size_t frame_bytes = (size_t)w * h * 4 * es;
    bool integer = p->fps_den == 1;
    int time_step = integer ? 100 : p->fps_den;
    float s0, s1, wa;
    int a, exact, vq, interp;
    or_select(p, n, w, h, &s0, &s1, &a, &wa, &exact, &vq, &interp);
    // the FG matte frames are read straight (plugins/retime-fgbg/src/glue.rs:335, host.rs:311-314)
    TimeMap map;
    retime_map(p, &map);
    auto fetch = [&](const void* clip, int pos, bool straight) -> Image {
        long long idx = clip_frame(map, pos);
        if (idx < 0 || idx >= nframes) return Image(w, h, f);
        const uint8_t* fr = (const uint8_t*)clip + (size_t)idx * frame_bytes;
        return straight ? from_frame_straight(fr, w, h, f) : from_frame(fr, w, h, f);
    };
    Image A = fetch(frames, a, false), B = fetch(frames, a + 1, false), result;
    Selection sel;
    sel.s0 = s0; sel.s1 = s1; sel.a = a; sel.b = a + 1; sel.wa = wa; sel.exact = exact != 0;
    sel.vectors_quality = vq; sel.interp = interp;
    std::string e;
    if (display == 2) return fail(1, "the Source display composes no layer");
    int first, last;
    display_group(display, nfg, &first, &last);  // plugins/retime-fgbg/src/glue.rs:180
    std::vector<float> shrink;
    bool any_shrink = false;
    for (int k = 0; k < nfg; k++) {
        shrink.push_back(fixed_reader(float_to_fixed(fg_shrink[k]), 1.0f));
        any_shrink = any_shrink || shrink.back() != 0.0f;
    }
    // compose.rs (layered_exact): an FG layer with a shrink clears the exactness of the position
    if (vq != 0 && !(exact && !any_shrink)) {  // compose.rs:155-158: the layered vector path
        if (interp < 0 || interp > 2) return fail(1, "bad interpolation mode");
        LayerJob job;
        job.shrink = shrink;
        job.first = first;
        job.last = last;
        // layers.rs:571-590 (vector_path): the points on the motion path's rows, y -> (H - 1) - y
        float last_row = (float)h - 1.0f;
        for (auto& lp : points) {
            if (p->rows_reversed)
                for (auto& q : lp) { q[1] = last_row - q[1]; q[3] = last_row - q[3]; }
            job.points.push_back(lp);
        }
        for (int k = 0; k < nfg; k++) {
            std::vector<float> ma = extract_raw(fetch(matte_clips[k], a, true), fg_chan[k]);
            std::vector<float> mb = extract_raw(fetch(matte_clips[k], a + 1, true), fg_chan[k]);
            if (p->rows_reversed) { ma = flip_matte(ma, w, h); mb = flip_matte(mb, w, h); }
            job.mattes_a.push_back(std::move(ma));
            job.mattes_b.push_back(std::move(mb));
            job.sensitivity.push_back(fixed_reader(float_to_fixed(fg_sens[k]), 1.0f) / 100.0f);
        }
        job.sensitivity.push_back(fixed_reader(float_to_fixed(p->sensitivity), 1.0f) / 100.0f);
        job.fs.quality = vq;
        job.fs.hiq = p->quality_high != 0;
        job.fs.taps_above_first = p->taps_above_first != 0;
        job.fs.track_alpha = p->track_rgb_a != 0;
        job.fs.wrap = p->wrap_360 != 0;
        job.cs.wrap_360 = p->wrap_360 != 0;
        job.cs.quality_high = p->quality_high != 0;
        job.cs.blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
        job.cs.warp_mode = p->smart_blend;
        job.cs.gouraud = true;  // plugins/retime-fgbg/src/glue.rs:142-143: every forward warp is the Gouraud variant
        job.cs.taps_above_first = p->taps_above_first != 0;
        job.sel = sel;
        Image ar = p->rows_reversed ? rows_reversed(A) : A, br = p->rows_reversed ? rows_reversed(B) : B;
        Image o;
        int rc = compose_layers_plates(job, ar, br, &o, &e);
        if (rc) return fail(rc, e);
        result = p->rows_reversed ? rows_reversed(o) : o;
    } else if (first == 0 && last == nfg && !any_shrink) {
        // compose.rs:166-169 with the full group fast path (layers.rs:177-179): the plain one
        int rc = interpolate(sel, A, B, &result, &e);
        if (rc) return fail(rc, e);
    } else if (first == last) {
        // layers.rs:414-436: a single group display rebuilds the group's plate of each frame
        std::vector<std::vector<float>> ma, mb;
        for (int k = 0; k < nfg; k++) {
            ma.push_back(extract_raw(fetch(matte_clips[k], a, true), fg_chan[k]));
            mb.push_back(extract_raw(fetch(matte_clips[k], a + 1, true), fg_chan[k]));
        }
        Image ra, rb;
        bool rev = p->rows_reversed != 0, above = p->taps_above_first != 0;
        bool wrap = p->wrap_360 != 0;
        int rc = rebuilt_plate(A, ma, shrink, first, rev, above, &ra, &e, wrap);
        if (!rc) rc = rebuilt_plate(B, mb, shrink, first, rev, above, &rb, &e, wrap);
        if (!rc) rc = interpolate(sel, ra, rb, &result, &e);
        if (rc) return fail(rc, e);
    } else {
        return fail(1, "the full group of an unwarped frame with an inverse matte shrink is not restated");
    }
    to_frame(result, out);
    return 0;
}

// Renders `nout` output frames of the `retime` effect over a raw clip of `nframes` wire frames.
int or_retime_clip(const void* frames, int nframes, int w, int h, int fmt, const or_retime_params* p, int nout,
                   void* out) {
    Fmt f = (Fmt)fmt;
    size_t es = f == U8 ? 1 : f == U16 ? 2 : 4;
    size_t frame_bytes = (size_t)w * h * 4 * es;
    for (int n = 0; n < nout; n++) {
        int rc = or_retime_one(frames, nframes, w, h, fmt, p, n, (uint8_t*)out + (size_t)n * frame_bytes);
        if (rc) return rc;
    }
    return 0;
}

// ---- the masked solve of the layered paths (flow/extras.rs) -----------------------------------------

int or_mask_pyramid(const float* matte, int w, int h, int quality, int hiq, int above_first, float* out, int* sizes,
                    int cap_levels) {
    FlowSettings s;
    s.quality = quality;
    s.hiq = hiq != 0;
    s.taps_above_first = above_first != 0;
    std::vector<Plane> lv;
    std::string e;
    if (!mask_pyramid(matte, w, h, s, &lv, &e)) return -fail(1, e);
    size_t off = 0;
    for (size_t i = 0; i < lv.size() && (int)i < cap_levels; i++) {
        sizes[2 * i] = lv[i].w;
        sizes[2 * i + 1] = lv[i].h;
        std::memcpy(out + off, lv[i].d.data(), lv[i].d.size() * sizeof(float));
        off += lv[i].d.size();
    }
    return (int)lv.size();
}

void or_mask_gradient(float* grad, const float* mask, int w, int h) { mask_gradient(grad, mask, w, h); }

void or_calc_b_masked(const float* i1, const float* i0, const float* grad, const float* flow, int w, int h,
                      const float* mask_y, float* out) {
    std::vector<float> b = calc_b_masked(i1, i0, grad, flow, w, h, mask_y);
    std::memcpy(out, b.data(), b.size() * sizeof(float));
}

void or_block_match_gated(const float* a, const float* b, float* flow, int w, int h, const float* gate) {
    block_match_gated(a, b, flow, w, h, gate);
}

// flow/extras.rs:244-265 with the mask pyramids of two mattes (0..1 at the image size, either may
// be null: no masks) and the block matching gate on or off; out: the flow at the working size
int or_solve_masked(const void* x_eng, const void* y_eng, int w, int h, int fmt, int quality, int hiq, float sensitivity,
                    int above_first, const float* matte_x, const float* matte_y, int gate, float* out) {
    Image x(w, h, (Fmt)fmt), y(w, h, (Fmt)fmt);
    std::memcpy(x.data(), x_eng, x.bytes());
    std::memcpy(y.data(), y_eng, y.bytes());
    FlowSettings s;
    s.quality = quality;
    s.hiq = hiq != 0;
    s.sensitivity = sensitivity;
    s.taps_above_first = above_first != 0;
    Pyramid px, py;
    std::string e;
    if (!build_pyramid(x, s, &px, &e) || !build_pyramid(y, s, &py, &e)) return fail(1, e);
    std::vector<Plane> mx, my;
    bool masks = matte_x && matte_y;
    if (masks && (!mask_pyramid(matte_x, w, h, s, &mx, &e) || !mask_pyramid(matte_y, w, h, s, &my, &e))) return fail(1, e);
    FlowField f = solve_pyramids_masked(px, py, s, masks ? &mx : nullptr, masks ? &my : nullptr, gate != 0);
    std::memcpy(out, f.d.data(), f.d.size() * sizeof(float));
    return 0;
}

// ---- the layered composition with plates (layers/plates.rs) ------------------------------------------

// One layered output frame: engine images A and B, nfg FG mattes at A and at B (nfg * w * h floats
// each, FG1 first), nfg + 1 sensitivities (0..1), the selection weight / interpolation and the
// settings; out: the engine image
int or_compose_layers(const void* a_eng, const void* b_eng, int w, int h, int fmt, int nfg, const float* mattes_a,
                      const float* mattes_b, const float* sens, const float* shrink, int first, int last,
                      const float* pts, const int* npts, int quality, int hiq, int above_first, int warp_mode,
                      int video_360, int gouraud, float wa, int interp, void* out_eng) {
    Image a(w, h, (Fmt)fmt), b(w, h, (Fmt)fmt), out;
    std::memcpy(a.data(), a_eng, a.bytes());
    std::memcpy(b.data(), b_eng, b.bytes());
    LayerJob job;
    size_t n = (size_t)w * h;
    for (int j = 0; j < nfg; j++) {
        job.mattes_a.emplace_back(mattes_a + j * n, mattes_a + (j + 1) * n);
        job.mattes_b.emplace_back(mattes_b + j * n, mattes_b + (j + 1) * n);
    }
    job.sensitivity.assign(sens, sens + nfg + 1);
    if (shrink) job.shrink.assign(shrink, shrink + nfg);
    job.first = first;
    job.last = last;
    job.points.resize(nfg + 1);
    for (int k = 0, o = 0; pts && npts && k <= nfg; k++)
        for (int i = 0; i < npts[k]; i++, o++) job.points[k].push_back({pts[4 * o], pts[4 * o + 1], pts[4 * o + 2], pts[4 * o + 3]});
    job.fs.quality = quality;
    job.fs.hiq = hiq != 0;
    job.fs.video_range_luma = video_360 != 0;
    job.fs.taps_above_first = above_first != 0;
    job.cs.warp_mode = warp_mode;
    job.cs.video_360 = video_360 != 0;
    job.cs.taps_above_first = above_first != 0;
    job.cs.gouraud = gouraud != 0;
    job.sel.wa = wa;
    job.sel.interp = interp;
    job.sel.exact = false;
    job.sel.vectors_quality = quality;
    std::string e;
    int rc = compose_layers_plates(job, a, b, &out, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// ---- Create Vectors (plugins/create-vectors/src/glue.rs:488-569, one layer, Display Motion Vectors)

struct or_cv_params {
    int fps_num, fps_den;
    int quality_high;
    int vector_resolution;  // popup: 1 Normal (half res), 2 Full res
    double max_displace;    // Max Displace (16.16 reader)
    int track_frame;        // popup: 1 Previous, 2 Next
    double sensitivity;     // Main_BG: Sensitivity, 0..100 (16.16 reader)
    int track_rgb_a;
    int rows_reversed;      // the plugin turns the frames upside down for the engine (glue.rs:28-37)
    int taps_above_first;   // the solver's vertical border tap order
    int prep;               // Image Prep popup: 1 None, 2 Contrast/Edge Enhance, 3 Delinearize
    int display;            // Display popup: 2 Motion Vectors (0 reads as 2), 3 Debug
    int debug_view_method;  // Debug View Method: 1 Warp, 2 Blend, 3 Diff, 4 Detail Compare, 5 Edge Compare
    int debug_textured;     // the Debug warp textured (the revision the parity grid records); 0 the
                            // Gouraud variant of the reference's current code (glue.rs:39-42)
};

// vectors.rs:57-130 on a flow field; dst_fmt 0/1/2
int or_encode_vectors(void* out_eng, int w, int h, int fmt, const float* flow, int fw, int fh, float scale) {
    Image out(w, h, (Fmt)fmt);
    FlowField f(fw, fh);
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    std::string e;
    int rc = encode_vectors(out, f, scale, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out_eng, out.data(), out.bytes());
    return 0;
}

// Output frame n of the Create Vectors effect over a raw clip (wire frames back to back).
int or_create_vectors_one(const void* frames, int nframes, int w, int h, int fmt, const or_cv_params* p, int n,
                          const float* pts, int npts, void* out) {
    Fmt f = (Fmt)fmt;
    size_t es = f == U8 ? 1 : f == U16 ? 2 : 4;
    size_t frame_bytes = (size_t)w * h * 4 * es;
    int ts = p->fps_den == 1 ? 100 : p->fps_den;
    int ct = n * ts;
    // create_vectors.rs:59-62, :71-89, :92-97
    uint32_t frame = (uint32_t)cvtt64f((float)ct / (float)ts + 0.5f);
    float nf = (float)(int32_t)frame;
    float fa = nf, fb = nf;
    bool debug = p->display == 3;
    if (!debug) {
        if (p->track_frame == 1) fb = nf - 1.0f;
        else if (p->track_frame == 2) fb = nf + 1.0f;
    } else {  // create_vectors.rs:71-89: the Debug display swaps the roles
        if (p->track_frame == 1) fa = nf + 1.0f;
        else if (p->track_frame == 2) fa = nf - 1.0f;
    }
    int a = cvtt32(fa), b = cvtt32(fb);
    auto frame_time = [&](int k) {
        float tsf = (float)ts, x = (float)k;
        float t = x < 0.0f ? -((-x) * tsf + 0.5f) : tsf * x + 0.5f;
        return cvtt32(t);
    };
    auto fetch = [&](int t) -> Image {  // glue.rs:399-421: a tick outside the clip is transparent
        long long idx = t >= 0 ? t / ts : -(((long long)-t + ts - 1) / ts);
        if (idx < 0 || idx >= nframes) return Image(w, h, f);
        return from_frame((const uint8_t*)frames + (size_t)idx * frame_bytes, w, h, f);
    };
    Image x = fetch(frame_time(a)), y = fetch(frame_time(b));
    if (!(w >= 2 && h >= 2)) {  // glue.rs:537-540
        to_frame(zero_vectors_image(w, h, f), out);
        return 0;
    }
    if (p->rows_reversed) {
        x = rows_reversed(x);
        y = rows_reversed(y);
    }
    CreateVectorsSettings cs;
    cs.quality = p->vector_resolution == 2 ? 5 : 4;
    cs.hiq = p->quality_high != 0;
    cs.sensitivity = fixed_reader(float_to_fixed(p->sensitivity), 1.0f) / 100.0f;
    cs.track_rgb_a = p->track_rgb_a != 0;
    cs.max_displace = (1.0f / 1.0f) * fixed_reader(float_to_fixed(p->max_displace), 1.0f);
    cs.taps_above_first = p->taps_above_first != 0;
    cs.prep_contrast_edge = p->prep == 2;
    cs.prep_delinearize = p->prep == 3;
    Image enc;
    std::string e;
    int rc;
    if (debug) {
        // plugins/create-vectors/src/glue.rs:557-566: the flow X -> Y of the job (with the points'
        // user displacement), the view with the Gouraud forward warp (create_vectors.rs:408-416)
        FlowSettings fs;
        fs.quality = cs.quality;
        fs.hiq = cs.hiq;
        fs.sensitivity = cs.sensitivity;
        fs.track_alpha = cs.track_rgb_a;
        fs.taps_above_first = cs.taps_above_first;
        fs.prep_contrast_edge = cs.prep_contrast_edge;
        fs.prep_delinearize = cs.prep_delinearize;
        FlowField flow;
        if (pts && npts > 0) {
            std::vector<std::array<float, 4>> pairs;
            float last_row = (float)h - 1.0f;
            for (int i = 0; i < npts; i++) {
                float ay = pts[4 * i + 1], by = pts[4 * i + 3];
                if (p->rows_reversed) { ay = last_row - ay; by = last_row - by; }
                pairs.push_back({pts[4 * i], ay, pts[4 * i + 2], by});
            }
            Pyramid px, py;
            if (!build_pyramid(x, fs, &px, &e) || !build_pyramid(y, fs, &py, &e)) return fail(1, e);
            std::vector<UserLevel> u = user_displacement(pairs, px.geo, w, h);
            flow = solve_pyramids_masked(px, py, fs, nullptr, nullptr, false, &u);
        } else if (!solve(x, y, fs, &flow, &e)) {
            return fail(1, e);
        }
        int m = p->debug_view_method;
        int code = m == 1 ? 4 : m == 2 ? 0 : m == 3 ? 1 : m == 4 ? 2 : 3;  // glue.rs:120-130
        rc = debug_view(x, y, flow, code, p->debug_textured == 0, &enc, &e);
    } else if (pts && npts > 0) {
        // create_vectors.rs:321-351 (layer_flows_on, one layer): the solve X -> Y with the user
        // displacement of the points (plugins/create-vectors/src/glue.rs:550-553: on the rows of the
        // frames, y -> (H - 1) - y when they are turned)
        std::vector<std::array<float, 4>> pairs;
        float last_row = (float)h - 1.0f;
        for (int i = 0; i < npts; i++) {
            float ay = pts[4 * i + 1], by = pts[4 * i + 3];
            if (p->rows_reversed) { ay = last_row - ay; by = last_row - by; }
            pairs.push_back({pts[4 * i], ay, pts[4 * i + 2], by});
        }
        FlowSettings fs;
        fs.quality = cs.quality;
        fs.hiq = cs.hiq;
        fs.sensitivity = cs.sensitivity;
        fs.track_alpha = cs.track_rgb_a;
        fs.taps_above_first = cs.taps_above_first;
        fs.prep_contrast_edge = cs.prep_contrast_edge;
        fs.prep_delinearize = cs.prep_delinearize;
        Pyramid px, py;
        if (!build_pyramid(x, fs, &px, &e) || !build_pyramid(y, fs, &py, &e)) return fail(1, e);
        std::vector<UserLevel> u = user_displacement(pairs, px.geo, w, h);
        FlowField flow = solve_pyramids_masked(px, py, fs, nullptr, nullptr, false, &u);
        enc = Image(w, h, f);
        rc = encode_vectors(enc, flow, cs.max_displace, &e);
    } else {
        rc = create_vectors(x, y, cs, &enc, &e);
    }
    if (rc) return fail(rc, e);
    if (p->rows_reversed) enc = rows_reversed(enc);
    to_frame(enc, out);
    return 0;
}

int or_create_vectors_clip(const void* frames, int nframes, int w, int h, int fmt, const or_cv_params* p, int nout,
                           const float* pts, const int* npts, void* out) {
    Fmt f = (Fmt)fmt;
    size_t es = f == U8 ? 1 : f == U16 ? 2 : 4;
    size_t frame_bytes = (size_t)w * h * 4 * es;
    for (int n = 0, o = 0; n < nout; n++) {
        int np = pts && npts ? npts[n] : 0;
        int rc = or_create_vectors_one(frames, nframes, w, h, fmt, p, n, np ? pts + 4 * o : nullptr, np,
                                       (uint8_t*)out + (size_t)n * frame_bytes);
        if (rc) return rc;
        o += np;
    }
    return 0;
}

}  // extern "C"

// ---- Vectors In (plugins/vectors-in: glue.rs:440-495, vectorin.rs, timemap.rs) ----------------------

extern "C" {

// Parameters of one `vectors-in` render (plugins/vectors-in/src/lib.rs), popups 1-based. In FPS is
// Out FPS is on (the input rate 30, the output rate the composition's: timemap.rs, glue.rs:204-215).
struct or_vecin_params {
    int fps_num, fps_den;      // composition rate (--fps)
    int quality_high;
    double speed_percent;      // constant Speed %
    int nkeys;                 // keyed Speed % (0: constant)
    const double* key_frames;
    const double* key_values;
    const int* key_ease;       // per key: bit 0 ease, bit 1 hold
    int frame_interp;          // popup 1..3
    int warping;               // popup: 1 Inverse, 2 Forward (glue.rs:94-100)
    double blur_compensation;
    double max_displace;       // Vectors: Max Displace
    double vec_scale_x, vec_scale_y;
    // the orders of the plugin's render (glue.rs:44-63): bottom-up rows, the tap above first in the
    // vertical passes of the fills, the Gouraud forward warp
    int rows_reversed;
    int taps_above_first;
    int gouraud;
    // the presence of a vector layer: 0 a set layer is present at every time (vectorin.rs:41-58,
    // the reference's current code); 1 present only where its clip has a frame at the output
    // frame's time, the error fill when neither is (the revision the parity grid records)
    int probe_current_time;
    // Time Remap Mode (0 or 1 Speed, 2 Frame Number) and Frame Num, constant or keyed
    int remap_mode;
    double frame_num;
    int nfn_keys;
    const double* fn_key_frames;
    const double* fn_key_values;
    const int* fn_key_ease;    // per key: bit 0 ease, bit 1 hold
    int own_input_rate;        // In FPS is Out FPS off: the input rate Input: Frame Rate
    double input_frame_rate;
    // Src: Mark Segments (plugins/vectors-in/src/lib.rs:93), constant or keys held between keys
    int mark_segs;
    int nmark_keys;
    const double* mark_key_frames;
    const double* mark_key_values;
};

// compose/vector.rs:329-345 (flow_from_vector_image_with) over an engine image, for the tests
int or_flow_from_vectors(const void* vec_eng, int w, int h, int fmt, float max_displace, float sx, float sy,
                         int above_first, float* flow_out) {
    Image v(w, h, (Fmt)fmt);
    std::memcpy(v.data(), vec_eng, v.bytes());
    FlowField f;
    std::string e;
    int rc = flow_from_vector_image(v, max_displace, sx, sy, above_first != 0, &f, &e);
    if (rc) return fail(rc, e);
    std::memcpy(flow_out, f.d.data(), f.d.size() * sizeof(float));
    return 0;
}

// vectors.rs:474-522 alone
int or_decode_vectors(const void* vec_eng, int w, int h, int fmt, float max_displace, float* flow_out) {
    Image v(w, h, (Fmt)fmt);
    std::memcpy(v.data(), vec_eng, v.bytes());
    FlowField f = decode_vectors(v, max_displace);
    std::memcpy(flow_out, f.d.data(), f.d.size() * sizeof(float));
    return 0;
}

// holefill.rs:497-518 on an interleaved flow in place
int or_fill_flow_holes(float* flow, int w, int h, const void* mask, int mask_kind, int above_first) {
    FlowField f(w, h);
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    std::string e;
    int rc = fill_flow_holes(f, mask, mask_kind, above_first != 0, &e);
    if (rc) return fail(rc, e);
    std::memcpy(flow, f.d.data(), f.d.size() * sizeof(float));
    return 0;
}

// compose/vector.rs:370-397
int or_invert_flow(const float* flow, int w, int h, int pyramid, int above_first, float* out) {
    FlowField f(w, h), o;
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    std::string e;
    int rc = invert_flow(f, pyramid != 0, above_first != 0, &o, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out, o.d.data(), o.d.size() * sizeof(float));
    return 0;
}

// vectorin.rs:125-155 on an engine image in place
void or_matte_step(void* eng, int w, int h, int fmt, const float* matte) {
    Image v(w, h, (Fmt)fmt);
    std::memcpy(v.data(), eng, v.bytes());
    matte_step(v, std::vector<float>(matte, matte + (size_t)w * h));
    std::memcpy(eng, v.data(), v.bytes());
}

// The selection of output frame n of the Vectors In effect: plugin 01's Speed map with the plugin's
// rates (in 30, out the composition's: timemap.rs, glue.rs:204-215) and the constant quality 4.
// Returns the ticks per frame.
static int vecin_select(const or_vecin_params* p, int n, int w, int h, TimeMap* map, Selection* sel) {
    bool integer = p->fps_den == 1;
    int time_step = integer ? 100 : p->fps_den;
    double comp = (double)p->fps_num / (double)p->fps_den;
    double in = p->own_input_rate ? (double)((float)p->input_frame_rate * 1.0f) : 30.0;
    map->lts = time_step;
    map->in_fps = snap_rate(in);
    map->out_fps = snap_rate(comp);
    map->dur = (float)(((double)time_step * map->out_fps) / map->in_fps);
    map->speed.constant = p->speed_percent;
    map->speed.set(p->nkeys, p->key_frames, p->key_values, p->key_ease, time_step);
    map->remap_mode = p->remap_mode == 2 ? 2 : 1;
    map->frame_num.constant = p->frame_num;
    map->frame_num.set(p->nfn_keys, p->fn_key_frames, p->fn_key_values, p->fn_key_ease, time_step);
    int cur = n * time_step;
    float t0 = (float)cur / (float)time_step;
    float t1 = ((float)time_step + (float)cur) / (float)time_step;
    sel->s0 = map->src_pos(t0);
    sel->s1 = map->src_pos(t1);
    float blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
    sel->a = cvtt_i32_f(sel->s0);
    sel->b = sel->a + 1;
    sel->wa = 1.0f - (sel->s0 - (float)sel->a);
    sel->exact = exact_position(sel->s0, sel->s1, blur);
    sel->vectors_quality = (w >= 2 && h >= 2) ? 4 : 0;
    sel->interp = p->frame_interp - 1;
    // timeline.rs:418-441 (marker_override) with the effect's marker, Src: Mark Segments at
    // T(f) = trunc((f64)dur * (f64)f + 0.5) (plugins/vectors-in/src/timemap.rs:49-70)
    Curve marks;
    marks.constant = p->mark_segs > 0 ? p->mark_segs : 1;
    std::vector<int> hold(p->nmark_keys > 0 ? p->nmark_keys : 0, 2);
    marks.set(p->nmark_keys, p->mark_key_frames, p->mark_key_values, hold.data(), time_step);
    auto marker = [&](float f) {
        long long v = (long long)marks.at(cvtt_i32_d((double)map->dur * (double)f + 0.5));
        return v >= 1 && v <= 5 ? (int)v - 1 : 0;
    };
    int ma = marker((float)sel->a), mb = marker((float)cvtt_i32_d((double)sel->s0 + 1.0));
    if (ma != mb) { sel->vectors_quality = 0; sel->interp = 0; }
    if (ma == 3) { sel->vectors_quality = 0; sel->interp = 0; }
    if (ma == 4) { sel->vectors_quality = 0; sel->interp = 1; }
    return time_step;
}

// vecin_select for the tests: s0, s1, wa as floats, then a, exact, vectors quality, interp and the
// clip frames of A and B at T(A), T(B)
int or_vecin_select(const or_vecin_params* p, int n, int w, int h, float* f3, int* i6) {
    TimeMap map;
    Selection sel;
    int ts = vecin_select(p, n, w, h, &map, &sel);
    auto idx = [&](int pos) -> int {
        int time = cvtt_i32_d((double)map.dur * (double)(float)pos + 0.5);
        return (int)(time >= 0 ? time / ts : -(((long long)-time + ts - 1) / ts));
    };
    f3[0] = sel.s0; f3[1] = sel.s1; f3[2] = sel.wa;
    i6[0] = sel.a; i6[1] = sel.exact ? 1 : 0; i6[2] = sel.vectors_quality; i6[3] = sel.interp;
    i6[4] = idx(sel.a); i6[5] = idx(sel.b);
    return 0;
}

// Output frame n of the single layer `vectors-in` render (glue.rs:386-495 with nfg 0, Display not
// Source): the footage clip `frames` (nframes wire frames), the vector layers `Vectors: Next` and
// `Vectors: Prev` as wire clips of n_next / n_prev frames (NULL: the layer is not set; a frame past
// a set layer's end is transparent, vectorin.rs:41-58). F_AB is Next at T(A), F_BA Prev at T(B)
// (vectorin.rs:203-227); a missing one is the other's inversion when the composition reads it
// (compose/vector.rs:422-447). No vector layer: the plugin's size mismatch error fill.
int or_vectors_in_one(const void* frames, int nframes, const void* vec_next, int n_next, const void* vec_prev, int n_prev,
                      int w, int h, int fmt, const or_vecin_params* p, int n, void* out) {
    Fmt f = (Fmt)fmt;
    size_t es = f == U8 ? 1 : f == U16 ? 2 : 4;
    size_t frame_bytes = (size_t)w * h * 4 * es;
    if (p->probe_current_time) {  // the layer's clip at the output frame's time (clip index n)
        if (vec_next && (n < 0 || n >= n_next)) vec_next = nullptr;
        if (vec_prev && (n < 0 || n >= n_prev)) vec_prev = nullptr;
    }
    if (!vec_next && !vec_prev) {
        // the size mismatch error fill (image.rs:388-425), straight to the wire: red, alpha half
        size_t np = (size_t)w * h;
        if (f == U8) {
            uint8_t* o = (uint8_t*)out;
            for (size_t i = 0; i < np; i++) { o[i * 4] = 0xff; o[i * 4 + 1] = 0; o[i * 4 + 2] = 0; o[i * 4 + 3] = 0x80; }
        } else if (f == U16) {
            uint16_t* o = (uint16_t*)out;  // q15_to_u16 of 0x8000 and 0x4000 (crates/fx-core/src/frame.rs:139-141)
            for (size_t i = 0; i < np; i++) { o[i * 4] = 65535; o[i * 4 + 1] = 0; o[i * 4 + 2] = 0; o[i * 4 + 3] = 32768; }
        } else {
            float* o = (float*)out;  // planes G, B, R, A
            for (size_t i = 0; i < np; i++) { o[i] = 0.0f; o[np + i] = 0.0f; o[2 * np + i] = 1.0f; o[3 * np + i] = 0.5f; }
        }
        return 0;
    }
    TimeMap map;
    Selection sel;
    int time_step = vecin_select(p, n, w, h, &map, &sel);
    float blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
    // T(k) = trunc(dur * k + 0.5) (timemap.rs:45-50), then the clip frame of that tick
    auto clip_index = [&](int pos) -> long long {
        int time = cvtt_i32_d((double)map.dur * (double)(float)pos + 0.5);
        return time >= 0 ? time / time_step : -(((long long)-time + time_step - 1) / time_step);
    };
    auto fetch = [&](const void* clip, int count, int pos) -> Image {
        long long idx = clip_index(pos);
        if (idx < 0 || idx >= count) return Image(w, h, f);
        Image img = from_frame((const uint8_t*)clip + (size_t)idx * frame_bytes, w, h, f);
        return p->rows_reversed ? rows_reversed(img) : img;
    };
    Image A = fetch(frames, nframes, sel.a), B = fetch(frames, nframes, sel.b), result;
    std::string e;
    if (sel.vectors_quality != 0 && !sel.exact) {
        if (sel.interp < 0 || sel.interp > 2) return fail(1, "bad interpolation mode");
        float md = fixed_reader(float_to_fixed(p->max_displace), 1.0f);
        float sx = fixed_reader(float_to_fixed(p->vec_scale_x), 1.0f), sy = fixed_reader(float_to_fixed(p->vec_scale_y), 1.0f);
        FlowField fab, fba;
        bool have_ab = false, have_ba = false;
        if (vec_next) {
            if (int rc = flow_from_vector_image(fetch(vec_next, n_next, sel.a), md, sx, sy, p->taps_above_first != 0, &fab, &e)) return fail(rc, e);
            have_ab = true;
        }
        if (vec_prev) {
            if (int rc = flow_from_vector_image(fetch(vec_prev, n_prev, sel.b), md, sx, sy, p->taps_above_first != 0, &fba, &e)) return fail(rc, e);
            have_ba = true;
        }
        ComposeSettings cs;
        cs.quality_high = p->quality_high != 0;
        cs.blur = blur;
        cs.warp_mode = p->warping == 2 ? 2 : 0;
        cs.video_360 = false;
        cs.taps_above_first = p->taps_above_first != 0;
        cs.gouraud = p->gouraud != 0;
        // complete_flows: the derived flow only where the composition (or the blur tail, F_AB) reads it
        bool tail = (double)std::fabs(sel.s0 - sel.s1) > 1e-6 && (double)blur > 0.005;
        bool need_ab = true, need_ba = true;
        if (sel.interp == 0) {
            bool ab = nearest_uses_f_ab(sel.wa, cs.warp_mode);
            need_ab = ab || tail;
            need_ba = !ab;
        }
        if (!have_ab && need_ab) {
            if (int rc = invert_flow(fba, !cs.gouraud, cs.taps_above_first, &fab, &e)) return fail(rc, e);
            have_ab = true;
        } else if (!have_ba && need_ba) {
            if (int rc = invert_flow(fab, !cs.gouraud, cs.taps_above_first, &fba, &e)) return fail(rc, e);
            have_ba = true;
        }
        Image o;
        int rc = compose_vectors(cs, sel, A, B, have_ab ? &fab : nullptr, have_ba ? &fba : nullptr, &o, &e);
        if (rc) return fail(rc, e);
        result = p->rows_reversed ? rows_reversed(o) : o;
    } else {
        int rc = interpolate(sel, A, B, &result, &e);
        if (rc) return fail(rc, e);
        if (p->rows_reversed) result = rows_reversed(result);
    }
    to_frame(result, out);
    return 0;
}

}  // extern "C"

// ---- the Debug views of Create Vectors (debug.rs), for the tests --------------------------------

namespace orc {
Image debug_views_of(const Image& wp, const Image& y, int code);
std::vector<float> debug_luma_plane(const Image& img);
std::vector<float> debug_detail(const std::vector<float>& l, int w, int h);
std::vector<float> debug_edge(const std::vector<float>& l, int w, int h);
void debug_overlay(Image& out, const std::vector<float>& r, const std::vector<float>& g);
}

extern "C" {

static Image wrap_image(const void* eng, int w, int h, int fmt) {
    Image im(w, h, (Fmt)fmt);
    std::memcpy(im.data(), eng, im.bytes());
    return im;
}

// debug.rs:285-378 and :399-434: the luma plane, the detail and edge measures, the overlay
void or_debug_luma(const void* eng, int w, int h, int fmt, float* out) {
    std::vector<float> l = debug_luma_plane(wrap_image(eng, w, h, fmt));
    std::memcpy(out, l.data(), l.size() * sizeof(float));
}
void or_debug_detail(const float* plane, int w, int h, float* out) {
    std::vector<float> d = debug_detail(std::vector<float>(plane, plane + (size_t)w * h), w, h);
    std::memcpy(out, d.data(), d.size() * sizeof(float));
}
void or_debug_edge(const float* plane, int w, int h, float* out) {
    std::vector<float> d = debug_edge(std::vector<float>(plane, plane + (size_t)w * h), w, h);
    std::memcpy(out, d.data(), d.size() * sizeof(float));
}
void or_debug_overlay(const float* r, const float* g, int w, int h, int fmt, void* out) {
    Image o(w, h, (Fmt)fmt);
    size_t n = (size_t)w * h;
    debug_overlay(o, std::vector<float>(r, r + n), std::vector<float>(g, g + n));
    std::memcpy(out, o.data(), o.bytes());
}

// debug.rs:155-171: view code 0..3 of W' against Y
void or_debug_views_of(const void* wp, const void* y, int w, int h, int fmt, int code, void* out) {
    Image o = debug_views_of(wrap_image(wp, w, h, fmt), wrap_image(y, w, h, fmt), code);
    std::memcpy(out, o.data(), o.bytes());
}

// debug.rs:139-143 (compose_over): y OVER a transparent image, then w OVER that
void or_debug_compose_over(const void* wimg, const void* y, int w, int h, int fmt, void* out) {
    Image o(w, h, (Fmt)fmt);
    over_pl(o, wrap_image(y, w, h, fmt));
    over_pl(o, wrap_image(wimg, w, h, fmt));
    std::memcpy(out, o.data(), o.bytes());
}

// debug.rs:104-152: the whole view (code 4 Warp), the forward warp Gouraud or textured
int or_debug_view(const void* x, const void* y, int w, int h, int fmt, const float* flow, int fw, int fh, int code,
                  int gouraud, void* out) {
    FlowField f(fw, fh);
    std::memcpy(f.d.data(), flow, f.d.size() * sizeof(float));
    Image o;
    std::string e;
    int rc = debug_view(wrap_image(x, w, h, fmt), wrap_image(y, w, h, fmt), f, code, gouraud != 0, &o, &e);
    if (rc) return fail(rc, e);
    std::memcpy(out, o.data(), o.bytes());
    return 0;
}

}  // extern "C"
