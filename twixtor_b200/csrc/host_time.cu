// The time model of the retime effect (timeline.rs): the Speed map with keyed curves and the frame
// selection, host scalars.
#include "runtime.h"

// =======================================================================================================
// The time model (timeline.rs) of the Speed map, host scalars

namespace {

int32_t cvtt_i32_d(double x) {  // timeline.rs:43-49
    if (x > -2147483649.0 && x < 2147483648.0) return (int32_t)x;
    return INT32_MIN;
}
int32_t cvtt_i32_f(float x) {  // timeline.rs:52-58
    if (x > -2147483904.0f && x < 2147483648.0f) return (int32_t)x;
    return INT32_MIN;
}
int32_t float_to_fixed(double f) {  // crates/fx-core/src/fixed.rs:8-10 (Rust `as i32` saturates)
    double v = f * 65536.0 + (f < 0.0 ? -0.5 : 0.5);
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0) return INT32_MAX;
    if (v <= -2147483648.0) return INT32_MIN;
    return (int32_t)v;
}
float fixed_reader(int32_t fixed, float scale) { return (float)((double)fixed * (1.0 / 65536.0)) * scale; }

// crates/fx-core/src/curves.rs:282-310, :348-375, :537-544: a float curve, constant when it has no
// key, else its keys sorted by time (frame * lts rounded half away from zero, time.rs:117-119),
// linear or eased between keys, held after a hold key (flags bit 0 ease, bit 1 hold)
struct Curve {
    struct Key {
        long long t;
        double v;
        int flags;
    };
    double constant = 0.0;
    std::vector<Key> keys;
    Curve(double c, int n, const double* frames, const double* values, const int32_t* flags, int lts) : constant(c) {
        for (int i = 0; i < n; i++)
            keys.push_back({(long long)std::llround(frames[i] * (double)lts), values[i], flags ? flags[i] : 0});
        std::stable_sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) { return a.t < b.t; });
    }
    double at(long long t) const {
        if (keys.empty()) return constant;
        size_t last = keys.size() - 1;
        if (t <= keys[0].t) return keys[0].v;
        if (t >= keys[last].t) return keys[last].v;
        size_t i = 0;
        while (i + 1 < keys.size() && keys[i + 1].t <= t) i++;
        const Key &a = keys[i], &b = keys[i + 1];
        if (a.flags & 2) return a.v;
        double u = (double)(t - a.t) / (double)(b.t - a.t);
        bool ea = (a.flags & 1) != 0, eb = (b.flags & 1) != 0;
        double f = (!ea && !eb) ? u : (ea && eb) ? u * u * (3.0 - 2.0 * u) : ea ? u * u * (2.0 - u) : u * (1.0 + u * (1.0 - u));
        return a.v + (b.v - a.v) * f;
    }
};

// timeline.rs:69-76: a rate within 2e-5 (an f32 difference) of 29.97, 59.94 or 23.976 becomes it
double snap_rate(double rate) {
    for (double t : {29.97, 59.94, 23.976})
        if ((double)std::fabs((float)(rate - t)) < 2e-5) rate = t;
    return rate;
}

// The time map of the retime effect (timeline.rs:106-131, :204-344) for tw_time_params.
struct RetimeMap {
    int lts = 100;
    double in_fps = 30.0, out_fps = 30.0;
    float dur = 100.0f;
    double frame_time_k = 0.05;
    bool plain_frame_time = false;  // retime-fgbg's frame time: trunc(dur * k + 0.5) at every rate
    int mode = 1;
    Curve speed, frame_num, marks;
    // fields: the retime effect's Input: Fields (the Vectors In map has none)
    RetimeMap(const tw_time_params* p, bool fields)
        : lts(p->fps_den == 1 ? 100 : p->fps_den),  // crates/fx-core/src/time.rs:92-99
          speed(p->speed_percent, p->nkeys, p->key_frames, p->key_values, p->key_ease, lts),
          frame_num(p->frame_num, p->nfn_keys, p->fn_key_frames, p->fn_key_values, p->fn_key_flags, lts),
          marks(p->mark_segs > 0 ? p->mark_segs : 1, p->nmark_keys, p->mark_key_frames, p->mark_key_values, nullptr, lts) {
        for (auto& k : marks.keys) k.flags = 2;  // a popup holds its value between keys (curves.rs:362)
        double in = 30.0, out = 30.0;  // "In FPS is Out FPS" on: both 30 (timeline.rs:117-120)
        if (p->own_input_rate) {
            in = (double)((float)p->input_frame_rate * 1.0f);
            out = (double)p->fps_num / (double)p->fps_den;
        }
        in_fps = snap_rate(in);
        out_fps = snap_rate(out);
        if (fields && (p->input_fields == 2 || p->input_fields == 3)) in_fps *= 2.0;  // timeline.rs:123-125
        dur = (float)(((double)lts * out_fps) / in_fps);
        if (p->frame_time_bias > 0.0) frame_time_k = p->frame_time_bias;
        plain_frame_time = p->frame_time_plain != 0;
        mode = p->remap_mode == 2 ? 2 : 1;
    }
    bool rates_ok() const { return !(0.01 > out_fps || 0.01 >= in_fps); }  // timeline.rs:125-127
    // timeline.rs:266-331 (Src Time Offset 0)
    float src_pos(float t, bool* unsupported) const {
        float lts_f = (float)lts;
        double ratio = in_fps / out_fps;
        if (mode == 2) {  // Frame Number: the curve at trunc((lts * t) + K), times in / out
            int time = cvtt_i32_d((double)(lts_f * t) + 0.05);
            return (float)(ratio * (double)(float)frame_num.at(time));
        }
        float out = 0.0f;
        int n2 = cvtt_i32_f(t * 2.0f);
        if (n2 >= (1 << 24)) { *unsupported = true; return 0.0f; }
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
        return (float)(ratio * (double)out);
    }
    // timeline.rs:347-354 (base 0): Src: Mark Segments at trunc((f * dur) + 0.5), 1..5 as 0..4, else 0
    int marker(float f) const {
        int32_t time = cvtt_i32_d((double)(f * dur) + 0.5);
        double v = marks.at(time);
        return v >= 1.0 && v <= 5.0 ? (int)v - 1 : 0;
    }
    // timeline.rs:336-344 (base 0), then the clip frame of that tick
    int32_t clip_frame(int32_t pos) const {
        float d = (float)pos;
        int32_t time = plain_frame_time || std::fabs(in_fps - out_fps) < frame_time_k
                           ? cvtt_i32_d((double)d * (double)dur + 0.5)
                                                                   : cvtt_i32_d((double)(d * dur) + (double)dur * frame_time_k);
        long long idx = time >= 0 ? time / lts : -(((long long)-time + lts - 1) / lts);
        return (int32_t)std::max<long long>(std::min<long long>(idx, INT32_MAX), INT32_MIN);
    }
};

}  // namespace

extern "C" int tw_select(const tw_time_params* p, int32_t n, int32_t width, int32_t height, tw_selection* out) {
    if (!p || !out || p->fps_num <= 0 || p->fps_den <= 0) return TW_ERR_BAD_PARAM;
    if (p->nkeys > 0 && (!p->key_frames || !p->key_values)) return TW_ERR_BAD_PARAM;
    if (p->nfn_keys > 0 && (!p->fn_key_frames || !p->fn_key_values)) return TW_ERR_BAD_PARAM;
    if (p->remap_mode < 0 || p->remap_mode > 2) return TW_ERR_BAD_PARAM;
    if (p->nmark_keys > 0 && (!p->mark_key_frames || !p->mark_key_values)) return TW_ERR_BAD_PARAM;
    RetimeMap map(p, true);
    if (!map.rates_ok()) return TW_ERR_BAD_PARAM;
    int lts = map.lts;
    int cur = n * lts;
    float t0 = (float)cur / (float)lts;                  // timeline.rs:136-142
    float t1 = ((float)lts + (float)cur) / (float)lts;
    bool bad = false;
    float s0 = map.src_pos(t0, &bad);
    float s1 = map.src_pos(t1, &bad);
    if (bad) return TW_ERR_UNSUPPORTED;
    float blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
    int a = cvtt_i32_f(s0);
    float frac = s0 - (float)a;
    out->s0 = s0;
    out->s1 = s1;
    // the clip frames of positions a and a + 1 (host.rs:155-159)
    out->a = map.clip_frame(a);
    out->b = map.clip_frame((int32_t)((uint32_t)a + 1u));
    out->wa = 1.0f - frac;
    bool exact = true;  // timeline.rs:429-439
    float fr = s0 - std::floor(s0);
    if ((double)std::fabs(fr) > 0.005 && (double)std::fabs((float)((double)fr - 1.0)) > 0.005) exact = false;
    if ((double)std::fabs(s0 - s1) > 1e-6 && (double)blur > 0.005) exact = false;
    out->exact = exact ? 1 : 0;
    int vq = p->vectors - 1;
    vq = (width >= 2 && height >= 2) ? vq : 0;
    int ip = p->frame_interp - 1;
    // timeline.rs:418-441 (marker_override, the core's g = trunc(s0 + 1.0)): markers that differ give
    // (No Vectors, Nearest), then No MV Use Nearest (0, Nearest) and No MV Frame Blend (0, Blend)
    int ma = map.marker((float)a), mb = map.marker((float)cvtt_i32_d((double)s0 + 1.0));
    if (ma != mb) { vq = 0; ip = 0; }
    if (ma == 3) { vq = 0; ip = 0; }
    if (ma == 4) { vq = 0; ip = 1; }
    out->vectors_quality = vq;
    out->interp = ip;
    return TW_OK;
}

// plugins/vectors-in/src/timemap.rs and glue.rs:204-215: the Speed map of the retime effect with the
// rates of the Vectors In effect (In FPS is Out FPS: the input rate 30, the output rate the
// composition's), the constant vectors quality 4 (prep.rs:111-117 for sides of 1), and the clip
// frames of the pair at T(k) = trunc(dur * k + 0.5) ticks (timemap.rs:45-50).
extern "C" int tw_select_vectors_in(const tw_time_params* p, int32_t n, int32_t width, int32_t height,
                                    tw_selection* out, tw_vecin_frame* frame) {
    if (!p || !out || !frame || p->fps_num <= 0 || p->fps_den <= 0) return TW_ERR_BAD_PARAM;
    if (p->nkeys > 0 && (!p->key_frames || !p->key_values)) return TW_ERR_BAD_PARAM;
    if (p->nfn_keys > 0 && (!p->fn_key_frames || !p->fn_key_values)) return TW_ERR_BAD_PARAM;
    if (p->remap_mode < 0 || p->remap_mode > 2) return TW_ERR_BAD_PARAM;
    if (p->nmark_keys > 0 && (!p->mark_key_frames || !p->mark_key_values)) return TW_ERR_BAD_PARAM;
    tw_time_params q = *p;  // the effect's rates: the input rate (30 with In FPS is Out FPS), the composition's
    q.own_input_rate = 1;
    q.input_frame_rate = p->own_input_rate ? p->input_frame_rate : 30.0;
    RetimeMap map(&q, false);
    if (!map.rates_ok()) return TW_ERR_BAD_PARAM;
    int lts = map.lts;
    int cur = n * lts;
    float t0 = (float)cur / (float)lts;
    float t1 = ((float)lts + (float)cur) / (float)lts;
    bool bad = false;
    float s0 = map.src_pos(t0, &bad);
    float s1 = map.src_pos(t1, &bad);
    if (bad) return TW_ERR_UNSUPPORTED;
    float blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
    int a = cvtt_i32_f(s0);
    out->s0 = s0;
    out->s1 = s1;
    out->a = a;
    out->b = (int32_t)((uint32_t)a + 1u);
    out->wa = 1.0f - (s0 - (float)a);
    bool exact = true;
    float fr = s0 - std::floor(s0);
    if ((double)std::fabs(fr) > 0.005 && (double)std::fabs((float)((double)fr - 1.0)) > 0.005) exact = false;
    if ((double)std::fabs(s0 - s1) > 1e-6 && (double)blur > 0.005) exact = false;
    out->exact = exact ? 1 : 0;
    int vq = (width >= 2 && height >= 2) ? 4 : 0, ip = p->frame_interp - 1;
    // timeline.rs:418-441 (marker_override) with the effect's marker: Src: Mark Segments at
    // T(f) = trunc((f64)dur * (f64)f + 0.5) (plugins/vectors-in/src/timemap.rs:49-70)
    auto marker = [&](float f) {
        double v = map.marks.at(cvtt_i32_d((double)map.dur * (double)f + 0.5));
        return v >= 1.0 && v <= 5.0 ? (int)v - 1 : 0;
    };
    int ma = marker((float)a), mb = marker((float)cvtt_i32_d((double)s0 + 1.0));
    if (ma != mb) { vq = 0; ip = 0; }
    if (ma == 3) { vq = 0; ip = 0; }
    if (ma == 4) { vq = 0; ip = 1; }
    out->vectors_quality = vq;
    out->interp = ip;
    auto clip_index = [&](int32_t pos) -> int32_t {  // T(k) = trunc(dur * k + 0.5), timemap.rs:45-50
        int32_t time = cvtt_i32_d((double)map.dur * (double)(float)pos + 0.5);
        long long idx = time >= 0 ? time / lts : -(((long long)-time + lts - 1) / lts);
        return (int32_t)std::max<long long>(std::min<long long>(idx, INT32_MAX), INT32_MIN);
    };
    frame->a = clip_index(out->a);
    frame->b = clip_index(out->b);
    return TW_OK;
}

// ---- one clip over several GPUs ------------------------------------------------------------------

extern "C" int tw_shard(int32_t nout, int32_t nranks, int32_t rank, int32_t* lo, int32_t* hi) {
    if (!lo || !hi || nout < 0 || nranks < 1 || rank < 0 || rank >= nranks) return TW_ERR_BAD_PARAM;
    // contiguous ranges in rank order; the first nout % nranks ranks take one frame more
    int64_t base = nout / nranks, extra = nout % nranks;
    int64_t l = rank * base + std::min<int64_t>(rank, extra);
    *lo = (int32_t)l;
    *hi = (int32_t)(l + base + (rank < extra ? 1 : 0));
    return TW_OK;
}

extern "C" int tw_source_window(const tw_selection* sels, int32_t n, int32_t nframes, int32_t* first, int32_t* last) {
    if (!first || !last || n < 0 || nframes < 0 || (n > 0 && !sels)) return TW_ERR_BAD_PARAM;
    int64_t f = INT64_MAX, l = INT64_MIN;
    for (int32_t k = 0; k < n; k++)
        for (int32_t idx : {sels[k].a, sels[k].b})  // both frames of the pair are read, exact frames included
            if (idx >= 0 && idx < nframes) {
                f = std::min<int64_t>(f, idx);
                l = std::max<int64_t>(l, idx);
            }
    if (f > l) {  // nothing inside the clip
        *first = 0;
        *last = -1;
    } else {
        *first = (int32_t)f;
        *last = (int32_t)l;
    }
    return TW_OK;
}
