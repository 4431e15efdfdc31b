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

struct SpeedCurve {  // crates/fx-core/src/curves.rs:348-375, :537-544
    const tw_time_params* p;
    long long key_time(int i, int step) const { return (long long)std::llround(p->key_frames[i] * (double)step); }
    double at(long long t, int step) const {
        if (p->nkeys <= 0) return p->speed_percent;
        int last = p->nkeys - 1;
        if (t <= key_time(0, step)) return p->key_values[0];
        if (t >= key_time(last, step)) return p->key_values[last];
        int i = 0;
        while (i + 1 < p->nkeys && key_time(i + 1, step) <= t) i++;
        long long ta = key_time(i, step), tb = key_time(i + 1, step);
        bool ea = p->key_ease && p->key_ease[i], eb = p->key_ease && p->key_ease[i + 1];
        double u = (double)(t - ta) / (double)(tb - ta);
        double f = (!ea && !eb) ? u : (ea && eb) ? u * u * (3.0 - 2.0 * u) : ea ? u * u * (2.0 - u) : u * (1.0 + u * (1.0 - u));
        return p->key_values[i] + (p->key_values[i + 1] - p->key_values[i]) * f;
    }
};

// timeline.rs:266-331 (Speed mode, Src Time Offset 0); `ratio` is in_fps / out_fps (1 for the
// retime effect with "In FPS is Out FPS")
float src_pos(const SpeedCurve& c, int lts, float t, bool* unsupported, double ratio = 30.0 / 30.0) {
    float lts_f = (float)lts;
    float out = 0.0f;
    int n2 = cvtt_i32_f(t * 2.0f);
    if (n2 >= (1 << 24)) { *unsupported = true; return 0.0f; }
    float k = 1.0f;
    while ((float)n2 >= k) {
        int time = cvtt_i32_d((double)((lts_f * k) / 2.0f) + 0.05);
        float sp = (float)((double)float_to_fixed(c.at(time, lts)) / 6553600.0);
        out = (sp / 2.0f) + out;
        k += 1.0f;
    }
    float tt = t * 2.0f;
    float rem = tt - (k + -1.0f);
    if ((double)rem > 0.0001) {
        int time = cvtt_i32_d((double)((tt * lts_f) / 2.0f) + 0.05);
        float sp = (float)((double)float_to_fixed(c.at(time, lts)) / 6553600.0);
        out = ((rem * sp) / 2.0f) + out;
    }
    return (float)(ratio * (double)out);
}

}  // namespace

extern "C" int tw_select(const tw_time_params* p, int32_t n, int32_t width, int32_t height, tw_selection* out) {
    if (!p || !out || p->fps_num <= 0 || p->fps_den <= 0) return TW_ERR_BAD_PARAM;
    if (p->nkeys > 0 && (!p->key_frames || !p->key_values)) return TW_ERR_BAD_PARAM;
    int lts = p->fps_den == 1 ? 100 : p->fps_den;  // crates/fx-core/src/time.rs:92-99
    SpeedCurve c{p};
    int cur = n * lts;
    float t0 = (float)cur / (float)lts;                  // timeline.rs:136-142
    float t1 = ((float)lts + (float)cur) / (float)lts;
    bool bad = false;
    float s0 = src_pos(c, lts, t0, &bad);
    float s1 = src_pos(c, lts, t1, &bad);
    if (bad) return TW_ERR_UNSUPPORTED;
    float blur = fixed_reader(float_to_fixed(p->blur_compensation), 1.0f);
    int a = cvtt_i32_f(s0);
    float frac = s0 - (float)a;
    out->s0 = s0;
    out->s1 = s1;
    out->a = a;
    out->b = (int32_t)((uint32_t)a + 1u);
    out->wa = 1.0f - frac;
    bool exact = true;  // timeline.rs:429-439
    float fr = s0 - std::floor(s0);
    if ((double)std::fabs(fr) > 0.005 && (double)std::fabs((float)((double)fr - 1.0)) > 0.005) exact = false;
    if ((double)std::fabs(s0 - s1) > 1e-6 && (double)blur > 0.005) exact = false;
    out->exact = exact ? 1 : 0;
    int vq = p->vectors - 1;
    out->vectors_quality = (width >= 2 && height >= 2) ? vq : 0;
    out->interp = p->frame_interp - 1;
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
    int lts = p->fps_den == 1 ? 100 : p->fps_den;
    double comp = (double)p->fps_num / (double)p->fps_den;
    if (0.01 > comp) return TW_ERR_BAD_PARAM;  // timeline.rs:125-127 (the rate check)
    double ratio = 30.0 / comp;
    float dur = (float)(((double)lts * comp) / 30.0);  // timeline.rs:128
    SpeedCurve c{p};
    int cur = n * lts;
    float t0 = (float)cur / (float)lts;
    float t1 = ((float)lts + (float)cur) / (float)lts;
    bool bad = false;
    float s0 = src_pos(c, lts, t0, &bad, ratio);
    float s1 = src_pos(c, lts, t1, &bad, ratio);
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
    out->vectors_quality = (width >= 2 && height >= 2) ? 4 : 0;
    out->interp = p->frame_interp - 1;
    auto clip_index = [&](int32_t pos) -> int32_t {  // the clip frame shown at T(pos) ticks
        int32_t time = cvtt_i32_d((double)dur * (double)(float)pos + 0.5);
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
