// CPU oracle of the layered composition with plates (plugins/retime-engine/src/layers/plates.rs,
// matte.rs) for the FG matte layers of retime-fgbg. TEST INFRASTRUCTURE ONLY (see oracle_core.h).
//
// Restated scope: warping codes 0 to 3, Nearest, Blend and Weighted Blend, the display groups and the
// inverse matte shrink (the plugin's choke of the cut), no tracking points, no wrap-around.
#include "oracle_layers.h"
#include "oracle_forward.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "oracle_smart.h"

namespace orc {

static const float PL_K8 = bits_f(0x3b808081u);   // matte.rs:921
static const float PL_K16 = bits_f(0x37800080u);  // matte.rs:922

static float white_of(Fmt f) { return f == U8 ? 255.0f : f == U16 ? 65535.0f : 1.0f; }

// Rust's saturating float -> i64 cast (`as i64`: NaN gives 0)
static int64_t as_i64(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 9223372036854775808.0f) return INT64_MAX;
    if (x < -9223372036854775808.0f) return INT64_MIN;
    return (int64_t)x;
}

LPlane raw_plane(const float* m, size_t n, Fmt fmt) {  // plates.rs:50-57
    LPlane p;
    p.white = white_of(fmt);
    p.v.assign(m, m + n);
    if (fmt == F32) return p;
    bool in = true;  // matte.rs:106-112 (in_range): the clamp only when a value leaves 0..1
    for (float x : p.v) in = in && x >= 0.0f && x <= 1.0f;
    for (float& x : p.v) {
        float c = x;
        if (!in) c = x > 1.0f ? 1.0f : (x >= 0.0f ? x : 0.0f);  // matte.rs:94-102
        x = (float)as_i64(c * p.white + 0.5f);
    }
    return p;
}

static float cut(float c, float v, float white, bool isf) {  // plates.rs:63-78
    float x = (float)((1.0 - (double)v) * (double)c);
    if (0.0f > x) x = 0.0f;
    else if (x > white) x = white;
    if (isf) return x + 0.0f;
    return (float)as_i64(x + 0.5f);
}

static float clamp_pl(float v) {  // matte.rs:350-359
    if (0.0f > v) return 0.0f;
    if (v >= 1.0f) return 1.0f;
    return v;
}

void display_group(int display, int nfg, int* first, int* last) {  // layers.rs:120-129
    if (display >= 3 && display <= 5) *first = *last = std::min(display - 3, nfg);
    else if (display == 6) *first = *last = nfg;
    else { *first = 0; *last = nfg; }
}

// matte.rs:337-341 (invert_pl_value)
static float invert_pl_value(float v) {
    float x = (float)(1.0 - (double)v);
    return x > 0.999f ? 1.0f : x;
}

// matte.rs:366-385 (blur_pl): the Gaussian of radius r with the runtime's powf taps, column pass above first
static void blur_pl(std::vector<float>& d, int w, int h, float r) {
    if ((double)r < 0.001 || d.empty()) return;  // conv.rs:52 (BLUR_RADIUS_EPS)
    int n = std::max((int)r + 1, 0);
    float s3 = r / 3.0f, dd = s3 * s3, sum = 0.0f;
    std::vector<float> k(n);
    for (int i = 0; i < n; i++) {
        float fi = (float)i;
        k[i] = crt_powf(2.0f, -((fi * fi) / dd));
        sum += k[i];
    }
    float den = sum * 2.0f - k[0];
    for (float& v : k) v /= den;
    convolve(d.data(), w, h, 1, k.data(), n, true);
}

// matte.rs:418-430 (choke_geometry): the half width r and the weight of the shrink step by a > 0
static void choke_geometry(float a, float* r_out, float* wgt) {
    float r = std::ceil(a + 1.0f);
    float fr = (float)((double)r - ((double)a + 1.0));
    if (fr < 0.01f) {
        a = a + 0.01f;
        r = std::ceil(a + 1.0f);
        fr = (float)((double)r - ((double)a + 1.0));
    }
    *r_out = r;
    *wgt = (float)(1.0 - (double)fr);
}

// matte.rs:441-484 (shrink_pl): one shrink step by the whole number of pixels a
static void shrink_pl(std::vector<float>& d, int w, int h, float a) {
    if (!(a > 0.0f) || d.empty()) return;
    float r, wgt;
    choke_geometry(a, &r, &wgt);
    blur_pl(d, w, h, wgt + r);
    long long n = (long long)r;
    float sigma = (float)((double)r / 3.0), s2 = sigma * sigma;
    size_t size = (size_t)(2 * n + 1);
    std::vector<float> k(size);
    float sum = 0.0f;
    for (size_t j = 0; j < size; j++) {
        float x = (float)std::llabs((long long)j - n);
        k[j] = crt_powf(2.0f, -((x * x) / s2));
        sum += k[j];
    }
    for (float& v : k) v /= sum;
    auto tail = [&](size_t from) {
        float acc = 0.0f;
        for (size_t j = from; j < size; j++) acc += k[j];
        return acc;
    };
    float s2sum = tail(2), s3sum = tail(3);
    float t = (s2sum - s3sum) * wgt + s3sum;
    double den = 1.0 - (double)t;
    for (float& v : d) {
        if (t > v) { v = 0.0f; continue; }
        float o = (float)((double)(v - t) / den);
        v = std::fabs((double)o - 1.0) < 1e-4 ? 1.0f : o;
    }
}

void choke_pl(std::vector<float>& m, int w, int h, float amount) {  // matte.rs:280-310
    if (!std::isfinite(amount)) return;
    bool grow = amount < 0.0f;
    float a = grow ? -amount : amount;
    if (a > 65536.0f) a = 65536.0f;  // matte.rs:190 (CHOKE_MAX)
    if (grow) for (float& v : m) v = invert_pl_value(v);
    float lo = std::floor(a), hi = std::ceil(a);
    if (lo == hi) {
        shrink_pl(m, w, h, lo);
    } else {
        std::vector<float> c = m;
        shrink_pl(m, w, h, lo);
        shrink_pl(c, w, h, hi);
        float t = a - lo;
        for (size_t i = 0; i < m.size(); i++) {  // matte.rs:326-345 (mix_pl)
            float x = (c[i] - m[i]) * t + m[i];
            if (x >= 1.0f) x = 1.0f;
            else if (0.0f > x) x = 0.0f;
            m[i] = x;
        }
    }
    if (grow) for (float& v : m) v = invert_pl_value(v);
    for (float& v : m) v = clamp_pl(v);
}

// plates.rs:80-90 (cut_matte): the FG matte as the cut reads it, choked by minus its inverse matte shrink
static std::vector<float> cut_matte(const LPlane& raw, float shrink, int w, int h) {
    float kk = 1.0f / raw.white;
    std::vector<float> v(raw.v.size());
    for (size_t i = 0; i < v.size(); i++) v[i] = raw.v[i] * kk;
    choke_pl(v, w, h, -shrink);
    return v;
}

LPlane comp_plane(const std::vector<LPlane>& raws, const std::vector<float>& shrink, int k, Fmt fmt, int w,
                  int h) {  // plates.rs:95-107
    float white = white_of(fmt);
    bool isf = fmt == F32;
    size_t n = (size_t)w * h;
    LPlane c;
    c.white = white;
    if (k == (int)raws.size()) c.v.assign(n, white);
    else c = raws[k];
    for (int j = k - 1; j >= 0; j--) {
        std::vector<float> v = cut_matte(raws[j], shrink.empty() ? 0.0f : shrink[j], w, h);
        for (size_t i = 0; i < n; i++) c.v[i] = cut(c.v[i], v[i], white, isf);
    }
    return c;
}

Image layer_times(const Image& src, const LPlane& p) {  // plates.rs:128-156
    Image out(src.w, src.h, src.fmt);
    size_t n = (size_t)src.w * src.h;
    for (size_t i = 0; i < n; i++) {
        for (int c = 0; c < 4; c++) {
            size_t j = i * 4 + c;
            if (src.fmt == U8) out.u8[j] = (uint8_t)as_i64((float)src.u8[j] * (p.v[i] * PL_K8) + 0.5f);
            else if (src.fmt == U16) out.u16[j] = (uint16_t)as_i64((float)src.u16[j] * (p.v[i] * PL_K16) + 0.5f);
            else out.f32[j] = nr::mul(p.v[i], src.f32[j]);
        }
    }
    return out;
}

// plates.rs:296-309: 1 where no layer above covers layer k; empty when it is 1 everywhere
bool solver_mask(const std::vector<LPlane>& raws, const LPlane& comp, int k, size_t n, std::vector<float>* out) {
    float white = comp.white;
    out->resize(n);
    bool all_one = true;
    for (size_t i = 0; i < n; i++) {
        float r = k == (int)raws.size() ? white : raws[k].v[i];
        float v = (white - (r - comp.v[i])) / white;
        (*out)[i] = v;
        all_one = all_one && v == 1.0f;
    }
    return !all_one;
}

static void unpremultiply_pl(Image& img) {  // plates.rs:160-187
    size_t n = (size_t)img.w * img.h;
    for (size_t i = 0; i < n; i++) {
        if (img.fmt == U8) {
            uint8_t o[4];
            unpremultiply_u8(&img.u8[i * 4], o);
            for (int c = 0; c < 4; c++) img.u8[i * 4 + c] = o[c];
        } else if (img.fmt == U16) {
            uint16_t* p = &img.u16[i * 4];
            if (p[0] == 0) continue;
            float inv = 65535.0f / (float)p[0];
            for (int c = 1; c < 4; c++) {
                float v = (float)p[c] * inv;
                if (65535.0f < v) v = 65535.0f;
                p[c] = (uint16_t)q(v);
            }
        } else {
            float* p = &img.f32[i * 4];
            if (1e-7 > (double)p[0]) continue;
            float inv = 1.0f / p[0];
            for (int c = 1; c < 4; c++) p[c] = nr::mul(inv, p[c]);
        }
    }
}

static void premultiply_pl(Image& img) {  // plates.rs:191-208
    size_t n = (size_t)img.w * img.h;
    for (size_t i = 0; i < n; i++) {
        if (img.fmt == U8) {
            uint8_t o[4];
            premultiply_u8(&img.u8[i * 4], o);
            for (int c = 0; c < 4; c++) img.u8[i * 4 + c] = o[c];
        } else if (img.fmt == U16) {
            uint16_t* p = &img.u16[i * 4];
            float f = (float)p[0] * PL_K16;
            for (int c = 1; c < 4; c++) p[c] = (uint16_t)q((float)p[c] * f);
        } else {
            float o[4];
            premultiply_f32(&img.f32[i * 4], o);
            for (int c = 0; c < 4; c++) img.f32[i * 4 + c] = o[c];
        }
    }
}

// plates.rs:245-256: unpremultiply, fill the colour where the plate is not opaque (holes:
// white - alpha), the alpha replaced by the layer's raw matte plane or (frame != null) the frame's
// alpha, premultiply
// is360: the 360 passes of the fill (plates.rs:252-263)
static int refill(Image& img, const LPlane* plane, const Image* frame, bool above_first, std::string* err,
                  bool is360 = false) {
    unpremultiply_pl(img);
    size_t n = (size_t)img.w * img.h;
    int rc;
    if (img.fmt == U8) {
        std::vector<uint8_t> m(n);
        for (size_t i = 0; i < n; i++) m[i] = (uint8_t)(0xffu - img.u8[i * 4]);
        rc = fill_holes(img, m.data(), 1, above_first, err, is360);
    } else if (img.fmt == U16) {
        std::vector<uint16_t> m(n);
        for (size_t i = 0; i < n; i++) m[i] = (uint16_t)(0xffffu - img.u16[i * 4]);
        rc = fill_holes(img, m.data(), 2, above_first, err, is360);
    } else {
        std::vector<float> m(n);
        for (size_t i = 0; i < n; i++) m[i] = 1.0f - img.f32[i * 4];
        rc = fill_holes(img, m.data(), 3, above_first, err, is360);
    }
    if (rc) return rc;
    for (size_t i = 0; i < n; i++) {  // plates.rs:211-239 (set_alpha)
        if (frame) {
            if (img.fmt == U8) img.u8[i * 4] = frame->u8[i * 4];
            else if (img.fmt == U16) img.u16[i * 4] = frame->u16[i * 4];
            else img.f32[i * 4] = frame->f32[i * 4];
        } else {
            float v = plane->v[i];
            if (img.fmt == U8) img.u8[i * 4] = (uint8_t)std::min<int64_t>(std::max<int64_t>(as_i64(v), 0), 255);
            else if (img.fmt == U16) img.u16[i * 4] = (uint16_t)std::min<int64_t>(std::max<int64_t>(as_i64(v), 0), 65535);
            else img.f32[i * 4] = v;
        }
    }
    premultiply_pl(img);
    return 0;
}

void over_pl(Image& d, const Image& s) {  // matte.rs:923-1030
    size_t n = (size_t)d.w * d.h;
    for (size_t i = 0; i < n; i++) {
        if (d.fmt == U8) {
            uint8_t* dp = &d.u8[i * 4];
            const uint8_t* sp = &s.u8[i * 4];
            uint8_t sa = sp[0];
            if (sa == 0) continue;
            if (sa == 255) { for (int c = 0; c < 4; c++) dp[c] = sp[c]; continue; }
            float saf = (float)sa, f = 1.0f - saf * PL_K8;
            uint8_t da = dp[0];
            for (int c = 1; c < 4; c++) dp[c] = (uint8_t)as_i64((float)dp[c] * f + (float)sp[c] + 0.5f);
            dp[0] = (uint8_t)as_i64((float)(255 - da) * saf * PL_K8 + (float)da + 0.5f);
        } else if (d.fmt == U16) {
            uint16_t* dp = &d.u16[i * 4];
            const uint16_t* sp = &s.u16[i * 4];
            uint16_t sa = sp[0];
            if (sa == 0) continue;
            if (sa == 65535) { for (int c = 0; c < 4; c++) dp[c] = sp[c]; continue; }
            float saf = (float)sa, f = 1.0f - saf * PL_K16;
            uint16_t da = dp[0];
            for (int c = 1; c < 4; c++) dp[c] = (uint16_t)as_i64((float)dp[c] * f + (float)sp[c] + 0.5f);
            dp[0] = (uint16_t)as_i64((float)(65535 - (int32_t)da) * saf * PL_K16 + (float)da + 0.5f);
        } else {
            float* dp = &d.f32[i * 4];
            const float* sp = &s.f32[i * 4];
            float sa = sp[0];
            if (sa == 0.0f) continue;
            if (sa == 1.0f) { for (int c = 0; c < 4; c++) dp[c] = sp[c]; continue; }
            float f = nr::sub(1.0f, sa);
            float da = dp[0];
            for (int c = 1; c < 4; c++) dp[c] = nr::add(nr::add(nr::mul(f, dp[c]), sp[c]), 0.0f);
            dp[0] = nr::add(nr::add(nr::mul(nr::sub(1.0f, da), sa), da), 0.0f);
        }
    }
}

static bool nearest_takes_a(int code, float wa) {  // layers.rs:697-703
    if (code == 0) return 0.5f <= wa;
    return !(0.5f > wa);
}

int compose_layers_plates(const LayerJob& job, const Image& a, const Image& b, Image* out, std::string* err) {
    int w = a.w, h = a.h;
    size_t n = (size_t)w * h;
    Fmt fmt = a.fmt;
    int nfg = (int)job.mattes_a.size();
    std::vector<LPlane> raws_a, raws_b;
    for (int j = 0; j < nfg; j++) {
        raws_a.push_back(raw_plane(job.mattes_a[j].data(), n, fmt));
        raws_b.push_back(raw_plane(job.mattes_b[j].data(), n, fmt));
    }
    const Selection& sel = job.sel;
    int code = job.cs.warp_mode;
    if (code < 0 || code > 3) { *err = "plates: warping code not 0 to 3"; return 1; }
    if (sel.interp < 0 || sel.interp > 2) { *err = "plates: bad interpolation mode"; return 1; }
    int first = job.first, last = job.last < 0 ? nfg : job.last;
    if (first < 0 || first > last || last > nfg) { *err = "plates: bad layer group"; return 1; }
    // plates.rs:330-370: the solves of the group's layers, one after the other
    std::vector<FlowField> f_ab(nfg + 1), f_ba(nfg + 1);
    std::vector<bool> has_ab(nfg + 1, false), has_ba(nfg + 1, false);
    for (int k = first; k <= last; k++) {
        FlowSettings fs = job.fs;
        fs.track_alpha = false;
        fs.sensitivity = job.sensitivity[k];
        LPlane ca = comp_plane(raws_a, job.shrink, k, fmt, w, h), cb = comp_plane(raws_b, job.shrink, k, fmt, w, h);
        Pyramid pa, pb;
        // plates.rs:319-323 (layer_solve_settings): Track RGB+A puts the luma pyramids (only) in the 360
        // mode of the filters; the luma itself gets no alpha
        FlowSettings fp = fs;
        fp.wrap = job.fs.wrap || job.fs.track_alpha;
        if (!build_pyramid(layer_times(a, ca), fp, &pa, err) || !build_pyramid(layer_times(b, cb), fp, &pb, err)) return 1;
        std::vector<float> ma, mb;
        bool hm_a = solver_mask(raws_a, ca, k, n, &ma), hm_b = solver_mask(raws_b, cb, k, n, &mb);
        std::vector<Plane> mpa, mpb;
        bool masks = hm_a || hm_b;
        if (masks) {
            if (!hm_a) ma.assign(n, 1.0f);
            if (!hm_b) mb.assign(n, 1.0f);
            if (!mask_pyramid(ma.data(), w, h, fs, &mpa, err) || !mask_pyramid(mb.data(), w, h, fs, &mpb, err)) return 1;
        }
        bool need_ab = true, need_ba = true;
        if (sel.interp == 0) {
            need_ab = nearest_uses_f_ab(sel.wa, code);
            need_ba = !need_ab;
        }
        // layers.rs:247-280 (solve_layer): the solve with X = A takes the pairs (at A, at B), the other
        // (at B, at A), as their user displacement
        const std::vector<std::array<float, 4>>* pts = (int)job.points.size() > k ? &job.points[k] : nullptr;
        std::vector<UserLevel> u_ab, u_ba;
        if (pts && !pts->empty()) {
            std::vector<std::array<float, 4>> fwd, bwd;
            for (const auto& p : *pts) {
                fwd.push_back({p[0], p[1], p[2], p[3]});
                bwd.push_back({p[2], p[3], p[0], p[1]});
            }
            u_ab = user_displacement(fwd, pa.geo, w, h);
            u_ba = user_displacement(bwd, pa.geo, w, h);
        }
        const std::vector<UserLevel>* uab = u_ab.empty() ? nullptr : &u_ab;
        const std::vector<UserLevel>* uba = u_ba.empty() ? nullptr : &u_ba;
        if (need_ab) { f_ab[k] = solve_pyramids_masked(pa, pb, fs, masks ? &mpa : nullptr, masks ? &mpb : nullptr, false, uab); has_ab[k] = true; }
        if (need_ba) { f_ba[k] = solve_pyramids_masked(pb, pa, fs, masks ? &mpb : nullptr, masks ? &mpa : nullptr, false, uba); has_ba[k] = true; }
    }
    // plates.rs:373-412: the composition of the group, bottom layer first, over an empty image
    Image res(w, h, fmt);
    for (int k = last; k >= first; k--) {
        const FlowField* fab = has_ab[k] ? &f_ab[k] : nullptr;
        const FlowField* fba = has_ba[k] ? &f_ba[k] : nullptr;
        const LPlane* pl_a = k == nfg ? nullptr : &raws_a[k];
        const LPlane* pl_b = k == nfg ? nullptr : &raws_b[k];
        const Image* fr_a = k == nfg ? &a : nullptr;
        const Image* fr_b = k == nfg ? &b : nullptr;
        Image la = layer_times(a, comp_plane(raws_a, job.shrink, k, fmt, w, h));
        Image lb = layer_times(b, comp_plane(raws_b, job.shrink, k, fmt, w, h));
        Image r;
        if (sel.interp == 0) {
            bool takes_a = nearest_takes_a(code, sel.wa);
            Image p = takes_a ? la : lb;
            int rc = refill(p, takes_a ? pl_a : pl_b, takes_a ? fr_a : fr_b, job.cs.taps_above_first, err, job.cs.wrap_360);
            if (rc) return rc;
            rc = compose_vectors(job.cs, sel, p, p, fab, fba, &r, err);
            if (rc) return rc;
        } else {
            // plates.rs:268-288: each side's plate is its own layer image OVER the other side's brought
            // to its time with amount 1: the inverse warp with hold edges (codes 0 and 1, A's plate reads
            // F_AB), the forward warp without coverage (codes 2 and 3, each side pushed by its own flow)
            WarpOpts o;
            o.is360 = job.cs.wrap_360;  // plates.rs:268-276 (warp_full)
            Image pa(w, h, fmt), pb(w, h, fmt);
            int rc = code >= 2 ? forward_warp(pa, lb, *fba, 1.0f, !job.cs.gouraud, nullptr, err) : inv_warp(pa, lb, *fab, 1.0f, o, nullptr, err);
            if (rc) return rc;
            over_pl(pa, la);
            rc = code >= 2 ? forward_warp(pb, la, *fab, 1.0f, !job.cs.gouraud, nullptr, err) : inv_warp(pb, la, *fba, 1.0f, o, nullptr, err);
            if (rc) return rc;
            over_pl(pb, lb);
            rc = refill(pa, pl_a, fr_a, job.cs.taps_above_first, err, job.cs.wrap_360);
            if (rc) return rc;
            rc = refill(pb, pl_b, fr_b, job.cs.taps_above_first, err, job.cs.wrap_360);
            if (rc) return rc;
            rc = compose_vectors(job.cs, sel, pa, pb, fab, fba, &r, err);
            if (rc) return rc;
        }
        if (k == nfg) res = std::move(r);
        else over_pl(res, r);
    }
    *out = std::move(res);
    return 0;
}

int rebuilt_plate(const Image& frame, const std::vector<std::vector<float>>& mattes, const std::vector<float>& shrink,
                  int k, bool reversed, bool above_first, Image* out, std::string* err, bool is360) {
    int w = frame.w, h = frame.h, nfg = (int)mattes.size();
    size_t n = (size_t)w * h;
    std::vector<LPlane> raws;
    for (const auto& m : mattes) raws.push_back(raw_plane(m.data(), n, frame.fmt));
    Image l = layer_times(frame, comp_plane(raws, shrink, k, frame.fmt, w, h));
    Image p = l;
    over_pl(p, l);  // the degenerate plate of an exact frame: the layer image OVER itself
    Image q = reversed ? rows_reversed(p) : p;
    int rc;
    if (k == nfg) {
        Image fa = reversed ? rows_reversed(frame) : frame;
        rc = refill(q, nullptr, &fa, above_first, err, is360);
    } else {
        LPlane rp = raws[k];
        if (reversed)
            for (int y = 0; y < h; y++)
                std::memcpy(&rp.v[(size_t)y * w], &raws[k].v[(size_t)(h - 1 - y) * w], sizeof(float) * w);
        rc = refill(q, &rp, nullptr, above_first, err, is360);
    }
    if (rc) return rc;
    p = reversed ? rows_reversed(q) : q;
    if (k == nfg) {
        *out = std::move(p);
        return 0;
    }
    Image o(w, h, frame.fmt);
    over_pl(o, p);
    *out = std::move(o);
    return 0;
}

}  // namespace orc
