// The layered composition with plates of retime-fgbg (layers/plates.rs:330-412): matte planes,
// chokes, refills, the per layer solves and compositions, and the layered clip call.
#include "runtime.h"

namespace tw {

// ---- the layered composition with plates (layers/plates.rs:330-412) ---------------------------------

// The settings the layered path serves (warping codes 0 to 3, Nearest, Blend or Weighted Blend, no
// 360 filters).
static int layers_check(tw_ctx* ctx, const tw_retime_settings& s, const tw_selection& sel) {
    const tw_engine_settings& cs = s.compose;
    if (cs.warp_mode < 0 || cs.warp_mode > 3) return ctx->fail(TW_ERR_BAD_PARAM, "layers: warping code %d is not 0 to 3", cs.warp_mode);
    if (sel.interp < 0 || sel.interp > 2)
        return ctx->fail(TW_ERR_BAD_PARAM, "layers: interpolation mode %d is not 0 to 2", sel.interp);
    if (cs.wrap_360 || s.flow.wrap)
        return ctx->fail(TW_ERR_UNSUPPORTED, "layers: the wrap-around (360) solve is not on the device");
    return TW_OK;
}

static int layer_job_check(tw_ctx* ctx, const tw_layer_job* job) {
    if (!job || job->nfg < 0 || job->nfg > 3) return ctx->fail(TW_ERR_BAD_PARAM, "layers: a job of 0 to 3 FG layers");
    if (job->display == 2) return ctx->fail(TW_ERR_BAD_PARAM, "layers: the Source display composes no layer");
    return TW_OK;
}

// layers.rs:120-129 (LayerJob::display_group): the group first..=last the Display popup shows
static void display_group(int display, int nfg, int* first, int* last) {
    if (display >= 3 && display <= 5) *first = *last = std::min(display - 3, nfg);
    else if (display == 6) *first = *last = nfg;
    else { *first = 0; *last = nfg; }
}

static bool any_shrink(const tw_layer_job& job) {
    for (int j = 0; j < job.nfg; j++)
        if (job.shrink[j] != 0.0f) return true;
    return false;
}

// The state a layered frame leaves in the flags, read after the stream is drained.
static int layers_status(tw_ctx* ctx) {
    int hf[4];
    CHECK(finish(ctx, hf, 4));
    if (hf[0]) return ctx->fail(TW_ERR_NAN_OUTPUT, "a solved flow holds a NaN");
    if (hf[1]) return bad_fail(ctx, hf[1]);
    if (hf[3]) return ctx->fail(TW_ERR_UNSUPPORTED, "hole fill of an image with a side of 1 pixel that has a hole");
    return TW_OK;
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

// The host scalars of one shrink step by the whole number of pixels a (matte.rs:366-385 blur_pl and
// 441-484 shrink_pl): the half kernel of its blur and its threshold, both from the runtime's powf.
struct ShrinkStep {
    bool blur = false;
    WideTaps taps{};
    float t = 0.0f;
    double den = 1.0;
};

static int shrink_step(tw_ctx* ctx, float a, ShrinkStep* st) {
    if (!(a > 0.0f)) return TW_OK;  // a step by 0 is the identity
    float r, wgt;
    choke_geometry(a, &r, &wgt);
    float radius = wgt + r;  // at least 2: the blur always runs
    int n = std::max((int)radius + 1, 0);
    if (n > MAX_WIDE_TAPS)
        return ctx->fail(TW_ERR_UNSUPPORTED, "layers: an inverse matte shrink of %g pixels (at most 13 on the device)",
                         (double)a);
    float s3 = radius / 3.0f, d = s3 * s3, sum = 0.0f;
    for (int i = 0; i < n; i++) {
        float fi = (float)i;
        st->taps.k[i] = crt_powf_host(2.0f, -((fi * fi) / d));
        sum += st->taps.k[i];
    }
    float den = sum * 2.0f - st->taps.k[0];
    for (int i = 0; i < n; i++) st->taps.k[i] /= den;
    st->taps.n = n;
    long long hn = (long long)r;
    float sigma = (float)((double)r / 3.0), s2 = sigma * sigma;
    std::vector<float> k((size_t)(2 * hn + 1));
    float ksum = 0.0f;
    for (size_t j = 0; j < k.size(); j++) {
        float x = (float)std::llabs((long long)j - hn);
        k[j] = crt_powf_host(2.0f, -((x * x) / s2));
        ksum += k[j];
    }
    for (float& v : k) v /= ksum;
    auto tail = [&](size_t from) {
        float acc = 0.0f;
        for (size_t j = from; j < k.size(); j++) acc += k[j];
        return acc;
    };
    float s2sum = tail(2), s3sum = tail(3);
    st->t = (s2sum - s3sum) * wgt + s3sum;
    st->den = 1.0 - (double)st->t;
    st->blur = true;
    return TW_OK;
}

// plates.rs:80-90 (cut_matte): FG j's raw plane `raw` (units of the depth) as the cut reads it, the
// plugin's choke by minus its inverse matte shrink (matte.rs:280-310) in the row order given, into
// `out`; scr: 4 planes of scratch.
static int choke_dev(tw_ctx* ctx, const float* raw, int W, int H, int fmt, float shrink, float* out, float* scr) {
    long n = (long)W * H;
    float white = fmt == TW_U8 ? 255.0f : fmt == TW_U16 ? 65535.0f : 1.0f;
    float kk = 1.0f / white;
    float amount = -shrink;
    float* base = scr;
    float* tmp = scr + n;
    float* b_lo = scr + 2 * n;
    float* b_hi = scr + 3 * n;
    if (!std::isfinite(amount)) {  // matte.rs:282-284: the plane as it is, not even clamped
        LAUNCH(ctx, k_choke_base, grid1(n), TB, 0, raw, n, kk, false, out);
        return TW_OK;
    }
    ChokeStep st{};
    st.grow = amount < 0.0f;
    float a = st.grow ? -amount : amount;
    if (a > 65536.0f) a = 65536.0f;  // matte.rs:190 (CHOKE_MAX)
    float lo = std::floor(a), hi = std::ceil(a);
    ShrinkStep s_lo, s_hi;
    CHECK(shrink_step(ctx, lo, &s_lo));
    st.mix = lo != hi;
    if (st.mix) CHECK(shrink_step(ctx, hi, &s_hi));
    st.lo_blur = s_lo.blur;
    st.hi_blur = st.mix && s_hi.blur;
    st.t_lo = s_lo.t;
    st.den_lo = s_lo.den;
    st.t_hi = s_hi.t;
    st.den_hi = s_hi.den;
    st.t = a - lo;
    LAUNCH(ctx, k_choke_base, grid1(n), TB, 0, raw, n, kk, st.grow, base);
    // blur_pl: the separable Gaussian with the column pass above first (conv.rs:598-615)
    if (st.lo_blur) {
        LAUNCH(ctx, k_conv_h_wide, grid2(W, H), TB, 0, (const float*)base, tmp, W, H, s_lo.taps);
        LAUNCH(ctx, k_conv_v_wide, grid2(W, H), TB, 0, (const float*)tmp, b_lo, W, H, s_lo.taps, true);
    }
    if (st.hi_blur) {
        LAUNCH(ctx, k_conv_h_wide, grid2(W, H), TB, 0, (const float*)base, tmp, W, H, s_hi.taps);
        LAUNCH(ctx, k_conv_v_wide, grid2(W, H), TB, 0, (const float*)tmp, b_hi, W, H, s_hi.taps, true);
    }
    LAUNCH(ctx, k_choke_finish, grid1(n), TB, 0, (const float*)base, (const float*)b_lo, (const float*)b_hi, st, n, out);
    return TW_OK;
}

// plates.rs:50-57: the raw planes of one side (each matte clamped when one of its values leaves
// 0..1) and, when a layer has an inverse matte shrink, the choked cut planes of every FG layer
static int raw_and_cut_planes(tw_ctx* ctx, const tw_layer_job& job, const float* mat, int side, int W, int H, int fmt,
                              float* raw, float* cuts, float* scr, int* range_flags) {
    long n = (long)W * H;
    int nfg = job.nfg;
    for (int j = 0; j < nfg; j++) {
        const float* m = mat + ((size_t)side * nfg + j) * n;
        int* fl_ = range_flags + side * 4 + j;
        LAUNCH(ctx, k_matte_out_of_range, grid1(n), TB, 0, m, n, fl_);
        LAUNCH(ctx, k_raw_plane, grid1(n), TB, 0, m, n, fmt, fl_, raw + (size_t)j * n);
    }
    if (cuts)
        for (int j = 0; j < nfg; j++) CHECK(choke_dev(ctx, raw + (size_t)j * n, W, H, fmt, job.shrink[j], cuts + (size_t)j * n, scr));
    return TW_OK;
}

// plates.rs:245-256 (refill) of the plate p of layer k at one side: unpremultiply, the pull-push fill
// where the plate is not opaque, the alpha replaced by the layer's raw plane (plane) or the frame's
// alpha (frame), premultiply
// holes: w*h bytes of scratch for the hole mask; hole_flag / side1_flag: the "some hole" flag of this
// fill and the refused fill of an image with a side of 1
static int refill_dev(tw_ctx* ctx, void* p, int W, int H, int fmt, const float* plane, const void* frame,
                      bool above_first, uint8_t* holes, int* hole_flag, int* side1_flag, DevBuf& fillbuf) {
    long n = (long)W * H;
    CHECK(ctx->cuda(cudaMemsetAsync(hole_flag, 0, sizeof(int), ctx->cur), "holes flag"));
    LAUNCH(ctx, k_refill_pre, grid1(n), TB, 0, p, fmt, n, holes, hole_flag);
    if (W < 2 || H < 2) LAUNCH(ctx, k_hole_side1, 1, 1, 0, hole_flag, side1_flag);
    else CHECK(fill_dev(ctx, p, W, H, fmt, holes, hole_flag, above_first, fillbuf));
    LAUNCH(ctx, k_refill_post, grid1(n), TB, 0, p, fmt, n, plane, frame);
    return TW_OK;
}

// One layered frame on ctx->stream: the engine images A and B in ctx->eng[0] / ctx->eng[1] (motion
// row order), `mat` the 2 x nfg raw mattes on the device (A's, then B's; FG1 first). The layers of
// the job's display group are solved and composed. Clears the flags first; *res_out receives the
// engine result (device).

static int layers_dev(tw_ctx* ctx, const tw_retime_settings& s, const tw_selection& sel_, const tw_layer_job& job,
                      const float* mat, int W, int H, int fmt, void** res_out, const tw_user_point* pts = nullptr,
                      const int32_t* npts = nullptr, bool flip_points = false) {
    const tw_selection* sel = &sel_;
    const tw_engine_settings& cs = s.compose;
    CHECK(layers_check(ctx, s, sel_));
    CHECK(layer_job_check(ctx, &job));
    int nfg = job.nfg;
    int first, last;
    display_group(job.display, nfg, &first, &last);
    bool shrink = any_shrink(job);
    long n = (long)W * H;
    size_t px = 4 * sample_bytes(fmt), ib = (size_t)n * px;
    tw_flow_settings fs0 = s.flow;
    fs0.quality = sel->vectors_quality;
    fs0.track_alpha = 0;  // plates.rs:319-323: the layered solves add no alpha to the luma,
    // Track RGB+A puts their luma pyramids (only) in the 360 mode of the filters
    bool pyramid_wrap = s.flow.wrap || s.flow.track_alpha;
    Geo g;
    CHECK(geometry(fs0, W, H, &g, &ctx->err));
    size_t pf = pyramid_floats(g);
    size_t fb = (size_t)g.w * g.h * 2;
    int L = nfg + 1;
    // one block: raw and cut planes (2 sides x nfg), comp planes (2 x L), layer images (2 x L), two
    // plates, the result, the flows (2 x L), per solved layer and side its pyramids, mask pyramid,
    // solver matte and scratch, and the user displacements
    size_t fl = 0;
    auto take = [&](size_t floats) { size_t o = fl; fl += (floats + 63) & ~(size_t)63; return o; };
    size_t o_raw = take(2 * (size_t)nfg * n), o_cut = take(shrink ? 2 * (size_t)nfg * n : 0), o_comp = take(2 * (size_t)L * n);
    size_t o_img = take(2 * (size_t)L * ib / 4 + 1), o_plate = take(2 * ib / 4 + 1);
    int G = last - first + 1;  // the layers solved, each on its own pair of streams with its own buffers
    size_t o_res = take(ib / 4 + 1), o_flow = take(2 * (size_t)L * fb), o_pyr = take(4 * pf * G), o_mpyr = take(2 * pf * G);
    size_t lres_floats = (ib + 255) / 256 * 64;  // one layer's composition, 256-byte aligned (8 and 16 B pixels)
    size_t o_scr = take(4 * (size_t)n), o_sides = take(10 * (size_t)n * G), o_lres = take(G * lres_floats);
    bool any_points = false;
    for (int k = 0; pts && npts && k <= nfg; k++) any_points = any_points || npts[k] > 0;
    size_t o_user = take(any_points ? 6 * pf * G : 0);
    CHECK(ctx->ensure(ctx->lay_mem, fl * sizeof(float), "layer buffers"));
    CHECK(ctx->ensure(ctx->holes, (size_t)n, "holes mask"));
    CHECK(ctx->ensure(ctx->eng[2], ib, "layer result"));
    float* M = ctx->lay_mem.as<float>();
    float* user = any_points ? M + o_user : nullptr;  // du, dv, uw of F_AB's solve, then of F_BA's
    float* raw = M + o_raw;
    float* cuts = shrink ? M + o_cut : nullptr;
    float* comp = M + o_comp;
    auto img = [&](int side, int k) { return (void*)((char*)(M + o_img) + ((size_t)side * L + k) * ib); };
    void* plate[2] = {(void*)(M + o_plate), (void*)((char*)(M + o_plate) + ib)};
    void* res = (void*)(M + o_res);
    auto flow = [&](int dir, int k) { return M + o_flow + ((size_t)dir * L + k) * fb; };  // dir 0: F_AB, 1: F_BA
    // layer g of the group (g = k - first), side 0 (A) or 1 (B): its band pyramid (with the transposed
    // copy), its mask pyramid, its solver matte plus four planes of scratch, its user displacement
    auto pyr = [&](int g, int side) { return M + o_pyr + ((size_t)g * 2 + side) * 2 * pf; };
    auto mpyr = [&](int g, int side) { return M + o_mpyr + ((size_t)g * 2 + side) * pf; };
    auto sides = [&](int g, int side) { return M + o_sides + ((size_t)g * 2 + side) * 5 * (size_t)n; };
    float* scr = M + o_scr;
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    CHECK(ctx->cuda(cudaMemsetAsync(flags + FL_ONE, 0x01, sizeof(int), ctx->stream), "flags"));
    const void* frame[2] = {ctx->eng[0].p, ctx->eng[1].p};
    // the raw planes, the cut planes of a shrink (in the motion path's rows, as the plates run), the
    // per-level range flags are not in use yet
    for (int side = 0; side < 2; side++)
        CHECK(raw_and_cut_planes(ctx, job, mat, side, W, H, fmt, raw + (size_t)side * nfg * n,
                                 cuts ? cuts + (size_t)side * nfg * n : nullptr, scr, flags + FL_ANY0));
    // the composition planes and the layer images of the group's layers at both sides
    for (int side = 0; side < 2; side++)
        for (int k = first; k <= last; k++) {
            float* c = comp + ((size_t)side * L + k) * n;
            LAUNCH(ctx, k_comp_plane, grid1(n), TB, 0, raw + (size_t)side * nfg * n,
                   cuts ? (const float*)(cuts + (size_t)side * nfg * n) : (const float*)nullptr, nfg, k, n, fmt, c);
            LAUNCH(ctx, k_layer_times, grid1(n), TB, 0, frame[side], c, img(side, k), fmt, n);
        }
    // the solves (plates.rs:340-369): each layer's own layer images, masked by its solver masks
    bool need_ab = true, need_ba = true;
    if (sel->interp == 0) {
        bool use_ab = (sel->wa < 0.5f && (unsigned)cs.warp_mode < 2) || (0.5f <= sel->wa && (unsigned)cs.warp_mode > 1);
        need_ab = use_ab;
        need_ba = !use_ab;
    }
    int pt_first[4] = {0, 0, 0, 0};
    for (int k = 1; pts && npts && k <= nfg; k++) pt_first[k] = pt_first[k - 1] + npts[k - 1];
    // The layers of the group are independent until the composition, a layer's two sides until its
    // solves, and its two solves of each other: layer g runs on the two streams of lane g (side A's
    // pyramids and F_AB on the first, side B's and F_BA on the second) with its own buffers and range
    // flags; the lanes fork from the context's stream here and join it before the composition.
    // warping codes 0 and 1 compose every layer on its lane too (codes 2 and 3 read the forward warp's
    // hit counts back and compose on the context's stream)
    bool lane_compose = cs.warp_mode < 2;
    CHECK(ctx->cuda(cudaEventRecord(ctx->ev_start, ctx->stream), "event"));
    for (int k = first; k <= last; k++) {
        int g = k - first;
        Lane& LL = ctx->lanes[g];
        CHECK(lane_ready(ctx, LL));
        cudaStream_t st[2] = {LL.s[0], LL.s[1]};
        for (int i = 0; i < 2; i++) CHECK(ctx->cuda(cudaStreamWaitEvent(st[i], ctx->ev_start, 0), "event"));
        tw_flow_settings fs = fs0;
        fs.sensitivity = job.sensitivity[k];
        Geo gk;
        CHECK(geometry(fs, W, H, &gk, &ctx->err));
        tw_flow_settings fp = fs;
        fp.wrap = pyramid_wrap ? 1 : 0;
        // layers.rs:257-270 (solve_layer): a layer with points solves with their user displacement
        int np_k = pts && npts ? npts[k] : 0;
        const float* ud[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};  // F_AB's, F_BA's
        for (int side = 0; side < 2; side++) {
            ctx->cur = st[side];
            float* sm = sides(g, side);
            float* sc = sm + n;
            CHECK(build_pyramid_dev(ctx, img(side, k), W, H, fmt, fp, gk, pyr(g, side), pyr(g, side) + pf, LL.scratch[side]));
            LAUNCH(ctx, k_solver_mask, grid1(n), TB, 0, raw + (size_t)side * nfg * n, nfg, k,
                   comp + ((size_t)side * L + k) * n, n, fmt, sm);
            CHECK(build_mask_pyramid_dev(ctx, sm, W, H, fs, gk, mpyr(g, side), sc, sc + n, flags + FL_ONE));
            if (np_k > 0 && (side == 0 ? need_ab : need_ba)) {
                UserPairs pr;
                float* u = user + ((size_t)g * 2 + side) * 3 * pf;
                CHECK(user_pairs(ctx, pts + pt_first[k], np_k, side == 0, flip_points, H, &pr));
                CHECK(build_user_dev(ctx, pr, gk, W, H, u, u + pf, u + 2 * pf, sc));
                ud[side][0] = u; ud[side][1] = u + pf; ud[side][2] = u + 2 * pf;
            }
        }
        // both sides' pyramids before either solve
        CHECK(ctx->cuda(cudaEventRecord(LL.ev_pyr[0], st[0]), "event"));
        CHECK(ctx->cuda(cudaEventRecord(LL.ev_pyr[1], st[1]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(st[1], LL.ev_pyr[0], 0), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(st[0], LL.ev_pyr[1], 0), "event"));
        int* lf = LL.flags.as<int>();
        if (need_ab) {
            ctx->cur = st[0];
            CHECK(solve_pyramids_dev(ctx, pyr(g, 0), pyr(g, 1), pyr(g, 0) + pf, pyr(g, 1) + pf, gk, fs, LL.work[0],
                                     flow(0, k), lf + FL_ANY0, flags + FL_NAN, mpyr(g, 0), mpyr(g, 1), ud[0][0], ud[0][1],
                                     ud[0][2]));
        }
        if (need_ba) {
            ctx->cur = st[1];
            CHECK(solve_pyramids_dev(ctx, pyr(g, 1), pyr(g, 0), pyr(g, 1) + pf, pyr(g, 0) + pf, gk, fs, LL.work[1],
                                     flow(1, k), lf + FL_ANY1, flags + FL_NAN, mpyr(g, 1), mpyr(g, 0), ud[1][0], ud[1][1],
                                     ud[1][2]));
        }
        CHECK(ctx->cuda(cudaEventRecord(LL.ev_solve1, st[1]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(st[0], LL.ev_solve1, 0), "event"));  // lane stream 0 after both solves
        if (!lane_compose) {
            CHECK(ctx->cuda(cudaEventRecord(LL.ev_done, st[0]), "event"));
            CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->stream, LL.ev_done, 0), "event"));
        }
    }
    ctx->cur = ctx->stream;
    // the composition of the group, bottom layer first, over an empty image (plates.rs:373-412): each
    // layer's own composition, then OVER
    auto layer_res = [&](int k) { return (void*)(M + o_lres + (size_t)(k - first) * lres_floats); };
    // one layer's composition into dst on ctx->cur, with the scratch given
    auto compose_layer = [&](int k, void* const* plate, void* dst, const SmartScratch& sc, uint8_t* holes,
                             int* hole_flag, DevBuf& fillbuf) -> int {
        const float* fab = need_ab ? flow(0, k) : nullptr;
        const float* fba = need_ba ? flow(1, k) : nullptr;
        auto refill = [&](void* p, int side) -> int {
            const float* plane = k == nfg ? nullptr : raw + ((size_t)side * nfg + k) * n;
            return refill_dev(ctx, p, W, H, fmt, plane, frame[side], cs.taps_above_first != 0, holes, hole_flag,
                              flags + FL_SIDE1, fillbuf);
        };
        if (sel->interp == 0) {
            bool takes_a = cs.warp_mode == 0 ? 0.5f <= sel->wa : !(0.5f > sel->wa);  // layers.rs:697-703
            int side = takes_a ? 0 : 1;
            CHECK(ctx->cuda(cudaMemcpyAsync(plate[0], img(side, k), ib, cudaMemcpyDeviceToDevice, ctx->cur), "plate"));
            CHECK(refill(plate[0], side));
            return compose_dev(ctx, cs, *sel, plate[0], plate[0], fab, fba, g.w, g.h, W, H, fmt, dst, false, false,
                               flags + FL_BAD, &sc);
        }
        // plates.rs:268-288: PA = LA OVER LB brought to A, PB = LB OVER LA brought to B, amount 1: the
        // inverse warp with hold edges for codes 0 and 1 (LB read through F_AB), the forward warp without
        // coverage for codes 2 and 3 (each side pushed by its own flow, LB by F_BA)
        if (cs.warp_mode >= 2) {
            CHECK(forward_warp_dev(ctx, img(1, k), fba, g.w, g.h, W, H, fmt, 1.0f, cs.gouraud == 0, plate[0], nullptr));
            CHECK(forward_warp_dev(ctx, img(0, k), fab, g.w, g.h, W, H, fmt, 1.0f, cs.gouraud == 0, plate[1], nullptr));
        } else {
            WarpParams pa_ = warp_params(img(1, k), fab, g.w, g.h, 1.0f, W, H, true);
            WarpParams pb_ = warp_params(img(0, k), fba, g.w, g.h, 1.0f, W, H, true);
            LAUNCH(ctx, k_inv_warp, grid2(W, H), TB, 0, pa_, fmt, plate[0], (uint8_t*)nullptr, W, H, flags + FL_BAD);
            LAUNCH(ctx, k_inv_warp, grid2(W, H), TB, 0, pb_, fmt, plate[1], (uint8_t*)nullptr, W, H, flags + FL_BAD);
        }
        LAUNCH(ctx, k_over_pl, grid1(n), TB, 0, plate[0], img(0, k), fmt, n);
        LAUNCH(ctx, k_over_pl, grid1(n), TB, 0, plate[1], img(1, k), fmt, n);
        CHECK(refill(plate[0], 0));
        CHECK(refill(plate[1], 1));
        return compose_dev(ctx, cs, *sel, plate[0], plate[1], fab, fba, g.w, g.h, W, H, fmt, dst, false, false,
                           flags + FL_BAD, &sc);
    };
    if (lane_compose) {
        for (int k = first; k <= last; k++) {
            Lane& LL = ctx->lanes[k - first];
            ctx->cur = LL.s[0];
            for (int i = 0; i < 2; i++) CHECK(ctx->ensure(LL.eng[i], ib, "layer plates"));
            CHECK(ctx->ensure(LL.comp, (size_t)n, "refill holes"));
            int* lf = LL.flags.as<int>();
            WbScratch wl = wb_scratch(LL.wb_wt, LL.wb_tmp, LL.wb_mask, LL.wb_cov);
            SmartScratch sl{nullptr, &LL.holes, &LL.fill, lf + FL_HOLE, flags + FL_SIDE1, &wl, lf + FL_WB, &LL.pre_blur};
            void* plates_l[2] = {LL.eng[0].p, LL.eng[1].p};
            CHECK(compose_layer(k, plates_l, layer_res(k), sl, LL.comp.as<uint8_t>(), lf + FL_HOLE, LL.work[0]));
            CHECK(ctx->cuda(cudaEventRecord(LL.ev_done, LL.s[0]), "event"));
            CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->stream, LL.ev_done, 0), "event"));
        }
        ctx->cur = ctx->stream;
        if (last == nfg) {
            res = layer_res(last);  // Main_BG's composition is the bottom of the stack
        } else {
            CHECK(ctx->cuda(cudaMemsetAsync(res, 0, ib, ctx->stream), "empty result"));
            LAUNCH(ctx, k_over_pl, grid1(n), TB, 0, res, layer_res(last), fmt, n);
        }
        for (int k = last - 1; k >= first; k--) LAUNCH(ctx, k_over_pl, grid1(n), TB, 0, res, layer_res(k), fmt, n);
    } else {
        WbScratch wbs = wb_scratch(ctx->wb_wt, ctx->wb_tmp, ctx->wb_mask, ctx->wb_cov);
        SmartScratch ss{nullptr, &ctx->masks, &ctx->fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB,
                        &ctx->pre_blur};
        if (last != nfg) CHECK(ctx->cuda(cudaMemsetAsync(res, 0, ib, ctx->stream), "empty result"));
        for (int k = last; k >= first; k--) {
            void* dst = k == nfg ? res : ctx->eng[2].p;
            CHECK(compose_layer(k, plate, dst, ss, ctx->holes.as<uint8_t>(), flags + FL_HOLE, ctx->work[1]));
            if (k != nfg) LAUNCH(ctx, k_over_pl, grid1(n), TB, 0, res, dst, fmt, n);
        }
    }
    *res_out = res;
    return TW_OK;
}

// layers.rs:414-436 and 497-528 (rebuilt_plate): a single group display of an unwarped frame. For
// each side the group's layer image (host rows: the frames in ctx->eng[0] / [1] and the raw mattes
// `mat` as the host delivers them) OVER itself, refilled in the rows of the motion path (`reversed`)
// and, for an FG layer, laid OVER an empty image; then the interpolation without flows into the wire
// frame `out`. Clears the flags first.
static int rebuilt_frame_dev(tw_ctx* ctx, const tw_retime_settings& s, const tw_selection& sel, const tw_layer_job& job,
                             const float* mat, int W, int H, int fmt, void* out) {
    CHECK(layer_job_check(ctx, &job));
    int nfg = job.nfg, k, last;
    display_group(job.display, nfg, &k, &last);
    if (k != last) return ctx->fail(TW_ERR_UNSUPPORTED, "layers: the full group of an unwarped frame with a shrink");
    bool shrink = any_shrink(job), reversed = s.motion_rows_reversed != 0;
    long n = (long)W * H;
    size_t px = 4 * sample_bytes(fmt), ib = (size_t)n * px;
    size_t fl = 0;
    auto take = [&](size_t floats) { size_t o = fl; fl += (floats + 63) & ~(size_t)63; return o; };
    size_t o_raw = take((size_t)nfg * n), o_cut = take(shrink ? (size_t)nfg * n : 0), o_comp = take((size_t)n);
    size_t o_l = take(ib / 4 + 1), o_p = take(ib / 4 + 1), o_q = take(ib / 4 + 1), o_alpha = take(ib / 4 + 1);
    size_t img_floats = (ib + 255) / 256 * 64;  // an engine image, 256-byte aligned (8 and 16 B pixels)
    size_t o_r = take(2 * img_floats), o_scr = take(4 * (size_t)n);
    CHECK(ctx->ensure(ctx->lay_mem, fl * sizeof(float), "layer buffers"));
    CHECK(ctx->ensure(ctx->holes, (size_t)n, "holes mask"));
    float* M = ctx->lay_mem.as<float>();
    float* raw = M + o_raw;
    float* cuts = shrink ? M + o_cut : nullptr;
    float* comp = M + o_comp;
    void* l = M + o_l;
    void* p = M + o_p;
    void* q = M + o_q;
    void* alpha = M + o_alpha;
    void* r[2] = {(void*)(M + o_r), (void*)(M + o_r + img_floats)};
    float* scr = M + o_scr;
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    const void* frame[2] = {ctx->eng[0].p, ctx->eng[1].p};
    for (int side = 0; side < 2; side++) {
        CHECK(raw_and_cut_planes(ctx, job, mat, side, W, H, fmt, raw, cuts, scr, flags + FL_ANY0));
        LAUNCH(ctx, k_comp_plane, grid1(n), TB, 0, raw, (const float*)cuts, nfg, k, n, fmt, comp);
        LAUNCH(ctx, k_layer_times, grid1(n), TB, 0, frame[side], comp, l, fmt, n);
        CHECK(ctx->cuda(cudaMemcpyAsync(p, l, ib, cudaMemcpyDeviceToDevice, ctx->stream), "plate"));
        LAUNCH(ctx, k_over_pl, grid1(n), TB, 0, p, l, fmt, n);  // the degenerate plate: LA OVER LA
        void* fillme = p;
        const float* plane = k == nfg ? nullptr : raw + (size_t)k * n;
        const void* fa = frame[side];
        if (reversed) {
            LAUNCH(ctx, k_flip_rows, grid1(n * (long)(px / 4)), TB, 0, (const void*)p, q, W, H, (int)px);
            if (k == nfg) {
                LAUNCH(ctx, k_flip_rows, grid1(n * (long)(px / 4)), TB, 0, frame[side], alpha, W, H, (int)px);
                fa = alpha;
            } else {
                LAUNCH(ctx, k_flip_rows, grid1(n), TB, 0, (const void*)plane, alpha, W, H, 4);
                plane = (const float*)alpha;
            }
            fillme = q;
        }
        CHECK(refill_dev(ctx, fillme, W, H, fmt, k == nfg ? nullptr : plane, k == nfg ? fa : nullptr,
                         s.compose.taps_above_first != 0, ctx->holes.as<uint8_t>(), flags + FL_HOLE, flags + FL_SIDE1,
                         ctx->work[1]));
        if (reversed) LAUNCH(ctx, k_flip_rows, grid1(n * (long)(px / 4)), TB, 0, (const void*)q, p, W, H, (int)px);
        if (k == nfg) {
            CHECK(ctx->cuda(cudaMemcpyAsync(r[side], p, ib, cudaMemcpyDeviceToDevice, ctx->stream), "plate"));
        } else {
            CHECK(ctx->cuda(cudaMemsetAsync(r[side], 0, ib, ctx->stream), "empty layer"));
            LAUNCH(ctx, k_over_pl, grid1(n), TB, 0, r[side], p, fmt, n);
        }
    }
    WbScratch wbs = wb_scratch(ctx->wb_wt, ctx->wb_tmp, ctx->wb_mask, ctx->wb_cov);
    SmartScratch ss{&ctx->eng[2], &ctx->masks, &ctx->fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB};
    return interpolate_dev(ctx, sel, r[0], r[1], W, H, fmt, out, true, flags + FL_BAD, &ss);
}


// One frame of the plain vector path (compose/vector.rs:289-321) on ctx->stream: the engine images in
// ctx->eng[0] / ctx->eng[1] (motion row order), the solves the interpolation needs, compose_vectors
// into `res` (an engine image). The serial form of retime_frame_lane, for the compositions that
// read counts back (the forward warps).
static int vector_frame_dev(tw_ctx* ctx, const tw_retime_settings& s, const tw_selection& sel, int W, int H, int fmt,
                            void* res, const tw_user_point* pts = nullptr, int npts = 0, bool flip_points = false) {
    tw_flow_settings fs = s.flow;
    fs.quality = sel.vectors_quality;
    if (fs.wrap) return ctx->fail(TW_ERR_UNSUPPORTED, "the wrap-around (360) solve is not on the device");
    Geo g;
    CHECK(geometry(fs, W, H, &g, &ctx->err));
    size_t pf = pyramid_floats(g);
    CHECK(ctx->ensure(ctx->pyr[0], 2 * pf * 4, "pyramid"));
    CHECK(ctx->ensure(ctx->pyr[1], 2 * pf * 4, "pyramid"));
    float* px_ = ctx->pyr[0].as<float>();
    float* py_ = ctx->pyr[1].as<float>();
    CHECK(build_pyramid_dev(ctx, ctx->eng[0].p, W, H, fmt, fs, g, px_, px_ + pf, ctx->plane));
    CHECK(build_pyramid_dev(ctx, ctx->eng[1].p, W, H, fmt, fs, g, py_, py_ + pf, ctx->plane));
    size_t fb = (size_t)g.w * g.h * 2 * sizeof(float);
    CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
    CHECK(ctx->ensure(ctx->flow[1], fb, "flow"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    bool need_ab = true, need_ba = true;
    if (sel.interp == 0) {
        bool use_ab = (sel.wa < 0.5f && (unsigned)s.compose.warp_mode < 2) || (0.5f <= sel.wa && (unsigned)s.compose.warp_mode > 1);
        need_ab = use_ab;
        need_ba = !use_ab;
    }
    // layers.rs:310-336 (single_layer_with_points): with tracking points the solves take their user
    // displacement
    const float *uab[3] = {nullptr, nullptr, nullptr}, *uba[3] = {nullptr, nullptr, nullptr};
    if (pts && npts > 0) {
        size_t np0 = (size_t)g.w * g.h;
        CHECK(ctx->ensure(ctx->lay_mem, (6 * pf + 4 * np0) * sizeof(float), "user displacement"));
        float* u = ctx->lay_mem.as<float>();
        float* scr = u + 6 * pf;
        UserPairs pr;
        if (need_ab) {
            CHECK(user_pairs(ctx, pts, npts, true, flip_points, H, &pr));
            CHECK(build_user_dev(ctx, pr, g, W, H, u, u + pf, u + 2 * pf, scr));
            uab[0] = u; uab[1] = u + pf; uab[2] = u + 2 * pf;
        }
        if (need_ba) {
            CHECK(user_pairs(ctx, pts, npts, false, flip_points, H, &pr));
            CHECK(build_user_dev(ctx, pr, g, W, H, u + 3 * pf, u + 4 * pf, u + 5 * pf, scr));
            uba[0] = u + 3 * pf; uba[1] = u + 4 * pf; uba[2] = u + 5 * pf;
        }
    }
    if (need_ab)
        CHECK(solve_pyramids_dev(ctx, px_, py_, px_ + pf, py_ + pf, g, fs, ctx->work[0], ctx->flow[0].as<float>(),
                                 flags + FL_ANY0, flags + FL_NAN, nullptr, nullptr, uab[0], uab[1], uab[2]));
    if (need_ba)
        CHECK(solve_pyramids_dev(ctx, py_, px_, py_ + pf, px_ + pf, g, fs, ctx->work[1], ctx->flow[1].as<float>(),
                                 flags + FL_ANY1, flags + FL_NAN, nullptr, nullptr, uba[0], uba[1], uba[2]));
    WbScratch wbs = wb_scratch(ctx->wb_wt, ctx->wb_tmp, ctx->wb_mask, ctx->wb_cov);
    SmartScratch ss{nullptr, &ctx->holes, &ctx->fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB, &ctx->pre_blur};
    return compose_dev(ctx, s.compose, sel, ctx->eng[0].p, ctx->eng[1].p, need_ab ? ctx->flow[0].as<float>() : nullptr,
                       need_ba ? ctx->flow[1].as<float>() : nullptr, g.w, g.h, W, H, fmt, res, false, false, flags + FL_BAD,
                       &ss);
}

}  // namespace tw

extern "C" {

int tw_compose_layers(tw_ctx* ctx, const tw_retime_settings* s, const tw_selection* sel, const tw_image* a,
                      const tw_image* b, const tw_layer_job* job, const float* mattes_a, const float* mattes_b,
                      tw_image_mut* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sel || !job || !out || !out->data)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    CHECK(check_out(ctx, out, "compose_layers output"));
    CHECK(layer_job_check(ctx, job));
    int nfg = job->nfg;
    if (nfg > 0 && (!mattes_a || !mattes_b)) return ctx->fail(TW_ERR_BAD_PARAM, "bad argument: no mattes");
    CHECK(check_image(ctx, a, "layers"));
    CHECK(check_image(ctx, b, "layers"));
    if (!same_shape(a, b) || out->width != a->width || out->height != a->height || out->fmt != a->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "layers: images of different shapes");
    CHECK(layers_check(ctx, *s, *sel));
    int W = a->width, H = a->height, fmt = a->fmt;
    size_t n = (size_t)W * H, ib = n * 4 * sample_bytes(fmt);
    CHECK(ctx->ensure(ctx->lay_in, std::max<size_t>(2 * (size_t)nfg * n, 1) * sizeof(float), "mattes"));
    float* mat = ctx->lay_in.as<float>();
    CHECK(upload_image(ctx, ctx->eng[0], a));
    CHECK(upload_image(ctx, ctx->eng[1], b));
    if (nfg > 0) {
        CHECK(ctx->cuda(cudaMemcpyAsync(mat, mattes_a, (size_t)nfg * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream),
                        "matte upload"));
        CHECK(ctx->cuda(cudaMemcpyAsync(mat + (size_t)nfg * n, mattes_b, (size_t)nfg * n * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream), "matte upload"));
    }
    void* res = nullptr;
    CHECK(layers_dev(ctx, *s, *sel, *job, mat, W, H, fmt, &res, job->points, job->npoints, false));
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, res, ib, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    return layers_status(ctx);
}

// retime-fgbg with FG matte layers over a clip in host memory: per output frame the footage and
// matte frames are uploaded, the in-between frames run the layered path in the motion path's row
// order and the exact frames the interpolation without flows (the full group fast path,
// layers.rs:177-179), each frame on the context's stream.
int tw_retime_layers_clip(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                          const tw_layer_job* job, const void* const* matte_clips, const int32_t* matte_nframes,
                          const tw_selection* sels, int32_t nout, int32_t width, int32_t height, int32_t fmt, void* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    bool no_points = true;
    if (job && job->nfg >= 0 && job->nfg <= 3 && job->points && job->npoints && nout > 0)
        for (long i = 0; i < (long)nout * (job->nfg + 1); i++)
            if (job->npoints[i] != 0) no_points = false;
    if (job && job->nfg == 0 && job->display != 2 && sels && s && s->compose.warp_mode < 2 && no_points)
        return tw_retime_clip(ctx, s, frames, nframes, sels, nout, width, height, fmt, out);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sels || !frames || !out || !job || (job->nfg > 0 && !matte_clips) || fmt < 0 || fmt > 2 || width <= 0 ||
        height <= 0 || nout < 0 || nframes < 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    CHECK(layer_job_check(ctx, job));
    int nfg = job->nfg;
    const int32_t* matte_chan = job->matte_chan;
    int first, last;
    display_group(job->display, nfg, &first, &last);
    bool shrink = any_shrink(*job);
    for (int j = 0; j < nfg; j++)
        if (!matte_clips[j] || (matte_nframes && matte_nframes[j] < 0)) return ctx->fail(TW_ERR_BAD_PARAM, "bad matte clip");
    int W = width, H = height;
    long n = (long)W * H;
    size_t bytes = (size_t)n * 4 * sample_bytes(fmt);
    for (int i = 0; i < 3; i++) CHECK(ctx->ensure(ctx->wire[i], bytes, "wire staging"));
    for (int i = 0; i < 3; i++) CHECK(ctx->ensure(ctx->eng[i], bytes, "engine images"));
    CHECK(ctx->ensure(ctx->lay_in, 2 * (size_t)nfg * n * sizeof(float), "mattes"));
    CHECK(ctx->ensure(ctx->flags, FLAGS_BYTES, "flags"));
    float* mat = ctx->lay_in.as<float>();
    int* flags = ctx->flags.as<int>();
    if (!ctx->up) CHECK(ctx->cuda(cudaStreamCreateWithFlags(&ctx->up, cudaStreamNonBlocking), "copy stream"));
    for (int i = 0; i < 2; i++) {
        if (!ctx->lay_up[i]) CHECK(ctx->cuda(cudaEventCreateWithFlags(&ctx->lay_up[i], cudaEventDisableTiming), "event"));
        if (!ctx->lay_free[i]) CHECK(ctx->cuda(cudaEventCreateWithFlags(&ctx->lay_free[i], cudaEventDisableTiming), "event"));
        for (int j = 0; j < 2 + 2 * nfg; j++) CHECK(ctx->ensure(ctx->lay_stage[i][j], bytes, "staging"));
    }
    // how output frame k is rendered: the vector path, the rebuilt plates of a single layer display or
    // the interpolation of the two frames (compose.rs:209-211: with FG layers a shrink clears the
    // exactness of a position)
    auto is_vector = [&](const tw_selection& sel) {
        bool exact = sel.exact && !(nfg > 0 && shrink);
        return sel.vectors_quality != 0 && !exact;
    };
    auto is_rebuilt = [&](const tw_selection& sel) {
        return !is_vector(sel) && nfg > 0 && !(first == 0 && last == nfg && !shrink);
    };
    // a frame of a clip into a staging buffer on the copy stream, or a blank frame outside the clip
    // (host.rs:338-352)
    auto upload = [&](const void* clip, int count, int f, void* dst) -> int {
        if (f >= 0 && f < count)
            return ctx->cuda(cudaMemcpyAsync(dst, (const uint8_t*)clip + (size_t)f * bytes, bytes, cudaMemcpyHostToDevice,
                                             ctx->up), "upload");
        return ctx->cuda(cudaMemsetAsync(dst, 0, bytes, ctx->up), "blank");
    };
    // the uploads of output frame k into staging slot k % 2, once the frame before the last is done
    // reading that slot: the footage pair, and each FG layer's matte frames at A and at B
    auto stage = [&](int k) -> int {
        const tw_selection& sel = sels[k];
        int slot = k & 1;
        CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->up, ctx->lay_free[slot], 0), "event"));
        CHECK(upload(frames, nframes, sel.a, ctx->lay_stage[slot][0].p));
        CHECK(upload(frames, nframes, sel.b, ctx->lay_stage[slot][1].p));
        if (is_vector(sel) || is_rebuilt(sel))
            for (int side = 0; side < 2; side++)
                for (int j = 0; j < nfg; j++) {
                    int count = matte_nframes ? matte_nframes[j] : nframes;
                    CHECK(upload(matte_clips[j], count, side ? sel.b : sel.a, ctx->lay_stage[slot][2 + side * nfg + j].p));
                }
        return ctx->cuda(cudaEventRecord(ctx->lay_up[slot], ctx->up), "event");
    };
    // a frame's FG mattes at A and at B from its staging slot, read straight (matte.rs:141-188) in the
    // row order given
    auto mattes = [&](int slot, bool flip) -> int {
        for (int side = 0; side < 2; side++)
            for (int j = 0; j < nfg; j++)
                LAUNCH(ctx, k_matte_extract, grid1(n), TB, 0, ctx->lay_stage[slot][2 + side * nfg + j].p, fmt, matte_chan[j],
                       W, H, flip, mat + ((size_t)side * nfg + j) * n);
        return TW_OK;
    };
    if (nout > 0) CHECK(stage(0));
    long pt_off = 0;  // the first point of output frame k in job->points
    for (int k = 0; k < nout; k++) {
        const tw_selection& sel = sels[k];
        const int32_t* npts = job->points && job->npoints ? job->npoints + (size_t)k * (nfg + 1) : nullptr;
        const tw_user_point* pts = npts ? job->points + pt_off : nullptr;
        for (int j = 0; npts && j <= nfg; j++) {
            if (npts[j] < 0) return ctx->fail(TW_ERR_BAD_PARAM, "a negative point count");
            pt_off += npts[j];
        }
        if (k + 1 < nout) CHECK(stage(k + 1));  // the next frame's uploads overlap this frame's work
        int slot = k & 1;
        bool vector = is_vector(sel);
        bool flip = vector && s->motion_rows_reversed != 0;
        CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->stream, ctx->lay_up[slot], 0), "event"));
        from_frame_dev(ctx, ctx->lay_stage[slot][0].p, ctx->eng[0].p, W, H, fmt, flip);
        from_frame_dev(ctx, ctx->lay_stage[slot][1].p, ctx->eng[1].p, W, H, fmt, flip);
        bool rebuilt = is_rebuilt(sel);
        if (vector || rebuilt) CHECK(mattes(slot, flip));
        CHECK(ctx->cuda(cudaEventRecord(ctx->lay_free[slot], ctx->stream), "event"));  // the slot is read
        uint8_t* dst = (uint8_t*)out + (size_t)k * bytes;
        if (rebuilt) {
            // layers.rs:414-436: a single group display of an unwarped frame rebuilds its plates
            CHECK(rebuilt_frame_dev(ctx, *s, sel, *job, mat, W, H, fmt, ctx->wire[2].p));
        } else if (!vector) {
            CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
            WbScratch wbs = wb_scratch(ctx->wb_wt, ctx->wb_tmp, ctx->wb_mask, ctx->wb_cov);
            SmartScratch ss{&ctx->eng[2], &ctx->holes, &ctx->fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB};
            CHECK(interpolate_dev(ctx, sel, ctx->eng[0].p, ctx->eng[1].p, W, H, fmt, ctx->wire[2].p, true, flags + FL_BAD, &ss));
        } else {
            void* res = ctx->eng[2].p;
            bool fp = s->motion_rows_reversed != 0;  // layers.rs:348-351: points on the motion path's rows
            if (nfg > 0) CHECK(layers_dev(ctx, *s, sel, *job, mat, W, H, fmt, &res, pts, npts, fp));
            else CHECK(vector_frame_dev(ctx, *s, sel, W, H, fmt, res, pts, npts ? npts[0] : 0, fp));  // compose.rs:155-164
            if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_to_frame_u8, grid1(n), TB, 0, (const uint8_t*)res, ctx->wire[2].as<uint8_t>(), W, H, flip);
            else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_to_frame_u16, grid1(n), TB, 0, (const uint16_t*)res, ctx->wire[2].as<uint16_t>(), W, H, flip);
            else LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, (const float*)res, ctx->wire[2].as<float>(), W, H, flip);
        }
        CHECK(ctx->cuda(cudaMemcpyAsync(dst, ctx->wire[2].p, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download"));
        CHECK(layers_status(ctx));
    }
    return TW_OK;
}

}  // extern "C"
