// Vectors In on the device: the flow of a vector layer image (compose/vector.rs:323-345), the flow
// inversion (compose/vector.rs:347-397), and the single layer render of the `vectors-in` effect
// (plugins/vectors-in/src/glue.rs:386-495 with compose.rs:101-131 and compose/vector.rs:399-447)
// for one frame and over clips.
#include "runtime.h"

namespace tw {

// The flow of an engine vector image on ctx->cur (compose/vector.rs:335-345): the decode with its
// hole flags, the flow fill of the holes (is360 off; nothing runs without a hole), Vec Scale.
// *any must be 0 on entry; the image has sides of at least 2.
int vec_flow_dev(tw_ctx* ctx, const void* vec, int W, int H, int fmt, float md, float sx, float sy, bool above_first,
                 float* flow, uint8_t* holes, int* any, DevBuf& fillbuf) {
    long n = (long)W * H;
    double es = fmt == TW_U8 ? 4.0 : fmt == TW_U16 ? 8.0 : 16.0;
    LAUNCHB(ctx, n * (es + 8.0 + 1.0), k_vec_decode, grid1(n), TB, 0, vec, fmt, md, (float2*)flow, holes, n, any);
    CHECK(fill_dev(ctx, flow, W, H, FILL_FLOW, holes, any, above_first, fillbuf));
    LAUNCHB(ctx, n * 16.0, k_vec_scale, grid1(n), TB, 0, (float2*)flow, n, sx, sy);
    return TW_OK;
}

// The inversion of a W x H flow on ctx->cur (compose/vector.rs:370-397): T = -(1, fx, fy, 1) pushed
// along the flow at amount 1 (textured, or the Gouraud variant when !pyramid) with its coverage,
// channels 1 and 2 of the pushed image with the inverted coverage as holes, the flow fill. `t` and
// `pushed` hold W x H float pixels each; *any must be 0 on entry. The forward warp synchronises
// ctx->cur and uses the context's forward warp buffers.
int invert_flow_dev(tw_ctx* ctx, const float* flow, int W, int H, bool pyramid, bool above_first, float* out,
                    float* t, float* pushed, uint8_t* holes, int* any, DevBuf& fillbuf) {
    long n = (long)W * H;
    LAUNCHB(ctx, n * 24.0, k_invert_prep, grid1(n), TB, 0, (const float2*)flow, (float4*)t, n);
    CHECK(forward_warp_dev(ctx, t, flow, W, H, W, H, TW_F32, 1.0f, pyramid, pushed, nullptr));
    LAUNCHB(ctx, n * 25.0, k_invert_take, grid1(n), TB, 0, (const float4*)pushed, ctx->fw_cov.as<uint8_t>(),
            (float2*)out, holes, n, any);
    return fill_dev(ctx, out, W, H, FILL_FLOW, holes, any, above_first, fillbuf);
}

// image.rs:388-425 (error_frame, SizeMismatch) written to a wire frame: red, alpha half
__global__ void k_error_fill(void* __restrict__ wire, int fmt, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fmt == TW_U8) ((uchar4*)wire)[i] = make_uchar4(0xff, 0, 0, 0x80);
    else if (fmt == TW_U16) ((ushort4*)wire)[i] = make_ushort4(65535, 0, 0, 32768);  // q15_to_u16 of 0x8000, 0x4000
    else {
        float* p = (float*)wire;  // planes G, B, R, A
        p[i] = 0.0f;
        p[n + i] = 0.0f;
        p[2 * n + i] = 1.0f;
        p[3 * n + i] = 0.5f;
    }
}

namespace {

// compose/vector.rs:422-447 (complete_flows): which flows the composition (or the blur tail,
// which reads F_AB) reads
void flows_needed(const tw_engine_settings& cs, const tw_selection& sel, bool* need_ab, bool* need_ba) {
    bool tail = (double)std::fabs(sel.s0 - sel.s1) > 1e-6 && (double)cs.blur > 0.005;
    *need_ab = *need_ba = true;
    if (sel.interp == 0) {
        bool ab = (sel.wa < 0.5f && (unsigned)cs.warp_mode < 2) || (0.5f <= sel.wa && (unsigned)cs.warp_mode > 1);
        *need_ab = ab || tail;
        *need_ba = !ab;
    }
}

// Whether a frame of the clip runs the forward warp (warping codes 2 and 3, or a flow inversion):
// those frames use the context's forward warp buffers and run on one lane.
bool uses_forward_warp(const tw_engine_settings& cs, const tw_selection& sel, const tw_vecin_frame& vf) {
    if (sel.vectors_quality == 0 || sel.exact || (!vf.has_next && !vf.has_prev)) return false;
    if (cs.warp_mode >= 2) return true;
    bool need_ab, need_ba;
    flows_needed(cs, sel, &need_ab, &need_ba);
    return (need_ab && !vf.has_next) || (need_ba && !vf.has_prev);
}

}  // namespace

// One output frame of the single layer Vectors In render on lane L from device wire frames (nullptr
// = a blank frame); vnext / vprev the vector layers' wire frames at T(A) and T(B) (nullptr with the
// layer present: a transparent frame). The frame's end is L.ev_done on stream 0.
static int vecin_frame_body(tw_ctx* ctx, Lane& L, const tw_retime_settings& s, const tw_selection& sel,
                            const tw_vecin_frame& vf, float md, const void* wa, const void* wb, const void* vnext,
                            const void* vprev, int W, int H, int fmt, void* out_wire) {
    size_t bytes = (size_t)W * H * 4 * sample_bytes(fmt);
    long n = (long)W * H;
    int* flags = L.flags.as<int>();
    if (L.used) CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[1], L.ev_done, 0), "lane order"));
    L.used = true;
    ctx->cur = L.s[0];
    if (!vf.has_next && !vf.has_prev) {  // glue.rs:417-423: the size mismatch fill, no engine call
        LAUNCHB(ctx, (double)bytes, k_error_fill, grid1(n), TB, 0, out_wire, fmt, n);
        return ctx->cuda(cudaEventRecord(L.ev_done, L.s[0]), "event");
    }
    const tw_engine_settings& cs = s.compose;
    bool vector = sel.vectors_quality != 0 && !sel.exact;
    bool flip = vector && s.motion_rows_reversed != 0;  // the plugin's bottom-up rows (glue.rs:44-48)
    CHECK(ctx->ensure(L.eng[0], bytes, "engine A"));
    CHECK(ctx->ensure(L.eng[1], bytes, "engine B"));
    if (wa) from_frame_dev(ctx, wa, L.eng[0].p, W, H, fmt, flip);
    else CHECK(ctx->cuda(cudaMemsetAsync(L.eng[0].p, 0, bytes, ctx->cur), "blank"));
    ctx->cur = L.s[1];
    if (wb) from_frame_dev(ctx, wb, L.eng[1].p, W, H, fmt, flip);
    else CHECK(ctx->cuda(cudaMemsetAsync(L.eng[1].p, 0, bytes, ctx->cur), "blank"));
    WbScratch wbs = wb_scratch(L.wb_wt, L.wb_tmp, L.wb_mask, L.wb_cov);
    if (!vector) {  // compose.rs:218-231: the fast path, no vector layer read
        CHECK(ctx->cuda(cudaEventRecord(L.ev_pyr[1], L.s[1]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[0], L.ev_pyr[1], 0), "event"));
        ctx->cur = L.s[0];
        SmartScratch ss{&L.comp, &L.holes, &L.fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB};
        CHECK(interpolate_dev(ctx, sel, L.eng[0].p, L.eng[1].p, W, H, fmt, out_wire, true, flags + FL_BAD, &ss));
        return ctx->cuda(cudaEventRecord(L.ev_done, L.s[0]), "event");
    }
    if (sel.interp < 0 || sel.interp > 2)
        return ctx->fail(TW_ERR_BAD_PARAM, "interpolation mode %d is not 0 (Nearest), 1 (Blend) or 2 (Weighted Blend)", sel.interp);
    // the vector layers' flows: Next on stream 0 into F_AB, Prev on stream 1 into F_BA
    size_t fb = (size_t)n * 2 * sizeof(float);
    bool af = cs.taps_above_first != 0;
    for (int side = 0; side < 2; side++) {
        bool has = side == 0 ? vf.has_next != 0 : vf.has_prev != 0;
        if (!has) continue;
        ctx->cur = L.s[side];
        const void* vw = side == 0 ? vnext : vprev;
        CHECK(ctx->ensure(L.pyr[side], bytes, "vector layer"));
        CHECK(ctx->ensure(L.flow[side], fb, "vector flow"));
        CHECK(ctx->ensure(L.scratch[side][0], (size_t)n, "vector holes"));
        if (vw) from_frame_dev(ctx, vw, L.pyr[side].p, W, H, fmt, flip);
        else CHECK(ctx->cuda(cudaMemsetAsync(L.pyr[side].p, 0, bytes, ctx->cur), "transparent"));
        int* any = flags + FL_ANY0 + side;
        CHECK(ctx->cuda(cudaMemsetAsync(any, 0, sizeof(int), ctx->cur), "holes flag"));
        const float* sc = side == 0 ? vf.next_scale : vf.prev_scale;
        CHECK(vec_flow_dev(ctx, L.pyr[side].p, W, H, fmt, md, sc[0], sc[1], af, L.flow[side].as<float>(),
                           L.scratch[side][0].as<uint8_t>(), any, L.work[side]));
    }
    CHECK(ctx->cuda(cudaEventRecord(L.ev_solve1, L.s[1]), "event"));
    CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[0], L.ev_solve1, 0), "event"));
    ctx->cur = L.s[0];
    // complete_flows: the missing flow is the inversion of the other where something reads it
    bool need_ab, need_ba;
    flows_needed(cs, sel, &need_ab, &need_ba);
    bool have_ab = vf.has_next != 0, have_ba = vf.has_prev != 0;
    if ((!have_ab && need_ab) || (!have_ba && need_ba)) {
        int from = have_ab ? 0 : 1, to = 1 - from;
        CHECK(ctx->ensure(L.flow[to], fb, "inverted flow"));
        CHECK(ctx->ensure(L.scratch[0][1], (size_t)n * 16, "inversion image"));
        CHECK(ctx->ensure(L.scratch[0][2], (size_t)n * 16, "inversion pushed"));
        CHECK(ctx->ensure(L.scratch[0][0], (size_t)n, "inversion holes"));
        int* any = flags + FL_ANY0 + 2;
        CHECK(ctx->cuda(cudaMemsetAsync(any, 0, sizeof(int), ctx->cur), "holes flag"));
        CHECK(invert_flow_dev(ctx, L.flow[from].as<float>(), W, H, cs.gouraud == 0, af, L.flow[to].as<float>(),
                              L.scratch[0][1].as<float>(), L.scratch[0][2].as<float>(), L.scratch[0][0].as<uint8_t>(), any,
                              L.work[0]));
        (to == 0 ? have_ab : have_ba) = true;
    }
    SmartScratch ss{&L.comp, &L.holes, &L.fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB, &L.pre_blur};
    const float* fab = have_ab ? L.flow[0].as<float>() : nullptr;
    const float* fba = have_ba ? L.flow[1].as<float>() : nullptr;
    if (cs.warp_mode >= 2) {  // the forward compositions write an engine image: then the wire frame
        CHECK(ctx->ensure(L.pyr[0], bytes, "forward composite"));
        void* eng = L.pyr[0].p;  // the Next layer's image is no longer read
        CHECK(compose_dev(ctx, cs, sel, L.eng[0].p, L.eng[1].p, fab, fba, W, H, W, H, fmt, eng, false, false, flags + FL_BAD,
                          &ss));
        to_frame_dev(ctx, eng, out_wire, W, H, fmt, flip);
    } else {
        CHECK(compose_dev(ctx, cs, sel, L.eng[0].p, L.eng[1].p, fab, fba, W, H, W, H, fmt, out_wire, true, flip, flags + FL_BAD,
                          &ss));
    }
    return ctx->cuda(cudaEventRecord(L.ev_done, L.s[0]), "event");
}

// The clip body on device wire clips: output frame k reads footage frames vfs[k].a / .b, Vectors:
// Next frame vfs[k].a and Vectors: Prev frame vfs[k].b (outside a clip: blank, and transparent for
// a present vector layer); frames that run the forward warp go one at a time on lane 0.
static int vecin_clip_dev(tw_ctx* ctx, const tw_retime_settings& s, const uint8_t* frames, int nframes,
                          const uint8_t* next, int n_next, const uint8_t* prev, int n_prev, const tw_selection* sels,
                          const tw_vecin_frame* vfs, int nout, float md, int W, int H, int fmt, uint8_t* out) {
    size_t bytes = (size_t)W * H * 4 * sample_bytes(fmt);
    bool fw = false;
    for (int k = 0; k < nout; k++) fw = fw || uses_forward_warp(s.compose, sels[k], vfs[k]);
    const int nl = fw ? 1 : std::min(MAX_LANES, std::max(1, ctx->nlanes));
    CHECK(lanes_begin(ctx, nl));
    int rc = TW_OK;
    auto at = [&](const uint8_t* clip, int count, int i) -> const void* {
        return clip && i >= 0 && i < count ? clip + (size_t)i * bytes : nullptr;
    };
    for (int k = 0; k < nout && rc == TW_OK; k++) {
        const tw_vecin_frame& vf = vfs[k];
        rc = vecin_frame_body(ctx, ctx->lanes[k % nl], s, sels[k], vf, md, at(frames, nframes, vf.a),
                              at(frames, nframes, vf.b), at(next, n_next, vf.a), at(prev, n_prev, vf.b), W, H, fmt,
                              out + (size_t)k * bytes);
    }
    int rc2 = lanes_end(ctx, nl);
    return rc ? rc : rc2;
}

static bool vecin_args_ok(const tw_vecin_frame* vfs, int nout, const void* next, const void* prev) {
    for (int k = 0; k < nout; k++)
        if ((vfs[k].has_next && !next) || (vfs[k].has_prev && !prev)) return false;
    return true;
}

}  // namespace tw

using namespace tw;

extern "C" {

int tw_decode_vectors(tw_ctx* ctx, const tw_image* vec, float max_displace, tw_flow* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, vec, "decode vectors"));
    if (!out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    if (out->width != vec->width || out->height != vec->height)
        return ctx->fail(TW_ERR_MISMATCH, "decode vectors: a %dx%d flow for a %dx%d image", out->width, out->height,
                         vec->width, vec->height);
    long n = (long)vec->width * vec->height;
    CHECK(upload_image(ctx, ctx->eng[0], vec));
    CHECK(ctx->ensure(ctx->flow[0], (size_t)n * 8, "flow"));
    CHECK(ctx->ensure(ctx->holes, (size_t)n, "holes"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    LAUNCH(ctx, k_vec_decode, grid1(n), TB, 0, ctx->eng[0].p, vec->fmt, max_displace, ctx->flow[0].as<float2>(),
           ctx->holes.as<uint8_t>(), n, flags + FL_HOLE);
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->flow[0].p, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

int tw_flow_from_vectors(tw_ctx* ctx, const tw_image* vec, float max_displace, float scale_x, float scale_y,
                         int32_t taps_above_first, tw_flow* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, vec, "vector layer"));
    if (!out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    int W = vec->width, H = vec->height;
    if (out->width != W || out->height != H)
        return ctx->fail(TW_ERR_MISMATCH, "vector layer: a %dx%d flow for a %dx%d image", out->width, out->height, W, H);
    long n = (long)W * H;
    CHECK(upload_image(ctx, ctx->eng[0], vec));
    CHECK(ctx->ensure(ctx->flow[0], (size_t)n * 8, "flow"));
    CHECK(ctx->ensure(ctx->holes, (size_t)n, "holes"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    if (W < 2 || H < 2) {  // the decode, and a hole is refused by the fill (holefill.rs:273-277)
        LAUNCH(ctx, k_vec_decode, grid1(n), TB, 0, ctx->eng[0].p, vec->fmt, max_displace, ctx->flow[0].as<float2>(),
               ctx->holes.as<uint8_t>(), n, flags + FL_HOLE);
        LAUNCH(ctx, k_hole_side1, 1, 1, 0, flags + FL_HOLE, flags + FL_SIDE1);
        LAUNCH(ctx, k_vec_scale, grid1(n), TB, 0, ctx->flow[0].as<float2>(), n, scale_x, scale_y);
    } else {
        CHECK(vec_flow_dev(ctx, ctx->eng[0].p, W, H, vec->fmt, max_displace, scale_x, scale_y, taps_above_first != 0,
                           ctx->flow[0].as<float>(), ctx->holes.as<uint8_t>(), flags + FL_HOLE, ctx->fill));
    }
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->flow[0].p, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[4];
    CHECK(finish(ctx, hf, 4));
    if (hf[3]) return ctx->fail(TW_ERR_UNSUPPORTED, "hole fill of a %dx%d flow: the pyramid resample divides by zero", W, H);
    return TW_OK;
}

int tw_fill_flow_holes(tw_ctx* ctx, tw_flow* flow, const void* mask, int32_t mask_kind, int32_t taps_above_first) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!flow || !flow->data || !mask || flow->width <= 0 || flow->height <= 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    if (mask_kind < 1 || mask_kind > 3)
        return ctx->fail(TW_ERR_BAD_PARAM, "hole fill: mask kind %d is not 1 (u8), 2 (u16) or 3 (f32)", mask_kind);
    int W = flow->width, H = flow->height;
    long n = (long)W * H;
    size_t mb = (size_t)n * (mask_kind == 1 ? 1 : mask_kind == 2 ? 2 : 4);
    CHECK(ctx->ensure(ctx->flow[0], (size_t)n * 8, "flow"));
    CHECK(ctx->ensure(ctx->eng[1], mb, "hole fill mask"));
    CHECK(ctx->ensure(ctx->holes, (size_t)n, "holes"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[0].p, flow->data, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->eng[1].p, mask, mb, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    LAUNCH(ctx, k_mask_holes, grid1(n), TB, 0, ctx->eng[1].p, mask_kind, ctx->holes.as<uint8_t>(), n, flags + FL_HOLE);
    if (W < 2 || H < 2) LAUNCH(ctx, k_hole_side1, 1, 1, 0, flags + FL_HOLE, flags + FL_SIDE1);
    else CHECK(fill_dev(ctx, ctx->flow[0].p, W, H, FILL_FLOW, ctx->holes.as<uint8_t>(), flags + FL_HOLE, taps_above_first != 0,
                        ctx->fill));
    CHECK(ctx->cuda(cudaMemcpyAsync(flow->data, ctx->flow[0].p, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[4];
    CHECK(finish(ctx, hf, 4));
    if (hf[3]) return ctx->fail(TW_ERR_UNSUPPORTED, "hole fill of a %dx%d flow: the pyramid resample divides by zero", W, H);
    return TW_OK;
}

int tw_invert_flow(tw_ctx* ctx, const tw_flow* in, int32_t pyramid, int32_t taps_above_first, tw_flow* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!in || !in->data || !out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    int W = in->width, H = in->height;
    if (out->width != W || out->height != H)
        return ctx->fail(TW_ERR_MISMATCH, "flow inversion: a %dx%d output for a %dx%d flow", out->width, out->height, W, H);
    if (W < 2 || H < 2) return ctx->fail(TW_ERR_MISMATCH, "flow inversion: the forward warp needs a flow of at least 2x2");
    long n = (long)W * H;
    CHECK(ctx->ensure(ctx->flow[0], (size_t)n * 8, "flow"));
    CHECK(ctx->ensure(ctx->flow[1], (size_t)n * 8, "inverted flow"));
    CHECK(ctx->ensure(ctx->eng[0], (size_t)n * 16, "inversion image"));
    CHECK(ctx->ensure(ctx->eng[1], (size_t)n * 16, "inversion pushed"));
    CHECK(ctx->ensure(ctx->holes, (size_t)n, "holes"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[0].p, in->data, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    CHECK(invert_flow_dev(ctx, ctx->flow[0].as<float>(), W, H, pyramid != 0, taps_above_first != 0, ctx->flow[1].as<float>(),
                          ctx->eng[0].as<float>(), ctx->eng[1].as<float>(), ctx->holes.as<uint8_t>(), flags + FL_HOLE,
                          ctx->fill));
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->flow[1].p, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

int tw_retime_frame_vectors(tw_ctx* ctx, const tw_retime_settings* s, const tw_selection* sel, const tw_vecin_frame* vf,
                            float max_displace, const void* wire_a, const void* wire_b, const void* wire_next,
                            const void* wire_prev, int32_t width, int32_t height, int32_t fmt, void* wire_out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sel || !vf || !wire_out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    if (s->compose.wrap_360) return ctx->fail(TW_ERR_UNSUPPORTED, "the 360 inverse warp is not on the device");
    size_t bytes = (size_t)width * height * 4 * sample_bytes(fmt);
    const void* host[4] = {wire_a, wire_b, vf->has_next ? wire_next : nullptr, vf->has_prev ? wire_prev : nullptr};
    const void* dev[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int i = 0; i < 4; i++) {
        if (!host[i]) continue;
        DevBuf& b = ctx->vi_wire[i];
        CHECK(ctx->ensure(b, bytes, "wire frame"));
        CHECK(ctx->cuda(cudaMemcpyAsync(b.p, host[i], bytes, cudaMemcpyHostToDevice, ctx->stream), "upload"));
        dev[i] = b.p;
    }
    CHECK(ctx->ensure(ctx->vi_wire[4], bytes, "wire out"));
    CHECK(lanes_begin(ctx, 1));
    int rc = vecin_frame_body(ctx, ctx->lanes[0], *s, *sel, *vf, max_displace, dev[0], dev[1], dev[2], dev[3], width, height,
                              fmt, ctx->vi_wire[4].p);
    int rc2 = lanes_end(ctx, 1);
    if (rc) return rc;
    if (rc2) return rc2;
    CHECK(ctx->cuda(cudaMemcpyAsync(wire_out, ctx->vi_wire[4].p, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "download");
}

int tw_vectors_in_clip_device(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                              const void* next, int32_t n_next, const void* prev, int32_t n_prev,
                              const tw_selection* sels, const tw_vecin_frame* vfs, int32_t nout, float max_displace,
                              int32_t width, int32_t height, int32_t fmt, void* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sels || !vfs || !out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0 || nout < 0 || nframes < 0 ||
        n_next < 0 || n_prev < 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    if (!vecin_args_ok(vfs, nout, next, prev)) return ctx->fail(TW_ERR_BAD_PARAM, "a present vector layer without its clip");
    if (s->compose.wrap_360) return ctx->fail(TW_ERR_UNSUPPORTED, "the 360 inverse warp is not on the device");
    return vecin_clip_dev(ctx, *s, (const uint8_t*)frames, nframes, (const uint8_t*)next, n_next, (const uint8_t*)prev,
                          n_prev, sels, vfs, nout, max_displace, width, height, fmt, (uint8_t*)out);
}

int tw_vectors_in_clip(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes, const void* next,
                       int32_t n_next, const void* prev, int32_t n_prev, const tw_selection* sels,
                       const tw_vecin_frame* vfs, int32_t nout, float max_displace, int32_t width, int32_t height,
                       int32_t fmt, void* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sels || !vfs || !out || !frames || fmt < 0 || fmt > 2 || width <= 0 || height <= 0 || nout < 0 ||
        nframes < 0 || n_next < 0 || n_prev < 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    if (!vecin_args_ok(vfs, nout, next, prev)) return ctx->fail(TW_ERR_BAD_PARAM, "a present vector layer without its clip");
    if (s->compose.wrap_360) return ctx->fail(TW_ERR_UNSUPPORTED, "the 360 inverse warp is not on the device");
    size_t bytes = (size_t)width * height * 4 * sample_bytes(fmt);
    // the three clips go to the device whole, the output comes back whole
    const void* src[3] = {frames, next, prev};
    int cnt[3] = {nframes, next ? n_next : 0, prev ? n_prev : 0};
    const uint8_t* dev[3] = {nullptr, nullptr, nullptr};
    for (int i = 0; i < 3; i++) {
        if (!src[i] || cnt[i] == 0) continue;
        CHECK(ctx->ensure(ctx->vi_clip[i], (size_t)cnt[i] * bytes, "vector clip"));
        CHECK(ctx->cuda(cudaMemcpyAsync(ctx->vi_clip[i].p, src[i], (size_t)cnt[i] * bytes, cudaMemcpyHostToDevice, ctx->stream),
                        "upload"));
        dev[i] = ctx->vi_clip[i].as<uint8_t>();
    }
    CHECK(ctx->ensure(ctx->vi_out, std::max<size_t>((size_t)nout * bytes, 1), "output clip"));
    int rc = vecin_clip_dev(ctx, *s, dev[0], nframes, dev[1], cnt[1], dev[2], cnt[2], sels, vfs, nout, max_displace, width,
                            height, fmt, ctx->vi_out.as<uint8_t>());
    if (rc) return rc;
    if (nout > 0)
        CHECK(ctx->cuda(cudaMemcpyAsync(out, ctx->vi_out.p, (size_t)nout * bytes, cudaMemcpyDeviceToHost, ctx->stream),
                        "download"));
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "download");
}

}  // extern "C"

// ---- the Debug views of Create Vectors (debug.rs:104-171) ------------------------------------------

namespace tw {

// The view `code` (0 Blend, 1 Diff, 2 Detail Compare, 4 Warp, any other Edge Compare) of engine images
// x and y by the flow (fw x fh, interleaved) into the engine image `out`, on ctx->cur: the forward warp
// of x at amount 1 (Gouraud, or textured when !gouraud), then W' = (y OVER cleared) with W OVER it,
// then the view. Sides of 1: the zero vector image. The forward warp synchronises ctx->cur and uses
// the context's forward warp buffers.
int debug_view_dev(tw_ctx* ctx, const void* x, const void* y, const float* flow, int fw, int fh, int W, int H, int fmt,
                   int code, bool gouraud, void* out, DevBuf& warped, DevBuf& wp, DevBuf& luma) {
    long n = (long)W * H;
    size_t bytes = (size_t)n * 4 * sample_bytes(fmt);
    if (W < 2 || H < 2) {
        LAUNCH(ctx, k_encode_vectors, grid2(W, H), TB, 0, (const float*)nullptr, 0, 0, out, W, H, fmt, 0.0f, 0.0f, 0.0f,
               0.0f, 1);
        return TW_OK;
    }
    if (code == 4) return forward_warp_dev(ctx, x, flow, fw, fh, W, H, fmt, 1.0f, !gouraud, out, nullptr);
    CHECK(ctx->ensure(warped, bytes, "debug warp"));
    CHECK(ctx->ensure(wp, bytes, "debug composite"));
    CHECK(forward_warp_dev(ctx, x, flow, fw, fh, W, H, fmt, 1.0f, !gouraud, warped.p, nullptr));
    CHECK(ctx->cuda(cudaMemsetAsync(wp.p, 0, bytes, ctx->cur), "clear"));
    double pb = 3.0 * (double)bytes;
    LAUNCHB(ctx, pb, k_over_pl, grid1(n), TB, 0, wp.p, y, fmt, n);
    LAUNCHB(ctx, pb, k_over_pl, grid1(n), TB, 0, wp.p, (const void*)warped.p, fmt, n);
    if (code == 0) {
        LAUNCHB(ctx, pb, k_debug_blend, grid1(n), TB, 0, (const void*)wp.p, y, fmt, out, n);
    } else if (code == 1) {
        LAUNCHB(ctx, pb, k_debug_diff, grid1(n), TB, 0, (const void*)wp.p, y, fmt, out, n);
    } else {
        CHECK(ctx->ensure(luma, 2 * (size_t)n * sizeof(float), "debug luma"));
        float* lw = luma.as<float>();
        float* ly = lw + n;
        double lb = (double)bytes + 4.0 * n;
        LAUNCHB(ctx, lb, k_debug_luma, grid1(n), TB, 0, (const void*)wp.p, fmt, lw, n);
        LAUNCHB(ctx, lb, k_debug_luma, grid1(n), TB, 0, y, fmt, ly, n);
        LAUNCHB(ctx, 8.0 * n + (double)bytes, k_debug_overlay, grid2(W, H), TB, 0, (const float*)lw, (const float*)ly, W, H,
                fmt, code == 2 ? 0 : 1, out);
    }
    return TW_OK;
}

}  // namespace tw

extern "C" int tw_debug_view(tw_ctx* ctx, const tw_image* x, const tw_image* y, const tw_flow* flow, int32_t code,
                             int32_t gouraud, tw_image_mut* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, x, "debug view"));
    CHECK(check_image(ctx, y, "debug view"));
    if (!flow || !flow->data || !out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "debug view output"));
    if (!same_shape(x, y) || out->width != x->width || out->height != x->height || out->fmt != x->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "debug view: incompatible frames");
    int W = x->width, H = x->height;
    if ((W >= 2 && H >= 2) && (flow->width < 2 || flow->height < 2))
        return ctx->fail(TW_ERR_MISMATCH, "debug view: the forward warp needs a flow of at least 2x2");
    size_t bytes = (size_t)W * H * 4 * sample_bytes(x->fmt);
    size_t fb = (size_t)std::max(flow->width * flow->height, 1) * 2 * sizeof(float);
    CHECK(upload_image(ctx, ctx->vi_wire[0], x));
    CHECK(upload_image(ctx, ctx->vi_wire[1], y));
    CHECK(ctx->ensure(ctx->vi_wire[2], fb, "flow"));
    CHECK(ctx->ensure(ctx->vi_wire[3], bytes, "debug output"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->vi_wire[2].p, flow->data, (size_t)flow->width * flow->height * 2 * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream), "flow upload"));
    CHECK(debug_view_dev(ctx, ctx->vi_wire[0].p, ctx->vi_wire[1].p, ctx->vi_wire[2].as<float>(), flow->width, flow->height,
                         W, H, x->fmt, code, gouraud != 0, ctx->vi_wire[3].p, ctx->eng[0], ctx->eng[1], ctx->plane[0]));
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->vi_wire[3].p, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "kernel execution");
}
