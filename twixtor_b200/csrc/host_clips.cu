// Whole output frames: the per frame pipeline on a lane (two streams), the host buffer clip driver
// with its device frame cache and copy streams, the device clip and batch calls, and Create Vectors.
#include "runtime.h"

namespace tw {

void from_frame_dev(tw_ctx* ctx, const void* wire, void* eng, int W, int H, int fmt, bool flip) {
    long n = (long)W * H;
    if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_from_frame_u8, grid1(n), TB, 0, (const uint8_t*)wire, (uint8_t*)eng, W, H, flip);
    else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_from_frame_u16, grid1(n), TB, 0, (const uint16_t*)wire, (uint16_t*)eng, W, H, flip);
    else LAUNCHB(ctx, 2.0 * 16 * n, k_from_frame_f32, grid1(n), TB, 0, (const float*)wire, (float*)eng, W, H, flip);
}

// image.rs:213-245 on ctx->cur: an engine image to a wire frame (upside down with flip)
void to_frame_dev(tw_ctx* ctx, const void* eng, void* wire, int W, int H, int fmt, bool flip) {
    long n = (long)W * H;
    if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_to_frame_u8, grid1(n), TB, 0, (const uint8_t*)eng, (uint8_t*)wire, W, H, flip);
    else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_to_frame_u16, grid1(n), TB, 0, (const uint16_t*)eng, (uint16_t*)wire, W, H, flip);
    else LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, (const float*)eng, (float*)wire, W, H, flip);
}

// One output frame on lane L from two device-resident wire frames (nullptr = a blank frame outside
// the clip); writes the output wire frame to out_wire (device). Both lane streams must already be
// ordered after the caller's work (ctx->ev_start); the frame's end is L.ev_done on stream 0.
static int retime_frame_body(tw_ctx* ctx, Lane& L, const tw_retime_settings& s, const tw_selection& sel, const void* wa,
                             const void* wb, int W, int H, int fmt, void* out_wire) {
    size_t bytes = (size_t)W * H * 4 * sample_bytes(fmt);
    int* flags = L.flags.as<int>();
    CHECK(ctx->ensure(L.eng[0], bytes, "engine A"));
    CHECK(ctx->ensure(L.eng[1], bytes, "engine B"));
    bool vector = sel.vectors_quality != 0 && !sel.exact;
    bool flip = vector && s.motion_rows_reversed != 0;
    // stream 1 reuses this lane's buffers: it waits for the lane's previous frame (a captured frame
    // forks stream 1 from stream 0 instead: the graph runs after the lane's previous work on stream 0)
    if (ctx->gmode == GRAPH_CAPTURE) {
        CHECK(ctx->cuda(cudaEventRecord(L.ev_fork, L.s[0]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[1], L.ev_fork, 0), "event"));
    } else if (ctx->gmode == GRAPH_OFF && L.used) {
        CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[1], L.ev_done, 0), "lane order"));
    }
    L.used = true;
    // a frame outside the clip is blank (host.rs:338-352); blank images are all zero in every depth
    ctx->cur = L.s[0];
    if (wa) from_frame_dev(ctx, wa, L.eng[0].p, W, H, fmt, flip);
    else CHECK(ctx->cuda(cudaMemsetAsync(L.eng[0].p, 0, bytes, ctx->cur), "blank"));
    ctx->cur = L.s[1];
    if (wb) from_frame_dev(ctx, wb, L.eng[1].p, W, H, fmt, flip);
    else CHECK(ctx->cuda(cudaMemsetAsync(L.eng[1].p, 0, bytes, ctx->cur), "blank"));
    if (!vector) {
        CHECK(ctx->cuda(cudaEventRecord(L.ev_pyr[1], L.s[1]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[0], L.ev_pyr[1], 0), "event"));
        ctx->cur = L.s[0];
        WbScratch wbs = wb_scratch(L.wb_wt, L.wb_tmp, L.wb_mask, L.wb_cov);
        SmartScratch ss{&L.comp, &L.holes, &L.fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB};
        CHECK(interpolate_dev(ctx, sel, L.eng[0].p, L.eng[1].p, W, H, fmt, out_wire, true, flags + FL_BAD, &ss));
        if (ctx->inject_now(TW_INJECT_STATUS)) LAUNCH(ctx, k_set_flag, 1, 1, 0, flags, FL_BOUND);
        CHECK(ctx->cuda(cudaEventRecord(L.ev_done, L.s[0]), "event"));
        return TW_OK;
    }
    // the vector path (compose/vector.rs:163-178 solve_flows, then compose_vectors)
    tw_flow_settings fs = s.flow;
    fs.quality = sel.vectors_quality;
    if (fs.wrap) return ctx->fail(TW_ERR_UNSUPPORTED, "the wrap-around (360) solve is not on the device");
    Geo g;
    CHECK(geometry(fs, W, H, &g, &ctx->err));
    size_t pf = pyramid_floats(g);
    CHECK(ctx->ensure(L.pyr[0], 2 * pf * 4, "pyramid"));
    CHECK(ctx->ensure(L.pyr[1], 2 * pf * 4, "pyramid"));
    float* px_ = L.pyr[0].as<float>();
    float* py_ = L.pyr[1].as<float>();
    size_t fb = (size_t)g.w * g.h * 2 * sizeof(float);
    CHECK(ctx->ensure(L.flow[0], fb, "flow"));
    CHECK(ctx->ensure(L.flow[1], fb, "flow"));
    ctx->cur = L.s[0];
    CHECK(build_pyramid_dev(ctx, L.eng[0].p, W, H, fmt, fs, g, px_, px_ + pf, L.scratch[0]));
    CHECK(GOP(ctx, ctx->cuda(cudaEventRecord(L.ev_pyr[0], L.s[0]), "event")));
    ctx->cur = L.s[1];
    CHECK(build_pyramid_dev(ctx, L.eng[1].p, W, H, fmt, fs, g, py_, py_ + pf, L.scratch[1]));
    CHECK(GOP(ctx, ctx->cuda(cudaEventRecord(L.ev_pyr[1], L.s[1]), "event")));
    CHECK(GOP(ctx, ctx->cuda(cudaStreamWaitEvent(L.s[0], L.ev_pyr[1], 0), "event")));
    CHECK(GOP(ctx, ctx->cuda(cudaStreamWaitEvent(L.s[1], L.ev_pyr[0], 0), "event")));
    bool need_ab = true, need_ba = true;
    if (sel.interp == 0) {
        bool use_ab = (sel.wa < 0.5f && (unsigned)s.compose.warp_mode < 2) || (0.5f <= sel.wa && (unsigned)s.compose.warp_mode > 1);
        need_ab = use_ab;
        need_ba = !use_ab;
    } else if (sel.interp != 1 && sel.interp != 2) {
        return ctx->fail(TW_ERR_BAD_PARAM, "interpolation mode %d is not 0 (Nearest), 1 (Blend) or 2 (Weighted Blend)", sel.interp);
    }
    if (need_ab) {
        ctx->cur = L.s[0];
        CHECK(solve_pyramids_dev(ctx, px_, py_, px_ + pf, py_ + pf, g, fs, L.work[0], L.flow[0].as<float>(),
                                 flags + FL_ANY0, flags + FL_NAN));
    }
    if (need_ba) {
        ctx->cur = L.s[1];
        CHECK(solve_pyramids_dev(ctx, py_, px_, py_ + pf, px_ + pf, g, fs, L.work[1], L.flow[1].as<float>(),
                                 flags + FL_ANY1, flags + FL_NAN));
    }
    CHECK(GOP(ctx, ctx->cuda(cudaEventRecord(L.ev_solve1, L.s[1]), "event")));
    CHECK(GOP(ctx, ctx->cuda(cudaStreamWaitEvent(L.s[0], L.ev_solve1, 0), "event")));
    ctx->cur = L.s[0];
    WbScratch wbs = wb_scratch(L.wb_wt, L.wb_tmp, L.wb_mask, L.wb_cov);
    SmartScratch ss{&L.comp, &L.holes, &L.fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB, &L.pre_blur};
    CHECK(compose_dev(ctx, s.compose, sel, L.eng[0].p, L.eng[1].p, need_ab ? L.flow[0].as<float>() : nullptr,
                      need_ba ? L.flow[1].as<float>() : nullptr, g.w, g.h, W, H, fmt, out_wire, true, flip,
                      flags + FL_BAD, &ss));
    if (ctx->inject_now(TW_INJECT_STATUS)) LAUNCH(ctx, k_set_flag, 1, 1, 0, flags, FL_BOUND);
    if (ctx->gmode == GRAPH_OFF) CHECK(ctx->cuda(cudaEventRecord(L.ev_done, L.s[0]), "event"));
    return TW_OK;
}

// The shape of a frame that decides every launch and stream operation of its pipeline: the frame
// size and depth, the settings, and the selection's vector quality, interpolation and flow choice.
static std::string frame_key(const tw_retime_settings& s, const tw_selection& sel, int W, int H, int fmt) {
    int v[6] = {W, H, fmt, sel.vectors_quality, sel.interp, sel.interp == 0 ? (sel.wa < 0.5f ? 1 : 2) : 0};
    std::string k((const char*)v, sizeof v);
    k.append((const char*)&s, sizeof s);
    return k;
}

// One output frame on lane L (retime_frame_body), as a CUDA graph where the frame allows it: the
// vector path of warping code 0 with Nearest or Blend, both source frames in the clip, no Blur
// Compensation. The first frame of a shape runs as it is (its buffers come to exist), the second is
// captured into the lane's graph of that shape, and every later one re-issues the same host code
// in replay mode, which launches nothing and updates the kernel nodes whose arguments changed (the
// source and output frames, the blend weights), then launches the graph on the lane's first stream.
static int retime_frame_lane(tw_ctx* ctx, Lane& L, const tw_retime_settings& s, const tw_selection& sel, const void* wa,
                             const void* wb, int W, int H, int fmt, void* out_wire) {
    bool vector = sel.vectors_quality != 0 && !sel.exact;
    bool eligible = ctx->graphs_on && !ctx->serial && !ctx->prof.on && ctx->inject_kind == 0 && vector && wa && wb &&
                    s.compose.warp_mode == 0 && (sel.interp == 0 || sel.interp == 1) && !((double)s.compose.blur > 0.005) &&
                    !s.flow.wrap && !s.compose.wrap_360;
    if (!eligible) return retime_frame_body(ctx, L, s, sel, wa, wb, W, H, fmt, out_wire);
    FrameGraph& G = L.graphs[frame_key(s, sel, W, H, fmt)];
    if (G.exec && G.alloc_gen != ctx->alloc_gen) {  // a buffer moved since the capture
        drop_graph(G);
        G.seen = true;
    }
    if (!G.seen) {
        G.seen = true;
        return retime_frame_body(ctx, L, s, sel, wa, wb, W, H, fmt, out_wire);
    }
    if (!G.exec) {  // capture
        ctx->gmode = GRAPH_CAPTURE;
        ctx->gcur = &G;
        ctx->gfail = false;
        cudaError_t e = cudaStreamBeginCapture(L.s[0], cudaStreamCaptureModeRelaxed);
        int rc = e == cudaSuccess ? retime_frame_body(ctx, L, s, sel, wa, wb, W, H, fmt, out_wire) : TW_OK;
        cudaGraph_t g = nullptr;
        cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(L.s[0], &g) : e;
        bool failed = ctx->gfail || e != cudaSuccess || e2 != cudaSuccess || !g;
        ctx->gmode = GRAPH_OFF;
        ctx->gcur = nullptr;
        ctx->gfail = false;
        if (!failed) {
            G.graph = g;
            failed = cudaGraphInstantiate(&G.exec, g, 0) != cudaSuccess;
        } else if (g) {
            cudaGraphDestroy(g);
        }
        if (rc || failed) {  // nothing of the frame ran: drop the graph for good, issue it directly
            cudaGetLastError();
            drop_graph(G);
            G.seen = true;
            ctx->graphs_on = rc ? ctx->graphs_on : false;
            if (rc) return rc;
            return retime_frame_body(ctx, L, s, sel, wa, wb, W, H, fmt, out_wire);
        }
        G.alloc_gen = ctx->alloc_gen;
    } else {  // replay
        ctx->gmode = GRAPH_REPLAY;
        ctx->gcur = &G;
        ctx->gi = 0;
        ctx->gfail = false;
        int rc = retime_frame_body(ctx, L, s, sel, wa, wb, W, H, fmt, out_wire);
        bool ok = !ctx->gfail && ctx->gi == G.nodes.size() && G.alloc_gen == ctx->alloc_gen;
        ctx->gmode = GRAPH_OFF;
        ctx->gcur = nullptr;
        ctx->gfail = false;
        if (rc) return rc;
        if (!ok) {
            drop_graph(G);
            G.seen = true;
            return retime_frame_body(ctx, L, s, sel, wa, wb, W, H, fmt, out_wire);
        }
    }
    CHECK(ctx->cuda(cudaGraphLaunch(G.exec, L.s[0]), "graph launch"));
    return ctx->cuda(cudaEventRecord(L.ev_done, L.s[0]), "event");
}

// The Create Vectors pass on lane L (create_vectors.rs:162-183): the engine images X and Y are in
// L.eng[0] (ready on stream 0) and L.eng[1] (ready on stream 1), in the engine's row order. The
// pyramids run on both streams, the solve X -> Y and the encode on stream 0; `out` receives the
// engine image, or with to_wire the wire frame (rows turned back when flip). The frame's end is
// L.ev_done on stream 0.
static int vectors_lane(tw_ctx* ctx, Lane& L, const tw_vectors_settings& s, int W, int H, int fmt, void* out,
                        bool to_wire, bool flip, const tw_user_point* pts = nullptr, int npts = 0) {
    int* flags = L.flags.as<int>();
    size_t bytes = (size_t)W * H * 4 * sample_bytes(fmt);
    void* eng_out = out;
    if (to_wire) {
        CHECK(ctx->ensure(L.comp, bytes, "encoded vectors"));
        eng_out = L.comp.p;
    }
    bool searchable = W >= 2 && H >= 2;  // prep.rs:100-102
    tw_flow_settings fs = s.flow;
    fs.video_range_luma = 0;
    fs.skip_refine = 0;
    if (fs.wrap) return ctx->fail(TW_ERR_UNSUPPORTED, "the wrap-around (360) solve is not on the device");
    if (!searchable) {
        CHECK(ctx->cuda(cudaEventRecord(L.ev_pyr[1], L.s[1]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[0], L.ev_pyr[1], 0), "event"));
        ctx->cur = L.s[0];
        LAUNCH(ctx, k_encode_vectors, grid2(W, H), TB, 0, (const float*)nullptr, 0, 0, eng_out, W, H, fmt, 0.0f, 0.0f, 0.0f,
               0.0f, 1);
    } else {
        Geo g;
        CHECK(geometry(fs, W, H, &g, &ctx->err));
        size_t pf = pyramid_floats(g);
        CHECK(ctx->ensure(L.pyr[0], 2 * pf * 4, "pyramid"));
        CHECK(ctx->ensure(L.pyr[1], 2 * pf * 4, "pyramid"));
        CHECK(ctx->ensure(L.flow[0], (size_t)g.w * g.h * 2 * sizeof(float), "flow"));
        float* px_ = L.pyr[0].as<float>();
        float* py_ = L.pyr[1].as<float>();
        ctx->cur = L.s[0];
        CHECK(build_pyramid_dev(ctx, L.eng[0].p, W, H, fmt, fs, g, px_, px_ + pf, L.scratch[0]));
        ctx->cur = L.s[1];
        CHECK(build_pyramid_dev(ctx, L.eng[1].p, W, H, fmt, fs, g, py_, py_ + pf, L.scratch[1]));
        CHECK(ctx->cuda(cudaEventRecord(L.ev_pyr[1], L.s[1]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[0], L.ev_pyr[1], 0), "event"));
        ctx->cur = L.s[0];
        // create_vectors.rs:336-351 (layer_flows_on, one layer): tracking points give the solve X -> Y
        // their user displacement, the pairs (at X, at Y) on the rows of the motion path
        const float* u = nullptr;
        if (pts && npts > 0) {
            size_t np0 = (size_t)g.w * g.h;
            CHECK(ctx->ensure(L.user, (3 * pf + 4 * np0) * sizeof(float), "user displacement"));
            UserPairs pr;
            CHECK(user_pairs(ctx, pts, npts, true, flip, H, &pr));
            u = L.user.as<float>();
            CHECK(build_user_dev(ctx, pr, g, W, H, (float*)u, (float*)u + pf, (float*)u + 2 * pf, (float*)u + 3 * pf));
        }
        CHECK(solve_pyramids_dev(ctx, px_, py_, px_ + pf, py_ + pf, g, fs, L.work[0], L.flow[0].as<float>(), flags + FL_ANY0,
                                 flags + FL_NAN, nullptr, nullptr, u, u ? u + pf : nullptr, u ? u + 2 * pf : nullptr));
        if (s.display == 3) {  // glue.rs:557-566: the Debug view of the pair's flow
            CHECK(debug_view_dev(ctx, L.eng[0].p, L.eng[1].p, L.flow[0].as<float>(), g.w, g.h, W, H, fmt, s.debug_view,
                                 s.debug_textured == 0, eng_out, L.wb_wt[0], L.wb_wt[1], L.wb_tmp[0]));
        } else {
        // vectors.rs:78-83, host scalars in single precision
        float dw1 = (float)(W - 1), dh1 = (float)(H - 1), fw1 = (float)(g.w - 1), fh1 = (float)(g.h - 1);
        float sx = fw1 / dw1, sy = fh1 / dh1;
        float kx = (dw1 / fw1) / s.max_displace, ky = (dh1 / fh1) / s.max_displace;
        LAUNCH(ctx, k_encode_vectors, grid2(W, H), TB, 0, L.flow[0].as<float>(), g.w, g.h, eng_out, W, H, fmt, sx, sy, kx, ky, 0);
        }
    }
    if (to_wire) {
        long n = (long)W * H;
        if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_to_frame_u8, grid1(n), TB, 0, (const uint8_t*)eng_out, (uint8_t*)out, W, H, flip);
        else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_to_frame_u16, grid1(n), TB, 0, (const uint16_t*)eng_out, (uint16_t*)out, W, H, flip);
        else LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, (const float*)eng_out, (float*)out, W, H, flip);
    }
    CHECK(ctx->cuda(cudaEventRecord(L.ev_done, L.s[0]), "event"));
    return TW_OK;
}

}  // namespace tw

extern "C" {

int tw_retime_frame(tw_ctx* ctx, const tw_retime_settings* s, const tw_selection* sel, const void* wire_a,
                    const void* wire_b, int32_t width, int32_t height, int32_t fmt, void* wire_out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sel || !wire_out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    size_t bytes = (size_t)width * height * 4 * sample_bytes(fmt);
    CHECK(ctx->ensure(ctx->wire[0], bytes, "wire A"));
    CHECK(ctx->ensure(ctx->wire[1], bytes, "wire B"));
    CHECK(ctx->ensure(ctx->wire[2], bytes, "wire out"));
    if (wire_a) CHECK(ctx->cuda(cudaMemcpyAsync(ctx->wire[0].p, wire_a, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    if (wire_b) CHECK(ctx->cuda(cudaMemcpyAsync(ctx->wire[1].p, wire_b, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    CHECK(lanes_begin(ctx, 1));
    int rc = retime_frame_lane(ctx, ctx->lanes[0], *s, *sel, wire_a ? ctx->wire[0].p : nullptr,
                               wire_b ? ctx->wire[1].p : nullptr, width, height, fmt, ctx->wire[2].p);
    int rc2 = lanes_end(ctx, 1);
    if (rc) return rc;
    if (rc2) return rc2;
    CHECK(ctx->cuda(cudaMemcpyAsync(wire_out, ctx->wire[2].p, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "download");
}

// tw_retime_clip: output frame k runs on lane k % nl. Its two source frames come from the device
// frame cache (uploaded on the `up` stream once, in order of first use; a slot is reused only after
// the frames that read it are done); the frame is composed into the lane's output buffer and copied
// down on the `down` stream, which the lane's next frame waits for before it writes that buffer.
// The host-buffer clip driver shared by tw_retime_clip and tw_create_vectors_clip: output frame k
// reads clip frames src(k) = (a, b) (an index outside the clip is a blank frame) through the device
// frame cache (uploaded once on the copy stream), runs frame_fn(k, lane, device A or null, device B
// or null, device output) on lane k % nl, and copies the output back on the other copy stream.
extern "C++" {
template <typename Src, typename FrameFn>
static int clip_host(tw_ctx* ctx, const void* frames, int nframes, int nout, int W, int H, int fmt, void* out, Src src,
                     FrameFn frame_fn) {
    size_t bytes = (size_t)W * H * 4 * sample_bytes(fmt);
    const int nl = std::min(MAX_LANES, std::max(1, ctx->nlanes));
    const int NS = tw_ctx::CACHE_SLOTS;
    // the copy streams and the cache events are made on first use; the layered clip call may have
    // made the upload stream already, so each is checked on its own
    if (!ctx->up) CHECK(ctx->cuda(cudaStreamCreateWithFlags(&ctx->up, cudaStreamNonBlocking), "copy stream"));
    if (!ctx->down) CHECK(ctx->cuda(cudaStreamCreateWithFlags(&ctx->down, cudaStreamNonBlocking), "copy stream"));
    if (!ctx->cache_ready[0]) {
        for (int i = 0; i < NS; i++) {
            CHECK(ctx->cuda(cudaEventCreateWithFlags(&ctx->cache_ready[i], cudaEventDisableTiming), "event"));
            for (int j = 0; j < MAX_LANES; j++)
                CHECK(ctx->cuda(cudaEventCreateWithFlags(&ctx->cache_free[i][j], cudaEventDisableTiming), "event"));
        }
        for (int i = 0; i < MAX_LANES; i++)
            CHECK(ctx->cuda(cudaEventCreateWithFlags(&ctx->out_free[i], cudaEventDisableTiming), "event"));
    }
    for (int i = 0; i < NS; i++) {
        CHECK(ctx->ensure(ctx->cache[i], bytes, "frame cache"));
        ctx->cache_frame[i] = -1;
    }
    for (int i = 0; i < nl; i++) CHECK(ctx->ensure(ctx->outbuf[i], bytes, "output buffer"));
    CHECK(lanes_begin(ctx, nl));
    CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->up, ctx->ev_start, 0), "event"));
    CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->down, ctx->ev_start, 0), "event"));
    std::vector<int> last_use(NS, -1);   // the last output frame that reads each slot
    std::vector<unsigned> readers(NS, 0);  // lanes that read each slot since its upload
    std::vector<bool> out_used(nl, false);
    auto frame_slot = [&](int f, int k, int keep) -> int {  // the slot holding source frame f (uploaded if absent)
        for (int i = 0; i < NS; i++)
            if (ctx->cache_frame[i] == f) { last_use[i] = k; return i; }
        int best = -1;
        for (int i = 0; i < NS; i++) {  // the least recently used slot that the current frame does not hold
            if (i == keep) continue;
            if (best < 0 || last_use[i] < last_use[best]) best = i;
        }
        for (int j = 0; j < nl; j++)  // every frame that read the old contents has finished
            if (readers[best] & (1u << j)) cudaStreamWaitEvent(ctx->up, ctx->cache_free[best][j], 0);
        readers[best] = 0;
        cudaMemcpyAsync(ctx->cache[best].p, (const uint8_t*)frames + (size_t)f * bytes, bytes, cudaMemcpyHostToDevice, ctx->up);
        cudaEventRecord(ctx->cache_ready[best], ctx->up);
        ctx->cache_frame[best] = f;
        last_use[best] = k;
        return best;
    };
    int rc = TW_OK;
    for (int k = 0; k < nout && rc == TW_OK; k++) {
        int fa, fb;
        src(k, &fa, &fb);
        int li = k % nl;
        Lane& L = ctx->lanes[li];
        int sa = (fa >= 0 && fa < nframes) ? frame_slot(fa, k, -1) : -1;
        int sb = (fb >= 0 && fb < nframes) ? (fb == fa ? sa : frame_slot(fb, k, sa)) : -1;
        for (int st = 0; st < 2; st++) {
            if (sa >= 0) cudaStreamWaitEvent(L.s[st], ctx->cache_ready[sa], 0);
            if (sb >= 0) cudaStreamWaitEvent(L.s[st], ctx->cache_ready[sb], 0);
        }
        if (out_used[li]) cudaStreamWaitEvent(L.s[0], ctx->out_free[li], 0);
        rc = frame_fn(k, L, sa >= 0 ? ctx->cache[sa].p : nullptr, sb >= 0 ? ctx->cache[sb].p : nullptr, ctx->outbuf[li].p);
        if (rc) break;
        // the frame's reads of its slots end with the lane's frame (both streams joined at ev_done)
        if (sa >= 0) { cudaEventRecord(ctx->cache_free[sa][li], L.s[0]); readers[sa] |= 1u << li; }
        if (sb >= 0) { cudaEventRecord(ctx->cache_free[sb][li], L.s[0]); readers[sb] |= 1u << li; }
        cudaStreamWaitEvent(ctx->down, L.ev_done, 0);
        cudaMemcpyAsync((uint8_t*)out + (size_t)k * bytes, ctx->outbuf[li].p, bytes, cudaMemcpyDeviceToHost, ctx->down);
        cudaEventRecord(ctx->out_free[li], ctx->down);
        out_used[li] = true;
    }
    // the caller's stream waits for the uploads and downloads too
    cudaEvent_t e_up = ctx->cache_ready[0];
    CHECK(ctx->cuda(cudaEventRecord(e_up, ctx->up), "event"));
    CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->stream, e_up, 0), "event"));
    cudaEvent_t e_down = ctx->out_free[0];
    CHECK(ctx->cuda(cudaEventRecord(e_down, ctx->down), "event"));
    CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->stream, e_down, 0), "event"));
    int rc2 = lanes_end(ctx, nl);
    if (rc) return rc;
    if (rc2) return rc2;
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "download");
}
}  // extern "C++"

int tw_retime_clip(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                   const tw_selection* sels, int32_t nout, int32_t width, int32_t height, int32_t fmt, void* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sels || !frames || !out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0 || nout < 0 || nframes < 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    return clip_host(
        ctx, frames, nframes, nout, width, height, fmt, out,
        [&](int k, int* a, int* b) {
            *a = sels[k].a;
            *b = sels[k].b;
        },
        [&](int k, Lane& L, const void* wa, const void* wb, void* ow) {
            return retime_frame_lane(ctx, L, *s, sels[k], wa, wb, width, height, fmt, ow);
        });
}

// ---- Create Vectors ----------------------------------------------------------------------------------

int tw_encode_vectors(tw_ctx* ctx, tw_image_mut* out, const tw_flow* flow, float scale) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!out || !out->data || !flow || !flow->data || out->fmt < 0 || out->fmt > 2)
        return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "encode_vectors output"));
    int W = out->width, H = out->height;
    if (W < 2 || H < 2 || flow->width < 2 || flow->height < 2)
        return ctx->fail(TW_ERR_MISMATCH, "vector encode needs images and a flow of at least 2x2 (image %dx%d, flow %dx%d)", W,
                         H, flow->width, flow->height);
    size_t fb = (size_t)flow->width * flow->height * 2 * sizeof(float);
    size_t ob = (size_t)W * H * 4 * sample_bytes(out->fmt);
    CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
    CHECK(ctx->ensure(ctx->eng[2], ob, "encoded vectors"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[0].p, flow->data, fb, cudaMemcpyHostToDevice, ctx->stream), "flow upload"));
    float dw1 = (float)(W - 1), dh1 = (float)(H - 1), fw1 = (float)(flow->width - 1), fh1 = (float)(flow->height - 1);
    float sx = fw1 / dw1, sy = fh1 / dh1, kx = (dw1 / fw1) / scale, ky = (dh1 / fh1) / scale;
    LAUNCH(ctx, k_encode_vectors, grid2(W, H), TB, 0, ctx->flow[0].as<float>(), flow->width, flow->height, ctx->eng[2].p, W,
           H, out->fmt, sx, sy, kx, ky, 0);
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[2].p, ob, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

int tw_create_vectors(tw_ctx* ctx, const tw_vectors_settings* s, const tw_image* x, const tw_image* y,
                      tw_image_mut* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "create_vectors output"));
    CHECK(check_image(ctx, x, "create vectors"));
    CHECK(check_image(ctx, y, "create vectors"));
    if (!same_shape(x, y) || out->width != x->width || out->height != x->height || out->fmt != x->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "create vectors: incompatible inputs (%dx%d fmt %d against %dx%d fmt %d)", x->width,
                         x->height, x->fmt, y->width, y->height, y->fmt);
    int W = x->width, H = x->height, fmt = x->fmt;
    size_t bytes = (size_t)W * H * 4 * sample_bytes(fmt);
    Lane& L = ctx->lanes[0];
    CHECK(lanes_begin(ctx, 1));
    CHECK(ctx->ensure(L.eng[0], bytes, "engine X"));
    CHECK(ctx->ensure(L.eng[1], bytes, "engine Y"));
    CHECK(ctx->ensure(ctx->eng[2], bytes, "encoded vectors"));
    L.used = true;
    CHECK(ctx->cuda(cudaMemcpyAsync(L.eng[0].p, x->data, bytes, cudaMemcpyHostToDevice, L.s[0]), "upload"));
    CHECK(ctx->cuda(cudaMemcpyAsync(L.eng[1].p, y->data, bytes, cudaMemcpyHostToDevice, L.s[1]), "upload"));
    int rc = vectors_lane(ctx, L, *s, W, H, fmt, ctx->eng[2].p, false, false);
    int rc2 = lanes_end(ctx, 1);
    if (rc) return rc;
    if (rc2) return rc2;
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[2].p, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "download");
}

int tw_vectors_pair(int32_t n, int32_t time_step, int32_t track_frame, int32_t* a, int32_t* b) {
    return tw_vectors_frame_pair(n, time_step, track_frame, 0, a, b);
}

int tw_vectors_frame_pair(int32_t n, int32_t time_step, int32_t track_frame, int32_t debug, int32_t* a, int32_t* b) {
    if (!a || !b || time_step <= 0) return TW_ERR_BAD_PARAM;
    int64_t ct = (int64_t)n * time_step;
    if (ct > INT32_MAX || ct < INT32_MIN) return TW_ERR_BAD_PARAM;
    // create_vectors.rs:59-62: the frame number of the current time
    float q = (float)(int32_t)ct / (float)time_step + 0.5f;
    uint32_t frame = (uint32_t)(int64_t)q;
    // :71-89: the pair (the Debug display swaps the roles)
    float nf = (float)(int32_t)frame, fa = nf, fb = nf;
    if (!debug) {
        if (track_frame == 1) fb = nf - 1.0f;
        else if (track_frame == 2) fb = nf + 1.0f;
    } else {
        if (track_frame == 1) fa = nf + 1.0f;
        else if (track_frame == 2) fa = nf - 1.0f;
    }
    auto cvtt = [](float v) { return (v > -2147483904.0f && v < 2147483648.0f) ? (int32_t)v : INT32_MIN; };
    // :92-97 and the clip frame of that tick (a layer time divided by the frame length, rounded down)
    auto clip_index = [&](int32_t k) {
        float tsf = (float)time_step, x = (float)k;
        float t = x < 0.0f ? -((-x) * tsf + 0.5f) : tsf * x + 0.5f;
        int64_t ticks = cvtt(t);
        int64_t idx = ticks >= 0 ? ticks / time_step : -((-ticks + time_step - 1) / time_step);
        return (int32_t)std::max<int64_t>(std::min<int64_t>(idx, INT32_MAX), INT32_MIN);
    };
    *a = clip_index(cvtt(fa));
    *b = clip_index(cvtt(fb));
    return TW_OK;
}

int tw_create_vectors_clip(tw_ctx* ctx, const tw_vectors_settings* s, const void* frames, int32_t nframes,
                           const int32_t* pairs, int32_t nout, const tw_user_point* points, const int32_t* npoints,
                           int32_t width, int32_t height, int32_t fmt, void* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !pairs || !frames || !out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0 || nout < 0 || nframes < 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    std::vector<long> pt_first((size_t)nout + 1, 0);  // the first point of output frame k
    for (int k = 0; points && npoints && k < nout; k++) {
        if (npoints[k] < 0) return ctx->fail(TW_ERR_BAD_PARAM, "a negative point count");
        pt_first[k + 1] = pt_first[k] + npoints[k];
    }
    size_t bytes = (size_t)width * height * 4 * sample_bytes(fmt);
    bool flip = s->rows_reversed != 0 && width >= 2 && height >= 2;
    // the Debug views' forward warp reads its hit total back and uses the context's buffers: one lane
    int saved_lanes = ctx->nlanes;
    if (s->display == 3) ctx->nlanes = 1;
    int rc = clip_host(
        ctx, frames, nframes, nout, width, height, fmt, out,
        [&](int k, int* a, int* b) {
            *a = pairs[2 * k];
            *b = pairs[2 * k + 1];
        },
        [&](int k, Lane& L, const void* wa, const void* wb, void* ow) {
            CHECK(ctx->ensure(L.eng[0], bytes, "engine X"));
            CHECK(ctx->ensure(L.eng[1], bytes, "engine Y"));
            if (L.used) CHECK(ctx->cuda(cudaStreamWaitEvent(L.s[1], L.ev_done, 0), "lane order"));
            L.used = true;
            ctx->cur = L.s[0];
            if (wa) from_frame_dev(ctx, wa, L.eng[0].p, width, height, fmt, flip);
            else CHECK(ctx->cuda(cudaMemsetAsync(L.eng[0].p, 0, bytes, ctx->cur), "blank"));
            ctx->cur = L.s[1];
            if (wb) from_frame_dev(ctx, wb, L.eng[1].p, width, height, fmt, flip);
            else CHECK(ctx->cuda(cudaMemsetAsync(L.eng[1].p, 0, bytes, ctx->cur), "blank"));
            bool with_points = points && npoints && npoints[k] > 0;
            return vectors_lane(ctx, L, *s, width, height, fmt, ow, true, flip, with_points ? points + pt_first[k] : nullptr,
                                with_points ? npoints[k] : 0);
        });
    ctx->nlanes = saved_lanes;
    return rc;
}

int tw_retime_clip_device(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                          const tw_selection* sels, int32_t nout, int32_t width, int32_t height, int32_t fmt, void* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !sels || !frames || !out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0 || nout < 0 || nframes < 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    size_t bytes = (size_t)width * height * 4 * sample_bytes(fmt);
    const int nl = std::min(MAX_LANES, std::max(1, ctx->nlanes));
    CHECK(lanes_begin(ctx, nl));
    int rc = TW_OK;
    for (int k = 0; k < nout && rc == TW_OK; k++) {
        const tw_selection& sel = sels[k];
        const uint8_t* base = (const uint8_t*)frames;
        const void* fa = (sel.a >= 0 && sel.a < nframes) ? base + (size_t)sel.a * bytes : nullptr;
        const void* fb = (sel.b >= 0 && sel.b < nframes) ? base + (size_t)sel.b * bytes : nullptr;
        rc = retime_frame_lane(ctx, ctx->lanes[k % nl], *s, sel, fa, fb, width, height, fmt, (uint8_t*)out + (size_t)k * bytes);
    }
    int rc2 = lanes_end(ctx, nl);
    return rc ? rc : rc2;
}

int tw_retime_batch_device(tw_ctx* ctx, const tw_clip_job* jobs, int32_t njobs) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!jobs || njobs < 0) return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    for (int j = 0; j < njobs; j++) {
        const tw_clip_job& J = jobs[j];
        if (!J.settings || !J.sels || !J.frames || !J.out || J.fmt < 0 || J.fmt > 2 || J.width <= 0 || J.height <= 0 ||
            J.nout < 0 || J.nframes < 0)
            return ctx->fail(TW_ERR_BAD_PARAM, "batch job %d: bad argument", j);
    }
    // the deal: round k takes output frame k of every clip that has one, the largest frames first
    std::vector<int> order(njobs);
    for (int j = 0; j < njobs; j++) order[j] = j;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        return (long)jobs[x].width * jobs[x].height * sample_bytes(jobs[x].fmt) >
               (long)jobs[y].width * jobs[y].height * sample_bytes(jobs[y].fmt);
    });
    int rounds = 0;
    for (int j = 0; j < njobs; j++) rounds = std::max(rounds, jobs[j].nout);
    const int nl = std::min(MAX_LANES, std::max(1, ctx->nlanes));
    CHECK(lanes_begin(ctx, nl));
    int rc = TW_OK;
    long slot = 0;
    for (int k = 0; k < rounds && rc == TW_OK; k++)
        for (int j : order) {
            const tw_clip_job& J = jobs[j];
            if (k >= J.nout) continue;
            size_t bytes = (size_t)J.width * J.height * 4 * sample_bytes(J.fmt);
            const tw_selection& sel = J.sels[k];
            const uint8_t* base = (const uint8_t*)J.frames;
            const void* fa = (sel.a >= 0 && sel.a < J.nframes) ? base + (size_t)sel.a * bytes : nullptr;
            const void* fb = (sel.b >= 0 && sel.b < J.nframes) ? base + (size_t)sel.b * bytes : nullptr;
            rc = retime_frame_lane(ctx, ctx->lanes[slot++ % nl], *J.settings, sel, fa, fb, J.width, J.height, J.fmt,
                                   (uint8_t*)J.out + (size_t)k * bytes);
            if (rc) break;
        }
    int rc2 = lanes_end(ctx, nl);
    return rc ? rc : rc2;
}


}  // extern "C"
