// The library context (tw_open / tw_close), its profiler and lanes, and the checks every entry point
// shares.
#include "runtime.h"

namespace tw {

// Every kernel launch of the library goes through LAUNCHB (LAUNCH passes no byte count): it counts
// the launch and, when the kernel is the one being profiled, brackets it with events.
bool prof_match(tw_ctx* ctx, const char* kernel) {
    return ctx->prof.on && (ctx->prof.name == kernel || ctx->prof.name == "*");
}
// Events come from a pool that the context keeps (created before a profiled region, reused by
// every session), so a profiled launch costs two event records, no event creation.
void prof_mark(tw_ctx* ctx) {
    if (ctx->prof.pooled == ctx->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->ev_pool.push_back(e);
    }
    cudaEvent_t e = ctx->ev_pool[ctx->prof.pooled++];
    cudaEventRecord(e, ctx->cur);
    ctx->prof.ev.push_back(e);
}


__global__ void k_set_flag(int* flags, int idx) { flags[idx] = 1; }

// A kernel launch while a lane captures its frame graph (launched into the capture; its node and
// arguments recorded) or replays it (nothing launched: the node's arguments are updated in the
// executable graph when they differ from the last ones). A launch that does not line up with the
// captured graph marks the replay as failed, and the frame is issued again without the graph.
void graph_kernel(tw_ctx* ctx, const void* func, dim3 grid, dim3 block, size_t smem, void** argv, std::string&& packed) {
    FrameGraph* G = ctx->gcur;
    if (ctx->gfail || !G) return;
    if (ctx->gmode == GRAPH_CAPTURE) {
        if (cudaLaunchKernel(func, grid, block, argv, smem, ctx->cur) != cudaSuccess) {
            ctx->gfail = true;
            return;
        }
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        if (cudaStreamGetCaptureInfo(ctx->cur, &st, nullptr, nullptr, &deps, &nd) != cudaSuccess || nd != 1 ||
            st != cudaStreamCaptureStatusActive) {
            ctx->gfail = true;
            return;
        }
        G->nodes.push_back(deps[0]);
        G->funcs.push_back(func);
        G->args.push_back(std::move(packed));
        return;
    }
    size_t i = ctx->gi++;
    if (i >= G->nodes.size() || G->funcs[i] != func) {
        ctx->gfail = true;
        return;
    }
    if (G->args[i] != packed) {
        cudaKernelNodeParams kp{};
        kp.func = (void*)func;
        kp.gridDim = grid;
        kp.blockDim = block;
        kp.sharedMemBytes = (unsigned)smem;
        kp.kernelParams = argv;
        kp.extra = nullptr;
        if (cudaGraphExecKernelNodeSetParams(G->exec, G->nodes[i], &kp) != cudaSuccess) {
            ctx->gfail = true;
            return;
        }
        G->args[i] = std::move(packed);
    }
}

void drop_graph(FrameGraph& G) {
    if (G.exec) cudaGraphExecDestroy(G.exec);
    if (G.graph) cudaGraphDestroy(G.graph);
    G = FrameGraph();
}

__global__ void k_selfcheck(int* out) {
    // the x86 truncation rules the strict kernels rely on
    float vals[6] = {-2.5f, 2.5f, 2147483648.0f, -2147483904.0f, __int_as_float(0x7fc00000), -0.0f};
    int want[6] = {-2, 2, INT32_MIN, INT32_MIN, INT32_MIN, 0};
    int ok = 1;
    for (int i = 0; i < 6; i++) ok &= cvtt32(vals[i]) == want[i];
    ok &= sat_u8(300.0f) == 255 && sat_u8(-3.0f) == 0 && sat_u8(__int_as_float(0x7fc00000)) == 255;
    ok &= qround(254.5f) == 255;
    out[0] = ok;
}

int upload_image(tw_ctx* ctx, DevBuf& b, const tw_image* im) {
    size_t bytes = (size_t)im->width * im->height * 4 * sample_bytes(im->fmt);
    CHECK(ctx->ensure(b, bytes, "image upload"));
    return ctx->cuda(cudaMemcpyAsync(b.p, im->data, bytes, cudaMemcpyHostToDevice, ctx->stream), "image upload");
}

int finish(tw_ctx* ctx, int* flags_host, int n) {
    cudaError_t e = cudaMemcpyAsync(flags_host, (int*)ctx->flags.p + FL_NAN, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    return ctx->cuda(e, "kernel execution");
}

bool same_shape(const tw_image* a, const tw_image* b) {
    return a->width == b->width && a->height == b->height && a->fmt == b->fmt;
}

int check_image(tw_ctx* ctx, const tw_image* im, const char* what) {
    if (!im || !im->data) return ctx->fail(TW_ERR_MISMATCH, "%s: no image", what);
    if (im->fmt < 0 || im->fmt > 2) return ctx->fail(TW_ERR_BAD_PARAM, "%s: format %d is not 0..2", what, im->fmt);
    if (im->width <= 0 || im->height <= 0) return ctx->fail(TW_ERR_MISMATCH, "%s: empty image", what);
    size_t need = image_bytes(im->width, im->height, im->fmt);
    if (im->bytes < need)
        return ctx->fail(TW_ERR_BAD_PARAM, "%s: the buffer holds %zu bytes, a %dx%d image needs %zu", what, im->bytes,
                         im->width, im->height, need);
    return TW_OK;
}

// An output image: the checks of an input image on the caller's writable buffer.
int check_out(tw_ctx* ctx, const tw_image_mut* im, const char* what) {
    if (!im) return ctx->fail(TW_ERR_BAD_PARAM, "%s: no output image", what);
    tw_image c{im->width, im->height, im->fmt, im->data, im->bytes};
    return check_image(ctx, &c, what);
}


// The refusal a composition's bad flag carries: bit 2 the motion blur, else the inverse warp.
int bad_fail(tw_ctx* ctx, int v) {
    if (v & 2)
        return ctx->fail(TW_ERR_UNSUPPORTED, "motion blur: a tap coordinate is NaN or a vector needs more than 65536 taps, "
                                             "which is not supported");
    return ctx->fail(TW_ERR_UNSUPPORTED, "inverse warp: a sample coordinate is NaN or never converges, which is not supported");
}

// Creates the lane's streams and events once; every call then points the lane's working streams at
// its own pair, or in serial mode at the context's stream (every kernel in issue order, so that each
// launch's events time that kernel alone).
int lane_ready(tw_ctx* ctx, Lane& L) {
    if (!L.own[0]) {
        for (int i = 0; i < 2; i++) {
            CHECK(ctx->cuda(cudaStreamCreateWithFlags(&L.own[i], cudaStreamNonBlocking), "lane stream"));
            CHECK(ctx->cuda(cudaEventCreateWithFlags(&L.ev_pyr[i], cudaEventDisableTiming), "lane event"));
        }
        CHECK(ctx->cuda(cudaEventCreateWithFlags(&L.ev_solve1, cudaEventDisableTiming), "lane event"));
        CHECK(ctx->cuda(cudaEventCreateWithFlags(&L.ev_done, cudaEventDisableTiming), "lane event"));
        CHECK(ctx->cuda(cudaEventCreateWithFlags(&L.ev_fork, cudaEventDisableTiming), "lane event"));
        CHECK(ctx->ensure(L.flags, FLAGS_BYTES, "lane flags"));
    }
    for (int i = 0; i < 2; i++) L.s[i] = ctx->serial ? ctx->stream : L.own[i];
    return TW_OK;
}

// Orders the first `nl` lanes' streams after the caller's work on ctx->stream (flags cleared first).
int lanes_begin(tw_ctx* ctx, int nl) {
    for (int i = 0; i < nl; i++) {
        Lane& L = ctx->lanes[i];
        CHECK(lane_ready(ctx, L));
        CHECK(ctx->cuda(cudaMemsetAsync(L.flags.p, 0, FLAGS_BYTES, ctx->stream), "flags"));
    }
    CHECK(ctx->cuda(cudaEventRecord(ctx->ev_start, ctx->stream), "event"));
    for (int i = 0; i < nl; i++)
        for (int k = 0; k < 2; k++) CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->lanes[i].s[k], ctx->ev_start, 0), "event"));
    return TW_OK;
}

// The caller's stream waits for the lanes; then their flags are checked (this synchronises).
int lanes_end(tw_ctx* ctx, int nl) {
    for (int i = 0; i < nl; i++) {
        Lane& L = ctx->lanes[i];
        if (!L.used) continue;
        CHECK(ctx->cuda(cudaEventRecord(L.ev_solve1, L.s[1]), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->stream, L.ev_solve1, 0), "event"));
        CHECK(ctx->cuda(cudaStreamWaitEvent(ctx->stream, L.ev_done, 0), "event"));
    }
    ctx->cur = ctx->stream;
    int hf[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < nl; i++) {
        Lane& L = ctx->lanes[i];
        if (!L.used) continue;
        int f[8];
        CHECK(ctx->cuda(cudaMemcpyAsync(f, (int*)L.flags.p + FL_NAN, sizeof f, cudaMemcpyDeviceToHost, ctx->stream), "flags"));
        CHECK(ctx->cuda(cudaStreamSynchronize(ctx->stream), "kernel execution"));
        for (int k = 0; k < 8; k++) hf[k] |= f[k];
        L.used = false;
    }
    CHECK(ctx->cuda(cudaGetLastError(), "kernel execution"));
    if (hf[0]) return ctx->fail(TW_ERR_NAN_OUTPUT, "a solved flow holds a NaN");
    if (hf[1]) return bad_fail(ctx, hf[1]);
    if (hf[3]) return ctx->fail(TW_ERR_UNSUPPORTED, "hole fill of an image with a side of 1 pixel that has a hole");
    if (hf[FL_BOUND - FL_NAN]) return ctx->fail(TW_ERR_DEVICE_BOUND, "a device loop reached its bound");
    return TW_OK;
}

}  // namespace tw

extern "C" {

int tw_open(int device, tw_ctx** out) {
    if (!out) return TW_ERR_BAD_PARAM;
    *out = nullptr;
    tw_ctx* ctx = new tw_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete ctx; return TW_ERR_CUDA; }
    e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete ctx; return TW_ERR_CUDA; }
    ctx->stream = ctx->own;
    ctx->cur = ctx->stream;
    if (cudaEventCreateWithFlags(&ctx->ev_start, cudaEventDisableTiming) != cudaSuccess) { tw_close(ctx); return TW_ERR_CUDA; }
    ctx->g7 = gaussian_taps(7.0f);
    ctx->g5 = gaussian_taps(5.0f);
    ctx->g2 = gaussian_taps(2.0f);
    ctx->b5 = binomial5();
    // block matching keeps one line of the field in shared memory (up to BM_MAX_LINE elements)
    e = cudaFuncSetAttribute(k_bm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bm_smem_bytes(BM_MAX_LINE));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_bm_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bm_smem_bytes(BM_MAX_LINE));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_level_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)level_init_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_level_iter_32x32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)level_iter_smem(LEVEL_TILE_32x32));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_level_iter_64x32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)level_iter_smem(LEVEL_TILE_64x32));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_level_iter_64x64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)level_iter_smem(LEVEL_TILE_64x64));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_solve_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_smem_bytes());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fill_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(FILL_COARSE_MAX_FLOATS * sizeof(float)));
    // the fast mode's builds of the same kernels
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fast::k_bm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bm_smem_bytes(BM_MAX_LINE));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fast::k_bm_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bm_smem_bytes(BM_MAX_LINE));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fast::k_level_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)level_init_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fast::k_level_iter_32x32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)level_iter_smem(LEVEL_TILE_32x32));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fast::k_level_iter_64x32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)level_iter_smem(LEVEL_TILE_64x32));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fast::k_level_iter_64x64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)level_iter_smem(LEVEL_TILE_64x64));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fast::k_solve_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_smem_bytes());
    if (e != cudaSuccess) { tw_close(ctx); return TW_ERR_CUDA; }
    if (ctx->ensure(ctx->flags, FLAGS_BYTES, "flags") != TW_OK) { tw_close(ctx); return TW_ERR_CUDA; }
    k_selfcheck<<<1, 1, 0, ctx->stream>>>(ctx->flags.as<int>());
    ctx->launches++;
    int ok = 0;
    e = cudaMemcpyAsync(&ok, ctx->flags.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess || ok != 1) { tw_close(ctx); return e != cudaSuccess ? TW_ERR_CUDA : TW_ERR_UNSUPPORTED; }
    *out = ctx;
    return TW_OK;
}

void tw_close(tw_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (auto* b : {&ctx->flags, &ctx->host_stage, &ctx->holes, &ctx->fill, &ctx->masks, &ctx->lay_mem, &ctx->lay_in, &ctx->fc_img[0], &ctx->fc_img[1], &ctx->fc_cov[0], &ctx->fc_cov[1], &ctx->wb_wt[0], &ctx->wb_wt[1],
                    &ctx->wb_tmp[0], &ctx->wb_tmp[1], &ctx->wb_mask[0], &ctx->wb_mask[1], &ctx->wb_cov[0], &ctx->wb_cov[1], &ctx->pre_blur, &ctx->comp_e, &ctx->logf_tab, &ctx->fw_vx, &ctx->fw_vy,
                    &ctx->fw_vd, &ctx->fw_pyr, &ctx->fw_tmp[0], &ctx->fw_tmp[1], &ctx->fw_cnt, &ctx->fw_off,
                    &ctx->fw_fill, &ctx->fw_sums, &ctx->fw_keys, &ctx->fw_cols, &ctx->fw_scratch, &ctx->fw_longq,
                    &ctx->fw_flags, &ctx->fw_cov})
        b->release(&ctx->held);
    for (int i = 0; i < 3; i++) { ctx->eng[i].release(&ctx->held); ctx->wire[i].release(&ctx->held); }
    for (int i = 0; i < 2; i++) { ctx->pyr[i].release(&ctx->held); ctx->work[i].release(&ctx->held); ctx->flow[i].release(&ctx->held); }
    for (int i = 0; i < 4; i++) ctx->plane[i].release(&ctx->held);
    for (int i = 0; i < 3; i++) ctx->vi_clip[i].release(&ctx->held);
    for (int i = 0; i < 5; i++) ctx->vi_wire[i].release(&ctx->held);
    ctx->vi_out.release(&ctx->held);
    for (auto& L : ctx->lanes) {
        for (auto& kv : L.graphs) drop_graph(kv.second);
        if (L.ev_fork) cudaEventDestroy(L.ev_fork);
        for (int i = 0; i < 2; i++) {
            L.eng[i].release(&ctx->held); L.pyr[i].release(&ctx->held); L.work[i].release(&ctx->held);
            L.flow[i].release(&ctx->held);
            for (int j = 0; j < 3; j++) L.scratch[i][j].release(&ctx->held);
            if (i == 0) { L.comp.release(&ctx->held); L.holes.release(&ctx->held); L.fill.release(&ctx->held); }
            for (DevBuf* b : {&L.wb_wt[i], &L.wb_tmp[i], &L.wb_mask[i], &L.wb_cov[i]}) b->release(&ctx->held);
            if (i == 0) { L.pre_blur.release(&ctx->held); L.user.release(&ctx->held); }
            if (L.own[i]) cudaStreamDestroy(L.own[i]);
            if (L.ev_pyr[i]) cudaEventDestroy(L.ev_pyr[i]);
        }
        L.flags.release(&ctx->held);
        if (L.ev_solve1) cudaEventDestroy(L.ev_solve1);
        if (L.ev_done) cudaEventDestroy(L.ev_done);
    }
    if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
    for (int i = 0; i < tw_ctx::CACHE_SLOTS; i++) {
        ctx->cache[i].release(&ctx->held);
        if (ctx->cache_ready[i]) cudaEventDestroy(ctx->cache_ready[i]);
        for (int j = 0; j < MAX_LANES; j++)
            if (ctx->cache_free[i][j]) cudaEventDestroy(ctx->cache_free[i][j]);
    }
    for (int i = 0; i < MAX_LANES; i++) {
        ctx->outbuf[i].release(&ctx->held);
        if (ctx->out_free[i]) cudaEventDestroy(ctx->out_free[i]);
    }
    for (int i = 0; i < 2; i++) {
        for (auto& b : ctx->lay_stage[i]) b.release(&ctx->held);
        if (ctx->lay_up[i]) cudaEventDestroy(ctx->lay_up[i]);
        if (ctx->lay_free[i]) cudaEventDestroy(ctx->lay_free[i]);
    }
    if (ctx->up) cudaStreamDestroy(ctx->up);
    if (ctx->down) cudaStreamDestroy(ctx->down);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    for (auto e : ctx->ev_pool) cudaEventDestroy(e);
    delete ctx;
}

size_t tw_last_error(const tw_ctx* ctx, char* buf, size_t cap) {
    if (!ctx) return 0;
    size_t n = ctx->err.size();
    if (buf && cap) {
        size_t m = std::min(n, cap - 1);
        std::memcpy(buf, ctx->err.data(), m);
        buf[m] = 0;
    }
    return n;
}

int tw_stats(const tw_ctx* ctx, uint64_t* kernel_launches, uint64_t* device_bytes) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    if (kernel_launches) *kernel_launches = ctx->launches;
    if (device_bytes) *device_bytes = ctx->held;
    return TW_OK;
}

int tw_profile_begin(tw_ctx* ctx, const char* kernel) {
    if (!ctx || !kernel) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    ctx->prof = KernelProfile();
    ctx->prof.on = true;
    ctx->prof.name = kernel;
    while (ctx->ev_pool.size() < 8192) {  // enough for a timed region of a few thousand launches
        cudaEvent_t e;
        CHECK(ctx->cuda(cudaEventCreate(&e), "profile events"));
        ctx->ev_pool.push_back(e);
    }
    return TW_OK;
}

int tw_profile_end(tw_ctx* ctx, double* total_ms, uint64_t* launches, double* bytes) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(ctx->cuda(cudaStreamSynchronize(ctx->stream), "profile sync"));
    double ms = 0.0;
    for (size_t i = 0; i + 1 < ctx->prof.ev.size(); i += 2) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, ctx->prof.ev[i], ctx->prof.ev[i + 1]);
        ms += t;
    }
    if (total_ms) *total_ms = ms;
    if (launches) *launches = ctx->prof.launches;
    if (bytes) *bytes = ctx->prof.bytes;
    ctx->prof = KernelProfile();
    return TW_OK;
}

size_t tw_profile_report(tw_ctx* ctx, char* buf, size_t cap) {
    if (!ctx) return 0;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return 0;
    struct Row { double ms = 0.0, bytes = 0.0; uint64_t n = 0; };
    std::vector<std::pair<std::string, Row>> rows;
    double total = 0.0;
    for (size_t i = 0; i + 1 < ctx->prof.ev.size(); i += 2) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, ctx->prof.ev[i], ctx->prof.ev[i + 1]);
        const std::string& k = ctx->prof.who[i / 2];
        auto it = std::find_if(rows.begin(), rows.end(), [&](const std::pair<std::string, Row>& r) { return r.first == k; });
        if (it == rows.end()) { rows.push_back({k, Row()}); it = rows.end() - 1; }
        it->second.ms += t;
        it->second.bytes += ctx->prof.nbytes[i / 2];
        it->second.n++;
        total += t;
    }
    std::sort(rows.begin(), rows.end(), [](const auto& a, const auto& b) { return a.second.ms > b.second.ms; });
    std::string out;
    char line[256];
    snprintf(line, sizeof line, "%-20s %8s %10s %8s %7s %10s\n", "kernel", "launches", "ms", "us/launch", "share", "alg GB/s");
    out += line;
    for (auto& r : rows) {
        snprintf(line, sizeof line, "%-20s %8llu %10.3f %8.2f %6.1f%% %10.1f\n", r.first.c_str(),
                 (unsigned long long)r.second.n, r.second.ms, 1e3 * r.second.ms / std::max<uint64_t>(r.second.n, 1),
                 100.0 * r.second.ms / std::max(total, 1e-9), r.second.ms > 0 ? r.second.bytes / (r.second.ms * 1e6) : 0.0);
        out += line;
    }
    if (buf && cap) {
        size_t m = std::min(out.size(), cap - 1);
        std::memcpy(buf, out.data(), m);
        buf[m] = 0;
    }
    return out.size();
}

int tw_set_lanes(tw_ctx* ctx, int32_t lanes) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (lanes < 0 || lanes > MAX_LANES) return ctx->fail(TW_ERR_BAD_PARAM, "lanes %d is not in 0..%d", lanes, MAX_LANES);
    ctx->serial = lanes == 0;
    ctx->nlanes = lanes == 0 ? 1 : lanes;
    return TW_OK;
}

int tw_debug_inject(tw_ctx* ctx, int32_t kind, int32_t n) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (kind < TW_INJECT_NONE || kind > TW_INJECT_STATUS || (kind != TW_INJECT_NONE && n < 1))
        return ctx->fail(TW_ERR_BAD_PARAM, "failure injection: kind %d with count %d", kind, n);
    ctx->inject_kind = kind;
    ctx->inject_n = kind == TW_INJECT_NONE ? 0 : n;
    return TW_OK;
}

int tw_set_graphs(tw_ctx* ctx, int32_t on) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->graphs_on = on != 0;
    if (!ctx->graphs_on)
        for (auto& L : ctx->lanes)
            for (auto& kv : L.graphs) drop_graph(kv.second);
    return TW_OK;
}

int tw_set_stream(tw_ctx* ctx, void* stream) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    ctx->stream = (cudaStream_t)stream;
    ctx->cur = ctx->stream;
    ctx->own_stream = false;
    return TW_OK;
}

}  // extern "C"
