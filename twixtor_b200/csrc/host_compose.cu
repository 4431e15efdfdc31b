// compose_vectors and its stages: inverse and forward warps, blends, Smart Blend, Weighted Blend,
// Blur Compensation and the pull-push hole fill (compose/vector.rs:117-284), with their entry points.
#include "runtime.h"

namespace tw {

// blend.rs:55-78: which branch blend(out, a, b, w) takes
int blend_mode(float w) {
    if (0.005 > (double)std::fabs(w)) return 1;
    if (0.005 > std::fabs((double)w - 1.0)) return 2;
    if (w < 0.0f || w > 1.0f) return 3;
    return 0;
}

// warp.rs:751-764: the |amount| early outs of inv_warp (a plain copy)
bool warp_copy_only(float amount, int fw, int width) {
    float a = amount < 0.0f ? -amount : amount;
    if (0.005 > (double)a) return true;
    float r = (float)(fw - 1) / (float)(width - 1);
    float q = (float)((double)amount / (double)r);
    if (q < 0.0f) q = -q;
    return 0.0001 > (double)q;
}

WarpParams warp_params(const void* src, const float* flow_interleaved, int fw, int fh, float amount, int width, int height,
                       bool hold) {
    WarpParams p{};
    p.src = src;
    p.fu = flow_interleaved;
    p.fv = flow_interleaved ? flow_interleaved + 1 : nullptr;
    p.fstride = 2;
    p.fw = fw;
    p.fh = fh;
    p.amount = amount;
    if (flow_interleaved) {
        p.rx = (float)(fw - 1) / (float)(width - 1);
        p.ry = (float)(fh - 1) / (float)(height - 1);
        p.sx = amount / p.rx;
        p.sy = amount / p.ry;
    }
    p.hold = hold;
    p.copy_only = flow_interleaved ? warp_copy_only(amount, fw, width) : true;
    return p;
}

// ---- the hole fill (holefill.rs) ------------------------------------------------------------------------
struct FillGeo {
    int dims[40][2];
    int top = 0;
};

FillGeo fill_geometry(int w, int h) {  // holefill.rs:140-171
    FillGeo g;
    long a = w, b = h;
    int count = 1;
    for (;;) {
        a /= 2;
        b /= 2;
        if (a < 2) a = 2;
        if (b < 2) b = 2;
        count += 1;
        if (!(a > 1 && b > 1 && (a != 2 || b != 2))) break;
    }
    int cw = w, ch = h;
    for (int k = 0; k <= count && k < 40; k++) {
        g.dims[k][0] = cw;
        g.dims[k][1] = ch;
        cw = std::max(cw / 2, 2);
        ch = std::max(ch / 2, 2);
    }
    g.top = count - 1;
    return g;
}

// one blur of a stack of planes, out of place (src stays as it is): both passes in one tiled launch
void fill_blur(tw_ctx* ctx, const float* src, float* dst, int w, int h, long stride, int planes, const Taps& t, int n,
               bool above_first, int rule, const int* any) {
    dim3 g((unsigned)((w + 31) / 32), (unsigned)((h + 31) / 32), (unsigned)planes);
    double pb = 8.0 * w * h * planes;  // every plane read once and written once
    LAUNCHB(ctx, pb, k_stack_blur, g, 256, 0, src, dst, w, h, stride, t, n, above_first ? 1 : 0, rule, any);
}

void fill_resample(tw_ctx* ctx, const float* src, int sw, int sh, float* dst, int dw, int dh, int planes, int rule,
                   const int* any) {
    dim3 g((unsigned)((dw + TB - 1) / TB), (unsigned)dh, (unsigned)planes);
    LAUNCHB(ctx, 4.0 * planes * ((double)sw * sh + (double)dw * dh), k_stack_resample, g, TB, 0, src, sw, sh, (long)sw * sh, dst,
            dw, dh, (long)dw * dh, rule, any);
}

// The pull-push fill of an engine image in place (holefill.rs:260-350, :452-491) with the u8
// holes mask; every kernel returns at once when *any (no hole) is 0. Per level a stack of the
// channels' value planes and the weights: five planes for an engine image, three for an
// interleaved flow (fmt FILL_FLOW, holefill.rs:497-518). Float images and flows run the NaN rule
// arithmetic (for numbers the plain arithmetic bit for bit, and where a NaN reaches the result the
// bits of the reference's repeat with the rule).
int fill_dev(tw_ctx* ctx, void* img, int W, int H, int fmt, const uint8_t* holes, const int* any, bool above_first,
             DevBuf& fb) {
    int rule = fmt == TW_F32 || fmt == FILL_FLOW;
    int nc = fmt == FILL_FLOW ? 2 : 4;  // value planes; the weights are plane nc
    int np = nc + 1;
    FillGeo g = fill_geometry(W, H);
    long n0 = (long)W * H;
    size_t offs[40];
    size_t tot = 0;
    for (int k = 0; k <= g.top; k++) { offs[k] = tot; tot += np * (size_t)g.dims[k][0] * g.dims[k][1]; }
    size_t o_ta = tot, o_sa = tot + np * n0, o_sb = o_sa + nc * n0;
    tot = o_sb + nc * n0;
    CHECK(ctx->ensure(fb, tot * sizeof(float), "hole fill planes"));
    float* base = fb.as<float>();
    float* ta = base + o_ta;
    LAUNCH(ctx, k_fill_load, grid1(n0), TB, 0, img, fmt, holes, base + offs[0], n0, any);
    // the coarse levels k0 .. top (every stack of them fits one block's shared memory) run in one
    // launch, k_fill_coarse: the finest such level k0 >= 1 is built by the pull below, the launch
    // pulls on from it, pushes down to it and leaves the push's level k0 - 1 in the solution planes
    int k0 = g.top + 1;
    for (int k = 1; k <= g.top; k++)
        if (fill_coarse_floats(g.dims, k, g.top, np, nc) <= FILL_COARSE_MAX_FLOATS) { k0 = k; break; }
    const int pull_to = k0 <= g.top ? k0 : g.top;
    for (int k = 1; k <= pull_to; k++) {  // pull: blur5 and the resample of the values and the weights
        int pw = g.dims[k - 1][0], ph = g.dims[k - 1][1], cw = g.dims[k][0], chh = g.dims[k][1];
        long pn = (long)pw * ph;
        // the level k - 1 planes stay for the push: the blur writes ta
        fill_blur(ctx, base + offs[k - 1], ta, pw, ph, pn, np, ctx->b5, 3, above_first, rule, any);
        fill_resample(ctx, ta, pw, ph, base + offs[k], cw, chh, np, rule, any);
    }
    float* sol = base + o_sa;
    float* nxt = base + o_sb;
    int push_from = g.top;
    if (k0 <= g.top) {
        FillCoarseJob J{};
        J.s_k0 = base + offs[k0];
        J.out = sol;
        for (int k = 0; k <= g.top; k++) {
            J.dims[k][0] = g.dims[k][0];
            J.dims[k][1] = g.dims[k][1];
        }
        J.k0 = k0;
        J.top = g.top;
        J.np = np;
        J.nc = nc;
        J.rule = rule;
        J.above_first = above_first;
        J.b5 = ctx->b5;
        J.g5 = ctx->g5;
        J.any = any;
        // the stack of level k0 read, the push's level k0 - 1 written
        double b = 4.0 * ((double)np * g.dims[k0][0] * g.dims[k0][1] + (double)nc * g.dims[k0 - 1][0] * g.dims[k0 - 1][1]);
        LAUNCHB(ctx, b, k_fill_coarse, 1, FILL_COARSE_THREADS, fill_coarse_floats(g.dims, k0, g.top, np, nc) * sizeof(float), J);
        push_from = k0 - 1;
    } else {
        long tn = (long)g.dims[g.top][0] * g.dims[g.top][1];
        LAUNCH(ctx, k_stack_zero, grid1(nc * tn), TB, 0, sol, nc * tn, any);
    }
    for (int lv = push_from; lv >= 0; lv--) {  // push
        int lw = g.dims[lv][0], lh = g.dims[lv][1];
        long ln = (long)lw * lh;
        LAUNCH(ctx, k_fill_combine, grid1(ln), TB, 0, sol, base + offs[lv], ln, nc, rule, any);
        fill_blur(ctx, sol, ta, lw, lh, ln, nc, ctx->g5, 6, above_first, rule, any);  // the blurred solution in ta
        if (lv == 0) {
            LAUNCH(ctx, k_fill_combine, grid1(ln), TB, 0, ta, base + offs[0], ln, nc, rule, any);
            sol = ta;
        } else {
            fill_resample(ctx, ta, lw, lh, nxt, g.dims[lv - 1][0], g.dims[lv - 1][1], nc, rule, any);
            std::swap(sol, nxt);
        }
    }
    LAUNCH(ctx, k_fill_store, grid1(n0), TB, 0, img, fmt, sol, n0, any);
    return TW_OK;
}

// ---- the forward warp (forward.rs:229-373) -----------------------------------------------------------

// The glibc logf exception table embedded by the build (csrc/logf_table.S), uploaded once.
int logf_table(tw_ctx* ctx, const uint2** tab, int* n) {
    size_t bytes = (size_t)((const char*)tw_logf_table_end - (const char*)tw_logf_table);
    *n = (int)(bytes / sizeof(uint2));
    if (!ctx->logf_tab.p) {
        CHECK(ctx->ensure(ctx->logf_tab, bytes, "logf table"));
        CHECK(ctx->cuda(cudaMemcpy(ctx->logf_tab.p, tw_logf_table, bytes, cudaMemcpyHostToDevice), "logf table upload"));
    }
    *tab = ctx->logf_tab.as<uint2>();
    return TW_OK;
}

int fw_level_count(int w, int h) {  // forward/pyramid.rs:20-36
    int n = 1, a = std::max(w, 2), b = std::max(h, 2);
    for (;;) {
        a /= 2;
        if (a < 2) break;
        b /= 2;
        if (b < 2) break;
        n++;
    }
    return n;
}

// fw_flags ints: [0] outside, [1] bad texture coordinate, [2] flow not zero, [3] long lists,
// [4] longest list, [6..7] the total number of hits (64 bit)
enum { FW_OUTSIDE = 0, FW_BAD = 1, FW_NONZERO = 2, FW_NLONG = 3, FW_MAXC = 4, FW_TOTAL = 6 };

// forward.rs:229-320 on device buffers, on ctx->cur: src (engine image) pushed by flow (fw x fh,
// interleaved) times amount into out (engine image, not src) and the coverage bytes into cov
// (nullptr: none). Textured (pyramid) or the Gouraud variant. The zero-flow early out and the hit
// total are read back, so the call synchronises ctx->cur.
int forward_warp_dev(tw_ctx* ctx, const void* src, const float* flow, int fw, int fh, int W, int H, int fmt,
                     float amount, bool pyramid, void* out, uint8_t* cov) {
    if (W < 2 || H < 2 || fw < 2 || fh < 2)
        return ctx->fail(TW_ERR_MISMATCH, "forward warp needs images and a flow of at least 2x2 (image %dx%d, flow %dx%d)", W, H,
                         fw, fh);
    long n = (long)W * H;
    size_t px = 4 * sample_bytes(fmt);
    CHECK(ctx->ensure(ctx->fw_flags, 64, "forward warp flags"));
    CHECK(ctx->ensure(ctx->fw_cov, (size_t)n, "coverage"));
    if (!cov) cov = ctx->fw_cov.as<uint8_t>();
    int* ff = ctx->fw_flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(ff, 0, 64, ctx->cur), "flags"));
    // early outs (forward.rs:252-257): |amount| below 1e-5 as a double, or a flow of zeros
    float a = 0.0f > amount ? -amount : amount;
    bool early = 1e-05 > (double)a;
    long nf = (long)fw * fh * 2;
    if (!early) {
        LAUNCH(ctx, k_fw_flow_nonzero, grid1(nf), TB, 0, flow, nf, ff + FW_NONZERO);
        int nz = 0;
        CHECK(ctx->cuda(cudaMemcpyAsync(&nz, ff + FW_NONZERO, sizeof nz, cudaMemcpyDeviceToHost, ctx->cur), "flags"));
        CHECK(ctx->cuda(cudaStreamSynchronize(ctx->cur), "kernel execution"));
        early = nz == 0;
    }
    if (early) {  // blend::copy and a full coverage
        CHECK(ctx->cuda(cudaMemcpyAsync(out, src, (size_t)n * px, cudaMemcpyDeviceToDevice, ctx->cur), "copy"));
        return ctx->cuda(cudaMemsetAsync(cov, 0xff, (size_t)n, ctx->cur), "coverage");
    }
    // 1. the vertex grid and the mip levels (forward/mesh.rs)
    FwGrid g;
    g.w = W;
    g.h = H;
    g.rx = (float)(fw - 1) / (float)(W - 1);
    g.ry = (float)(fh - 1) / (float)(H - 1);
    g.sx = amount / g.rx;
    g.sy = amount / g.ry;
    int levels = fw_level_count(W, H);
    bool mips = pyramid && levels > 1;
    if (levels > FW_MAX_LEVELS) return ctx->fail(TW_ERR_TOO_LARGE, "forward warp: %d pyramid levels", levels);
    CHECK(ctx->ensure(ctx->fw_vx, n * sizeof(float), "vertices"));
    CHECK(ctx->ensure(ctx->fw_vy, n * sizeof(float), "vertices"));
    if (mips) CHECK(ctx->ensure(ctx->fw_vd, n * sizeof(float), "mip levels"));
    const uint2* tab = nullptr;
    int ntab = 0;
    if (mips) CHECK(logf_table(ctx, &tab, &ntab));
    float inv_ln2 = 1.0f / logf(2.0f);  // mesh.rs:89, the host libm like the reference's
    LAUNCH(ctx, k_fw_vertices, grid1(n), TB, 0, flow, fw, fh, g,
           ctx->fw_vx.as<float>(), ctx->fw_vy.as<float>(), mips ? ctx->fw_vd.as<float>() : (float*)nullptr, inv_ln2, tab,
           ntab);
    // 2. the mip pyramid (forward/pyramid.rs:39-70); level 0 is the source
    FwLevels L{};
    L.p[0] = src;
    L.w[0] = W;
    L.h[0] = H;
    L.count = pyramid ? levels : 1;
    if (pyramid && levels > 1) {
        size_t tot = 0;
        int cw = W, chh = H;
        size_t offs[FW_MAX_LEVELS];
        for (int i = 1; i < levels; i++) {
            cw = std::max(cw / 2, 2);
            chh = std::max(chh / 2, 2);
            offs[i] = tot;
            tot += (size_t)cw * chh * px;
            L.w[i] = cw;
            L.h[i] = chh;
        }
        CHECK(ctx->ensure(ctx->fw_pyr, tot, "mip pyramid"));
        CHECK(ctx->ensure(ctx->fw_tmp[0], (size_t)n * px, "mip blur"));
        CHECK(ctx->ensure(ctx->fw_tmp[1], (size_t)n * px, "mip blur"));
        for (int i = 1; i < levels; i++) {
            L.p[i] = (char*)ctx->fw_pyr.p + offs[i];
            int pw = L.w[i - 1], ph = L.h[i - 1];
            dim3 gb((unsigned)((pw + 127) / 128), (unsigned)ph);
            LAUNCH(ctx, k_fwp_blur, gb, 128, 0, L.p[i - 1], ctx->fw_tmp[0].p, pw, ph, 0, fmt);
            LAUNCH(ctx, k_fwp_blur, gb, 128, 0, ctx->fw_tmp[0].p, ctx->fw_tmp[1].p, pw, ph, 1, fmt);
            dim3 gr((unsigned)((L.w[i] + 127) / 128), (unsigned)L.h[i]);
            LAUNCH(ctx, k_fwp_resample, gr, 128, 0, ctx->fw_tmp[1].p, pw, ph, (void*)L.p[i], L.w[i], L.h[i], fmt);
        }
    }
    // 3. count the hits of every pixel, then their offsets
    CHECK(ctx->ensure(ctx->fw_cnt, n * sizeof(uint32_t), "hit counts"));
    CHECK(ctx->ensure(ctx->fw_off, n * sizeof(uint32_t), "hit offsets"));
    CHECK(ctx->ensure(ctx->fw_fill, n * sizeof(uint32_t), "hit fill"));
    int nb = (int)((n + FW_SCAN_BLOCK - 1) / FW_SCAN_BLOCK);
    CHECK(ctx->ensure(ctx->fw_sums, (size_t)nb * sizeof(uint32_t), "scan sums"));
    CHECK(ctx->ensure(ctx->fw_longq, n * sizeof(uint32_t), "long lists"));
    CHECK(ctx->cuda(cudaMemsetAsync(ctx->fw_cnt.p, 0, n * sizeof(uint32_t), ctx->cur), "counts"));
    CHECK(ctx->cuda(cudaMemsetAsync(ctx->fw_fill.p, 0, n * sizeof(uint32_t), ctx->cur), "fill"));
    FwRaster R{};
    R.w = W;
    R.h = H;
    R.fmt = fmt;
    R.pyramid = pyramid != 0;
    R.vx = ctx->fw_vx.as<float>();
    R.vy = ctx->fw_vy.as<float>();
    R.vd = mips ? ctx->fw_vd.as<float>() : nullptr;
    R.levels = L;
    R.cnt = ctx->fw_cnt.as<uint32_t>();
    R.off = ctx->fw_off.as<uint32_t>();
    R.fill = ctx->fw_fill.as<uint32_t>();
    R.out = out;
    R.cov = cov;
    R.outside = ff + FW_OUTSIDE;
    R.bad = ff + FW_BAD;
    R.nlong = (uint32_t*)(ff + FW_NLONG);
    R.longq = ctx->fw_longq.as<uint32_t>();
    long tris = 2L * (W - 1) * (H - 1);
    unsigned gt = (unsigned)((tris + 127) / 128);
    // algorithmic bytes: the vertices (20 per source pixel) read by the two scan conversions; the hit
    // list (key and colour, 20 per hit) written by the emit and read by the resolve, which writes the
    // output pixel and its coverage
    const double vbytes = 20.0 * W * H;
    LAUNCHB(ctx, vbytes, k_fw_count, gt, 128, 0, R);
    LAUNCH(ctx, k_scan_block, (unsigned)nb, 256, 0, R.cnt, R.off, n, ctx->fw_sums.as<uint32_t>(), (uint32_t*)(ff + FW_MAXC));
    LAUNCH(ctx, k_scan_sums, 1, 1024, 0, ctx->fw_sums.as<uint32_t>(), nb, (unsigned long long*)(ff + FW_TOTAL));
    LAUNCH(ctx, k_scan_add, grid1(n), TB, 0, R.off, n, ctx->fw_sums.as<uint32_t>());
    int hf[8];
    CHECK(ctx->cuda(cudaMemcpyAsync(hf, ff, sizeof hf, cudaMemcpyDeviceToHost, ctx->cur), "flags"));
    CHECK(ctx->cuda(cudaStreamSynchronize(ctx->cur), "kernel execution"));
    if (hf[FW_OUTSIDE])
        return ctx->fail(TW_ERR_UNSUPPORTED, "forward warp: the degenerate last row pass of the rasteriser would write outside "
                                             "the image, which is not supported");
    unsigned long long total;
    std::memcpy(&total, hf + FW_TOTAL, sizeof total);
    uint32_t maxc = (uint32_t)hf[FW_MAXC];
    if (total >= (1ull << 31)) return ctx->fail(TW_ERR_TOO_LARGE, "forward warp: %llu covered pixel hits", total);
    // 4. the hit lists
    size_t nt = total ? (size_t)total : 1;
    CHECK(ctx->ensure(ctx->fw_keys, nt * sizeof(uint32_t), "hit keys"));
    CHECK(ctx->ensure(ctx->fw_cols, nt * sizeof(float4), "hit colours"));
    if (maxc > 4096) CHECK(ctx->ensure(ctx->fw_scratch, 2 * nt * sizeof(uint2), "long list scratch"));
    R.keys = ctx->fw_keys.as<uint32_t>();
    R.cols = ctx->fw_cols.as<float4>();
    R.scratch = maxc > 4096 ? ctx->fw_scratch.as<uint2>() : nullptr;
    R.total = (uint32_t)total;
    if (R.pyramid) LAUNCHB(ctx, vbytes + 20.0 * (double)total, k_fw_emit_tex, gt, 128, 0, R);
    else LAUNCHB(ctx, vbytes + 20.0 * (double)total, k_fw_emit, gt, 128, 0, R);
    // 5. the running mean of every pixel in triangle order, the depth conversion, the coverage
    LAUNCHB(ctx, 20.0 * (double)total + 17.0 * W * H, k_fw_resolve, grid1(n), TB, 0, R);
    LAUNCH(ctx, k_fw_resolve_long, 296, 512, FW_LONG_SMEM_BYTES, R);
    CHECK(ctx->cuda(cudaMemcpyAsync(hf, ff, sizeof hf, cudaMemcpyDeviceToHost, ctx->cur), "flags"));
    CHECK(ctx->cuda(cudaStreamSynchronize(ctx->cur), "kernel execution"));
    CHECK(ctx->cuda(cudaGetLastError(), "kernel execution"));
    if (hf[FW_BAD]) return ctx->fail(TW_ERR_UNSUPPORTED, "forward warp: a texture coordinate outside the image");
    return TW_OK;
}

// warp/blurcomp.rs:42-130 (blur_compensation with is360 off): the amount from the two source
// positions and the slider, clamped; the motion blur of img (engine image) into dst with the post
// step of its sign. Returns TW_OK with *ran false when the compensation does nothing (dst untouched).
int blur_comp_dev(tw_ctx* ctx, const void* img, void* dst, const float* flow, int fw, int fh, float s0, float s1,
                  float blur, bool hiq, int W, int H, int fmt, int* bad, bool* ran) {
    *ran = false;
    float a = std::fabs(s0 - s1);
    if (!((double)a > 1e-6) || !((double)blur > 0.005)) return TW_OK;
    float amount = (a - 1.0f) * blur;
    if (20.0f < amount) amount = 20.0f;
    else if (amount < -10.0f) amount = -10.0f;
    if ((double)std::fabs(amount) < 1e-6) return TW_OK;
    if (W < 2 || H < 2 || fw < 2 || fh < 2)
        return ctx->fail(TW_ERR_MISMATCH, "motion blur needs images and a flow of at least 2x2 (image %dx%d, flow %dx%d)", W, H, fw, fh);
    MotionBlur B{};
    B.src = img;
    B.dst = dst;
    B.flow = warp_params(img, flow, fw, fh, 0.0f, W, H, true);
    B.fmt = fmt;
    B.w = W;
    B.h = H;
    B.rx = (float)(fw - 1) / (float)(W - 1);
    B.ry = (float)(fh - 1) / (float)(H - 1);
    float eff = 0.0f < amount ? amount : 0.5f;  // a negative amount blurs by 0.5 and lerps
    B.kx = (0.5f / B.rx) * eff;
    B.ky = (0.5f / B.ry) * eff;
    B.shifted = false;  // shutter 0.5
    B.k = 0.5f * 2.0f - 1.0f;
    B.bilinear = hiq;
    B.post = 0.0f < amount ? 1 : 2;
    B.lerp_w = amount;
    B.bad = bad;
    LAUNCH(ctx, k_motion_blur, grid1((long)W * H), TB, 0, B);
    *ran = true;
    return TW_OK;
}


WbScratch wb_scratch(DevBuf* wt, DevBuf* tmp, DevBuf* mask, DevBuf* cov) {
    return WbScratch{{&wt[0], &wt[1]}, {&tmp[0], &tmp[1]}, {&mask[0], &mask[1]}, {&cov[0], &cov[1]}};
}

// filters.rs:627-631 (sharpen_weight), in double precision as the reference computes it
float sharpen_weight(float t) {
    double x = 1.0 - std::fabs(0.5 - (double)t) * 2.0;
    float neg = -(float)x;
    return (float)((double)neg * 0.5);
}

// filters.rs:649-657 (sharpen_step_with): frame (an engine image, in place) against the unwarped
// orig, on ctx->cur. gate: see filters.cu (nullptr: always).
int sharpen_dev(tw_ctx* ctx, void* frame, const void* orig, int W, int H, int fmt, float t, bool above_first,
                const WbScratch& ws, const int* gate) {
    long n = (long)W * H;
    size_t ib = (size_t)n * 4 * sample_bytes(fmt);
    for (int i = 0; i < 2; i++) {
        CHECK(ctx->ensure(*ws.tmp[i], ib, "sharpening planes"));
        CHECK(ctx->ensure(*ws.mask[i], (size_t)n, "sharpening mask"));
    }
    uint8_t* cur = ws.mask[0]->as<uint8_t>();
    uint8_t* nxt = ws.mask[1]->as<uint8_t>();
    float white = fmt == TW_U8 ? 255.0f : fmt == TW_U16 ? 65535.0f : 1.0f;
    float limit = 0.4f * white * 0.4f * 0.4f * 3.0f;  // filters.rs:293-295, MASK_THRESHOLD 0.4
    LAUNCH(ctx, k_wb_diff_mask, grid1(n), TB, 0, frame, orig, fmt, n, limit, cur, gate);
    // filters.rs:507-520: prune 254 and 509, dilate, fill 254 -> 255 twice, 254 -> 128, 127 -> 64
    if (W >= 3 && H >= 3) {
        auto step = [&]() { std::swap(cur, nxt); };
        if (H >= 5) {
            LAUNCH(ctx, k_mask_prune, grid1(n), TB, 0, cur, nxt, W, H, 254, gate);
            step();
            LAUNCH(ctx, k_mask_prune, grid1(n), TB, 0, cur, nxt, W, H, 509, gate);
            step();
        }
        LAUNCH(ctx, k_mask_dilate, grid1(n), TB, 0, cur, nxt, W, H, gate);
        step();
        const int fills[4][2] = {{254, 255}, {254, 255}, {254, 128}, {127, 64}};
        for (auto& f : fills) {
            LAUNCH(ctx, k_mask_fill_border, grid1(n), TB, 0, cur, nxt, W, H, f[0], f[1], gate);
            step();
        }
    } else {
        LAUNCH(ctx, k_mask_clean_small, 1, 1, 0, cur, nxt, W, H, gate);
    }
    // the blur (radius 3.0, filters.rs:75-93: taps 1, 1/2, 1/16, 1/512 over their sum, from powf)
    WbTaps T{};
    {
        float sum = 0.0f, wv[4];
        for (int i = 0; i < 4; i++) {
            float fi = (float)i;
            float x = -((fi * fi) / 1.0f);
            wv[i] = powf(2.0f, x);
            sum += wv[i];
        }
        float denom = sum * 2.0f - wv[0];
        for (int i = 0; i < 4; i++) T.w[i] = wv[i] / denom;
        T.count = 4;
    }
    void* t0 = ws.tmp[0]->p;
    void* t1 = ws.tmp[1]->p;
    LAUNCH(ctx, k_wb_blur, grid1(n), TB, 0, frame, t0, fmt, W, H, T, false, false, gate);
    LAUNCH(ctx, k_wb_blur, grid1(n), TB, 0, t0, t1, fmt, W, H, T, true, above_first, gate);
    LAUNCH(ctx, k_wb_finish, grid1(n), TB, 0, frame, t1, cur, fmt, n, sharpen_weight(t), gate);
    return TW_OK;
}

// smartblend.rs:427-456 (weighted_tail) on ctx->cur: ta / tb sharpened against a / b, then with
// coverage (c0 != nullptr) the plain Smart Blend into out, the combined inverted coverage and the
// fill; without coverage the blend. out: an engine image.
int weighted_tail_dev(tw_ctx* ctx, void* out, void* ta, const void* a, void* tb, const void* b, float wa, int W, int H,
                      int fmt, const uint8_t* c0, const uint8_t* c1, bool above_first, const SmartScratch& ss, int* bad) {
    long n = (long)W * H;
    float frac = 1.0f - wa;
    CHECK(sharpen_dev(ctx, ta, a, W, H, fmt, frac, above_first, *ss.wb, nullptr));
    CHECK(sharpen_dev(ctx, tb, b, W, H, fmt, wa, above_first, *ss.wb, nullptr));
    if (!c0) {
        WarpParams pa = warp_params(ta, nullptr, 0, 0, 0.0f, W, H, true);
        WarpParams pb = warp_params(tb, nullptr, 0, 0, 0.0f, W, H, true);
        LAUNCH(ctx, k_compose_blend, grid2(W, H), TB, 0, pa, pb, fmt, frac, blend_mode(frac), out, W, H, false, false, bad);
        return TW_OK;
    }
    LAUNCH(ctx, k_smart_blend, grid1(n), TB, 0, ta, tb, fmt, frac, false, out, n);
    CHECK(ctx->ensure(*ss.holes, (size_t)n, "holes mask"));
    CHECK(ctx->cuda(cudaMemsetAsync(ss.any_hole, 0, sizeof(int), ctx->cur), "holes flag"));
    LAUNCH(ctx, k_cov_holes, grid1(n), TB, 0, c0, c1, ss.holes->as<uint8_t>(), n, ss.any_hole);
    if (W < 2 || H < 2) {
        LAUNCH(ctx, k_hole_side1, 1, 1, 0, ss.any_hole, ss.side1);
        return TW_OK;
    }
    return fill_dev(ctx, out, W, H, fmt, ss.holes->as<uint8_t>(), ss.any_hole, above_first, *ss.fill);
}

// compose/vector.rs:117-147 (compose_forward) with forward.rs:384-496: warping codes 2 (coverage,
// the Smart Blend composite or its binary variant, the combined and inverted coverage, the hole
// fill) and 3 (no coverage, the plain blend), Nearest and Blend, on ctx->cur (the forward warps
// read their counts back). The pushed frame uses its own flow (A by F_AB); cs.gouraud selects the
// Gouraud forward warp (stages::GouraudForward). out: an engine image.
int compose_forward_dev(tw_ctx* ctx, const tw_engine_settings& cs, const tw_selection& sel, const void* eng_a,
                        const void* eng_b, const float* f_ab, const float* f_ba, int fw, int fh, int W, int H, int fmt,
                        void* out, int* bad, const SmartScratch* ss) {
    if (!ss) return ctx->fail(TW_ERR_UNSUPPORTED, "the forward compositions need their scratch");
    bool fill = cs.warp_mode == 2;
    bool pyramid = cs.gouraud == 0;
    float wa = sel.wa, frac = 1.0f - wa;
    long n = (long)W * H;
    size_t ib = (size_t)n * 4 * sample_bytes(fmt);
    for (int i = 0; i < 2; i++) {
        CHECK(ctx->ensure(ctx->fc_img[i], ib, "forward composition"));
        CHECK(ctx->ensure(ctx->fc_cov[i], (size_t)n, "forward coverage"));
    }
    uint8_t* c0 = ctx->fc_cov[0].as<uint8_t>();
    uint8_t* c1 = ctx->fc_cov[1].as<uint8_t>();
    auto finish_fill = [&](const uint8_t* second) -> int {  // smartblend.rs:335-345 / forward.rs:430-432
        CHECK(ctx->ensure(*ss->holes, (size_t)n, "holes mask"));
        CHECK(ctx->cuda(cudaMemsetAsync(ss->any_hole, 0, sizeof(int), ctx->cur), "holes flag"));
        LAUNCH(ctx, k_cov_holes, grid1(n), TB, 0, c0, second, ss->holes->as<uint8_t>(), n, ss->any_hole);
        return fill_dev(ctx, out, W, H, fmt, ss->holes->as<uint8_t>(), ss->any_hole, cs.taps_above_first != 0, *ss->fill);
    };
    if (sel.interp == 0) {
        bool use_ab = (wa < 0.5f && (unsigned)cs.warp_mode < 2) || (0.5f <= wa && (unsigned)cs.warp_mode > 1);
        const float* flow = use_ab ? f_ab : f_ba;
        if (!flow) return ctx->fail(TW_ERR_MISMATCH, "the composition needs the flow %s but it was not computed", use_ab ? "F_AB" : "F_BA");
        bool take_a = !(0.5f > wa);  // a NaN weight takes A
        CHECK(forward_warp_dev(ctx, take_a ? eng_a : eng_b, flow, fw, fh, W, H, fmt, take_a ? 1.0f - wa : wa, pyramid, out,
                               fill ? c0 : nullptr));
        return fill ? finish_fill(nullptr) : TW_OK;
    }
    if (sel.interp == 1) {
        if (!f_ab || !f_ba) return ctx->fail(TW_ERR_MISMATCH, "the composition needs both flows");
        void* ta = ctx->fc_img[0].p;
        void* tb = ctx->fc_img[1].p;
        CHECK(forward_warp_dev(ctx, eng_a, f_ab, fw, fh, W, H, fmt, frac, pyramid, ta, fill ? c0 : nullptr));
        CHECK(forward_warp_dev(ctx, eng_b, f_ba, fw, fh, W, H, fmt, wa, pyramid, tb, fill ? c1 : nullptr));
        if (!fill) {  // blend_tail without coverage: blend(tA, tB, frac)
            WarpParams pa = warp_params(ta, nullptr, 0, 0, 0.0f, W, H, true);
            WarpParams pb = warp_params(tb, nullptr, 0, 0, 0.0f, W, H, true);
            LAUNCH(ctx, k_compose_blend, grid2(W, H), TB, 0, pa, pb, fmt, frac, blend_mode(frac), out, W, H, false, false, bad);
            return TW_OK;
        }
        LAUNCH(ctx, k_smart_blend, grid1(n), TB, 0, ta, tb, fmt, frac, cs.video_360 != 0, out, n);
        return finish_fill(c1);
    }
    if (sel.interp == 2) {  // forward.rs:498-572: the two pushes, then weighted_tail
        if (!ss->wb) return ctx->fail(TW_ERR_UNSUPPORTED, "Weighted Blend needs its scratch");
        if (!f_ab || !f_ba) return ctx->fail(TW_ERR_MISMATCH, "the composition needs both flows");
        void* ta = ctx->fc_img[0].p;
        void* tb = ctx->fc_img[1].p;
        CHECK(forward_warp_dev(ctx, eng_a, f_ab, fw, fh, W, H, fmt, frac, pyramid, ta, fill ? c0 : nullptr));
        CHECK(forward_warp_dev(ctx, eng_b, f_ba, fw, fh, W, H, fmt, wa, pyramid, tb, fill ? c1 : nullptr));
        return weighted_tail_dev(ctx, out, ta, eng_a, tb, eng_b, wa, W, H, fmt, fill ? c0 : nullptr, fill ? c1 : nullptr,
                                 cs.taps_above_first != 0, *ss, bad);
    }
    return ctx->fail(TW_ERR_BAD_PARAM, "interpolation mode %d is not 0 (Nearest), 1 (Blend) or 2 (Weighted Blend)", sel.interp);
}

// compose_vectors (compose/vector.rs:209-284): warping code 0 and the fast path blends
// (compose.rs:218-231) as one fused kernel launch, code 1 as the Smart Blend kernel and the fill,
// codes 2 and 3 through compose_forward_dev (engine output only). eng_a/eng_b/f_ab/f_ba are device
// pointers.
int compose_dev(tw_ctx* ctx, const tw_engine_settings& cs, const tw_selection& sel, const void* eng_a,
                const void* eng_b, const float* f_ab, const float* f_ba, int fw, int fh, int W, int H, int fmt,
                void* out, bool to_wire, bool flip_out, int* bad, const SmartScratch* ss) {
    if (cs.warp_mode < 0 || cs.warp_mode > 3) return ctx->fail(TW_ERR_BAD_PARAM, "warping code %d is not 0 to 3", cs.warp_mode);
    if (cs.wrap_360) return ctx->fail(TW_ERR_UNSUPPORTED, "the 360 inverse warp is not on the device");
    // the Blur Compensation tail (compose/vector.rs:276-281, warp/blurcomp.rs:42-48): when
    // |s0 - s1| > 1e-6 and the slider > 0.005, the composition goes to an engine image first and
    // the motion blur along F_AB (else the single flow) writes the output
    float d = std::fabs(sel.s0 - sel.s1);
    const float* bflow = f_ab ? f_ab : f_ba;
    if ((double)d > 1e-6 && (double)cs.blur > 0.005 && bflow) {
        if (!ss || !ss->blur || (to_wire && !ss->comp))
            return ctx->fail(TW_ERR_UNSUPPORTED, "Blur Compensation needs its scratch");
        size_t ib = (size_t)W * H * 4 * sample_bytes(fmt);
        CHECK(ctx->ensure(*ss->blur, ib, "composite before the blur"));
        tw_engine_settings c2 = cs;
        c2.blur = 0.0f;
        void* pre = ss->blur->p;
        CHECK(compose_dev(ctx, c2, sel, eng_a, eng_b, f_ab, f_ba, fw, fh, W, H, fmt, pre, false, false, bad, ss));
        void* post = out;
        if (to_wire) {
            CHECK(ctx->ensure(*ss->comp, ib, "composite"));
            post = ss->comp->p;
        }
        bool ran = false;
        CHECK(blur_comp_dev(ctx, pre, post, bflow, fw, fh, sel.s0, sel.s1, cs.blur, cs.quality_high != 0, W, H, fmt, bad, &ran));
        const void* res = ran ? post : pre;
        long n = (long)W * H;
        if (to_wire) {
            if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_to_frame_u8, grid1(n), TB, 0, (const uint8_t*)res, (uint8_t*)out, W, H, flip_out);
            else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_to_frame_u16, grid1(n), TB, 0, (const uint16_t*)res, (uint16_t*)out, W, H, flip_out);
            else LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, (const float*)res, (float*)out, W, H, flip_out);
        } else if (!ran) {
            CHECK(ctx->cuda(cudaMemcpyAsync(out, pre, ib, cudaMemcpyDeviceToDevice, ctx->cur), "copy"));
        }
        return TW_OK;
    }
    if (cs.warp_mode >= 2) {
        if (to_wire)
            return ctx->fail(TW_ERR_UNSUPPORTED, "the forward warps compose on the context's stream only (tw_compose_vectors, "
                                                 "tw_retime_layers_clip)");
        return compose_forward_dev(ctx, cs, sel, eng_a, eng_b, f_ab, f_ba, fw, fh, W, H, fmt, out, bad, ss);
    }
    if (W < 2 || H < 2 || fw < 2 || fh < 2)
        return ctx->fail(TW_ERR_MISMATCH, "inverse warp needs images and a flow of at least 2x2 (image %dx%d, flow %dx%d)", W, H, fw, fh);
    float wa = sel.wa;
    float frac = 1.0f - wa;
    WarpParams pa{}, pb{};
    float wb = 0.0f;
    int mode;
    if (cs.warp_mode == 1) {  // Smart Blend (smartblend.rs:350-393): warps without hold, coverage, fill
        if (!ss) return ctx->fail(TW_ERR_UNSUPPORTED, "Smart Blend needs its scratch");
        int smode;
        if (sel.interp == 0) {
            bool use_ab = (wa < 0.5f && 1u < 2) || (0.5f <= wa && 1u > 1);
            const float* flow = use_ab ? f_ab : f_ba;
            if (!flow) return ctx->fail(TW_ERR_MISMATCH, "the composition needs the flow %s but it was not computed", use_ab ? "F_AB" : "F_BA");
            // the A branch unless 0.5 > wa (a NaN weight takes A)
            if (!(0.5f > wa)) pa = warp_params(eng_a, flow, fw, fh, 1.0f - wa, W, H, false);
            else pa = warp_params(eng_b, flow, fw, fh, wa, W, H, false);
            pb = pa;
            smode = 0;
        } else if (sel.interp == 1) {
            if (!f_ab || !f_ba) return ctx->fail(TW_ERR_MISMATCH, "the composition needs both flows");
            pa = warp_params(eng_a, f_ba, fw, fh, frac, W, H, false);
            pb = warp_params(eng_b, f_ab, fw, fh, wa, W, H, false);
            smode = 1;
        } else if (sel.interp == 2) {
            // smartblend.rs:400-420 (weighted_blend_smart): the warps without hold and with coverage,
            // then weighted_tail (sharpening, the plain Smart Blend, the fill)
            if (!ss->wb) return ctx->fail(TW_ERR_UNSUPPORTED, "Weighted Blend needs its scratch");
            if (!f_ab || !f_ba) return ctx->fail(TW_ERR_MISMATCH, "the composition needs both flows");
            const WbScratch& ws = *ss->wb;
            size_t px = (size_t)W * H, ib = px * 4 * sample_bytes(fmt);
            for (int i = 0; i < 2; i++) {
                CHECK(ctx->ensure(*ws.wt[i], ib, "warped frame"));
                CHECK(ctx->ensure(*ws.cov[i], px, "coverage"));
            }
            pa = warp_params(eng_a, f_ba, fw, fh, frac, W, H, false);
            pb = warp_params(eng_b, f_ab, fw, fh, wa, W, H, false);
            LAUNCH(ctx, k_inv_warp, grid2(W, H), TB, 0, pa, fmt, ws.wt[0]->p, ws.cov[0]->as<uint8_t>(), W, H, bad);
            LAUNCH(ctx, k_inv_warp, grid2(W, H), TB, 0, pb, fmt, ws.wt[1]->p, ws.cov[1]->as<uint8_t>(), W, H, bad);
            void* comp = out;
            if (to_wire) {
                CHECK(ctx->ensure(*ss->comp, ib, "composite"));
                comp = ss->comp->p;
            }
            CHECK(weighted_tail_dev(ctx, comp, ws.wt[0]->p, eng_a, ws.wt[1]->p, eng_b, wa, W, H, fmt, ws.cov[0]->as<uint8_t>(),
                                    ws.cov[1]->as<uint8_t>(), cs.taps_above_first != 0, *ss, bad));
            if (to_wire) {
                long n = (long)px;
                if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_to_frame_u8, grid1(n), TB, 0, (const uint8_t*)comp, (uint8_t*)out, W, H, flip_out);
                else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_to_frame_u16, grid1(n), TB, 0, (const uint16_t*)comp, (uint16_t*)out, W, H, flip_out);
                else LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, (const float*)comp, (float*)out, W, H, flip_out);
            }
            return TW_OK;
        } else {
            return ctx->fail(TW_ERR_BAD_PARAM, "interpolation mode %d is not 0 (Nearest), 1 (Blend) or 2 (Weighted Blend)", sel.interp);
        }
        size_t px = (size_t)W * H;
        void* comp = out;
        if (to_wire) {
            CHECK(ctx->ensure(*ss->comp, px * 4 * sample_bytes(fmt), "composite"));
            comp = ss->comp->p;
        }
        CHECK(ctx->ensure(*ss->holes, px, "holes mask"));
        CHECK(ctx->cuda(cudaMemsetAsync(ss->any_hole, 0, sizeof(int), ctx->cur), "holes flag"));
        LAUNCH(ctx, k_compose_smart, grid2(W, H), TB, 0, pa, pb, fmt, smode, frac, cs.video_360 != 0, comp,
               ss->holes->as<uint8_t>(), W, H, ss->any_hole, bad);
        if (W < 2 || H < 2) LAUNCH(ctx, k_hole_side1, 1, 1, 0, ss->any_hole, ss->side1);
        else CHECK(fill_dev(ctx, comp, W, H, fmt, ss->holes->as<uint8_t>(), ss->any_hole, cs.taps_above_first != 0, *ss->fill));
        if (to_wire) {
            long n = (long)px;
            if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_to_frame_u8, grid1(n), TB, 0, (const uint8_t*)comp, (uint8_t*)out, W, H, flip_out);
            else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_to_frame_u16, grid1(n), TB, 0, (const uint16_t*)comp, (uint16_t*)out, W, H, flip_out);
            else LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, (const float*)comp, (float*)out, W, H, flip_out);
        }
        return TW_OK;
    }
    if (sel.interp == 0) {
        bool use_ab = (wa < 0.5f && (unsigned)cs.warp_mode < 2) || (0.5f <= wa && (unsigned)cs.warp_mode > 1);
        const float* flow = use_ab ? f_ab : f_ba;
        if (!flow) return ctx->fail(TW_ERR_MISMATCH, "the composition needs the flow %s but it was not computed", use_ab ? "F_AB" : "F_BA");
        if (0.5f <= wa) pa = warp_params(eng_a, flow, fw, fh, frac, W, H, true);
        else pa = warp_params(eng_b, flow, fw, fh, wa, W, H, true);
        pb = pa;
        mode = 1;
    } else if (sel.interp == 1) {
        if (!f_ab || !f_ba) return ctx->fail(TW_ERR_MISMATCH, "the composition needs both flows");
        pa = warp_params(eng_a, f_ba, fw, fh, frac, W, H, true);
        pb = warp_params(eng_b, f_ab, fw, fh, wa, W, H, true);
        wb = frac;
        mode = blend_mode(frac);
    } else if (sel.interp == 2) {
        // compose/vector.rs:255-272: the two warps with hold, each sharpened against its frame, blend
        if (!ss || !ss->wb) return ctx->fail(TW_ERR_UNSUPPORTED, "Weighted Blend needs its scratch");
        if (!f_ab || !f_ba) return ctx->fail(TW_ERR_MISMATCH, "the composition needs both flows");
        const WbScratch& ws = *ss->wb;
        size_t ib = (size_t)W * H * 4 * sample_bytes(fmt);
        for (int i = 0; i < 2; i++) CHECK(ctx->ensure(*ws.wt[i], ib, "warped frame"));
        WarpParams qa = warp_params(eng_a, f_ba, fw, fh, frac, W, H, true);
        WarpParams qb = warp_params(eng_b, f_ab, fw, fh, wa, W, H, true);
        LAUNCH(ctx, k_inv_warp, grid2(W, H), TB, 0, qa, fmt, ws.wt[0]->p, (uint8_t*)nullptr, W, H, bad);
        LAUNCH(ctx, k_inv_warp, grid2(W, H), TB, 0, qb, fmt, ws.wt[1]->p, (uint8_t*)nullptr, W, H, bad);
        CHECK(sharpen_dev(ctx, ws.wt[0]->p, eng_a, W, H, fmt, frac, cs.taps_above_first != 0, ws, nullptr));
        CHECK(sharpen_dev(ctx, ws.wt[1]->p, eng_b, W, H, fmt, wa, cs.taps_above_first != 0, ws, nullptr));
        pa = warp_params(ws.wt[0]->p, nullptr, 0, 0, 0.0f, W, H, true);
        pb = warp_params(ws.wt[1]->p, nullptr, 0, 0, 0.0f, W, H, true);
        wb = frac;
        mode = blend_mode(frac);
    } else {
        return ctx->fail(TW_ERR_BAD_PARAM, "interpolation mode %d is not 0 (Nearest), 1 (Blend) or 2 (Weighted Blend)", sel.interp);
    }
    // A and B read, the output written, the two flows read (at their own resolution)
    double px = (double)W * H * 4 * sample_bytes(fmt);
    LAUNCHB(ctx, 3.0 * px + 16.0 * fw * fh, k_compose_blend, grid2(W, H), TB, 0, pa, pb, fmt, wb, mode, out, W, H,
            to_wire, flip_out, bad);
    return TW_OK;
}

// compose.rs:218-231 (interpolate): the fast path without flows
int interpolate_dev(tw_ctx* ctx, const tw_selection& sel, const void* eng_a, const void* eng_b, int W, int H, int fmt,
                    void* out, bool to_wire, int* bad, const SmartScratch* ss) {
    WarpParams pa = warp_params(eng_a, nullptr, 0, 0, 0.0f, W, H, true);
    WarpParams pb = warp_params(eng_b, nullptr, 0, 0, 0.0f, W, H, true);
    int mode;
    float wb = 0.0f;
    if (sel.interp == 0) {
        mode = sel.wa >= 0.5f ? 1 : 2;
    } else if (sel.interp == 1) {
        wb = (float)(1.0 - (double)sel.wa);
        mode = blend_mode(wb);
    } else if (sel.interp == 2) {
        // blend.rs:276-296: equals blend(a, b, 1 - wa) for 8 and 16 bpc
        wb = 1.0f - sel.wa;
        mode = blend_mode(wb);
        if (fmt == TW_F32) {
            // float frames: blend(a + 0, b + 0, 1 - wa), unless a sample is NaN or above 1e30 in
            // magnitude; then the full sequence with every filter (weighted_blend_noflow_reference:
            // sharpen_step, the engine's tap order). The device decides: the sharpening kernels are
            // gated by the unsound flag.
            if (!ss || !ss->wb || !ss->wb_gate || (to_wire && !ss->comp))
                return ctx->fail(TW_ERR_UNSUPPORTED, "Weighted Blend without flows needs its scratch");
            const WbScratch& ws = *ss->wb;
            long n = (long)W * H;
            size_t ib = (size_t)n * 16;
            for (int i = 0; i < 2; i++) CHECK(ctx->ensure(*ws.wt[i], ib, "sharpened frame"));
            int* gate = ss->wb_gate;
            CHECK(ctx->cuda(cudaMemsetAsync(gate, 0, sizeof(int), ctx->cur), "flag"));
            LAUNCH(ctx, k_f32_unsound, grid1(4 * n), TB, 0, (const float*)eng_a, 4 * n, gate);
            LAUNCH(ctx, k_f32_unsound, grid1(4 * n), TB, 0, (const float*)eng_b, 4 * n, gate);
            LAUNCH(ctx, k_copy_gated, grid1(n), TB, 0, (const uint4*)eng_a, (uint4*)ws.wt[0]->p, n, gate);
            LAUNCH(ctx, k_copy_gated, grid1(n), TB, 0, (const uint4*)eng_b, (uint4*)ws.wt[1]->p, n, gate);
            CHECK(sharpen_dev(ctx, ws.wt[0]->p, eng_a, W, H, fmt, wb, false, ws, gate));
            CHECK(sharpen_dev(ctx, ws.wt[1]->p, eng_b, W, H, fmt, sel.wa, false, ws, gate));
            void* eo = out;
            if (to_wire) {
                CHECK(ctx->ensure(*ss->comp, ib, "composite"));
                eo = ss->comp->p;
            }
            LAUNCH(ctx, k_wb_noflow_f32, grid1(n), TB, 0, (const float*)eng_a, (const float*)eng_b, ws.wt[0]->as<float>(),
                   ws.wt[1]->as<float>(), gate, wb, (float)(1.0 - (double)wb), mode, (float*)eo, n);
            if (to_wire) LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, (const float*)eo, (float*)out, W, H, false);
            return TW_OK;
        }
    } else {
        return ctx->fail(TW_ERR_BAD_PARAM, "interpolation mode %d is not 0 (Nearest), 1 (Blend) or 2 (Weighted Blend)", sel.interp);
    }
    LAUNCH(ctx, k_compose_blend, grid2(W, H), TB, 0, pa, pb, fmt, wb, mode, out, W, H, to_wire, false, bad);
    return TW_OK;
}

}  // namespace tw

extern "C" {

int tw_compose_vectors(tw_ctx* ctx, const tw_engine_settings* settings, const tw_selection* sel, const tw_image* a,
                       const tw_image* b, const tw_flow* f_ab, const tw_flow* f_ba, tw_image_mut* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!settings || !sel || !out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "compose_vectors output"));
    CHECK(check_image(ctx, a, "compose"));
    CHECK(check_image(ctx, b, "compose"));
    if (!same_shape(a, b) || out->width != a->width || out->height != a->height || out->fmt != a->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "compose: images of different shapes");
    const tw_flow* f = f_ab ? f_ab : f_ba;
    if (!f) return ctx->fail(TW_ERR_MISMATCH, "compose: no flow");
    if (f_ab && f_ba && (f_ab->width != f_ba->width || f_ab->height != f_ba->height))
        return ctx->fail(TW_ERR_MISMATCH, "compose: flows of different sizes");
    int fw = f->width, fh = f->height;
    CHECK(upload_image(ctx, ctx->eng[0], a));
    CHECK(upload_image(ctx, ctx->eng[1], b));
    size_t fb = (size_t)fw * fh * 2 * sizeof(float);
    if (f_ab) {
        CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
        CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[0].p, f_ab->data, fb, cudaMemcpyHostToDevice, ctx->stream), "flow upload"));
    }
    if (f_ba) {
        CHECK(ctx->ensure(ctx->flow[1], fb, "flow"));
        CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[1].p, f_ba->data, fb, cudaMemcpyHostToDevice, ctx->stream), "flow upload"));
    }
    size_t ob = (size_t)a->width * a->height * 4 * sample_bytes(a->fmt);
    CHECK(ctx->ensure(ctx->eng[2], ob, "compose output"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    WbScratch wbs = wb_scratch(ctx->wb_wt, ctx->wb_tmp, ctx->wb_mask, ctx->wb_cov);
    SmartScratch ss{nullptr, &ctx->holes, &ctx->fill, flags + FL_HOLE, flags + FL_SIDE1, &wbs, flags + FL_WB, &ctx->pre_blur};
    CHECK(compose_dev(ctx, *settings, *sel, ctx->eng[0].p, ctx->eng[1].p, f_ab ? ctx->flow[0].as<float>() : nullptr,
                      f_ba ? ctx->flow[1].as<float>() : nullptr, fw, fh, a->width, a->height, a->fmt, ctx->eng[2].p,
                      false, false, flags + FL_BAD, &ss));
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[2].p, ob, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[4];
    CHECK(finish(ctx, hf, 4));
    if (hf[1]) return bad_fail(ctx, hf[1]);
    if (hf[3])
        return ctx->fail(TW_ERR_UNSUPPORTED, "hole fill of a %dx%d image: the pyramid resample divides by zero for a side of 1",
                         a->width, a->height);
    return TW_OK;
}

int tw_inv_warp(tw_ctx* ctx, tw_image_mut* out, const tw_image* src, const tw_flow* flow, float amount, int32_t hold,
                uint8_t* cov) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, src, "inv_warp"));
    if (!out || !out->data || !flow || !flow->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "inv_warp output"));
    if (out->width != src->width || out->height != src->height || out->fmt != src->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "inverse warp: destination and source differ");
    int W = src->width, H = src->height;
    if (W < 2 || H < 2 || flow->width < 2 || flow->height < 2)
        return ctx->fail(TW_ERR_MISMATCH, "inverse warp needs images and a flow of at least 2x2 (image %dx%d, flow %dx%d)", W, H,
                         flow->width, flow->height);
    CHECK(upload_image(ctx, ctx->eng[0], src));
    size_t fb = (size_t)flow->width * flow->height * 2 * sizeof(float);
    CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[0].p, flow->data, fb, cudaMemcpyHostToDevice, ctx->stream), "flow upload"));
    size_t ob = (size_t)W * H * 4 * sample_bytes(src->fmt);
    CHECK(ctx->ensure(ctx->eng[2], ob, "warp output"));
    CHECK(ctx->ensure(ctx->plane[3], (size_t)W * H, "coverage"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    WarpParams p = warp_params(ctx->eng[0].p, ctx->flow[0].as<float>(), flow->width, flow->height, amount, W, H, (hold & 1) != 0);
    p.is360 = (hold & 2) != 0;  // warp.rs:29-50: is360 takes precedence over hold
    uint8_t* dcov = cov ? ctx->plane[3].as<uint8_t>() : nullptr;
    LAUNCH(ctx, k_inv_warp, grid2(W, H), TB, 0, p, src->fmt, ctx->eng[2].p, dcov, W, H, flags + FL_BAD);
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[2].p, ob, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    if (cov) CHECK(ctx->cuda(cudaMemcpyAsync(cov, dcov, (size_t)W * H, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[2];
    CHECK(finish(ctx, hf, 2));
    if (hf[1]) return bad_fail(ctx, hf[1]);
    return TW_OK;
}

int tw_blend(tw_ctx* ctx, tw_image_mut* out, const tw_image* a, const tw_image* b, float w) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, a, "blend"));
    CHECK(check_image(ctx, b, "blend"));
    if (!out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "blend output"));
    if (!same_shape(a, b) || out->width != a->width || out->height != a->height || out->fmt != a->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "image primitives need equal size and format");
    int W = a->width, H = a->height;
    CHECK(upload_image(ctx, ctx->eng[0], a));
    CHECK(upload_image(ctx, ctx->eng[1], b));
    size_t ob = (size_t)W * H * 4 * sample_bytes(a->fmt);
    CHECK(ctx->ensure(ctx->eng[2], ob, "blend output"));
    WarpParams pa = warp_params(ctx->eng[0].p, nullptr, 0, 0, 0.0f, W, H, true);
    WarpParams pb = warp_params(ctx->eng[1].p, nullptr, 0, 0, 0.0f, W, H, true);
    int* flags = ctx->flags.as<int>();
    LAUNCH(ctx, k_compose_blend, grid2(W, H), TB, 0, pa, pb, a->fmt, w, blend_mode(w), ctx->eng[2].p, W, H, false, false,
           flags + FL_BAD);
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[2].p, ob, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

int tw_smart_blend(tw_ctx* ctx, tw_image_mut* out, const tw_image* p1, const tw_image* p2, float w, int32_t binary) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, p1, "smart blend"));
    CHECK(check_image(ctx, p2, "smart blend"));
    if (!out || !out->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "smart_blend output"));
    if (!same_shape(p1, p2) || out->width != p1->width || out->height != p1->height || out->fmt != p1->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "smart blend: images of %dx%d and %dx%d", p1->width, p1->height, p2->width,
                         p2->height);
    long n = (long)p1->width * p1->height;
    CHECK(upload_image(ctx, ctx->eng[0], p1));
    CHECK(upload_image(ctx, ctx->eng[1], p2));
    size_t ob = (size_t)n * 4 * sample_bytes(p1->fmt);
    CHECK(ctx->ensure(ctx->eng[2], ob, "smart blend output"));
    LAUNCH(ctx, k_smart_blend, grid1(n), TB, 0, ctx->eng[0].p, ctx->eng[1].p, p1->fmt, w, binary != 0, ctx->eng[2].p, n);
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[2].p, ob, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

int tw_fill_holes(tw_ctx* ctx, tw_image_mut* img, const void* mask, int32_t mask_kind, int32_t taps_above_first) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!img || !img->data || !mask) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    if (img->fmt < 0 || img->fmt > 2 || img->width <= 0 || img->height <= 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "hole fill: bad image");
    CHECK(check_out(ctx, img, "fill_holes image"));
    if (mask_kind < 1 || mask_kind > 3)
        return ctx->fail(TW_ERR_BAD_PARAM, "hole fill: mask kind %d is not 1 (u8), 2 (u16) or 3 (f32)", mask_kind);
    int W = img->width, H = img->height;
    long n = (long)W * H;
    size_t ib = (size_t)n * 4 * sample_bytes(img->fmt);
    size_t mb = (size_t)n * (mask_kind == 1 ? 1 : mask_kind == 2 ? 2 : 4);
    CHECK(ctx->ensure(ctx->eng[0], ib, "hole fill image"));
    CHECK(ctx->ensure(ctx->eng[1], mb, "hole fill mask"));
    CHECK(ctx->ensure(ctx->holes, (size_t)n, "holes mask"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->eng[0].p, img->data, ib, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->eng[1].p, mask, mb, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    LAUNCH(ctx, k_mask_holes, grid1(n), TB, 0, ctx->eng[1].p, mask_kind, ctx->holes.as<uint8_t>(), n, flags + FL_HOLE);
    if (W < 2 || H < 2) LAUNCH(ctx, k_hole_side1, 1, 1, 0, flags + FL_HOLE, flags + FL_SIDE1);
    else CHECK(fill_dev(ctx, ctx->eng[0].p, W, H, img->fmt, ctx->holes.as<uint8_t>(), flags + FL_HOLE, taps_above_first != 0, ctx->fill));
    CHECK(ctx->cuda(cudaMemcpyAsync(img->data, ctx->eng[0].p, ib, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[4];
    CHECK(finish(ctx, hf, 4));
    if (hf[3])
        return ctx->fail(TW_ERR_UNSUPPORTED, "hole fill of a %dx%d image: the pyramid resample divides by zero for a side of 1",
                         W, H);
    return TW_OK;
}

// ---- the forward warp (forward.rs:229-373) -----------------------------------------------------------

int tw_forward_warp(tw_ctx* ctx, tw_image_mut* out, const tw_image* src, const tw_flow* flow, float amount,
                    int32_t pyramid, uint8_t* cov) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, src, "forward warp"));
    if (!out || !out->data || !flow || !flow->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "forward_warp output"));
    if (out->width != src->width || out->height != src->height || out->fmt != src->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "forward warp: destination %dx%d fmt %d against source %dx%d fmt %d", out->width,
                         out->height, out->fmt, src->width, src->height, src->fmt);
    int W = src->width, H = src->height, fmt = src->fmt;
    long n = (long)W * H;
    size_t ib = (size_t)n * 4 * sample_bytes(fmt);
    long nf = (long)flow->width * flow->height * 2;
    CHECK(upload_image(ctx, ctx->eng[0], src));
    CHECK(ctx->ensure(ctx->flow[0], std::max(nf, 1L) * sizeof(float), "flow"));
    CHECK(ctx->ensure(ctx->eng[1], ib, "forward warp output"));
    CHECK(ctx->ensure(ctx->fw_cov, (size_t)n, "coverage"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[0].p, flow->data, nf * sizeof(float), cudaMemcpyHostToDevice, ctx->stream),
                    "flow upload"));
    CHECK(forward_warp_dev(ctx, ctx->eng[0].p, ctx->flow[0].as<float>(), flow->width, flow->height, W, H, fmt, amount,
                           pyramid != 0, ctx->eng[1].p, ctx->fw_cov.as<uint8_t>()));
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[1].p, ib, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    if (cov) CHECK(ctx->cuda(cudaMemcpyAsync(cov, ctx->fw_cov.p, (size_t)n, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "kernel execution");
}

int tw_motion_blur(tw_ctx* ctx, tw_image_mut* out, const tw_image* src, const tw_flow* flow, float amount,
                   int32_t hiq, float shutter) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, src, "motion blur"));
    if (!out || !out->data || !flow || !flow->data) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    CHECK(check_out(ctx, out, "motion_blur output"));
    if (out->width != src->width || out->height != src->height || out->fmt != src->fmt)
        return ctx->fail(TW_ERR_MISMATCH, "motion blur: destination and source differ in shape");
    int W = src->width, H = src->height, fmt = src->fmt;
    if (W < 2 || H < 2 || flow->width < 2 || flow->height < 2)
        return ctx->fail(TW_ERR_MISMATCH, "motion blur needs images and a flow of at least 2x2 (image %dx%d, flow %dx%d)", W, H,
                         flow->width, flow->height);
    size_t ib = (size_t)W * H * 4 * sample_bytes(fmt), fb = (size_t)flow->width * flow->height * 2 * sizeof(float);
    CHECK(upload_image(ctx, ctx->eng[0], src));
    CHECK(ctx->ensure(ctx->eng[1], ib, "motion blur output"));
    CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->flow[0].p, flow->data, fb, cudaMemcpyHostToDevice, ctx->stream), "flow upload"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    MotionBlur B{};
    B.src = ctx->eng[0].p;
    B.dst = ctx->eng[1].p;
    B.flow = warp_params(ctx->eng[0].p, ctx->flow[0].as<float>(), flow->width, flow->height, 0.0f, W, H, true);
    B.fmt = fmt;
    B.w = W;
    B.h = H;
    B.rx = (float)(flow->width - 1) / (float)(W - 1);
    B.ry = (float)(flow->height - 1) / (float)(H - 1);
    B.kx = (0.5f / B.rx) * amount;
    B.ky = (0.5f / B.ry) * amount;
    B.shifted = shutter != 0.5f;
    B.k = shutter * 2.0f - 1.0f;
    B.bilinear = hiq != 0;
    B.bad = flags + FL_BAD;
    LAUNCH(ctx, k_motion_blur, grid1((long)W * H), TB, 0, B);
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->eng[1].p, ib, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[2];
    CHECK(finish(ctx, hf, 2));
    if (hf[1]) return bad_fail(ctx, hf[1]);
    return TW_OK;
}

int tw_warp_blend_adjoint(tw_ctx* ctx, const float* a, const float* b, const float* f_ab, const float* f_ba,
                          int32_t width, int32_t height, int32_t flow_w, int32_t flow_h, int32_t batch, float wa,
                          const float* target, const float* grad_out, float* out, float* loss, float* da, float* db,
                          float* df_ab, float* df_ba) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!a || !b || !f_ab || !f_ba || batch < 0) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    if (width < 2 || height < 2 || flow_w < 2 || flow_h < 2)
        return ctx->fail(TW_ERR_MISMATCH, "warp + blend needs images and flows of at least 2x2 (image %dx%d, flow %dx%d)",
                         width, height, flow_w, flow_h);
    if (batch > 65535) return ctx->fail(TW_ERR_TOO_LARGE, "warp + blend: a batch of %d", batch);
    if (loss && !target) return ctx->fail(TW_ERR_BAD_PARAM, "warp + blend: a loss needs its target");
    if (batch == 0) return TW_OK;
    AdjParams P{};
    P.a = a;
    P.b = b;
    P.f_ab = f_ab;
    P.f_ba = f_ba;
    P.target = target;
    P.grad_out = grad_out;
    P.out = out;
    P.loss = loss;
    P.da = da;
    P.db = db;
    P.df_ab = df_ab;
    P.df_ba = df_ba;
    P.w = width;
    P.h = height;
    P.fw = flow_w;
    P.fh = flow_h;
    P.rx = (float)(flow_w - 1) / (float)(width - 1);
    P.ry = (float)(flow_h - 1) / (float)(height - 1);
    P.wa = wa;
    P.tiled = P.rx <= 1.0f && P.ry <= 1.0f;
    if (!ctx->adj_smem_set) {
        CHECK(ctx->cuda(cudaFuncSetAttribute(k_warp_blend_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, ADJ_SMEM),
                        "adjoint shared memory"));
        ctx->adj_smem_set = true;
    }
    dim3 grid((unsigned)((width + ADJ_TX - 1) / ADJ_TX), (unsigned)((height + ADJ_TY - 1) / ADJ_TY), (unsigned)batch);
    // algorithmic bytes: A, B and the target or output gradient read, the output and the four
    // gradients written once, the flows read once
    double img = 16.0 * width * height * batch, fl = 8.0 * flow_w * flow_h * batch;
    double bytes = img * (2 + (target || grad_out ? 1 : 0) + (out ? 1 : 0) + (da ? 1 : 0) + (db ? 1 : 0)) +
                   fl * (2 + (df_ab ? 1 : 0) + (df_ba ? 1 : 0));
    LAUNCHB(ctx, bytes, k_warp_blend_adjoint, grid, ADJ_THREADS, ADJ_SMEM, P);
    return ctx->cuda(cudaGetLastError(), "launch");
}

int tw_check_powf(tw_ctx* ctx, const float* x, const float* y, float* out, int64_t n) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!x || !y || !out || n < 0) return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    if (n == 0) return TW_OK;
    size_t b = (size_t)n * sizeof(float);
    CHECK(ctx->ensure(ctx->plane[0], b, "powf input"));
    CHECK(ctx->ensure(ctx->plane[1], b, "powf input"));
    CHECK(ctx->ensure(ctx->plane[2], b, "powf output"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->plane[0].p, x, b, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->plane[1].p, y, b, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    LAUNCH(ctx, k_check_powf, grid1(n), TB, 0, ctx->plane[0].as<float>(), ctx->plane[1].as<float>(), ctx->plane[2].as<float>(),
           (long)n);
    CHECK(ctx->cuda(cudaMemcpyAsync(out, ctx->plane[2].p, b, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    return ctx->cuda(cudaStreamSynchronize(ctx->stream), "kernel execution");
}

int tw_check_logf(tw_ctx* ctx, const float* x, float* out, int64_t n) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!x || !out || n < 0) return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    if (n == 0) return TW_OK;
    const uint2* tab;
    int ntab;
    CHECK(logf_table(ctx, &tab, &ntab));
    CHECK(ctx->ensure(ctx->fw_vx, (size_t)n * sizeof(float), "logf input"));
    CHECK(ctx->ensure(ctx->fw_vy, (size_t)n * sizeof(float), "logf output"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->fw_vx.p, x, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream), "upload"));
    LAUNCH(ctx, k_logf_glibc, grid1((long)n), TB, 0, ctx->fw_vx.as<float>(), ctx->fw_vy.as<float>(), (long)n, tab, ntab);
    CHECK(ctx->cuda(cudaMemcpyAsync(out, ctx->fw_vy.p, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream), "download"));
    CHECK(ctx->cuda(cudaStreamSynchronize(ctx->stream), "kernel execution"));
    return ctx->cuda(cudaGetLastError(), "kernel execution");
}

int tw_from_frame(tw_ctx* ctx, const void* wire, int32_t width, int32_t height, int32_t fmt, void* engine_out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!wire || !engine_out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0) return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    size_t bytes = (size_t)width * height * 4 * sample_bytes(fmt);
    CHECK(ctx->ensure(ctx->wire[0], bytes, "wire"));
    CHECK(ctx->ensure(ctx->eng[0], bytes, "engine"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->wire[0].p, wire, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    long n = (long)width * height;
    if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_from_frame_u8, grid1(n), TB, 0, ctx->wire[0].as<uint8_t>(), ctx->eng[0].as<uint8_t>(), width, height, false);
    else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_from_frame_u16, grid1(n), TB, 0, ctx->wire[0].as<uint16_t>(), ctx->eng[0].as<uint16_t>(), width, height, false);
    else LAUNCHB(ctx, 2.0 * 16 * n, k_from_frame_f32, grid1(n), TB, 0, ctx->wire[0].as<float>(), ctx->eng[0].as<float>(), width, height, false);
    CHECK(ctx->cuda(cudaMemcpyAsync(engine_out, ctx->eng[0].p, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

int tw_to_frame(tw_ctx* ctx, const void* engine, int32_t width, int32_t height, int32_t fmt, void* wire_out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!engine || !wire_out || fmt < 0 || fmt > 2 || width <= 0 || height <= 0) return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    size_t bytes = (size_t)width * height * 4 * sample_bytes(fmt);
    CHECK(ctx->ensure(ctx->wire[0], bytes, "wire"));
    CHECK(ctx->ensure(ctx->eng[0], bytes, "engine"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->eng[0].p, engine, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    long n = (long)width * height;
    if (fmt == TW_U8) LAUNCHB(ctx, 2.0 * 4 * n, k_to_frame_u8, grid1(n), TB, 0, ctx->eng[0].as<uint8_t>(), ctx->wire[0].as<uint8_t>(), width, height, false);
    else if (fmt == TW_U16) LAUNCHB(ctx, 2.0 * 8 * n, k_to_frame_u16, grid1(n), TB, 0, ctx->eng[0].as<uint16_t>(), ctx->wire[0].as<uint16_t>(), width, height, false);
    else LAUNCHB(ctx, 2.0 * 16 * n, k_to_frame_f32, grid1(n), TB, 0, ctx->eng[0].as<float>(), ctx->wire[0].as<float>(), width, height, false);
    CHECK(ctx->cuda(cudaMemcpyAsync(wire_out, ctx->wire[0].p, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

}  // extern "C"
