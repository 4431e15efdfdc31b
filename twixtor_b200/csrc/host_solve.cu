// The solver driver: geometry and host scalars, the band and mask pyramids, the user displacement
// of tracking points, block matching and the level loop (flow.rs:1258-1307), with the solve entry
// points.
#include "runtime.h"

namespace tw {

void flow_resolution(int q, bool hiq, int w, int h, int* r_out, int* w0, int* h0) {
    int r = (q <= 2) ? 3 : (q == 3) ? 2 : (q == 4) ? 1 : 0;
    if (!hiq) r = (r == 0) ? 1 : (r == 1) ? 2 : (r == 2) ? 3 : r;
    while (r > 0 && ((w >> r) < 2 || (h >> r) < 2)) r -= 1;
    int ww = w, hh = h;
    for (int i = 0; i < r; i++) { ww /= 2; hh /= 2; }
    *r_out = r; *w0 = ww; *h0 = hh;
}

int level_count(int w0, int h0, int min_size) {
    int levels = 1, w = w0, h = h0;
    for (;;) {
        w /= 2;
        if (w < min_size) break;
        h /= 2;
        if (h < min_size) break;
        if (w > 2 && h > 2 && !(w == 2 && h == 2)) levels += 1;
        else break;
    }
    return levels;
}

int geometry(const tw_flow_settings& s, int w, int h, Geo* g, std::string* err) {
    if (s.quality <= 0 || s.quality > 5) { *err = "flow quality is outside 1..=5 (0 disables the estimator)"; return TW_ERR_BAD_PARAM; }
    if (!(s.sensitivity >= 0.0f) || !std::isfinite(s.sensitivity)) { *err = "sensitivity must be finite and not negative"; return TW_ERR_BAD_PARAM; }
    flow_resolution(s.quality, s.hiq != 0, w, h, &g->reduction, &g->w, &g->h);
    if (g->w < 2 || g->h < 2) { *err = "optical flow: working size below 2x2 is not supported"; return TW_ERR_UNSUPPORTED; }
    if (g->w > BM_MAX_LINE || g->h > BM_MAX_LINE) { *err = "optical flow: a working size side above 6144 is not on the device"; return TW_ERR_UNSUPPORTED; }
    g->levels = std::min(level_count(g->w, g->h, 2), 32);
    int lw = g->w, lh = g->h;
    for (int i = 0; i < g->levels; i++) {
        g->sizes[i][0] = lw;
        g->sizes[i][1] = lh;
        lw = std::max(lw / 2, 2);
        lh = std::max(lh / 2, 2);
    }
    return TW_OK;
}

void start_level(float sensitivity, int levels, int* start, float* damp) {  // flow.rs:179-197
    float p = (float)std::pow((double)sensitivity, 2.0);
    float l1 = (float)std::log((double)p);
    float l2 = (float)std::log(2.0);
    float lv = (float)levels;
    float x = l1 / l2 + lv;
    if (0.0f <= x || std::isnan(x)) {
        if (x < lv || std::isnan(x)) {
            float f = std::floor(x);
            int s = (std::isnan(f) || f >= 2147483648.0f || f < -2147483648.0f) ? INT32_MIN : (int)f;
            int su = s < 0 ? 0 : s;
            *start = std::min(su, levels - 1);
            *damp = x - (float)su;
        } else {
            *start = levels - 1;
            *damp = 1.0f;
        }
    } else {
        *start = 0;
        *damp = 0.0f;
    }
}

Taps gaussian_taps(float r) {  // flow/conv.rs:64-86
    Taps t{};
    int ri = std::isnan(r) ? 0 : (int)r;
    int n = std::max(ri + 1, 0);
    n = std::min(n, MAX_TAPS);
    float s3 = r / 3.0f;
    float d = s3 * s3;
    float sum = 0.0f;
    for (int i = 0; i < n; i++) {
        float fi = (float)i;
        float tt = fi * fi;
        float e = -(tt / d);
        float v = (float)std::pow(2.0, (double)e);
        t.k[i] = v;
        sum += v;
    }
    t.n = n;
    if (n == 0) return t;
    float den = sum * 2.0f - t.k[0];
    for (int i = 0; i < n; i++) t.k[i] /= den;
    return t;
}

Taps binomial5() {  // flow/conv.rs:48
    Taps t{};
    t.k[0] = 0.375f;
    t.k[1] = 0.25f;
    t.k[2] = 0.0625f;
    t.n = 3;
    return t;
}

// ---- separable convolution of `c` planes in place (flow/conv.rs: convolve_above_first) --------------
void conv_planes(tw_ctx* ctx, float* const* planes, int c, int w, int h, const Taps& t, bool above_first, float* tmp) {
    bool multi = c > 1;
    for (int i = 0; i < c; i++) {
        double b = 8.0 * w * h;  // one plane read, one written
        LAUNCHB(ctx, b, k_conv_h, grid2(w, h), TB, 0, planes[i], tmp, w, h, t, multi);
        LAUNCHB(ctx, b, k_conv_v, grid2(w, h), TB, 0, tmp, planes[i], w, h, t, multi, above_first, (const float*)nullptr,
                (float*)nullptr);
    }
}

// One solver iteration (k_level_iter_*) with the tile shape and block size of the level's choice:
// B read from b_in; with b_out the next iteration's B written (planes of pitch bp, stride bplane).
// Algorithmic bytes per pixel: B (2), the tensor (3) and the flow (2) read, the flow (2) written;
// with b_out also I1, the I0 gather and the gradient (2) read and B (2) written.
void level_iter(tw_ctx* ctx, LevelTune ic, const float* A, const float* B, const float* gx, const float* gy,
                const float* a0, const float* a1, const float* a2, const float* fu, const float* fv, int w, int h, bool af,
                float* nu, float* nv, const float* mask_y, bool fast, const float* b_in, float* b_out, int bp,
                long bplane) {
    double b = (b_out ? 60.0 : 36.0) * w * h;
    size_t smem = level_iter_smem(ic.iter_tile);
    if (ic.iter_tile == LEVEL_TILE_64x64) {
        dim3 g((unsigned)((w + 63) / 64), (unsigned)((h + 63) / 64));
        LAUNCHV(ctx, fast, b, k_level_iter_64x64, g, ic.iter_threads, smem, b_in, bp, bplane, A, B, gx, gy, a0, a1, a2, fu, fv, w,
                h, ctx->g7, ctx->g5, af, nu, nv, mask_y, b_out);
    } else if (ic.iter_tile == LEVEL_TILE_64x32) {
        dim3 g((unsigned)((w + 63) / 64), (unsigned)((h + 31) / 32));
        LAUNCHV(ctx, fast, b, k_level_iter_64x32, g, ic.iter_threads, smem, b_in, bp, bplane, A, B, gx, gy, a0, a1, a2, fu, fv, w,
                h, ctx->g7, ctx->g5, af, nu, nv, mask_y, b_out);
    } else {
        LAUNCHV(ctx, fast, b, k_level_iter_32x32, tiles(w, h), ic.iter_threads, smem, b_in, bp, bplane, A, B, gx, gy, a0, a1, a2,
                fu, fv, w, h, ctx->g7, ctx->g5, af, nu, nv, mask_y, b_out);
    }
}

// The launch shapes at a level of w x h: the tuning table's entry when the autotuner measured this
// size, else the defaults: 32 x 32 iteration tiles with 512 threads for levels of few tiles
// (latency bound: fewer elements per thread per stage) and 256 otherwise; 256 threads per line of
// block matching.
LevelTune default_tune(int w, int h) {
    long tiles_n = (long)((w + 31) / 32) * ((h + 31) / 32);
    return LevelTune{LEVEL_TILE_32x32, tiles_n <= 296 ? 512 : 256, TB, TB};
}

LevelTune level_tune(tw_ctx* ctx, int w, int h) {
    auto it = ctx->tune_table.find(((uint64_t)(uint32_t)w << 32) | (uint32_t)h);
    return it != ctx->tune_table.end() ? it->second : default_tune(w, h);
}

// Threads per CTA of the tiled pyramid and tensor kernels: a level of few tiles is latency bound
// (every CTA walks its stages one after the other), so its CTAs get more threads and each thread
// fewer elements per stage; a level with tiles enough to fill the GPU keeps 256.
static int level_threads(int w, int h) {
    long tiles_n = (long)((w + 31) / 32) * ((h + 31) / 32);
    return tiles_n <= 148 ? 1024 : tiles_n <= 296 ? 512 : 256;
}

// ---- the pyramid of one engine image (flow.rs:242-275) ----------------------------------------------
// Builds the band pass levels into `out` (levels concatenated, finest first) and their transposes
// into out_t. Luma, the reduction steps (prep.rs:252-259) and each level's blur5 + band run as
// tiled kernels (k_blur5_band), each followed by the corner aligned resample to the next size.
int build_pyramid_dev(tw_ctx* ctx, const void* eng_dev, int W, int H, int fmt, const tw_flow_settings& s, const Geo& g,
                      float* out, float* out_t, DevBuf* scratch) {
    if (s.video_range_luma && s.track_alpha)
        return ctx->fail(TW_ERR_UNSUPPORTED, "optical flow luma: video range conversion together with Track RGB+A is not supported");
    int lmode = (s.track_alpha ? LUMA_TRACK_ALPHA : 0) | (s.video_range_luma ? LUMA_VIDEO_RANGE : 0);
    const bool fast = s.fast_mode != 0;  // the fast mode's build of the band pyramid's kernels
    size_t full = (size_t)W * H * sizeof(float);
    for (int i = 0; i < 3; i++) CHECK(ctx->ensure(scratch[i], full, "pyramid scratch"));
    float* cur = scratch[0].as<float>();
    float* tmp = scratch[1].as<float>();
    float* nxt = scratch[2].as<float>();
    bool af = s.taps_above_first != 0;
    int cw = W, ch = H;
    if (s.wrap) {
        // flow.rs:236-275 in the 360 mode of the filters (prep.rs:261-299): the luma, the reduction and
        // every level with the circular row pass, the equirectangular column pass and resample
        if (s.prep_contrast_edge)
            return ctx->fail(TW_ERR_UNSUPPORTED, "the 360 mode Contrast / Edge Enhance is not on the device");
        long n = (long)W * H;
        LAUNCH(ctx, k_luma, grid1(n), TB, 0, eng_dev, fmt, cur, W, H, s.track_alpha != 0, s.video_range_luma != 0);
        for (int r = 0; r < g.reduction; r++) {
            LAUNCH(ctx, k_conv_h_wrap, grid2(cw, ch), TB, 0, (const float*)cur, tmp, cw, ch, ctx->b5);
            LAUNCH(ctx, k_conv_v_sphere, grid2(cw, ch), TB, 0, (const float*)tmp, nxt, cw, ch, ctx->b5,
                   (const float*)nullptr, (float*)nullptr, (float*)nullptr);
            int nw = cw / 2, nh = ch / 2;
            LAUNCH(ctx, k_resample_sphere, grid2(nw, nh), TB, 0, (const float*)nxt, cw, ch, cur, nw, nh);
            cw = nw;
            ch = nh;
        }
        if (s.prep_delinearize) LAUNCH(ctx, k_delinearize, grid1((long)cw * ch), TB, 0, cur, (long)cw * ch);
        size_t off = 0;
        for (int i = 0; i < g.levels; i++) {
            int lw = g.sizes[i][0], lh = g.sizes[i][1];
            LAUNCH(ctx, k_conv_h_wrap, grid2(lw, lh), TB, 0, (const float*)cur, nxt, lw, lh, ctx->b5);
            LAUNCH(ctx, k_conv_v_sphere, grid2(lw, lh), TB, 0, (const float*)nxt, tmp, lw, lh, ctx->b5, (const float*)cur,
                   out + off, out_t ? out_t + off : (float*)nullptr);
            if (i + 1 < g.levels) {
                int nw = g.sizes[i + 1][0], nh = g.sizes[i + 1][1];
                LAUNCH(ctx, k_resample_sphere, grid2(nw, nh), TB, 0, (const float*)tmp, lw, lh, cur, nw, nh);
            }
            off += (size_t)lw * lh;
        }
        return TW_OK;
    }
    if (g.reduction == 0) {
        long n = (long)W * H;
        LAUNCH(ctx, k_luma, grid1(n), TB, 0, eng_dev, fmt, cur, W, H, s.track_alpha != 0, s.video_range_luma != 0);
    }
    for (int r = 0; r < g.reduction; r++) {  // prep.rs:252-259; the first step reads the luma on the fly
        LAUNCHV(ctx, fast, (r == 0 ? 4.0 * sample_bytes(fmt) : 4.0) * cw * ch + 4.0 * cw * ch, k_blur5_band, tiles(cw, ch),
                FUSED_THREADS, 0, r == 0 ? (const float*)nullptr : cur, r == 0 ? eng_dev : nullptr, fmt, lmode, cw, ch, af, tmp,
                (float*)nullptr, (float*)nullptr);
        int nw = cw / 2, nh = ch / 2;
        LAUNCHV(ctx, fast, 0, k_resample, grid2(nw, nh), TB, 0, tmp, cw, ch, nxt, nw, nh);
        std::swap(cur, nxt);
        cw = nw;
        ch = nh;
    }
    // flow.rs:248-253: the image prep of level 0, Delinearize then Contrast / Edge Enhance
    if (s.prep_delinearize) LAUNCH(ctx, k_delinearize, grid1((long)cw * ch), TB, 0, cur, (long)cw * ch);
    if (s.prep_contrast_edge) {
        conv_planes(ctx, &cur, 1, cw, ch, ctx->g2, af, tmp);  // prep.rs:329, the Gaussian of radius 2.0
        LAUNCH(ctx, k_edge_map, grid1((long)cw * ch), TB, 0, cur, nxt, cw, ch);
        std::swap(cur, nxt);
    }
    size_t off = 0;
    size_t pf = pyramid_floats(g);
    for (int i = 0; i < g.levels; i++) {
        int lw = g.sizes[i][0], lh = g.sizes[i][1];
        LAUNCHV(ctx, fast, 16.0 * lw * lh, k_blur5_band, tiles(lw, lh), level_threads(lw, lh), 0, cur, (const void*)nullptr, fmt, 0, lw,
                lh, af, tmp, out + off, out_t ? out_t + off : (float*)nullptr);
        if (i + 1 < g.levels) {
            int nw = g.sizes[i + 1][0], nh = g.sizes[i + 1][1];
            LAUNCHV(ctx, fast, 0, k_resample, grid2(nw, nh), TB, 0, tmp, lw, lh, cur, nw, nh);
        }
        off += (size_t)lw * lh;
    }
    (void)pf;
    return TW_OK;
}

size_t pyramid_floats(const Geo& g) {
    size_t n = 0;
    for (int i = 0; i < g.levels; i++) n += (size_t)g.sizes[i][0] * g.sizes[i][1];
    return n;
}

// The pairs of a solve from a layer's tracking points (layers.rs:254, UserPoint::pair): (at A, at B)
// for the solve with X = A, (at B, at A) for the other; `flip`: on the motion path's bottom-up rows,
// y -> (H - 1) - y (layers.rs:348-351). More than twelve points is refused.
int user_pairs(tw_ctx* ctx, const tw_user_point* pts, int n, bool x_is_a, bool flip, int H, UserPairs* out) {
    if (n > MAX_USER_PAIRS) return ctx->fail(TW_ERR_UNSUPPORTED, "%d tracking points on one layer (at most 12)", n);
    out->n = n;
    float last_row = (float)H - 1.0f;
    for (int i = 0; i < n; i++) {
        float ax = pts[i].at_a[0], ay = pts[i].at_a[1], bx = pts[i].at_b[0], by = pts[i].at_b[1];
        if (flip) {
            ay = last_row - ay;
            by = last_row - by;
        }
        out->p[i][0] = x_is_a ? ax : bx;
        out->p[i][1] = x_is_a ? ay : by;
        out->p[i][2] = x_is_a ? bx : ax;
        out->p[i][3] = x_is_a ? by : ay;
    }
    return TW_OK;
}

// points.rs:201-240 (user_displacement_with, no wrap): the user displacement of a solve, planes du,
// dv, uw laid out like the band pyramid; level 0 the splat of the pairs, normalised and negated,
// every coarser level the binomial blur of the level above (the two channels with the multi channel
// border rule, the column pass above first), the corner aligned resample and the scale of d by the
// ratio of the level sizes. scr: 4 planes of level 0's size.
int build_user_dev(tw_ctx* ctx, const UserPairs& pr, const Geo& g, int W, int H, float* du, float* dv, float* uw,
                          float* scr) {
    size_t pf = pyramid_floats(g);
    for (float* p : {du, dv, uw}) CHECK(ctx->cuda(cudaMemsetAsync(p, 0, pf * sizeof(float), ctx->cur), "user displacement"));
    int w0 = g.sizes[0][0], h0 = g.sizes[0][1];
    LAUNCH(ctx, k_user_splat, 1, 32, 0, pr, w0, h0, W, H, du, dv, uw);
    LAUNCH(ctx, k_user_finest, grid1((long)w0 * h0), TB, 0, du, dv, uw, (long)w0 * h0);
    size_t off = 0;
    for (int l = 1; l < g.levels; l++) {
        int pw = g.sizes[l - 1][0], ph = g.sizes[l - 1][1], nw = g.sizes[l][0], nh = g.sizes[l][1];
        size_t pn = (size_t)pw * ph, noff = off + pn;
        float* c[3] = {scr, scr + pn, scr + 2 * pn};
        float* tmp = scr + 3 * pn;
        CHECK(ctx->cuda(cudaMemcpyAsync(c[0], du + off, pn * sizeof(float), cudaMemcpyDeviceToDevice, ctx->cur), "user"));
        CHECK(ctx->cuda(cudaMemcpyAsync(c[1], dv + off, pn * sizeof(float), cudaMemcpyDeviceToDevice, ctx->cur), "user"));
        CHECK(ctx->cuda(cudaMemcpyAsync(c[2], uw + off, pn * sizeof(float), cudaMemcpyDeviceToDevice, ctx->cur), "user"));
        conv_planes(ctx, c, 2, pw, ph, ctx->b5, true, tmp);
        conv_planes(ctx, c + 2, 1, pw, ph, ctx->b5, true, tmp);
        LAUNCH(ctx, k_resample, grid2(nw, nh), TB, 0, c[0], pw, ph, du + noff, nw, nh);
        LAUNCH(ctx, k_resample, grid2(nw, nh), TB, 0, c[1], pw, ph, dv + noff, nw, nh);
        LAUNCH(ctx, k_resample, grid2(nw, nh), TB, 0, c[2], pw, ph, uw + noff, nw, nh);
        float sx = (float)(nw - 1) / (float)(pw - 1), sy = (float)(nh - 1) / (float)(ph - 1);
        LAUNCH(ctx, k_user_scale, grid1((long)nw * nh), TB, 0, du + noff, dv + noff, (long)nw * nh, sx, sy);
        off = noff;
    }
    return TW_OK;
}

// ---- block matching (flow.rs:551-622) -----------------------------------------------------------------
// Rows on the row-major planes; then the field is transposed, the column sweeps run on the
// transposed planes (AT, BT: the level's bands stored column by column), and the field goes back.
// uT, vT: scratch for the transposed field (w * h floats each).
void block_match(tw_ctx* ctx, const float* A, const float* B, const float* AT, const float* BT, float* fu, float* fv,
                 float* uT, float* vT, int w, int h, bool fast) {
    if (w < 3 || h < 3) return;  // callers refuse lines above BM_MAX_LINE before any launch
    double b = 24.0 * w * h;  // per launch (both sweeps): the field read and written (8 + 8), A and B read once (4 + 4)
    LevelTune t = level_tune(ctx, w, h);
    // the row sweeps write the transposed field the column sweeps read, and those write it back
    LAUNCHV(ctx, fast, b, k_bm_rows, h - 2, t.bm_rows_threads, bm_smem_bytes(w), A, B, fu, fv, w, h, uT, vT);
    LAUNCHV(ctx, fast, b, k_bm_cols, w - 2, t.bm_cols_threads, bm_smem_bytes(h), AT, BT, uT, vT, w, h, fu, fv);
}

// ---- one solve over two resident pyramids (flow.rs:1258-1307) ------------------------------------------
// x, y: band pass levels of X and Y; work: scratch for this solve; out: interleaved flow at level 0
// size (device). any: 32 ints of per-level "some pixel in range" flags; nan_flag: set when the
// result holds a NaN. Per level: one tiled kernel for the gradient and the blurred tensor, one per
// iteration (calc_b, blur7, new_disp, blur5 in shared memory, the flow ping-ponged), the block
// matching sweeps, the range check, and the reset / damping fused into the upsample.
// mx, my (may be null): the binary mask pyramids of a layered solve (flow/extras.rs:386-430), laid
// out like the band pyramids; the gradient is masked by X's level mask and the B step gated by Y's.
// The block matching is not gated (the effects build ungated masks, create_vectors.rs:360,
// layers/plates.rs:360).
int solve_pyramids_dev(tw_ctx* ctx, const float* x, const float* y, const float* xt, const float* yt, const Geo& g,
                       const tw_flow_settings& s, DevBuf& work, float* out, int* any, int* nan_flag,
                       const float* mx, const float* my, const float* udu,
                       const float* udv, const float* uww) {
    size_t np0 = (size_t)g.w * g.h;
    // planes: gx gy a0 a1 a2 u0 v0 u1 v1 uT vT, then two B buffers of two planes each, 16-byte
    // aligned, of pitch (w + 3) & ~3 at every level (plane stride bplane: the finest level's)
    const int NP = 11;
    const size_t boff = (np0 * NP + 3) & ~(size_t)3;
    const long bplane = (long)((g.w + 3) & ~3) * g.h;
    CHECK(ctx->ensure(work, (boff + 4 * (size_t)bplane) * sizeof(float), "solve scratch"));
    float* base = work.as<float>();
    float *gx = base, *gy = base + np0, *a0 = base + 2 * np0, *a1 = base + 3 * np0, *a2 = base + 4 * np0;
    float *fu = base + 5 * np0, *fv = base + 6 * np0, *nu = base + 7 * np0, *nv = base + 8 * np0;
    float *ut = base + 9 * np0, *vt = base + 10 * np0;
    float* bb[2] = {base + boff, base + boff + 2 * bplane};
    int start;
    float damp;
    start_level(s.sensitivity, g.levels, &start, &damp);
    size_t offs[32];
    size_t off = 0;
    for (int i = 0; i < g.levels; i++) { offs[i] = off; off += (size_t)g.sizes[i][0] * g.sizes[i][1]; }
    long ns = (long)g.sizes[start][0] * g.sizes[start][1];
    CHECK(GOP(ctx, ctx->cuda(cudaMemsetAsync(fu, 0, ns * sizeof(float), ctx->cur), "flow init")));
    CHECK(GOP(ctx, ctx->cuda(cudaMemsetAsync(fv, 0, ns * sizeof(float), ctx->cur), "flow init")));
    CHECK(GOP(ctx, ctx->cuda(cudaMemsetAsync(any, 0, 32 * sizeof(int), ctx->cur), "range flags")));
    bool af = s.taps_above_first != 0;
    bool damp_any = std::fabs((double)damp - 1.0) >= 1e-6;
    const bool fast = s.fast_mode != 0;
    // The coarse levels whose planes fit one block's shared memory run in one launch (coarse.cu),
    // for the plain solve; the masked and the tracked solves keep the kernel by kernel path.
    int first = start;
    if (!mx && !my && !udu) {
        int last = -1;
        for (int l = start; l >= 1; l--) {
            int w = g.sizes[l][0], h = g.sizes[l][1];
            if (w * h > COARSE_MAX_PIXELS || w > COARSE_MAX_LINE || h > COARSE_MAX_LINE) break;
            last = l;
        }
        if (last >= 1) {
            CoarseJob J{};
            J.x = x;
            J.y = y;
            for (int i = 0; i < g.levels; i++) {
                J.sizes[i][0] = g.sizes[i][0];
                J.sizes[i][1] = g.sizes[i][1];
                J.offs[i] = (int)offs[i];
            }
            J.start = start;
            J.last = last;
            J.damp_any = damp_any;
            J.damp = damp;
            J.refine = !s.skip_refine;
            J.af = af;
            J.g7 = ctx->g7;
            J.g5 = ctx->g5;
            J.any = any;
            J.fu_out = fu;
            J.fv_out = fv;
            double px = 0.0;
            for (int l = start; l >= last; l--) px += (double)g.sizes[l][0] * g.sizes[l][1];
            LAUNCHV(ctx, fast, 8.0 * px, k_solve_coarse, 1, COARSE_THREADS, coarse_smem_bytes(), J);
            first = last - 1;
        }
    }
    for (int l = first; l >= 0; l--) {
        int w = g.sizes[l][0], h = g.sizes[l][1];
        const float* A = x + offs[l];
        const float* B = y + offs[l];
        const float* AT = xt + offs[l];
        const float* BT = yt + offs[l];
        double px = (double)w * h;
        int lt = level_threads(w, h);
        const float* mask_x = mx ? mx + offs[l] : nullptr;
        const float* mask_y = my ? my + offs[l] : nullptr;
        // flow/extras.rs:198-215: the user displacement of the tracking points, flow = d / w, after the
        // start or the upsample, after the finest level's block matching and at the end of the level
        auto user = [&]() {
            if (udu) LAUNCH(ctx, k_apply_user, grid1((long)w * h), TB, 0, fu, fv, udu + offs[l], udv + offs[l], uww + offs[l],
                            (long)w * h);
        };
        user();
        LevelTune ic = level_tune(ctx, w, h);
        const int bp = (w + 3) & ~3;
        // the image read, the gradient and the tensor written; the flow, I0 (gather) read and B written
        LAUNCHV(ctx, fast, 44.0 * px, k_level_init, tiles(w, h), lt, level_init_smem(), A, w, h, ctx->g7, af, gx, gy, a0, a1, a2,
                mask_x, fu, fv, B, mask_y, bb[0], bp, bplane);
        for (int it = 0; it < 3; it++) {
            // iteration it reads B from bb[it & 1]; the next one's B comes from its epilogue, or after
            // the finest level's block matching from the pointwise pass
            const bool emit = it == 0 || (it == 1 && l != 0);
            level_iter(ctx, ic, A, B, gx, gy, a0, a1, a2, fu, fv, w, h, af, nu, nv, mask_y, fast, bb[it & 1],
                       emit ? bb[(it + 1) & 1] : nullptr, bp, bplane);
            std::swap(fu, nu);
            std::swap(fv, nv);
            if (it == 1 && l == 0) {
                if (!s.skip_refine) block_match(ctx, A, B, AT, BT, fu, fv, ut, vt, w, h, fast);
                user();
                LAUNCHV(ctx, fast, 32.0 * px, k_calc_b_pitched, grid2(w, h), TB, 0, A, B, gx, gy, fu, fv, w, h, mask_y, bb[0], bp,
                        bplane);
            }
        }
        if (l != 0 && !s.skip_refine) block_match(ctx, A, B, AT, BT, fu, fv, ut, vt, w, h, fast);
        user();
        LAUNCHV(ctx, fast, 0, k_range_any, grid2(w, h), TB, 0, fu, fv, w, h, any + l);
        bool damp_now = l == start && damp_any;
        if (l > 0) {
            int dw = g.sizes[l - 1][0], dh = g.sizes[l - 1][1];
            LAUNCHV(ctx, fast, 0, k_apply_upsample, grid2(dw, dh), TB, 0, fu, fv, w, h, any, l, start, damp_now, damp, nu, nv, dw, dh);
            std::swap(fu, nu);
            std::swap(fv, nv);
        } else {
            LAUNCHV(ctx, fast, 0, k_apply_negate, grid1((long)np0), TB, 0, fu, fv, (long)np0, any, start, damp_now, damp, out, nan_flag);
        }
    }
    return TW_OK;
}

// The binary mask pyramid of a matte (flow/extras.rs:76-123): binarize at 0.95, then per reduction
// step and per level the blur5 (the pyramid's tap order), the corner aligned resample, binarize.
// matte: w*h values 0..1 on the device (consumed); out: pyramid_floats(g) values, laid out like
// the band pyramid; scratch: two planes of w*h. `one` points at a nonzero device int (the stack
// passes run unconditionally).
int build_mask_pyramid_dev(tw_ctx* ctx, float* matte, int W, int H, const tw_flow_settings& s, const Geo& g, float* out,
                           float* scratch0, float* scratch1, const int* one) {
    float* cur = matte;
    float* tmp = scratch0;
    float* nxt = scratch1;
    bool af = s.taps_above_first != 0;
    // prep::blur5 of one plane into tmp: the band pyramid's tiled kernel (both passes in one launch)
    auto blur5 = [&](const float* p, int w, int h) {
        LAUNCHB(ctx, 8.0 * w * h, k_blur5_band, tiles(w, h), level_threads(w, h), 0, p, (const void*)nullptr, 0, 0, w, h,
                af, tmp, (float*)nullptr, (float*)nullptr);
    };
    auto resample = [&](const float* src, int sw, int sh, float* dst, int dw, int dh) {
        dim3 gp((unsigned)((dw + TB - 1) / TB), (unsigned)dh, 1);
        LAUNCH(ctx, k_stack_resample, gp, TB, 0, src, sw, sh, (long)sw * sh, dst, dw, dh, (long)dw * dh, 0, one);
        LAUNCH(ctx, k_binarize, grid1((long)dw * dh), TB, 0, dst, (long)dw * dh);
    };
    int cw = W, ch = H;
    LAUNCH(ctx, k_binarize, grid1((long)W * H), TB, 0, cur, (long)W * H);
    for (int r = 0; r < g.reduction; r++) {
        int nw = cw / 2, nh = ch / 2;
        blur5(cur, cw, ch);
        resample(tmp, cw, ch, nxt, nw, nh);
        std::swap(cur, nxt);
        cw = nw;
        ch = nh;
    }
    size_t off = 0;
    for (int i = 0; i < g.levels; i++) {
        int lw = g.sizes[i][0], lh = g.sizes[i][1];
        CHECK(ctx->cuda(cudaMemcpyAsync(out + off, cur, (size_t)lw * lh * sizeof(float), cudaMemcpyDeviceToDevice, ctx->cur),
                        "mask level"));
        off += (size_t)lw * lh;
        if (i + 1 < g.levels) {
            blur5(cur, lw, lh);
            resample(tmp, lw, lh, nxt, g.sizes[i + 1][0], g.sizes[i + 1][1]);
            std::swap(cur, nxt);
        }
    }
    return TW_OK;
}

}  // namespace tw

extern "C" {

int tw_flow_geometry(const tw_flow_settings* s, int32_t width, int32_t height, int32_t* flow_w, int32_t* flow_h,
                     int32_t* levels, int32_t* sizes, int32_t cap) {
    if (!s) return TW_ERR_BAD_PARAM;
    Geo g;
    std::string e;
    int rc = geometry(*s, width, height, &g, &e);
    if (rc) return rc;
    if (flow_w) *flow_w = g.w;
    if (flow_h) *flow_h = g.h;
    if (levels) *levels = g.levels;
    if (sizes)
        for (int i = 0; i < g.levels && i < cap; i++) { sizes[2 * i] = g.sizes[i][0]; sizes[2 * i + 1] = g.sizes[i][1]; }
    return TW_OK;
}

// flags layout (ints): [0..1] solve state of solve 0, [2..3] of solve 1, [4] NaN flag, [5] warp refused
static int solve_common(tw_ctx* ctx, const tw_image* a, const tw_image* b, const tw_flow_settings* s, tw_flow* f_ab,
                        tw_flow* f_ba, bool pair) {
    CHECK(check_image(ctx, a, "solve"));
    CHECK(check_image(ctx, b, "solve"));
    if (!s) return ctx->fail(TW_ERR_BAD_PARAM, "no flow settings");
    if (!same_shape(a, b))
        return ctx->fail(TW_ERR_MISMATCH, "optical flow: incompatible inputs (%dx%d fmt %d against %dx%d fmt %d)", a->width,
                         a->height, a->fmt, b->width, b->height, b->fmt);
    if (s->wrap) return ctx->fail(TW_ERR_UNSUPPORTED, "the wrap-around (360) solve is not on the device");
    Geo g;
    CHECK(geometry(*s, a->width, a->height, &g, &ctx->err));
    if (f_ab && (f_ab->width != g.w || f_ab->height != g.h || !f_ab->data))
        return ctx->fail(TW_ERR_MISMATCH, "flow buffer is not %dx%d", g.w, g.h);
    if (f_ba && (f_ba->width != g.w || f_ba->height != g.h || !f_ba->data))
        return ctx->fail(TW_ERR_MISMATCH, "flow buffer is not %dx%d", g.w, g.h);
    CHECK(upload_image(ctx, ctx->eng[0], a));
    CHECK(upload_image(ctx, ctx->eng[1], b));
    size_t pf = pyramid_floats(g);
    CHECK(ctx->ensure(ctx->pyr[0], 2 * pf * 4, "pyramid"));
    CHECK(ctx->ensure(ctx->pyr[1], 2 * pf * 4, "pyramid"));
    float* px_ = ctx->pyr[0].as<float>();
    float* py_ = ctx->pyr[1].as<float>();
    CHECK(build_pyramid_dev(ctx, ctx->eng[0].p, a->width, a->height, a->fmt, *s, g, px_, px_ + pf, ctx->plane));
    CHECK(build_pyramid_dev(ctx, ctx->eng[1].p, b->width, b->height, b->fmt, *s, g, py_, py_ + pf, ctx->plane));
    size_t fb = (size_t)g.w * g.h * 2 * sizeof(float);
    CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
    CHECK(ctx->ensure(ctx->flow[1], fb, "flow"));
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    // f_ab = solve(X = A, Y = B); f_ba = solve(X = B, Y = A)
    if (f_ab)
        CHECK(solve_pyramids_dev(ctx, px_, py_, px_ + pf, py_ + pf, g, *s, ctx->work[0], ctx->flow[0].as<float>(),
                                 flags + FL_ANY0, flags + FL_NAN));
    if (pair && f_ba)
        CHECK(solve_pyramids_dev(ctx, py_, px_, py_ + pf, px_ + pf, g, *s, ctx->work[1], ctx->flow[1].as<float>(),
                                 flags + FL_ANY1, flags + FL_NAN));
    if (f_ab) CHECK(ctx->cuda(cudaMemcpyAsync(f_ab->data, ctx->flow[0].p, fb, cudaMemcpyDeviceToHost, ctx->stream), "flow download"));
    if (pair && f_ba) CHECK(ctx->cuda(cudaMemcpyAsync(f_ba->data, ctx->flow[1].p, fb, cudaMemcpyDeviceToHost, ctx->stream), "flow download"));
    int hf[2];
    CHECK(finish(ctx, hf, 2));
    if (hf[0]) return ctx->fail(TW_ERR_NAN_OUTPUT, "the solved flow holds a NaN");
    return TW_OK;
}

int tw_solve_masked(tw_ctx* ctx, const tw_image* x, const tw_image* y, const tw_flow_settings* s, const float* matte_x,
                    const float* matte_y, tw_flow* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!out || !out->data || !s) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    if (!matte_x != !matte_y) return ctx->fail(TW_ERR_BAD_PARAM, "a masked solve needs the mattes of both images");
    CHECK(check_image(ctx, x, "solve"));
    CHECK(check_image(ctx, y, "solve"));
    if (!same_shape(x, y))
        return ctx->fail(TW_ERR_MISMATCH, "optical flow: incompatible inputs (%dx%d fmt %d against %dx%d fmt %d)", x->width,
                         x->height, x->fmt, y->width, y->height, y->fmt);
    if (s->wrap) return ctx->fail(TW_ERR_UNSUPPORTED, "the wrap-around (360) solve is not on the device");
    Geo g;
    CHECK(geometry(*s, x->width, x->height, &g, &ctx->err));
    if (out->width != g.w || out->height != g.h) return ctx->fail(TW_ERR_MISMATCH, "flow buffer is not %dx%d", g.w, g.h);
    int W = x->width, H = x->height;
    size_t n = (size_t)W * H;
    CHECK(upload_image(ctx, ctx->eng[0], x));
    CHECK(upload_image(ctx, ctx->eng[1], y));
    size_t pf = pyramid_floats(g);
    CHECK(ctx->ensure(ctx->pyr[0], 2 * pf * 4, "pyramid"));
    CHECK(ctx->ensure(ctx->pyr[1], 2 * pf * 4, "pyramid"));
    float* px_ = ctx->pyr[0].as<float>();
    float* py_ = ctx->pyr[1].as<float>();
    CHECK(build_pyramid_dev(ctx, ctx->eng[0].p, W, H, x->fmt, *s, g, px_, px_ + pf, ctx->plane));
    CHECK(build_pyramid_dev(ctx, ctx->eng[1].p, W, H, y->fmt, *s, g, py_, py_ + pf, ctx->plane));
    float *mx = nullptr, *my = nullptr;
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    if (matte_x) {
        CHECK(ctx->ensure(ctx->masks, 2 * pf * sizeof(float), "mask pyramids"));
        CHECK(ctx->ensure(ctx->holes, 4 * n * sizeof(float), "mattes"));
        float* mt = ctx->holes.as<float>();
        CHECK(ctx->cuda(cudaMemcpyAsync(mt, matte_x, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream), "matte upload"));
        CHECK(ctx->cuda(cudaMemcpyAsync(mt + n, matte_y, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream), "matte upload"));
        // a nonzero int for the stack passes' "run" flag
        CHECK(ctx->cuda(cudaMemsetAsync(flags + FL_ONE, 0x01, sizeof(int), ctx->stream), "flags"));
        mx = ctx->masks.as<float>();
        my = mx + pf;
        CHECK(build_mask_pyramid_dev(ctx, mt, W, H, *s, g, mx, mt + 2 * n, mt + 3 * n, flags + FL_ONE));
        CHECK(build_mask_pyramid_dev(ctx, mt + n, W, H, *s, g, my, mt + 2 * n, mt + 3 * n, flags + FL_ONE));
    }
    size_t fb = (size_t)g.w * g.h * 2 * sizeof(float);
    CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
    CHECK(solve_pyramids_dev(ctx, px_, py_, px_ + pf, py_ + pf, g, *s, ctx->work[0], ctx->flow[0].as<float>(), flags + FL_ANY0,
                             flags + FL_NAN, mx, my));
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->flow[0].p, fb, cudaMemcpyDeviceToHost, ctx->stream), "flow download"));
    int hf[2];
    CHECK(finish(ctx, hf, 2));
    if (hf[0]) return ctx->fail(TW_ERR_NAN_OUTPUT, "the solved flow holds a NaN");
    return TW_OK;
}

int tw_solve_pyramids(tw_ctx* ctx, const tw_flow_settings* s, int32_t width, int32_t height, const float* x_levels,
                      const float* y_levels, const float* mask_x, const float* mask_y, const float* user_d,
                      const float* user_w, tw_flow* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!s || !x_levels || !y_levels || !out || !out->data || width <= 0 || height <= 0)
        return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    if (!mask_x != !mask_y) return ctx->fail(TW_ERR_BAD_PARAM, "solve_pyramids: the mask pyramids of both images, or none");
    if (!user_d != !user_w) return ctx->fail(TW_ERR_BAD_PARAM, "solve_pyramids: the user displacement and its weights, or none");
    if (s->wrap) return ctx->fail(TW_ERR_UNSUPPORTED, "the wrap-around (360) solve is not on the device");
    Geo g;
    CHECK(geometry(*s, width, height, &g, &ctx->err));
    if (out->width != g.w || out->height != g.h) return ctx->fail(TW_ERR_MISMATCH, "flow buffer is not %dx%d", g.w, g.h);
    size_t pf = pyramid_floats(g);
    CHECK(ctx->ensure(ctx->pyr[0], 2 * pf * 4, "pyramid"));
    CHECK(ctx->ensure(ctx->pyr[1], 2 * pf * 4, "pyramid"));
    float* px_ = ctx->pyr[0].as<float>();
    float* py_ = ctx->pyr[1].as<float>();
    CHECK(ctx->cuda(cudaMemcpyAsync(px_, x_levels, pf * 4, cudaMemcpyHostToDevice, ctx->stream), "pyramid upload"));
    CHECK(ctx->cuda(cudaMemcpyAsync(py_, y_levels, pf * 4, cudaMemcpyHostToDevice, ctx->stream), "pyramid upload"));
    // the transposed levels of the column sweeps, as build_pyramid_dev writes them beside the bands
    size_t off = 0;
    for (int i = 0; i < g.levels; i++) {
        int lw = g.sizes[i][0], lh = g.sizes[i][1];
        LAUNCHB(ctx, 16.0 * lw * lh, k_transpose2, dim3((lw + 31) / 32, (lh + 31) / 32), dim3(32, 8), 0, px_ + off, py_ + off,
                px_ + pf + off, py_ + pf + off, lw, lh);
        off += (size_t)lw * lh;
    }
    const float *mx = nullptr, *my = nullptr, *udu = nullptr, *udv = nullptr, *uww = nullptr;
    if (mask_x) {
        CHECK(ctx->ensure(ctx->masks, 2 * pf * sizeof(float), "mask pyramids"));
        float* m = ctx->masks.as<float>();
        CHECK(ctx->cuda(cudaMemcpyAsync(m, mask_x, pf * 4, cudaMemcpyHostToDevice, ctx->stream), "mask upload"));
        CHECK(ctx->cuda(cudaMemcpyAsync(m + pf, mask_y, pf * 4, cudaMemcpyHostToDevice, ctx->stream), "mask upload"));
        mx = m;
        my = m + pf;
    }
    if (user_d) {  // UserLevel::d interleaved (dx, dy) and ::w per level -> the planes du, dv, w
        CHECK(ctx->ensure(ctx->lay_in, 5 * pf * sizeof(float), "user displacement"));
        float* u = ctx->lay_in.as<float>();
        CHECK(ctx->cuda(cudaMemcpyAsync(u + 3 * pf, user_d, 2 * pf * 4, cudaMemcpyHostToDevice, ctx->stream), "user upload"));
        CHECK(ctx->cuda(cudaMemcpyAsync(u + 2 * pf, user_w, pf * 4, cudaMemcpyHostToDevice, ctx->stream), "user upload"));
        LAUNCH(ctx, k_deinterleave, grid1((long)pf), TB, 0, (const float*)(u + 3 * pf), (long)pf, u, u + pf);
        udu = u;
        udv = u + pf;
        uww = u + 2 * pf;
    }
    int* flags = ctx->flags.as<int>();
    CHECK(ctx->cuda(cudaMemsetAsync(flags, 0, FLAGS_BYTES, ctx->stream), "flags"));
    size_t fb = (size_t)g.w * g.h * 2 * sizeof(float);
    CHECK(ctx->ensure(ctx->flow[0], fb, "flow"));
    CHECK(solve_pyramids_dev(ctx, px_, py_, px_ + pf, py_ + pf, g, *s, ctx->work[0], ctx->flow[0].as<float>(), flags + FL_ANY0,
                             flags + FL_NAN, mx, my, udu, udv, uww));
    CHECK(ctx->cuda(cudaMemcpyAsync(out->data, ctx->flow[0].p, fb, cudaMemcpyDeviceToHost, ctx->stream), "flow download"));
    int hf[2];
    CHECK(finish(ctx, hf, 2));
    if (hf[0]) return ctx->fail(TW_ERR_NAN_OUTPUT, "the solved flow holds a NaN");
    return TW_OK;
}

int tw_solve(tw_ctx* ctx, const tw_image* x, const tw_image* y, const tw_flow_settings* s, tw_flow* out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!out) return ctx->fail(TW_ERR_BAD_PARAM, "no output flow");
    return solve_common(ctx, x, y, s, out, nullptr, false);
}

int tw_solve_pair(tw_ctx* ctx, const tw_image* a, const tw_image* b, const tw_flow_settings* s, tw_flow* f_ab,
                  tw_flow* f_ba) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!f_ab || !f_ba) return ctx->fail(TW_ERR_BAD_PARAM, "no output flow");
    return solve_common(ctx, a, b, s, f_ab, f_ba, true);
}

int tw_build_pyramid(tw_ctx* ctx, const tw_image* img, const tw_flow_settings* s, float* levels_out) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    CHECK(check_image(ctx, img, "build_pyramid"));
    if (!s || !levels_out) return ctx->fail(TW_ERR_BAD_PARAM, "missing argument");
    Geo g;
    CHECK(geometry(*s, img->width, img->height, &g, &ctx->err));
    CHECK(upload_image(ctx, ctx->eng[0], img));
    size_t pf = pyramid_floats(g);
    CHECK(ctx->ensure(ctx->pyr[0], 2 * pf * 4, "pyramid"));
    CHECK(build_pyramid_dev(ctx, ctx->eng[0].p, img->width, img->height, img->fmt, *s, g, ctx->pyr[0].as<float>(),
                            ctx->pyr[0].as<float>() + pf, ctx->plane));
    CHECK(ctx->cuda(cudaMemcpyAsync(levels_out, ctx->pyr[0].p, pf * 4, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

int tw_block_match(tw_ctx* ctx, const float* a, const float* b, float* flow, int32_t width, int32_t height) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (!a || !b || !flow || width <= 0 || height <= 0) return ctx->fail(TW_ERR_BAD_PARAM, "bad argument");
    if (width > BM_MAX_LINE || height > BM_MAX_LINE) return ctx->fail(TW_ERR_UNSUPPORTED, "block matching: a side above 6144");
    size_t n = (size_t)width * height;
    CHECK(ctx->ensure(ctx->plane[0], n * 4, "plane A"));
    CHECK(ctx->ensure(ctx->plane[1], n * 4, "plane B"));
    CHECK(ctx->ensure(ctx->plane[2], n * 8, "flow"));
    CHECK(ctx->ensure(ctx->work[0], n * 4 * 6, "flow planes"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->plane[0].p, a, n * 4, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->plane[1].p, b, n * 4, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    CHECK(ctx->cuda(cudaMemcpyAsync(ctx->plane[2].p, flow, n * 8, cudaMemcpyHostToDevice, ctx->stream), "upload"));
    float* fu = ctx->work[0].as<float>();
    float* fv = fu + n;
    float *at = fv + n, *bt = at + n, *ut = bt + n, *vt = ut + n;
    LAUNCH(ctx, k_deinterleave, grid1((long)n), TB, 0, ctx->plane[2].as<float>(), (long)n, fu, fv);
    LAUNCH(ctx, k_transpose2, dim3((width + 31) / 32, (height + 31) / 32), dim3(32, 8), 0, ctx->plane[0].as<float>(),
           ctx->plane[1].as<float>(), at, bt, width, height);
    block_match(ctx, ctx->plane[0].as<float>(), ctx->plane[1].as<float>(), at, bt, fu, fv, ut, vt, width, height);
    LAUNCH(ctx, k_interleave, grid1((long)n), TB, 0, fu, fv, (long)n, ctx->plane[2].as<float>());
    CHECK(ctx->cuda(cudaMemcpyAsync(flow, ctx->plane[2].p, n * 8, cudaMemcpyDeviceToHost, ctx->stream), "download"));
    int hf[1];
    return finish(ctx, hf, 1);
}

}  // extern "C"
