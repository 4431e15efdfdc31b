// Declarations of the library's sm_100a kernels (strict mode) and their small device helpers.
//
// Layout in HBM: every multi channel buffer of the solver is PLANAR (one float plane per channel,
// row major, pitch = width), so each pass streams coalesced lanes and the separable filter runs
// the same code on each plane. The reference's interleaved layout only changes where samples
// live, never the arithmetic of an element, so results are bit identical. Engine images keep the
// reference's interleaved A, R, G, B samples (one 32-bit word per 8 bpc pixel).
#pragma once
#include <cstdint>

#include "strict.cuh"

// The solver's translation units (fused.cu, solver.cu, coarse.cu) are compiled twice: in strict mode,
// and for the fast mode (TW_FAST_VARIANT: FMA contraction, approximate division and square root,
// denormals flushed), whose kernels land in namespace tw::fast (declared in kernels_fast.cuh).
#ifdef TW_FAST_VARIANT
#define TW_VARIANT_BEGIN namespace fast {
#define TW_VARIANT_END }
#else
#define TW_VARIANT_BEGIN
#define TW_VARIANT_END
#endif

namespace tw {

constexpr int MAX_TAPS = 8;  // Gaussian r=7 has 8 half taps (flow/conv.rs:64-86)

struct Taps {
    float k[MAX_TAPS];
    int n;
};
// the half kernels of the matte choke's blur (matte.rs:366-385: radius a + 2.01 for a shrink of a
// pixels, n = a + 3 taps for a whole a); shrinks up to 13 pixels
constexpr int MAX_WIDE_TAPS = 16;
struct WideTaps {
    float k[MAX_WIDE_TAPS];
    int n;
};

// ---- image boundary and luma (image.rs, prep.rs) -------------------------------------------------
// wire -> engine, optionally reading the wire rows bottom up (the motion path's row order)
__global__ void k_from_frame_u8(const uint8_t* __restrict__ wire, uint8_t* __restrict__ eng, int w, int h, bool flip);
__global__ void k_from_frame_u16(const uint16_t* __restrict__ wire, uint16_t* __restrict__ eng, int w, int h, bool flip);
__global__ void k_from_frame_f32(const float* __restrict__ wire, float* __restrict__ eng, int w, int h, bool flip);
// engine -> wire, optionally reading the engine rows bottom up
__global__ void k_to_frame_u8(const uint8_t* __restrict__ eng, uint8_t* __restrict__ wire, int w, int h, bool flip);
__global__ void k_to_frame_u16(const uint16_t* __restrict__ eng, uint16_t* __restrict__ wire, int w, int h, bool flip);
__global__ void k_to_frame_f32(const float* __restrict__ eng, float* __restrict__ wire, int w, int h, bool flip);
__global__ void k_luma(const void* __restrict__ eng, int fmt, float* __restrict__ out, int w, int h, bool track_alpha,
                       bool video_range);

// ---- separable filters and resampling (flow/conv.rs, flow/sample.rs) -------------------------------
__global__ void k_conv_h(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t, bool multi);
// vertical pass; when band != nullptr it also writes band = orig - result (flow.rs:266-267)
__global__ void k_conv_v(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t, bool multi,
                         bool above_first, const float* __restrict__ orig, float* __restrict__ band);
__global__ void k_conv_h_wide(const float* __restrict__ src, float* __restrict__ dst, int w, int h, WideTaps t);
__global__ void k_conv_v_wide(const float* __restrict__ src, float* __restrict__ dst, int w, int h, WideTaps t,
                              bool above_first);
__global__ void k_resample(const float* __restrict__ src, int sw, int sh, float* __restrict__ dst, int dw, int dh);
// the 360 mode of the pyramid's filters: circular rows, equirectangular columns and resample
__global__ void k_conv_h_wrap(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t);
__global__ void k_conv_v_sphere(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t,
                                const float* __restrict__ orig, float* __restrict__ band, float* __restrict__ band_t);
__global__ void k_resample_sphere(const float* __restrict__ src, int sw, int sh, float* __restrict__ dst, int dw, int dh);

// ---- solver (flow.rs:277-442) ------------------------------------------------------------------------
// gradient (2 planes) and structure tensor (3 planes)
__global__ void k_grad_tensor(const float* __restrict__ img, int w, int h, float* __restrict__ gx,
                              float* __restrict__ gy, float* __restrict__ a0, float* __restrict__ a1,
                              float* __restrict__ a2);
__global__ void k_calc_b(const float* __restrict__ i1, const float* __restrict__ i0, const float* __restrict__ gx,
                         const float* __restrict__ gy, const float* __restrict__ fu, const float* __restrict__ fv,
                         int w, int h, float* __restrict__ bx, float* __restrict__ by);
__global__ void k_new_disp(float* __restrict__ fu, float* __restrict__ fv, const float* __restrict__ a0,
                           const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ bx,
                           const float* __restrict__ by, long n);
// sets *any_in_range when some pixel's x + u, y + v lies inside the level (flow.rs:430-442)
__global__ void k_range_any(const float* __restrict__ fu, const float* __restrict__ fv, int w, int h,
                            int* __restrict__ any_in_range);
// the range reset while the check is live, then the damping of the start level (flow.rs:1292-1300)
__global__ void k_range_apply(float* __restrict__ fu, float* __restrict__ fv, long n, int* __restrict__ state,
                              bool damp_now, float damp);
__global__ void k_range_init(int* __restrict__ state);
__global__ void k_range_next(int* __restrict__ state);
__global__ void k_upsample_flow(const float* __restrict__ su, const float* __restrict__ sv, int sw, int sh,
                                float* __restrict__ du, float* __restrict__ dv, int dw, int dh);
// the final negation (flow.rs:1305) into the interleaved FlowField layout
__global__ void k_negate_interleave(const float* __restrict__ fu, const float* __restrict__ fv, long n,
                                    float* __restrict__ out, int* __restrict__ nan_flag);
__global__ void k_fill(float* __restrict__ p, long n, float v);
__global__ void k_deinterleave(const float* __restrict__ in, long n, float* __restrict__ fu, float* __restrict__ fv);
__global__ void k_interleave(const float* __restrict__ fu, const float* __restrict__ fv, long n, float* __restrict__ out);

// block matching (flow.rs:447-622): the four sweeps; one CTA per row or column, bm_smem_bytes(line)
// shared. k_bm_rows: both sweeps of every row (left to right, then right to left) of (fu, fv), the
// result written into the transposes (uT, vT; element (x, y) at [x * h + y]); k_bm_cols: both
// sweeps of every column (top to bottom, then bottom to top) read from (uT, vT), with the
// transposes of A and B, the result written back into (fu, fv). Lines 0 and last are not swept.
__global__ void k_bm_rows(const float* __restrict__ A, const float* __restrict__ B, const float* __restrict__ fu,
                          const float* __restrict__ fv, int w, int h, float* __restrict__ uT, float* __restrict__ vT);
__global__ void k_bm_cols(const float* __restrict__ AT, const float* __restrict__ BT, const float* __restrict__ uT,
                          const float* __restrict__ vT, int w, int h, float* fu, float* fv);
// two w x h planes into their h x w transposes; block (32, 8), grid (ceil(w/32), ceil(h/32))
__global__ void k_transpose2(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ at,
                             float* __restrict__ bt, int w, int h);
size_t bm_smem_bytes(int len);
// longest row or column block matching keeps in shared memory (9 arrays of 4-byte values per element)
constexpr int BM_MAX_LINE = 6144;

// ---- warps and blends (warp.rs, blend.rs) ------------------------------------------------------------
struct WarpParams {
    const void* src;     // engine image
    const float* fu;     // flow u (element stride fstride)
    const float* fv;
    int fstride;
    int fw, fh;
    float amount;
    // warp.rs:636-651: the flow's ratios to the image, rx = (fw - 1) / (w - 1), ry likewise, and the
    // steps sx = amount / rx, sy = amount / ry, single precision, formed once on the host (the same
    // IEEE divisions the kernel made per pixel)
    float rx, ry, sx, sy;
    bool copy_only;      // the |amount| early outs of inv_warp (warp.rs:751-764)
    bool hold;
    bool is360;          // wrap-around: the point wrapped into the image, the pole reflection, the 360 sampler
};
// out = inv_warp(src, flow, amount); optional coverage
__global__ void k_inv_warp(WarpParams p, int fmt, void* __restrict__ out, uint8_t* __restrict__ cov, int w, int h,
                           int* __restrict__ bad);
// out = blend(a, b, w) for the common branch (blend.rs:81-114); the snap / extrapolation branches
// are decided on the host
__global__ void k_blend(const void* __restrict__ a, const void* __restrict__ b, void* __restrict__ out, int fmt,
                        long nsamples, float w);
// lerp(first, second, w) in place (blend.rs:144-258)
__global__ void k_lerp(void* __restrict__ first, const void* __restrict__ second, int fmt, long npx, float w);

// The fused Blend composition of warping code 0 (compose/vector.rs:262-276): both inverse warps,
// the blend and (to_wire) the unpremultiply + wire store of the finish, rows optionally read
// bottom up on the way out. `blend_mode`: 0 common branch, 1 copy of tA, 2 copy of tB.
__global__ void k_compose_blend(WarpParams pa, WarpParams pb, int fmt, float wblend, int blend_mode, void* __restrict__ out,
                                int w, int h, bool to_wire, bool flip_out, int* __restrict__ bad);

// ---- fused, shared-memory tiled kernels (fused.cu) -----------------------------------------------------
constexpr int FUSED_TILE_X = 32, FUSED_TILE_Y = 32, FUSED_THREADS = 256;
__global__ void k_blur5_band(const float* __restrict__ orig, const void* __restrict__ luma_src, int fmt, int luma_mode,
                             int w, int h, bool above_first, float* __restrict__ tmp_out, float* __restrict__ band_out,
                             float* __restrict__ band_t_out);
__global__ void k_level_init(const float* __restrict__ img, int w, int h, Taps g7, bool above_first,
                             float* __restrict__ gxo, float* __restrict__ gyo, float* __restrict__ a0o,
                             float* __restrict__ a1o, float* __restrict__ a2o, const float* __restrict__ mask,
                             const float* __restrict__ fu, const float* __restrict__ fv, const float* __restrict__ i0,
                             const float* __restrict__ mask_y, float* __restrict__ b_out, int bp, long bplane);
__global__ void k_calc_b_pitched(const float* __restrict__ i1, const float* __restrict__ i0,
                                 const float* __restrict__ gx, const float* __restrict__ gy,
                                 const float* __restrict__ fu, const float* __restrict__ fv, int w, int h,
                                 const float* __restrict__ mask_y, float* __restrict__ b_out, int bp, long bplane);
__global__ void k_binarize(float* __restrict__ p, long n);
size_t level_init_smem();
// One solver iteration (blur7 of B, new_disp, blur5 of the flow, then calc_b of the next iteration
// at its outputs when b_out is given) over TX x TY tiles: one kernel per tile shape; the host picks
// the shape per level size (its tuning table). B planes: pitch bp (a multiple of 4 floats), plane
// stride bplane, 16-byte aligned.
enum { LEVEL_TILE_32x32 = 0, LEVEL_TILE_64x32 = 1, LEVEL_TILE_64x64 = 2, LEVEL_TILE_COUNT = 3 };
constexpr int LEVEL_ITER_MAX_THREADS = 512;
#define TW_DECLARE_LEVEL_ITER(TX, TY)                                                                                 \
    __global__ void k_level_iter_##TX##x##TY(                                                                       \
        const float* __restrict__ b_in, int bp, long bplane, const float* __restrict__ i1,                          \
        const float* __restrict__ i0, const float* __restrict__ gx, const float* __restrict__ gy,                    \
        const float* __restrict__ a0, const float* __restrict__ a1, const float* __restrict__ a2,                    \
        const float* __restrict__ fu, const float* __restrict__ fv, int w, int h, Taps g7, Taps g5,                  \
        bool above_first, float* __restrict__ fu_out, float* __restrict__ fv_out, const float* __restrict__ mask_y,  \
        float* __restrict__ b_out);
TW_DECLARE_LEVEL_ITER(32, 32)
TW_DECLARE_LEVEL_ITER(64, 32)
TW_DECLARE_LEVEL_ITER(64, 64)
#undef TW_DECLARE_LEVEL_ITER
size_t level_iter_smem(int tile);

// The persistent coarse-level solve (coarse.cu): one block walks the levels start .. last of a solve
// whose planes fit its shared memory (at most COARSE_MAX_PIXELS pixels and COARSE_MAX_LINE per side;
// last >= 1), and writes the upsampled flow of level last - 1 (planar) for the tiled kernels.
constexpr int COARSE_THREADS = 1024;
constexpr int COARSE_MAX_PIXELS = 2048;
constexpr int COARSE_MAX_LINE = 128;
struct CoarseJob {
    const float* x;  // the band pyramids of X and Y, levels concatenated finest first
    const float* y;
    int sizes[32][2];
    int offs[32];  // the first element of each level
    int start, last;
    bool damp_any;  // the start level's damping differs from 1
    float damp;
    bool refine;  // block matching (not skip_refine)
    bool af;      // the vertical tap above first
    Taps g7, g5;
    int* any;  // the per level range flags (32 ints, zeroed before)
    float* fu_out;
    float* fv_out;
};
__global__ void k_solve_coarse(CoarseJob job);
size_t coarse_smem_bytes();
__global__ void k_apply_upsample(const float* __restrict__ su, const float* __restrict__ sv, int sw, int sh,
                                 const int* __restrict__ any, int l, int start, bool damp_now, float damp,
                                 float* __restrict__ du, float* __restrict__ dv, int dw, int dh);
__global__ void k_apply_negate(const float* __restrict__ fu, const float* __restrict__ fv, long n,
                               const int* __restrict__ any, int start, bool damp_now, float damp,
                               float* __restrict__ out, int* __restrict__ nan_flag);

// ---- warping code 1: Smart Blend and the hole fill (smart.cu) -----------------------------------------
// mode 0: Nearest (the warp pa only), 1: Blend (pa = A, pb = B, w = frac); binary: the binary alpha
// composite. Writes the engine image, the u8 holes mask and sets *any_hole when a pixel is a hole.
__global__ void k_compose_smart(WarpParams pa, WarpParams pb, int fmt, int mode, float w, bool binary,
                                void* __restrict__ out, uint8_t* __restrict__ holes, int W, int H,
                                int* __restrict__ any_hole, int* __restrict__ bad);
__global__ void k_smart_blend(const void* __restrict__ p1, const void* __restrict__ p2, int fmt, float w, bool binary,
                              void* __restrict__ out, long n);
__global__ void k_cov_holes(const uint8_t* __restrict__ c1, const uint8_t* __restrict__ c2, uint8_t* __restrict__ holes,
                            long n, int* __restrict__ any_hole);
__global__ void k_mask_holes(const void* __restrict__ mask, int kind, uint8_t* __restrict__ holes, long n,
                             int* __restrict__ any_hole);
// The format code of an interleaved 2 channel flow in the hole fill (k_fill_load, k_fill_store, fill_dev)
constexpr int FILL_FLOW = 3;
__global__ void k_fill_load(const void* __restrict__ img, int fmt, const uint8_t* __restrict__ holes,
                            float* __restrict__ stack, long n, const int* __restrict__ any_hole);
// both passes of the fill's blur (horizontal, then vertical, the vertical border taps above first
// with above_first) out of place, 32 x 32 output tiles per block and plane; 256 threads; n: 3
// (blur5) or 6 (Gaussian r5) taps; rule: the NaN rule arithmetic (float images and flows)
__global__ void k_stack_blur(const float* __restrict__ src, float* __restrict__ dst, int w, int h, long pstride, Taps t,
                             int n, int above_first, int rule, const int* __restrict__ any_hole);
__global__ void k_stack_resample(const float* __restrict__ src, int sw, int sh, long sstride, float* __restrict__ dst,
                                 int dw, int dh, long dstride, int rule, const int* __restrict__ any_hole);
__global__ void k_fill_combine(float* __restrict__ sol, const float* __restrict__ vals, long n, int nc, int rule,
                               const int* __restrict__ any_hole);
__global__ void k_fill_store(void* __restrict__ img, int fmt, const float* __restrict__ sol, long n,
                             const int* __restrict__ any_hole);
__global__ void k_stack_zero(float* __restrict__ p, long n, const int* __restrict__ any_hole);
__global__ void k_hole_side1(const int* __restrict__ any_hole, int* __restrict__ flag);
// The coarse levels of the pull-push fill in one block: the pull from level k0 (its stack given,
// np planes) up to the top level and the push from the top down to level k0, every stack of those
// levels in shared memory; the push's result resampled to level k0 - 1 goes to out (nc planes of
// that level). Level sizes as the fill's geometry (holefill.rs:140-171). fill_coarse_floats: the
// shared memory it needs, in floats.
constexpr int FILL_COARSE_THREADS = 1024;
constexpr int FILL_COARSE_MAX_FLOATS = 50 * 1024;  // 200 KB
struct FillCoarseJob {
    const float* s_k0;
    float* out;
    int dims[40][2];
    int k0, top, np, nc, rule, above_first;
    Taps b5, g5;
    const int* any;
};
__global__ void k_fill_coarse(FillCoarseJob J);
long fill_coarse_floats(const int dims[][2], int k0, int top, int np, int nc);

__global__ void k_encode_vectors(const float* __restrict__ flow, int fw, int fh, void* __restrict__ out, int W, int H,
                                 int fmt, float sx, float sy, float kx, float ky, int zero);

// ---- the layered composition with plates (layers.cu) -----------------------------------------------
__global__ void k_matte_extract(const void* __restrict__ wire, int fmt, int chan, int w, int h, bool flip,
                                float* __restrict__ out);
__global__ void k_matte_out_of_range(const float* __restrict__ m, long n, int* __restrict__ flag);
__global__ void k_raw_plane(const float* __restrict__ m, long n, int fmt, const int* __restrict__ clamp,
                            float* __restrict__ out);
__global__ void k_comp_plane(const float* __restrict__ raws, const float* __restrict__ cuts, int nfg, int k, long n,
                             int fmt, float* __restrict__ out);
// one choke of the cut (matte.rs:280-310): host scalars of its shrink steps
struct ChokeStep {
    bool grow, lo_blur, hi_blur, mix;
    float t_lo, t_hi, t;     // the thresholds of the steps by lo and hi; the mix weight a - lo
    double den_lo, den_hi;   // 1 - (double)threshold
};
__global__ void k_choke_base(const float* __restrict__ raw, long n, float kk, bool grow, float* __restrict__ out);
__global__ void k_choke_finish(const float* __restrict__ base, const float* __restrict__ b_lo,
                               const float* __restrict__ b_hi, ChokeStep st, long n, float* __restrict__ out);
__global__ void k_flip_rows(const void* __restrict__ src, void* __restrict__ dst, int w, int h, int px);
// ---- tracking points (points.rs:112-240, flow/extras.rs:181-215) -----------------------------------
constexpr int MAX_USER_PAIRS = 12;  // the twelve Track Points of the effects
struct UserPairs {
    int n;
    float p[MAX_USER_PAIRS][4];  // (from x, from y, to x, to y) in output pixels, point order
};
__global__ void k_user_splat(UserPairs pairs, int w0, int h0, int W, int H, float* __restrict__ du,
                             float* __restrict__ dv, float* __restrict__ uw);
__global__ void k_user_finest(float* __restrict__ du, float* __restrict__ dv, float* __restrict__ uw, long n);
__global__ void k_user_scale(float* __restrict__ du, float* __restrict__ dv, long n, float sx, float sy);
__global__ void k_apply_user(float* __restrict__ fu, float* __restrict__ fv, const float* __restrict__ du,
                             const float* __restrict__ dv, const float* __restrict__ uw, long n);
__global__ void k_solver_mask(const float* __restrict__ raws, int nfg, int k, const float* __restrict__ comp, long n,
                              int fmt, float* __restrict__ out);
__global__ void k_layer_times(const void* __restrict__ src, const float* __restrict__ p, void* __restrict__ out, int fmt,
                              long n);
__global__ void k_over_pl(void* __restrict__ dest, const void* __restrict__ src, int fmt, long n);
__global__ void k_refill_pre(void* __restrict__ img, int fmt, long n, uint8_t* __restrict__ holes,
                             int* __restrict__ any_hole);
__global__ void k_refill_post(void* __restrict__ img, int fmt, long n, const float* __restrict__ plane,
                              const void* __restrict__ frame);

// ---- the forward warp (forward.cu) ---------------------------------------------------------------------
struct FwGrid {  // forward/mesh.rs:11-26
    int w, h;
    float rx, ry, sx, sy;
};
constexpr int FW_MAX_LEVELS = 16;
struct FwLevels {  // level 0 is the source
    const void* p[FW_MAX_LEVELS];
    int w[FW_MAX_LEVELS], h[FW_MAX_LEVELS];
    int count;
};
struct FwRaster {
    int w, h, fmt;
    bool pyramid;                     // textured (true) or Gouraud
    const float *vx, *vy, *vd;        // vertex positions, mip levels (null: all 0)
    FwLevels levels;
    uint32_t *cnt, *off, *fill;       // per pixel: hit count, segment start, hits written
    uint32_t* keys;                   // per hit: triangle index
    float4* cols;                     // per hit: colour
    void* out;
    uint8_t* cov;                     // may be null
    int *outside, *bad;
    uint32_t *nlong, *longq;          // the queue of pixels with long hit lists
    uint2* scratch;                   // 2 * total pairs for lists above the shared memory sort
    uint32_t total;
};
__global__ void k_logf_glibc(const float* __restrict__ x, float* __restrict__ out, long n, const uint2* __restrict__ tab,
                             int ntab);
__global__ void k_fw_flow_nonzero(const float* __restrict__ flow, long n, int* __restrict__ flag);
__global__ void k_fw_vertices(const float* __restrict__ flow, int fw, int fh, FwGrid g, float* __restrict__ vx,
                              float* __restrict__ vy, float* __restrict__ vd, float inv_ln2,
                              const uint2* __restrict__ tab, int ntab);
__global__ void k_fwp_blur(const void* __restrict__ in, void* __restrict__ out, int w, int h, int vertical, int fmt);
__global__ void k_fwp_resample(const void* __restrict__ src, int sw, int sh, void* __restrict__ dst, int dw, int dh,
                               int fmt);
__global__ void k_fw_count(FwRaster R);
__global__ void k_fw_emit(FwRaster R);      // the Gouraud variant
__global__ void k_fw_emit_tex(FwRaster R);  // the textured variant (R.pyramid)
constexpr int FW_SCAN_BLOCK = 2048;
__global__ void k_scan_block(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, long n,
                             uint32_t* __restrict__ sums, uint32_t* __restrict__ maxc);
__global__ void k_scan_sums(uint32_t* __restrict__ sums, int nb, unsigned long long* __restrict__ total);
__global__ void k_scan_add(uint32_t* __restrict__ out, long n, const uint32_t* __restrict__ sums);
__global__ void k_fw_resolve(FwRaster R);
constexpr int FW_LONG_SMEM_BYTES = 4096 * 8;
__global__ void k_fw_resolve_long(FwRaster R);

// ---- the Weighted Blend filters (filters.cu, filters.rs) ----
struct WbTaps {  // the half kernel of the sharpening blur (filters.rs:75-93), w[0] the centre
    float w[8];
    int count;
};
__global__ void k_wb_blur(const void* __restrict__ src, void* __restrict__ dst, int fmt, int w, int h, WbTaps T, bool cols,
                          bool above_first, const int* __restrict__ gate);
__global__ void k_wb_diff_mask(const void* __restrict__ a, const void* __restrict__ b, int fmt, long n, float limit,
                               uint8_t* __restrict__ mask, const int* __restrict__ gate);
__global__ void k_mask_prune(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int w, int h, int limit,
                             const int* __restrict__ gate);
__global__ void k_mask_dilate(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int w, int h,
                              const int* __restrict__ gate);
__global__ void k_mask_fill_border(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int w, int h, int limit,
                                   int value, const int* __restrict__ gate);
__global__ void k_mask_clean_small(uint8_t* __restrict__ m, uint8_t* __restrict__ scratch, int w, int h,
                                   const int* __restrict__ gate);
__global__ void k_wb_finish(void* __restrict__ frame, const void* __restrict__ blurred, const uint8_t* __restrict__ mask,
                            int fmt, long n, float c, const int* __restrict__ gate);
__global__ void k_f32_unsound(const float* __restrict__ a, long n, int* __restrict__ flag);
__global__ void k_copy_gated(const uint4* __restrict__ src, uint4* __restrict__ dst, long n, const int* __restrict__ gate);
__global__ void k_wb_noflow_f32(const float* __restrict__ a, const float* __restrict__ b, const float* __restrict__ a1,
                                const float* __restrict__ b1, const int* __restrict__ unsound, float w, float wl, int mode,
                                float* __restrict__ out, long n);

// ---- the image prep (prep.cu, prep.rs) ----
__device__ float crt_powf(float x, float y);
// the same powf on the host (the matte choke's Gaussian taps)
float crt_powf_host(float x, float y);
__global__ void k_delinearize(float* __restrict__ p, long n);
__global__ void k_edge_map(const float* __restrict__ src, float* __restrict__ dst, int w, int h);
__global__ void k_check_powf(const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ out, long n);

// ---- Blur Compensation (filters.cu, warp/blurcomp.rs) ----
struct MotionBlur {
    const void* src;
    void* dst;
    WarpParams flow;  // the flow field of the blur (fu, fv, fstride, fw, fh)
    int fmt, w, h;
    float rx, ry, kx, ky, k;
    bool shifted, bilinear;
    int post;        // 0 none, 1 clear the colour of transparent pixels, 2 lerp(dst, src, lerp_w)
    float lerp_w;
    int* bad;        // bit 2: a NaN tap or a vector of more than 65536 taps
};
__global__ void k_motion_blur(MotionBlur B);

// ---- the adjoint of warp + blend (adjoint.cu) ----
struct AdjParams {
    const float* a;         // batch x (w x h x 4)
    const float* b;
    const float* f_ab;      // batch x (fw x fh x 2), interleaved
    const float* f_ba;
    const float* target;    // the L1 loss against it (nullptr: grad_out drives the backward)
    const float* grad_out;  // d loss / d out (nullptr with target == nullptr: forward only)
    float* out;             // the forward output (nullptr: not written)
    float* loss;            // batch sums of |out - target| (accumulated)
    float* da;              // the gradients (accumulated; nullptr: not computed)
    float* db;
    float* df_ab;
    float* df_ba;
    int w, h, fw, fh;
    float rx, ry, wa;
    bool tiled;             // rx <= 1 and ry <= 1: the flow gradients gather in shared memory first
};
constexpr int ADJ_TX = 32, ADJ_TY = 32, ADJ_THREADS = 256;  // the output tile of a CTA
constexpr int ADJ_BOX_PX = 1536;                            // the shared image gradient tile, per side
// dynamic shared memory: two image tiles (float4) and two flow tiles ((TX + 2) x (TY + 2) x 2 floats)
constexpr int ADJ_SMEM = 2 * ADJ_BOX_PX * 16 + 2 * (ADJ_TX + 2) * (ADJ_TY + 2) * 2 * 4;
__global__ void k_warp_blend_adjoint(AdjParams P);

// ---- Vectors In (vecin.cu) ----
// vectors.rs:474-528 + :555-561 with the hole rule of holefill.rs:124-133: the flow of an encoded
// engine image (interleaved) and its hole flags (the inverted alpha at or above eps), *any_hole set
// when one is a hole
__global__ void k_vec_decode(const void* __restrict__ vec, int fmt, float md, float2* __restrict__ flow,
                             uint8_t* __restrict__ holes, long n, int* __restrict__ any_hole);
// vectors.rs:573-578: Vec Scale
__global__ void k_vec_scale(float2* __restrict__ flow, long n, float sx, float sy);
// compose/vector.rs:376-384: T = (-1 * 1, -1 * fx, -1 * fy, -1 * 1)
__global__ void k_invert_prep(const float2* __restrict__ flow, float4* __restrict__ t, long n);
// compose/vector.rs:386-395: channels 1 and 2 of the pushed image as the flow, the inverted coverage
// as the holes (a hole where 255 - coverage is not 0)
__global__ void k_invert_take(const float4* __restrict__ pushed, const uint8_t* __restrict__ cov,
                              float2* __restrict__ flow, uint8_t* __restrict__ holes, long n, int* __restrict__ any_hole);
// plugins/vectors-in/src/vectorin.rs:125-155: the alpha of an engine image capped by a matte in
// the units of the depth
__global__ void k_matte_step(void* __restrict__ img, int fmt, const float* __restrict__ matte, long n);

// ---- the Debug views of Create Vectors (debug.cu, debug.rs) ----
// debug.rs:155-171 Blend: W' lerped towards Y by 0.5 (copy then lerp)
__global__ void k_debug_blend(const void* __restrict__ wp, const void* __restrict__ y, int fmt, void* __restrict__ out,
                              long n);
// debug.rs:437-476: the grey Diff of W' and Y
__global__ void k_debug_diff(const void* __restrict__ wp, const void* __restrict__ y, int fmt, void* __restrict__ out,
                             long n);
// debug.rs:285-310: the luma plane of the Detail and Edge views
__global__ void k_debug_luma(const void* __restrict__ img, int fmt, float* __restrict__ out, long n);
// debug.rs:318-434: the Detail (edge == 0) or Edge measure of both luma planes and the overlay
__global__ void k_debug_overlay(const float* __restrict__ lw, const float* __restrict__ ly, int w, int h, int fmt,
                                int edge, void* __restrict__ out);

}  // namespace tw
