/*
 * twixtor_b200: the retime hot path of baairon/twixtor (plugins/retime-engine) as sm_100a CUDA
 * behind a C ABI.
 *
 * Conventions
 *   - Images are engine images: 4 channels interleaved in the order A, R, G, B, colour
 *     PREMULTIPLIED by alpha, rows tightly packed, top row first; 8 bpc (uint8), 16 bpc (uint16,
 *     full range 0..65535) or 32 bpc (float, white 1.0). This is `image::Image`
 *     (plugins/retime-engine/src/image.rs:17-73).
 *   - Wire frames are the host's frames (crates/fx-core/src/frame.rs:79-131): 8 bpc RGBA
 *     interleaved, 16 bpc RGBA little endian interleaved (range 0..65535), 32 bpc planar in the
 *     plane order G, B, R, A.
 *   - Flows are `flow::FlowField` (flow.rs:37-76): width * height * 2 floats, (dx, dy) interleaved,
 *     at the working resolution of the estimator.
 *   - The caller owns every host buffer it passes; the library owns the device memory and the
 *     CUDA context state. Every call is synchronous at the ABI. One tw_ctx may be used from one
 *     thread at a time (the reference's device backend serialises its queue behind a mutex,
 *     device/exec/backend.rs:121-181; tw_ctx holds a mutex too).
 *   - Every call returns a tw_status; TW_OK is 0. tw_last_error() names the cause of the last
 *     failure on the context. Nothing is ever computed on the CPU: a stage the device cannot
 *     serve returns TW_ERR_UNSUPPORTED and the caller decides (the reference's executor reruns
 *     the CPU stage, device/exec/mod.rs:332-369).
 *
 * Strict mode: every kernel repeats the reference CPU engine's single precision operation order
 * with no FMA contraction, IEEE division, x86 truncating conversions and the reference's double
 * precision steps, so flows and output frames are bit identical to the CPU path on identical
 * inputs (finite inputs; a NaN anywhere in a solved flow returns TW_ERR_NAN_OUTPUT, as the
 * reference device path's download does, device/solver/mod.rs:575).
 */
#ifndef TWIXTOR_B200_H
#define TWIXTOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; map 1:1 onto the reference's `StageError` (device/image.rs:14-23): Cl -> TW_ERR_CUDA,
 * NanOutput -> TW_ERR_NAN_OUTPUT, Unsupported -> TW_ERR_UNSUPPORTED; TW_ERR_MISMATCH and
 * TW_ERR_BAD_PARAM are the CPU functions' FxError::Mismatch and FxError::BadParam. */
typedef enum tw_status {
    TW_OK = 0,
    TW_ERR_CUDA = 1,
    TW_ERR_NAN_OUTPUT = 2,
    TW_ERR_UNSUPPORTED = 3,
    TW_ERR_MISMATCH = 4,
    TW_ERR_BAD_PARAM = 5,
    TW_ERR_DEVICE_BOUND = 6, /* a data-dependent device loop reached its bound (never for finite data) */
    TW_ERR_TOO_LARGE = 7     /* tw_block_match_noalloc: width * height above TW_NOALLOC_MAX_PIXELS */
} tw_status;

typedef enum tw_fmt { TW_U8 = 0, TW_U16 = 1, TW_F32 = 2 } tw_fmt;

typedef struct tw_ctx tw_ctx;

/* An engine image (image.rs:66-71). `data` holds width * height * 4 samples of `fmt`; `bytes` is the
 * size of the caller's buffer behind `data`. A buffer shorter than the image needs is refused with
 * TW_ERR_BAD_PARAM before anything is read or written (the reference's slices carry their length;
 * a C pointer does not). */
typedef struct tw_image {
    int32_t width, height, fmt;
    const void* data;
    size_t bytes;
} tw_image;

typedef struct tw_image_mut {
    int32_t width, height, fmt;
    void* data;
    size_t bytes;
} tw_image_mut;

/* flow::FlowField (flow.rs:37-76). */
typedef struct tw_flow {
    int32_t width, height;
    float* data;
} tw_flow;

/* flow::FlowSettings (flow.rs:83-123), plus the vertical tap order of the solver's separable
 * filters: 1 = the tap above first (flow/conv.rs:598-615, the reference's order); 0 = below
 * first (the order of the reference revision its parity grid records). */
typedef struct tw_flow_settings {
    int32_t quality;          /* 1..5 */
    int32_t hiq;              /* high quality render */
    float sensitivity;        /* slider / 100 */
    int32_t prep_contrast_edge;
    int32_t prep_delinearize;
    int32_t track_alpha;
    int32_t video_range_luma;
    int32_t skip_refine;
    int32_t wrap;             /* 360 solve: TW_ERR_UNSUPPORTED */
    int32_t taps_above_first;
    int32_t fast_mode;        /* 0: strict (bit identical to the CPU path); 1: the solver's kernels (pyramid,
                                 iterations, block matching) as built with FMA contraction, approximate division
                                 and flushed denormals: not bit identical; the library's tests state its flow
                                 error in pixels and frame PSNR against a double precision CPU restatement */
} tw_flow_settings;

/* timeline::Selection (timeline.rs:391-414). */
typedef struct tw_selection {
    float s0, s1;
    int32_t a, b;
    float wa;
    int32_t exact;
    int32_t vectors_quality;
    int32_t interp;           /* 0 Nearest, 1 Blend, 2 Weighted Blend */
} tw_selection;

/* The part of host::EngineSettings (host.rs:20-100) that compose_vectors reads. */
typedef struct tw_engine_settings {
    int32_t warp_mode;        /* 0 inverse, 1 Smart Blend, 2 forward + fill, 3 forward */
    int32_t video_360;        /* "360 Video" checkbox */
    int32_t wrap_360;         /* engine wrap-around flag */
    int32_t quality_high;
    float blur;               /* Blur Compensation slider */
    int32_t taps_above_first; /* Stages::vertical_taps() of the stage set (stages.rs:66-70) */
    int32_t gouraud;          /* forward warps of codes 2/3 as the Gouraud variant: the stage set is
                                 wrapped in stages::GouraudForward (stages.rs:101-129), as retime-fgbg's
                                 is (plugins/retime-fgbg/src/glue.rs:142-143); 0 the textured warp */
} tw_engine_settings;

/* Everything one output frame of the `retime` effect needs beyond its selection: the flow
 * settings, the compose settings and the row order of the motion path
 * (EngineSettings::motion_rows_reversed, host.rs; plugin 01 sets it, plugins/retime/src/glue.rs:39-40). */
typedef struct tw_retime_settings {
    tw_flow_settings flow;
    tw_engine_settings compose;
    int32_t motion_rows_reversed;
} tw_retime_settings;

/* The Create Vectors pass of one layer (create_vectors.rs:97-135): the solver settings (quality 4
 * Normal (half res) or 5 Full res, hiq, sensitivity, track_alpha for Track RGB+A, the tap order;
 * video_range_luma, skip_refine and wrap are off), Max Displace in pixels of the output, and the
 * row order the engine sees (plugin 02 turns the frames upside down, glue.rs:28-37). */
typedef struct tw_vectors_settings {
    tw_flow_settings flow;
    float max_displace;
    int32_t rows_reversed;
    int32_t display;           /* Display popup: 2 Motion Vectors (0 reads as 2), 3 Debug (glue.rs:81-118) */
    int32_t debug_view;        /* the Debug view's engine code (glue.rs:120-130): 0 Blend, 1 Diff, 2 Detail
                                  Compare, 3 Edge Compare, 4 Warp */
    int32_t debug_textured;    /* the Debug forward warp textured (the revision the parity grid records);
                                  0 the Gouraud variant of the reference (glue.rs:39-42, :557-561) */
} tw_vectors_settings;

/* ---- context ------------------------------------------------------------------------------ */

/* Opens device `device` (the reference's `--device gpu=N` open, device/exec/open.rs:72-116).
 * Runs a small self check of the strict conversions on the device before returning. */
int tw_open(int device, tw_ctx** out);
void tw_close(tw_ctx* ctx);
/* Copies the message of the last failure into buf (NUL terminated); returns its full length. */
size_t tw_last_error(const tw_ctx* ctx, char* buf, size_t cap);
/* Per-stage counters: launches of the library's kernels since open, and device bytes held. */
int tw_stats(const tw_ctx* ctx, uint64_t* kernel_launches, uint64_t* device_bytes);

/* The number of output frames the clip calls keep in flight (1..8; default 4): each has its own
 * buffers and two streams, so their solves overlap on the GPU. 0 is the serial mode: one frame at a
 * time with all its work on the context's stream in issue order (nothing overlaps, so the profiler's
 * events time each kernel alone). A tuning knob only: the output bytes do not depend on it. */
int tw_set_lanes(tw_ctx* ctx, int32_t lanes);

/* Failure injection, for tests of the error paths (the reference's device tests fake failing
 * backends the same way, device/exec/tests.rs). Nothing faults, traps or hangs the GPU: with
 * TW_INJECT_ALLOC the n-th device allocation from now (a buffer that has to grow) fails as a
 * cudaMalloc out of memory would, leaving the buffer as it was, and the call returns TW_ERR_CUDA;
 * with TW_INJECT_STATUS a small kernel sets the device status word of the n-th output frame from
 * now, as a kernel whose bounded loop ran out sets it, and the clip or frame call that reads it
 * returns TW_ERR_DEVICE_BOUND. The context stays usable after either. TW_INJECT_NONE disarms. */
#define TW_INJECT_NONE 0
#define TW_INJECT_ALLOC 1
#define TW_INJECT_STATUS 2
int tw_debug_inject(tw_ctx* ctx, int32_t kind, int32_t n);

/* The autotuner (no counterpart in the reference, whose OpenCL kernels launch one shape): for every
 * level size of a solve of a width x height frame under settings s, it times on the device the
 * tile shapes (32x32, 64x32, 64x64) and block sizes (256, 512) of the solver iteration and the
 * block sizes (128, 256, 512 threads per line) of the row and the column block matching, on
 * stand-in planes of that size, and keeps the fastest of each in the context's table, which every
 * later solve on the context uses. With path != NULL the table is first read from that JSON file
 * (entries written by this library for a device of the same name; sizes found there are not
 * measured again) and then written back: the persistent cache of the tuned shapes. `measured`
 * (may be NULL) receives the number of level sizes timed. Every shape computes the same bytes. */
int tw_autotune(tw_ctx* ctx, const tw_flow_settings* s, int32_t width, int32_t height, const char* path,
                int32_t* measured);
/* The context's table as the JSON text tw_autotune writes (NUL terminated); returns its full length. */
size_t tw_tuning_table(tw_ctx* ctx, char* buf, size_t cap);
/* Sets the table entry of one level size by hand (iter_tile 0 32x32, 1 64x32, 2 64x64; block sizes
 * multiples of 32, at most 512 for the iteration and 1024 for block matching), or clears the
 * table (sizes without an entry take the defaults). */
int tw_tuning_set(tw_ctx* ctx, int32_t width, int32_t height, int32_t iter_tile, int32_t iter_threads,
                  int32_t bm_rows_threads, int32_t bm_cols_threads);
int tw_tuning_clear(tw_ctx* ctx);

/* CUDA graphs of the per-frame pipeline of the clip calls (on by default): a lane captures the
 * pipeline of an in-between frame (warping code 0 with Nearest or Blend, both source frames in the
 * clip, no Blur Compensation) the second time it renders a frame of that shape, then replays the
 * graph for every later one, updating only the kernel arguments that changed (the source and output
 * frames, the blend weights). The bytes do not depend on it. 0 turns it off and drops the graphs. */
int tw_set_graphs(tw_ctx* ctx, int32_t on);

/* Makes the context enqueue on `stream` (a cudaStream_t; NULL is the legacy default stream)
 * instead of its own, so a caller can order the library's work with its own and time it with its
 * own events. */
int tw_set_stream(tw_ctx* ctx, void* stream);

/* Live timing of one kernel by name (for example "k_conv_v"): between begin and end, every launch
 * of that kernel is bracketed with CUDA events on the context's stream; end returns the summed
 * device time, the launch count and the algorithmic bytes those launches move (each input plane
 * read once, each output written once). Replaces the reference's VFX_DEVICE_REPORT counters
 * (device/exec/mod.rs:141-322). */
int tw_profile_begin(tw_ctx* ctx, const char* kernel);
int tw_profile_end(tw_ctx* ctx, double* total_ms, uint64_t* launches, double* bytes);
/* With tw_profile_begin(ctx, "*") every kernel is timed: a text table per kernel (launches, device
 * ms, us per launch, share, algorithmic GB/s) of the launches since begin, written into buf; returns
 * its full length. Call it before tw_profile_end. */
size_t tw_profile_report(tw_ctx* ctx, char* buf, size_t cap);

/* ---- the Stages / Backend seam (stages.rs:33-71, device/exec/backend.rs:27-46) --------------- */

/* Working geometry of a solve (FlowSettings::geometry, flow.rs:129-151): the flow size and the
 * level count; sizes receives (w, h) per level, finest first, up to cap levels. */
int tw_flow_geometry(const tw_flow_settings* s, int32_t width, int32_t height, int32_t* flow_w, int32_t* flow_h,
                     int32_t* levels, int32_t* sizes, int32_t cap);

/* flow::solve (flow.rs:1328-1332): X(p) ~ Y(p + out(p)); `out` has the working size. Replaces
 * Backend::solve (device/exec/backend.rs:29). */
int tw_solve(tw_ctx* ctx, const tw_image* x, const tw_image* y, const tw_flow_settings* s, tw_flow* out);

/* flow::extras::solve_pyramids_with (flow/extras.rs:244-265) with the mask pyramids of a layer
 * (MaskPyramid::build_ungated, extras.rs:130-134, the masks the layered effects build): X(p) ~
 * Y(p + out(p)) with X's gradient masked by X's binary level mask and the B step gated by the
 * warped level mask of Y (flow.rs:737-845). matte_x, matte_y: width*height values 0..1 (the layer's
 * effective matte at X and at Y), both NULL for the plain solve. Replaces
 * Backend::solve_pyramids_with (device/exec/backend.rs:33) for the layers without tracking points. */
int tw_solve_masked(tw_ctx* ctx, const tw_image* x, const tw_image* y, const tw_flow_settings* s, const float* matte_x,
                    const float* matte_y, tw_flow* out);

/* flow::extras::solve_pyramids_with (flow/extras.rs:244-265) on the caller's pyramids: X(p) ~ Y(p +
 * out(p)) from the band pyramids of X and Y (x_levels, y_levels: the levels of the geometry of s for
 * a width x height frame concatenated finest first, as tw_build_pyramid returns them) with a
 * layer's SolveExtras (extras.rs:173-179): the mask pyramids of X and Y (laid out like the bands;
 * both NULL: none; the sweeps are not gated, as MaskPyramid::build_ungated, the masks the effects
 * build) and the user displacement of its tracking points (UserDisplacement, points.rs:201-240:
 * user_d the levels' (dx, dy) interleaved, user_w their weights, both laid out like the bands; both
 * NULL: none). All host buffers. Replaces Backend::solve_pyramids_with (device/exec/backend.rs:33)
 * one to one. */
int tw_solve_pyramids(tw_ctx* ctx, const tw_flow_settings* s, int32_t width, int32_t height, const float* x_levels,
                      const float* y_levels, const float* mask_x, const float* mask_y, const float* user_d,
                      const float* user_w, tw_flow* out);

/* flow::solve_pair (flow.rs:1347-1353): f_ab = solve(A, B), f_ba = solve(B, A), the pyramids built
 * once. Replaces Backend::solve_pair (device/exec/backend.rs:31). */
int tw_solve_pair(tw_ctx* ctx, const tw_image* a, const tw_image* b, const tw_flow_settings* s, tw_flow* f_ab,
                  tw_flow* f_ba);

/* compose::compose_vectors (compose/vector.rs:209-284): the warps, the composition and the blur
 * compensation tail of one vector frame. f_ab / f_ba may be NULL where the interpolation mode
 * does not read them. Replaces Backend::compose_vectors (device/exec/backend.rs:39). */
int tw_compose_vectors(tw_ctx* ctx, const tw_engine_settings* settings, const tw_selection* sel, const tw_image* a,
                       const tw_image* b, const tw_flow* f_ab, const tw_flow* f_ba, tw_image_mut* out);

/* ---- single stages, for callers that drive the engine step by step ------------------------ */

/* flow::build_pyramid (flow.rs:242-275): the band pass levels, concatenated finest first
 * (sum of w*h floats over the levels). */
int tw_build_pyramid(tw_ctx* ctx, const tw_image* img, const tw_flow_settings* s, float* levels_out);

/* flow::block_match (flow.rs:551-622): the four in-place sweeps over a level; a and b are the
 * band pass planes of X and Y (w*h floats), flow is interleaved (w*h*2 floats), updated in place. */
int tw_block_match(tw_ctx* ctx, const float* a, const float* b, float* flow, int32_t width, int32_t height);

/* Block matching for callers that cannot allocate device memory. No counterpart in the reference.
 *
 * Some hosts cannot call cudaMalloc: a plugin inside an application that owns the device memory
 * pool and hands out only its own frame buffers, or a real-time render thread where a driver
 * allocation can stall or is not allowed. This is tw_block_match with DEVICE pointers: a and b
 * (width * height floats each) and flow (width * height * 2 floats, interleaved, updated in place)
 * are the caller's device buffers, and the call allocates nothing (no cudaMalloc or cudaFree, no
 * context). Its scratch is a fixed device array inside the library, 6 * TW_NOALLOC_MAX_PIXELS
 * floats (12 MiB), which every GPU that loads the library holds until the process exits; frames
 * above TW_NOALLOC_MAX_PIXELS pixels (e.g. anything above a 960 x 540 working size plus a
 * little), or a side above 6144, return TW_ERR_TOO_LARGE. The work runs on `stream` (a
 * cudaStream_t, NULL for the default stream) in the CUDA context current on the calling thread,
 * and the call returns when it is done. Every call looks the array's address up in that context
 * and sets the sweep kernels' shared memory limit there (neither allocates), so a host may bind its
 * own context or reset the device between calls. The first call in a process or context may still
 * load the library's device code (lazy module loading, the CUDA default), which is when the array
 * and the kernels take their device memory: make one warm-up call off the real-time thread and
 * before any stream capture. All calls share the one array, which keeps the last call's contents
 * (each call writes every element it reads first): calls that overlap on the GPU (from several
 * host threads or streams at once) race on it and must be serialised by the caller. The status
 * covers this call's own launches and the completion of `stream`; an error that earlier launches
 * of the host left pending is neither reported as this call's nor cleared. */
#define TW_NOALLOC_MAX_PIXELS (1L << 19)
int tw_block_match_noalloc(const float* a, const float* b, float* flow, int32_t width, int32_t height, void* stream);

/* warp::inv_warp / inv_warp_coverage (warp.rs:693-786) with mode 1; `hold` carries WarpOpts: bit 0
 * hold, bit 1 is360 (the wrap by whole turns, the pole reflection and the 360 sampler, warp.rs:
 * 563-621; it takes precedence over hold and leaves the coverage at 255). cov may be NULL (no
 * coverage image) or width*height bytes. */
int tw_inv_warp(tw_ctx* ctx, tw_image_mut* out, const tw_image* src, const tw_flow* flow, float amount, int32_t hold,
                uint8_t* cov);

/* blend::blend (blend.rs:55-114). */
int tw_blend(tw_ctx* ctx, tw_image_mut* out, const tw_image* a, const tw_image* b, float w);

/* smartblend::smart_blend / smart_blend_binary (smartblend.rs:305-315): p1 over p2 and p2 over p1
 * blended at w, or (binary != 0) the binary alpha composite. */
int tw_smart_blend(tw_ctx* ctx, tw_image_mut* out, const tw_image* p1, const tw_image* p2, float w, int32_t binary);

/* One tracking point in use (points.rs:36-55, UserPoint): its position at the layer times of frame
 * A and of frame B, in output pixels (pixel centres at whole numbers). */
typedef struct tw_user_point {
    float at_a[2];
    float at_b[2];
} tw_user_point;

/* The FG matte layers of a layered render (layers.rs:71-129, LayerParams and LayerJob, as
 * plugins/retime-fgbg/src/glue.rs:160-193 reads them): FG1 .. FG nfg and Main_BG. */
typedef struct tw_layer_job {
    int32_t nfg;            /* FG matte layers, 0 to 3 */
    int32_t matte_chan[3];  /* fgN_matte_chan: 1 R, 2 G, 3 B, else alpha (read by tw_retime_layers_clip) */
    float sensitivity[4];   /* 0..1 per layer, FG1 first, Main_BG at index nfg */
    float shrink[3];        /* fgN_inv_matte_shrink in pixels (the 16.16 reader's value), at most 13 */
    int32_t display;        /* the Display popup: 1 all layers, 3 to 5 FG1 to FG3 alone, 6 Main_BG alone
                               (layers.rs:120-129); 2 (Source) composes no layer and is refused */
    /* The tracking points in use (plugins/retime-fgbg/src/glue.rs:196-211, user_points), as the host
     * evaluates its Track Points at the layer times of the pair: npoints[k] points of layer k (Main_BG
     * last), back to back in `points`, at most 12 per layer. tw_compose_layers: nfg + 1 counts, the
     * points in the rows of its images; tw_retime_layers_clip: nout * (nfg + 1) counts, output frame by
     * output frame, in host rows. NULL: no point. Each solve of a layer with points takes their user
     * displacement (points.rs:201-240, flow/extras.rs:181-215). */
    const tw_user_point* points;
    const int32_t* npoints;
} tw_layer_job;

/* The layered composition with plates (layers/plates.rs:330-412, solve_and_compose_plates) of one
 * in-between frame of the FG matte effects: every layer of the job's display group (FG1 .. FG nfg,
 * then Main_BG) solved on its own layer images with its solver masks (tw_solve_masked), its plates
 * (its layer image OVER the other frame's warped to its time) refilled, the single layer
 * composition of the warping code (codes 0 to 3; Nearest, Blend or Weighted Blend), and the layers
 * composed OVER from the bottom up, over an empty image when Main_BG is not in the group. The
 * composition planes cut each layer by the layers above it, each choked by minus its inverse matte
 * shrink (plates.rs:80-107, matte.rs:280-484). a, b: the engine images (also the tracking
 * frames); mattes_a / mattes_b: nfg raw mattes of width*height floats each at A and at B, FG1
 * first (0..1; a float matte as it is). No tracking point is in use; the caller hands the images
 * in the motion path's row order. Replaces the CPU compose::retime_layers vector path for those
 * settings. */
int tw_compose_layers(tw_ctx* ctx, const tw_retime_settings* s, const tw_selection* sel, const tw_image* a,
                      const tw_image* b, const tw_layer_job* job, const float* mattes_a, const float* mattes_b,
                      tw_image_mut* out);

/* forward::forward_warp_with (forward.rs:229-320) with the coverage image when cov != NULL (w*h
 * bytes, 255 where a triangle covered the pixel): the displaced triangle mesh of the flow
 * rasterised into a running mean, textured from the source's mip pyramid (pyramid != 0, the
 * compositor's default) or with the vertex colours interpolated (pyramid == 0, the Gouraud variant
 * `stages::GouraudForward` selects). The flow may have any size of at least 2x2. Replaces
 * Stages::forward_warp_with (stages.rs:33-71). TW_ERR_UNSUPPORTED where the reference refuses (the
 * degenerate last-row pass would write outside the image). */
int tw_forward_warp(tw_ctx* ctx, tw_image_mut* out, const tw_image* src, const tw_flow* flow, float amount,
                    int32_t pyramid, uint8_t* cov);

/* warp::blurcomp::motion_blur (warp/blurcomp.rs:176-559, is360 off): the flow directed motion blur
 * of Blur Compensation, the bilinear taps (hiq != 0) or the nearest ones, the shutter offset of
 * the centre. The compositions run it themselves after the composite (with the clear or the lerp
 * of compensate); this is the primitive alone. */
int tw_motion_blur(tw_ctx* ctx, tw_image_mut* out, const tw_image* src, const tw_flow* flow, float amount,
                   int32_t hiq, float shutter);

/* The adjoint of warp + blend (no reference counterpart: the differentiable twin of compose_vectors'
 * Blend with warping code 0, for photometric flow refinement). Forward: out = ta + (tb - ta) * w,
 * w = 1 - wa, ta = warp(a, f_ba, 1 - wa), tb = warp(b, f_ab, wa), warp(S, F, s)(p) = S sampled
 * bilinearly at p + F(p r) (s / r) (F sampled bilinearly at p r, r = (flow size - 1) / (image size -
 * 1) per axis, the step s / r formed once as warp.rs:636-651 forms it), the position clamped to the
 * image. Backward: from grad_out
 * (d loss / d out), or with target != NULL from the L1 loss sum |out - target| (its sum per batch
 * item added to loss[i]); the gradients are ADDED into da, db (w x h x 4), df_ab, df_ba (flow_w x
 * flow_h x 2), each NULL when not wanted; the forward output goes to out (NULL: not written).
 * All pointers are DEVICE pointers to float RGBA frames and interleaved flows, batch items back
 * to back. The work is enqueued on the context's stream and the call returns without waiting;
 * nothing of the forward pass is stored (the backward recomputes the samples). */
int tw_warp_blend_adjoint(tw_ctx* ctx, const float* a, const float* b, const float* f_ab, const float* f_ba,
                          int32_t width, int32_t height, int32_t flow_w, int32_t flow_h, int32_t batch, float wa,
                          const float* target, const float* grad_out, float* out, float* loss, float* da, float* db,
                          float* df_ab, float* df_ba);

/* The powf of the plugin's C runtime that the Delinearize prep calls (crt_powf.rs:229-268), over
 * n argument pairs: a check hook for the runtime's traced values, as tw_check_logf is for logf.
 * Bit exact on the prep's arguments (a base >= 0 or NaN, the exponent 1 / 2.2); a negative base
 * with an integer exponent and results that over- or underflow float are not the runtime's. */
int tw_check_powf(tw_ctx* ctx, const float* x, const float* y, float* out, int64_t n);

/* Self check of the device's logf of the forward warp's mip level (forward/mesh.rs:89-90), which
 * must equal the host C library's logf bit for bit: out[i] = logf(x[i]) computed on the device. */
int tw_check_logf(tw_ctx* ctx, const float* x, float* out, int64_t n);

/* vectors::encode_vectors (vectors.rs:57-130): the flow (any size of at least 2x2) encoded into
 * `out` (engine image, its size and format): R dx and G dy centred and scaled by `scale` (Max
 * Displace), B 0, A white. */
int tw_encode_vectors(tw_ctx* ctx, tw_image_mut* out, const tw_flow* flow, float scale);

/* create_vectors::create_vectors_on (create_vectors.rs:162-183) for one layer: solve(x, y) on the
 * device and the encode of the flow, engine images in and out (s->rows_reversed is ignored: the
 * caller hands the images in the engine's row order). A side of 1 gives the zero vector image. */
int tw_create_vectors(tw_ctx* ctx, const tw_vectors_settings* s, const tw_image* x, const tw_image* y,
                      tw_image_mut* out);

/* debug::debug_view_on (debug.rs:104-171): the view `code` (0 Blend, 1 Diff, 2 Detail Compare, 4 Warp,
 * any other Edge Compare) of engine images x and y by the flow X(p) ~ Y(p + flow(p)) (any size of at
 * least 2x2): the forward warp of x at amount 1 (the Gouraud variant with gouraud != 0, else the
 * textured one), W' = (y OVER a cleared image) with the warp OVER it (matte::over_pl), then the view;
 * frames with a side of 1 give the zero vector image. */
int tw_debug_view(tw_ctx* ctx, const tw_image* x, const tw_image* y, const tw_flow* flow, int32_t code,
                  int32_t gouraud, tw_image_mut* out);

/* create_vectors::frame_pair (create_vectors.rs:71-89) and the clip frames of the pair: as
 * tw_vectors_pair, with debug != 0 the Debug display's roles (Previous: a = n + 1, Next: a = n - 1). */
int tw_vectors_frame_pair(int32_t n, int32_t time_step, int32_t track_frame, int32_t debug, int32_t* a, int32_t* b);

/* The clip frames of output frame n of Create Vectors (create_vectors.rs:59-97, glue.rs:488-524):
 * a = n, b = n - 1 (track_frame 1, Previous) or n + 1 (2, Next); a frame outside the clip is
 * blank. time_step: ticks per frame (integer rates: 100). */
int tw_vectors_pair(int32_t n, int32_t time_step, int32_t track_frame, int32_t* a, int32_t* b);

/* The Create Vectors effect over a clip in HOST memory (wire frames back to back): output frame k
 * encodes the flow from clip frame pairs[2k] to pairs[2k + 1] (a frame index outside 0..nframes-1
 * is a blank frame), with the device frame cache, the lanes and the copy streams of
 * tw_retime_clip. The output wire frames go to out + k * frame_bytes. points / npoints: the
 * tracking points in use of each output frame (plugins/create-vectors/src/glue.rs:278-291,
 * layer_points, as the host evaluates them at the layer times of the pair; host rows), npoints[k]
 * of them for frame k, at most 12, back to back; they give the solve its user displacement
 * (create_vectors.rs:336-351). NULL: no point. */
int tw_create_vectors_clip(tw_ctx* ctx, const tw_vectors_settings* s, const void* frames, int32_t nframes,
                           const int32_t* pairs, int32_t nout, const tw_user_point* points, const int32_t* npoints,
                           int32_t width, int32_t height, int32_t fmt, void* out);

/* holefill::fill_holes_masked_with (holefill.rs:452-491) with is360 off: the pull-push fill of
 * `img` in place. `mask` holds width*height values of kind 1 (u8), 2 (u16) or 3 (f32); a pixel is
 * a hole when !(eps > m) (holefill.rs:124-133). taps_above_first: the vertical border tap order
 * (0: below first, the engine's order the unit tests use). A hole in an image with a side of 1
 * pixel is TW_ERR_UNSUPPORTED, as in the reference. */
int tw_fill_holes(tw_ctx* ctx, tw_image_mut* img, const void* mask, int32_t mask_kind, int32_t taps_above_first);

/* image::Image::from_frame / to_frame (image.rs:178-245): wire frame <-> engine image. */
int tw_from_frame(tw_ctx* ctx, const void* wire, int32_t width, int32_t height, int32_t fmt, void* engine_out);
int tw_to_frame(tw_ctx* ctx, const void* engine, int32_t width, int32_t height, int32_t fmt, void* wire_out);

/* ---- the time model of the `retime` effect (host scalars) ---------------------------------- */

/* The parameters the time map and the frame selection read (plugins/retime/src/lib.rs:59-99 as
 * frontend::read_settings reads them, frontend.rs:184-244; timeline.rs:106-131, :204-344). Popups
 * carry their raw 1-based values. A curve is constant (no key) or keyed at frame numbers, linear
 * between keys, eased at a key whose flag has bit 0, held after a key whose flag has bit 1
 * (crates/fx-core/src/curves.rs:282-310, :348-375, :537-544). Src Time Offset is 0. A zeroed tail
 * (remap_mode .. frame_time_plain) is the Speed mode with "In FPS is Out FPS" on. */
typedef struct tw_time_params {
    int32_t fps_num, fps_den;  /* the host's frame rate; integer rates get 100 ticks a frame */
    double speed_percent;
    int32_t nkeys;
    const double* key_frames;
    const double* key_values;
    const int32_t* key_ease;   /* per key flags: 1 ease, 2 hold */
    int32_t vectors;           /* Motion Vectors popup 1..5 */
    int32_t frame_interp;      /* Frame Interp popup 1..3 */
    double blur_compensation;
    int32_t remap_mode;        /* Time Remap Mode popup: 1 Speed (0 reads as 1), 2 Frame Number */
    double frame_num;          /* Frame Num (Frame Number mode), constant when nfn_keys == 0 */
    int32_t nfn_keys;
    const double* fn_key_frames;
    const double* fn_key_values;
    const int32_t* fn_key_flags;
    int32_t own_input_rate;    /* "In FPS is Out FPS" off: the input rate input_frame_rate (narrowed to
                                  float), the output rate fps; both snapped (timeline.rs:69-76) */
    double input_frame_rate;
    double frame_time_bias;    /* the bias of the frame time between unequal rates (timeline.rs:25): 0
                                  reads as 0.05, the reference's value; 0.1 the revision its parity
                                  grids record */
    int32_t frame_time_plain;  /* retime-fgbg's frame time: trunc(dur * k + 0.5) at every rate, no bias
                                  branch (timeline.rs:204-210) */
    int32_t input_fields;      /* Input: Fields popup (plugins/retime/src/lib.rs:70): 2 Upper Field First or
                                  3 Lower Field First double the source rate (timeline.rs:123-125); 0 and
                                  1 are None */
    int32_t mark_segs;         /* Src: Mark Segments popup (1 Cut A, 2 Cut B, 3 Cut C, 4 No MV Use Nearest,
                                  5 No MV Frame Blend), constant when nmark_keys == 0; 0 reads as 1 */
    int32_t nmark_keys;        /* its keys: a popup holds each key's value up to the next key */
    const double* mark_key_frames;
    const double* mark_key_values;
} tw_time_params;

/* The selection of output frame n of a clip of width x height (timeline::select, timeline.rs:
 * 451-469, with RemapTimeMap::src_pos :266-331, the segment override of Src: Mark Segments
 * marker_override :418-441 and the tiny-frame rule prep.rs:111-117). out->a and
 * out->b are the CLIP frames of the pair, the frames positions a and a + 1 show at frame_time
 * (host.rs:155-159, timeline.rs:336-344), which the clip calls read; with equal rates they are the
 * positions themselves. TW_ERR_BAD_PARAM for a rate at or below 0.01 (timeline.rs:125-127). */
int tw_select(const tw_time_params* p, int32_t n, int32_t width, int32_t height, tw_selection* out);

/* ---- Vectors In (plugins/vectors-in, compose/vector.rs:323-447) ----------------------------- */

/* One output frame of the Vectors In render beyond its selection (plugins/vectors-in/src/vectorin.rs:
 * 175-227): the clip frames of the pair (footage A and Vectors: Next at clip frame a, footage B and
 * Vectors: Prev at clip frame b), which vector layers are present (has_next / has_prev; a present
 * layer without a frame there is a transparent image, which decodes to the zero flow) and their
 * Vec Scale X / Y at the fetch times. */
typedef struct tw_vecin_frame {
    int32_t a, b;
    int32_t has_next, has_prev;
    float next_scale[2];
    float prev_scale[2];
} tw_vecin_frame;

/* The selection of output frame n of the Vectors In effect (plugins/vectors-in/src/timemap.rs,
 * glue.rs:204-215): the time map of tw_select with the input rate 30 (In FPS is Out FPS on; else
 * p->input_frame_rate) and the output rate the composition's, the vectors quality 4 (p->vectors is
 * not read), out->a / out->b the positions, and in frame->a / frame->b the clip frames of the pair
 * at T(k) = trunc(dur * k + 0.5) ticks. The other fields of `frame` are left as they are. */
int tw_select_vectors_in(const tw_time_params* p, int32_t n, int32_t width, int32_t height, tw_selection* out,
                         tw_vecin_frame* frame);

/* vectors::decode_vectors (vectors.rs:474-528): the flow of an encoded engine image of the same
 * size (R dx and G dy, 8 bpc ((c * 2) / 254 - 1) * md and 16 bpc with 65534 in double precision,
 * float (c * 2 - 1) * md; alpha 0 the zero vector). */
int tw_decode_vectors(tw_ctx* ctx, const tw_image* vec, float max_displace, tw_flow* out);

/* compose::flow_from_vector_image_with (compose/vector.rs:335-345): the decode, the pull-push fill
 * of the holes of the inverted alpha (holefill.rs:497-518, is360 off, the tap order
 * taps_above_first), then Vec Scale (vectors.rs:573-578). A hole in an image with a side of 1
 * pixel is TW_ERR_UNSUPPORTED, as in the reference. */
int tw_flow_from_vectors(tw_ctx* ctx, const tw_image* vec, float max_displace, float scale_x, float scale_y,
                         int32_t taps_above_first, tw_flow* out);

/* holefill::fill_flow_holes_with (holefill.rs:497-518) with is360 off: both components of `flow`
 * filled in place; the mask as in tw_fill_holes. */
int tw_fill_flow_holes(tw_ctx* ctx, tw_flow* flow, const void* mask, int32_t mask_kind, int32_t taps_above_first);

/* compose::invert_flow_on (compose/vector.rs:370-397): T = -(1, fx, fy, 1) pushed along the flow
 * at amount 1 with the forward warp (pyramid != 0 the textured warp, 0 the Gouraud variant), the
 * coverage inverted, channels 1 and 2 of the pushed image as the flow, the holes filled. `out` has
 * the flow's size (at least 2x2). */
int tw_invert_flow(tw_ctx* ctx, const tw_flow* in, int32_t pyramid, int32_t taps_above_first, tw_flow* out);

/* One output frame of the single layer Vectors In render (glue.rs:386-495 with nfg 0, Display not
 * Source; compose.rs:101-131): wire frames of the footage at A and B (NULL: blank), of Vectors: Next
 * at A and Vectors: Prev at B (read only for a present layer; NULL: transparent). Neither layer
 * present: the size mismatch error fill (image.rs:388-425), as the effect writes it. Else the
 * vector path when sel->vectors_quality != 0 and !sel->exact: each present layer's flow
 * (tw_flow_from_vectors with Max Displace `max_displace` and the frame's Vec Scale), the missing
 * one as the inversion of the other where the composition reads it (compose/vector.rs:422-447;
 * the forward warp Gouraud when s->compose.gouraud), then tw_compose_vectors' composition; else
 * the fast path. s->motion_rows_reversed turns every input of the vector path, the vector layers
 * included, upside down and the output back (glue.rs:44-48). The hole fills take
 * s->compose.taps_above_first. */
int tw_retime_frame_vectors(tw_ctx* ctx, const tw_retime_settings* s, const tw_selection* sel, const tw_vecin_frame* vf,
                            float max_displace, const void* wire_a, const void* wire_b, const void* wire_next,
                            const void* wire_prev, int32_t width, int32_t height, int32_t fmt, void* wire_out);

/* The same over clips in HOST memory: the footage (nframes wire frames back to back), Vectors: Next
 * (n_next frames; NULL when no frame has it) and Vectors: Prev (n_prev); output frame k from
 * sels[k] and vfs[k] goes to out + k * frame_bytes. A clip frame outside a clip is blank (footage)
 * or transparent (vector layer). The clips are uploaded whole; frames run on the lanes, except
 * that a call whose frames run the forward warp (warping codes 2 and 3, or a flow inversion) runs
 * them one at a time. */
int tw_vectors_in_clip(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes, const void* next,
                       int32_t n_next, const void* prev, int32_t n_prev, const tw_selection* sels,
                       const tw_vecin_frame* vfs, int32_t nout, float max_displace, int32_t width, int32_t height,
                       int32_t fmt, void* out);

/* The same with every clip and the output in DEVICE memory; enqueues on the context's stream and
 * returns after it completes. */
int tw_vectors_in_clip_device(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                              const void* next, int32_t n_next, const void* prev, int32_t n_prev,
                              const tw_selection* sels, const tw_vecin_frame* vfs, int32_t nout, float max_displace,
                              int32_t width, int32_t height, int32_t fmt, void* out);

/* ---- one clip over several GPUs ------------------------------------------------------------ */

/* The output frames [lo, hi) of a clip of nout output frames that rank `rank` of `nranks` renders:
 * contiguous ranges in rank order whose sizes differ by at most one. No counterpart in the reference,
 * whose renderer walks the output frames in order on one device (crates/fx-cli/src/temporal.rs:
 * 206-249); an output frame needs nothing from any other (timeline.rs:447-469), so the ranks
 * exchange nothing and the outputs concatenate in rank order. */
int tw_shard(int32_t nout, int32_t nranks, int32_t rank, int32_t* lo, int32_t* hi);

/* The clip frames [first, last] that selections sels[0 .. n) read inside a clip of nframes frames
 * (frames a and b of every selection; first > last when none lies inside the clip): the source
 * window one rank uploads. A frame at the boundary of two ranks' ranges lies in both windows, and
 * each rank builds its pyramid itself, which costs one frame per boundary and needs no exchange. */
int tw_source_window(const tw_selection* sels, int32_t n, int32_t nframes, int32_t* first, int32_t* last);

/* ---- whole output frames ------------------------------------------------------------------ */

/* One output frame of the `retime` effect's core (compose.rs:93-101 with vector_path,
 * compose/vector.rs:289-321, then the finish, frontend.rs:273-276): wire frames A and B of the
 * selection in, the output wire frame out. Runs the vector path when sel->vectors_quality != 0
 * and !sel->exact, else the fast path (compose.rs:218-231). A and B are the frames the host
 * fetched for sel->a and sel->b (a blank frame for one outside the clip). */
int tw_retime_frame(tw_ctx* ctx, const tw_retime_settings* s, const tw_selection* sel, const void* wire_a,
                    const void* wire_b, int32_t width, int32_t height, int32_t fmt, void* wire_out);

/* The same over a clip in HOST memory (page-locked memory makes the copies asynchronous):
 * `frames` holds nframes wire frames back to back, output frame k goes to out + k * frame_bytes.
 * Each source frame a selection references is uploaded once into a device frame cache (the
 * reference's device backend keeps resident frames the same way, device/exec/backend.rs:190-208),
 * several output frames are in flight at once, and uploads, kernels and downloads overlap on
 * separate streams. Returns after every output frame is in `out`. */
int tw_retime_clip(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                   const tw_selection* sels, int32_t nout, int32_t width, int32_t height, int32_t fmt, void* out);

/* The same over a clip resident in device memory: `frames` holds nframes wire frames back to
 * back, `sels` nout selections; output frame k goes to out + k * frame_bytes. Source frames
 * outside the clip are blank. All pointers are device pointers; the call enqueues on the
 * context's stream and returns after it completes. */
int tw_retime_clip_device(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                          const tw_selection* sels, int32_t nout, int32_t width, int32_t height, int32_t fmt,
                          void* out);

/* retime-fgbg with FG matte layers over a clip in HOST memory (plugins/retime-fgbg/src/glue.rs:
 * 275, render_temporal, with compose.rs:149-223 and layers.rs:410-567): output frame k of the
 * selections `sels`; footage in `frames` (nframes wire frames back to back), the FG matte layers
 * FG1 .. FG job->nfg in matte_clips[j] (wire frames of the footage's size and format,
 * matte_nframes[j] of them, or nframes when matte_nframes is NULL), each read through its channel
 * job->matte_chan[j]. The in-between frames run tw_compose_layers in the motion path's row order
 * (rows reversed when s->motion_rows_reversed); an FG layer with an inverse matte shrink makes
 * every position an in-between one (compose.rs:209-211). The unwarped frames take the
 * interpolation without flows, of the frames themselves for the full group, of the group's rebuilt
 * plates for a single layer display (layers.rs:414-528). A frame outside a clip is blank. No
 * tracking point is in use. s->compose.gouraud should be 1 (retime-fgbg's forward warps are the
 * Gouraud variant). nfg 0 with warping codes 0/1 is tw_retime_clip; codes 2/3 run the plain
 * vector path frame by frame on the context's stream. The full group of an unwarped frame with a
 * shrink (Vectors off) is TW_ERR_UNSUPPORTED. */
int tw_retime_layers_clip(tw_ctx* ctx, const tw_retime_settings* s, const void* frames, int32_t nframes,
                          const tw_layer_job* job, const void* const* matte_clips, const int32_t* matte_nframes,
                          const tw_selection* sels, int32_t nout, int32_t width, int32_t height, int32_t fmt,
                          void* out);

/* One clip of a batch: its settings, its source frames (nframes wire frames back to back, DEVICE
 * memory), its selections and its output (nout wire frames, DEVICE memory). */
typedef struct tw_clip_job {
    const tw_retime_settings* settings;
    const void* frames;
    int32_t nframes;
    const tw_selection* sels;
    int32_t nout;
    int32_t width, height, fmt;
    void* out;
} tw_clip_job;

/* Several clips of any sizes and depths in one call (the batched retime): the output frames of all
 * jobs are dealt round robin over the clips onto the lanes, so frames of different clips are in
 * flight together; each equals tw_retime_clip_device of its own clip. Returns when all are done. */
int tw_retime_batch_device(tw_ctx* ctx, const tw_clip_job* jobs, int32_t njobs);

#ifdef __cplusplus
}
#endif

#endif /* TWIXTOR_B200_H */
