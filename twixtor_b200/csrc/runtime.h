// Internal header of the library's host runtime: the device context, its buffers and lanes, the
// launch macro, and the functions the host translation units share. Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/twixtor_b200.h"
#include "kernels.cuh"
#include "kernels_fast.cuh"
#include "luma.cuh"

namespace tw {

// ---- host geometry (prep.rs:63-146, flow.rs:129-197) ---------------------------------------------

struct Geo {
    int reduction = 0, w = 0, h = 0, levels = 0;
    int sizes[32][2];
};

int geometry(const tw_flow_settings& s, int w, int h, Geo* g, std::string* err);
void start_level(float sensitivity, int levels, int* start, float* damp);
Taps gaussian_taps(float r);
Taps binomial5();
inline size_t sample_bytes(int fmt) { return fmt == TW_U8 ? 1 : fmt == TW_U16 ? 2 : 4; }
inline size_t image_bytes(int w, int h, int fmt) { return (size_t)w * h * 4 * sample_bytes(fmt); }

// ---- device buffers --------------------------------------------------------------------------------

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n, size_t* held) {
        if (n <= cap) return cudaSuccess;
        if (p) { cudaFree(p); *held -= cap; p = nullptr; cap = 0; }
        size_t want = std::max(n, (size_t)256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) { cap = want; *held += want; }
        return e;
    }
    void release(size_t* held) {
        if (p) { cudaFree(p); *held -= cap; }
        p = nullptr;
        cap = 0;
    }
    template <typename T> T* as() const { return (T*)p; }
};

}  // namespace tw

using namespace tw;

// Live per-kernel timing for the benchmark: CUDA events around every launch of one named kernel on
// the context's stream, with the algorithmic bytes each launch moves.
// The launch shapes at one level size (the autotuner's table entries): the solver iteration's tile
// shape and block size, and the block size of each block matching kernel (one block per line).
struct LevelTune {
    int iter_tile;        // LEVEL_TILE_*
    int iter_threads;     // a multiple of 32 up to LEVEL_ITER_MAX_THREADS
    int bm_rows_threads;  // a multiple of 32 up to 1024
    int bm_cols_threads;
};

struct KernelProfile {
    bool on = false;
    size_t pooled = 0;            // events of the context's pool in use by this session
    std::string name;             // one kernel, or "*" for every kernel
    std::vector<cudaEvent_t> ev;  // start, stop pairs
    std::vector<std::string> who; // the kernel of each pair
    std::vector<double> nbytes;   // the algorithmic bytes of each pair
    double bytes = 0.0;
    uint64_t launches = 0;
};

// One set of buffers for one output frame in flight, with two streams: the two pyramids and the
// two solves of a pair run concurrently (stream 0: A's pyramid, solve(A, B), the composition;
// stream 1: B's pyramid, solve(B, A)). Several lanes keep several output frames in flight.
// A captured per-frame pipeline of one lane (CUDA graph): its executable graph, the captured graph
// that owns the nodes, and each kernel node in launch order with its function and arguments (the last
// ones set), so that a later frame of the same shape updates only the nodes whose arguments changed.
struct FrameGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaGraphNode_t> nodes;
    std::vector<const void*> funcs;
    std::vector<std::string> args;
    uint64_t alloc_gen = 0;  // the context's allocation generation at capture (buffers moved since: stale)
    bool seen = false;       // a frame of this shape ran once without a graph (its buffers exist)
};
enum { GRAPH_OFF = 0, GRAPH_CAPTURE = 1, GRAPH_REPLAY = 2 };

struct Lane {
    std::map<std::string, FrameGraph> graphs;  // by frame shape
    cudaEvent_t ev_fork = nullptr;             // the second stream's entry into a capture
    cudaStream_t s[2] = {nullptr, nullptr};    // the streams this call uses: own[] or, serial, the context's
    cudaStream_t own[2] = {nullptr, nullptr};  // the lane's own streams
    cudaEvent_t ev_pyr[2] = {nullptr, nullptr};  // pyramid of A / B done
    cudaEvent_t ev_solve1 = nullptr;             // solve on stream 1 done
    cudaEvent_t ev_done = nullptr;               // the frame's composition done (stream 0)
    bool used = false;
    DevBuf eng[2], pyr[2], work[2], flow[2], scratch[2][3], flags;
    DevBuf comp, holes, fill;  // warping code 1: the composite, its holes mask, the fill's planes
    DevBuf wb_wt[2], wb_tmp[2], wb_mask[2], wb_cov[2];  // Weighted Blend: warped frames, blur planes, masks, coverage
    DevBuf pre_blur;  // Blur Compensation: the composite before the motion blur
    DevBuf user;      // tracking points: the user displacement of the solve and its scratch
};
constexpr int MAX_LANES = 8;

struct tw_ctx {
    int device = 0;
    KernelProfile prof;
    cudaStream_t cur = nullptr;  // the stream every launch goes to
    Lane lanes[MAX_LANES];
    int nlanes = 4;  // output frames in flight in the clip calls (tw_set_lanes)
    std::map<uint64_t, LevelTune> tune_table;  // (w << 32 | h) -> the measured launch shapes of that level size
    // CUDA graphs of the per-frame pipeline (tw_set_graphs): the mode of the launches being issued,
    // the graph they go to, the next kernel node of a replay, and a failure seen on the way
    bool graphs_on = true;
    int gmode = GRAPH_OFF;
    FrameGraph* gcur = nullptr;
    size_t gi = 0;
    bool gfail = false;
    uint64_t alloc_gen = 0;  // counts the device (re)allocations of the context's buffers
    bool serial = false;  // tw_set_lanes(ctx, 0): one lane whose work all runs on the context's stream
    cudaEvent_t ev_start = nullptr;
    // tw_retime_clip: a device cache of source frames, and the copy streams
    static constexpr int CACHE_SLOTS = 20;
    DevBuf cache[CACHE_SLOTS], outbuf[MAX_LANES];
    int cache_frame[CACHE_SLOTS];
    cudaEvent_t cache_ready[CACHE_SLOTS] = {}, out_free[MAX_LANES] = {};
    cudaEvent_t cache_free[CACHE_SLOTS][MAX_LANES] = {};  // per slot, the end of each lane's last read
    cudaStream_t up = nullptr, down = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t own = nullptr;  // the stream the context created
    bool own_stream = true;
    std::mutex mu;
    std::string err;
    uint64_t launches = 0;
    size_t held = 0;
    Taps g7{}, g5{}, b5{}, g2{};
    // engine images, wire staging, pyramids, solve work, flows
    DevBuf eng[3], wire[3], pyr[2], plane[4], work[2], flow[2], flags, holes, fill, masks;
    DevBuf lay_mem;  // the layered path: planes, layer images, plates, flows
    DevBuf lay_in;   // the layered path: the raw mattes at A and B
    // tw_retime_layers_clip: two staging slots (the footage pair and the matte frames of a frame),
    // filled on the copy stream one frame ahead; uploaded / last read events per slot
    DevBuf lay_stage[2][8];
    cudaEvent_t lay_up[2] = {nullptr, nullptr}, lay_free[2] = {nullptr, nullptr};
    DevBuf fc_img[2], fc_cov[2];  // the forward compositions: the two pushed frames and their coverage
    DevBuf wb_wt[2], wb_tmp[2], wb_mask[2], wb_cov[2];  // Weighted Blend (the calls on the context's stream)
    DevBuf pre_blur, comp_e;  // Blur Compensation: the composite before the blur, the engine result
    DevBuf vi_clip[3], vi_out, vi_wire[5];  // Vectors In: the clips on the device, the output clip, one frame's wires
    bool adj_smem_set = false;  // the adjoint kernel's dynamic shared memory limit is raised
    DevBuf host_stage;  // unused placeholder for pinned staging
    std::vector<cudaEvent_t> ev_pool;  // the profiler's events (KernelProfile)
    // the forward warp: vertices, mip pyramid, per pixel counts / offsets, hit lists, flags
    DevBuf logf_tab, fw_vx, fw_vy, fw_vd, fw_pyr, fw_tmp[2], fw_cnt, fw_off, fw_fill, fw_sums, fw_keys, fw_cols,
        fw_scratch, fw_longq, fw_flags, fw_cov;

    int fail(int code, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        err = buf;
        return code;
    }
    int cuda(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return TW_OK;
        return fail(TW_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    // tw_debug_inject: the kind of failure armed and the count of events before it fires
    int inject_kind = 0, inject_n = 0;
    bool inject_now(int kind) {  // true once, at the n-th event of the armed kind
        if (inject_kind != kind || inject_n <= 0) return false;
        if (--inject_n > 0) return false;
        inject_kind = 0;
        return true;
    }
    int ensure(DevBuf& b, size_t n, const char* what) {
        if (n > b.cap && inject_now(TW_INJECT_ALLOC))  // the buffer is left as it was, as a failed cudaMalloc leaves it
            return fail(TW_ERR_CUDA, "%s: out of memory (injected allocation failure)", what);
        if (n > b.cap) alloc_gen++;  // a buffer moves: captured graphs that name it are stale
        return cuda(b.ensure(n, &held), what);
    }
};

// The glibc logf exception table embedded by the build (csrc/logf_table.S).
extern "C" const uint32_t tw_logf_table[];
extern "C" const uint32_t tw_logf_table_end[];

namespace tw {

// Every kernel launch of the library goes through LAUNCHB (LAUNCH passes no byte count): it counts
// the launch and, when the kernel is the one being profiled, brackets it with events.
bool prof_match(tw_ctx* ctx, const char* kernel);
void prof_mark(tw_ctx* ctx);

// A kernel launch while a lane captures or replays its frame graph (host_context.cu).
void graph_kernel(tw_ctx* ctx, const void* func, dim3 grid, dim3 block, size_t smem, void** argv, std::string&& packed);
void drop_graph(FrameGraph& G);

template <typename T, size_t... I>
void launch_tuple(tw_ctx* ctx, const void* k, dim3 grid, dim3 block, size_t smem, T& t, std::index_sequence<I...>) {
    void* argv[] = {(void*)&std::get<I>(t)..., nullptr};
    if (ctx->gmode == GRAPH_OFF) {
        cudaLaunchKernel(k, grid, block, argv, smem, ctx->cur);
        return;
    }
    std::string packed;
    (packed.append((const char*)&std::get<I>(t), sizeof(std::get<I>(t))), ...);
    graph_kernel(ctx, k, grid, block, smem, argv, std::move(packed));
}

// One kernel launch: the arguments converted to the kernel's own parameter types, then launched on
// ctx->cur, or recorded into / updated in the lane's frame graph.
template <typename... P, typename... A>
void launch_kernel(tw_ctx* ctx, void (*k)(P...), dim3 grid, dim3 block, size_t smem, A&&... a) {
    std::tuple<P...> t(static_cast<P>(std::forward<A>(a))...);
    launch_tuple(ctx, (const void*)k, grid, block, smem, t, std::index_sequence_for<P...>{});
}

// A stream operation of the per-frame pipeline other than a kernel (a memset, an event): issued
// normally and while capturing (it becomes a node of the graph), skipped while replaying.
#define GOP(ctx, expr) ((ctx)->gmode == GRAPH_REPLAY ? (int)TW_OK : (expr))

#define LAUNCHB(ctx, nbytes_, kernel, grid, block, smem, ...)                        \
    do {                                                                           \
        bool _p = prof_match((ctx), #kernel);                                      \
        if (_p) prof_mark(ctx);                                                    \
        launch_kernel((ctx), kernel, dim3(grid), dim3(block), (size_t)(smem), __VA_ARGS__); \
        (ctx)->launches++;                                                         \
        if (_p) {                                                                  \
            prof_mark(ctx);                                                        \
            (ctx)->prof.bytes += (double)(nbytes_);                                \
            (ctx)->prof.launches++;                                                \
            (ctx)->prof.who.push_back(#kernel);                                    \
            (ctx)->prof.nbytes.push_back((double)(nbytes_));                       \
        }                                                                          \
    } while (0)
#define LAUNCH(ctx, kernel, grid, block, smem, ...) LAUNCHB(ctx, 0, kernel, grid, block, smem, __VA_ARGS__)
// The strict kernel, or with `fastv` its fast mode build (tw::fast, kernels_fast.cuh).
#define LAUNCHV(ctx, fastv, nbytes_, kernel, grid, block, smem, ...)                         \
    do {                                                                                   \
        if (fastv) LAUNCHB(ctx, nbytes_, fast::kernel, grid, block, smem, __VA_ARGS__);    \
        else LAUNCHB(ctx, nbytes_, kernel, grid, block, smem, __VA_ARGS__);                \
    } while (0)

#define CHECK(expr)                 \
    do {                            \
        int _rc = (expr);           \
        if (_rc != TW_OK) return _rc; \
    } while (0)

constexpr int TB = 256;
// device flags (ints): [0..31] per-level range flags of solve 0, [32..63] of solve 1, [64] NaN in a
// flow, [65] a warp refused a sample coordinate
constexpr int FL_ANY0 = 0, FL_ANY1 = 32, FL_NAN = 64, FL_BAD = 65, FL_HOLE = 66, FL_SIDE1 = 67, FL_ONE = 68, FL_WB = 69,
              FL_BOUND = 70;  // [70] a device loop reached its bound
constexpr size_t FLAGS_BYTES = 128 * sizeof(int);

inline dim3 grid2(int w, int h) { return dim3((unsigned)((w + TB - 1) / TB), (unsigned)h); }
inline unsigned grid1(long n) { return (unsigned)((n + TB - 1) / TB); }
inline dim3 tiles(int w, int h) { return dim3((unsigned)((w + FUSED_TILE_X - 1) / FUSED_TILE_X), (unsigned)((h + FUSED_TILE_Y - 1) / FUSED_TILE_Y)); }

// Scratch of the warping code 1 composition: the composite (engine image), its holes mask, the
// fill's planes, and the device flag "some pixel is a hole".
struct WbScratch {  // Weighted Blend: the two warped frames, the blur planes, the masks, the coverage
    DevBuf* wt[2];
    DevBuf* tmp[2];
    DevBuf* mask[2];
    DevBuf* cov[2];
};

struct SmartScratch {
    DevBuf* comp;
    DevBuf* holes;
    DevBuf* fill;
    int* any_hole;  // set by the composition when a pixel is a hole
    int* side1;     // set when an image with a side of 1 pixel has a hole (the fill refuses it)
    const WbScratch* wb = nullptr;  // Weighted Blend scratch (nullptr: Weighted Blend refused)
    int* wb_gate = nullptr;         // the unsound float flag of the Weighted Blend without flows
    DevBuf* blur = nullptr;         // Blur Compensation: the composite before the blur (nullptr: refused)
};

// ---- shared by the host translation units ---------------------------------------------------------

// host_context.cu
int upload_image(tw_ctx* ctx, DevBuf& b, const tw_image* im);
int finish(tw_ctx* ctx, int* flags_host, int n);
bool same_shape(const tw_image* a, const tw_image* b);
int check_image(tw_ctx* ctx, const tw_image* im, const char* what);
int check_out(tw_ctx* ctx, const tw_image_mut* im, const char* what);
int lane_ready(tw_ctx* ctx, Lane& L);
int lanes_begin(tw_ctx* ctx, int nl);
int lanes_end(tw_ctx* ctx, int nl);
int bad_fail(tw_ctx* ctx, int v);
__global__ void k_set_flag(int* flags, int idx);  // flags[idx] = 1 (the injected device status)

// host_solve.cu
LevelTune level_tune(tw_ctx* ctx, int w, int h);
LevelTune default_tune(int w, int h);
void block_match(tw_ctx* ctx, const float* A, const float* B, const float* AT, const float* BT, float* fu, float* fv,
                 float* uT, float* vT, int w, int h, bool fast = false);
void level_iter(tw_ctx* ctx, LevelTune ic, const float* A, const float* B, const float* gx, const float* gy,
                const float* a0, const float* a1, const float* a2, const float* fu, const float* fv, int w, int h, bool af,
                float* nu, float* nv, const float* mask_y, bool fast, const float* b_in, float* b_out, int bp,
                long bplane);
size_t pyramid_floats(const Geo& g);
int build_pyramid_dev(tw_ctx* ctx, const void* eng_dev, int W, int H, int fmt, const tw_flow_settings& s, const Geo& g,
                      float* out, float* out_t, DevBuf* scratch);
int user_pairs(tw_ctx* ctx, const tw_user_point* pts, int n, bool x_is_a, bool flip, int H, UserPairs* out);
int build_user_dev(tw_ctx* ctx, const UserPairs& pr, const Geo& g, int W, int H, float* du, float* dv, float* uw,
                   float* scr);
int solve_pyramids_dev(tw_ctx* ctx, const float* x, const float* y, const float* xt, const float* yt, const Geo& g,
                       const tw_flow_settings& s, DevBuf& work, float* out, int* any, int* nan_flag,
                       const float* mx = nullptr, const float* my = nullptr, const float* udu = nullptr,
                       const float* udv = nullptr, const float* uww = nullptr);
int build_mask_pyramid_dev(tw_ctx* ctx, float* matte, int W, int H, const tw_flow_settings& s, const Geo& g, float* out,
                           float* scratch0, float* scratch1, const int* one);

// host_compose.cu
bool warp_copy_only(float amount, int fw, int width);
WarpParams warp_params(const void* src, const float* flow_interleaved, int fw, int fh, float amount, int width, int height,
                       bool hold);
int fill_dev(tw_ctx* ctx, void* img, int W, int H, int fmt, const uint8_t* holes, const int* any, bool above_first,
             DevBuf& fb);
int forward_warp_dev(tw_ctx* ctx, const void* src, const float* flow, int fw, int fh, int W, int H, int fmt,
                     float amount, bool pyramid, void* out, uint8_t* cov);
WbScratch wb_scratch(DevBuf* wt, DevBuf* tmp, DevBuf* mask, DevBuf* cov);
int compose_dev(tw_ctx* ctx, const tw_engine_settings& cs, const tw_selection& sel, const void* eng_a,
                const void* eng_b, const float* f_ab, const float* f_ba, int fw, int fh, int W, int H, int fmt,
                void* out, bool to_wire, bool flip_out, int* bad, const SmartScratch* ss);
int interpolate_dev(tw_ctx* ctx, const tw_selection& sel, const void* eng_a, const void* eng_b, int W, int H, int fmt,
                    void* out, bool to_wire, int* bad, const SmartScratch* ss);

// host_clips.cu
void from_frame_dev(tw_ctx* ctx, const void* wire, void* eng, int W, int H, int fmt, bool flip);
void to_frame_dev(tw_ctx* ctx, const void* eng, void* wire, int W, int H, int fmt, bool flip);

// host_vecin.cu
int vec_flow_dev(tw_ctx* ctx, const void* vec, int W, int H, int fmt, float md, float sx, float sy, bool above_first,
                 float* flow, uint8_t* holes, int* any, DevBuf& fillbuf);
int invert_flow_dev(tw_ctx* ctx, const float* flow, int W, int H, bool pyramid, bool above_first, float* out,
                    float* t, float* pushed, uint8_t* holes, int* any, DevBuf& fillbuf);
int debug_view_dev(tw_ctx* ctx, const void* x, const void* y, const float* flow, int fw, int fh, int W, int H, int fmt,
                   int code, bool gouraud, void* out, DevBuf& warped, DevBuf& wp, DevBuf& luma);

}  // namespace tw

