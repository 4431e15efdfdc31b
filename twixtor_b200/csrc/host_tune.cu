// The autotuner: per level size of a solve, the launch shapes of the solver iteration (tile shape
// and block size) and of block matching (block size per line), measured on the device and kept in
// the context's table, with a JSON file as its persistent cache. Every shape computes the same
// bytes (each element keeps the reference's operation order whatever the tiling), so the table
// changes only the time.
#include "runtime.h"

namespace tw {

// Deterministic stand-in data for the timings: planes of band-like values (a hash of the index,
// centred on 0, amplitude `amp`) and a small flow.
__global__ void k_tune_fill(float* p, long n, uint32_t seed, float amp) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t x = (uint32_t)i * 2654435761u ^ seed;
    x ^= x >> 15;
    x *= 2246822519u;
    x ^= x >> 13;
    p[i] = ((float)(x & 0xffffff) / 16777216.0f - 0.5f) * amp;
}

uint64_t key(int w, int h) { return ((uint64_t)(uint32_t)w << 32) | (uint32_t)h; }
bool valid_threads(int t, int max) { return t >= 32 && t <= max && t % 32 == 0; }

namespace {

const char* tile_name(int t) { return t == LEVEL_TILE_64x64 ? "64x64" : t == LEVEL_TILE_64x32 ? "64x32" : "32x32"; }

// The table as JSON: the device's name, then one entry per level size.
std::string table_json(tw_ctx* ctx) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, ctx->device);
    std::string out = "{\n  \"device\": \"";
    out += prop.name;
    out += "\",\n  \"levels\": {\n";
    size_t k = 0;
    char line[256];
    for (auto& kv : ctx->tune_table) {
        int w = (int)(kv.first >> 32), h = (int)(kv.first & 0xffffffffu);
        const LevelTune& t = kv.second;
        snprintf(line, sizeof line,
                 "    \"%dx%d\": {\"iter_tile\": \"%s\", \"iter_threads\": %d, \"bm_rows_threads\": %d, "
                 "\"bm_cols_threads\": %d}%s\n",
                 w, h, tile_name(t.iter_tile), t.iter_threads, t.bm_rows_threads, t.bm_cols_threads,
                 ++k < ctx->tune_table.size() ? "," : "");
        out += line;
    }
    out += "  }\n}\n";
    return out;
}

// Reads the entries of a table this library wrote for the same device; other lines are ignored.
void load_table(tw_ctx* ctx, const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return;
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, ctx->device);
    char line[512];
    bool same_device = false;
    while (fgets(line, sizeof line, f)) {
        char dev[256];
        if (sscanf(line, " \"device\": \"%255[^\"]\"", dev) == 1) same_device = std::strcmp(dev, prop.name) == 0;
        int w, h, it, rt, ct;
        char tile[16];
        if (same_device &&
            sscanf(line, " \"%dx%d\": {\"iter_tile\": \"%15[0-9x]\", \"iter_threads\": %d, \"bm_rows_threads\": %d, "
                         "\"bm_cols_threads\": %d}",
                   &w, &h, tile, &it, &rt, &ct) == 6) {
            int t = std::strcmp(tile, "64x64") == 0 ? LEVEL_TILE_64x64 : std::strcmp(tile, "64x32") == 0 ? LEVEL_TILE_64x32
                                                                                                        : LEVEL_TILE_32x32;
            if (w > 0 && h > 0 && valid_threads(it, LEVEL_ITER_MAX_THREADS) && valid_threads(rt, 1024) &&
                valid_threads(ct, 1024))
                ctx->tune_table[key(w, h)] = LevelTune{t, it, rt, ct};
        }
    }
    fclose(f);
}

}  // namespace
}  // namespace tw

extern "C" {

int tw_autotune(tw_ctx* ctx, const tw_flow_settings* s, int32_t width, int32_t height, const char* path,
                int32_t* measured) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cur = ctx->stream;
    if (measured) *measured = 0;
    if (!s || width <= 0 || height <= 0) return ctx->fail(TW_ERR_BAD_PARAM, "autotune: bad argument");
    Geo g;
    CHECK(geometry(*s, width, height, &g, &ctx->err));
    if (path) load_table(ctx, path);
    std::vector<int> todo;
    for (int l = 0; l < g.levels; l++)
        if (!ctx->tune_table.count(key(g.sizes[l][0], g.sizes[l][1]))) todo.push_back(l);
    if (!todo.empty()) {
        // stand-in planes of the largest level: A, B, the gradient, the tensor, the flow in and out,
        // the transposes, and a copy of the flow that block matching updates in place
        size_t n0 = (size_t)g.w * g.h;
        DevBuf buf;
        size_t held = 0;
        const int NP = 16;
        // and two B buffers (two planes each) of pitch (w + 3) & ~3, 16-byte aligned
        const size_t boff = (NP * n0 + 3) & ~(size_t)3;
        const long bplane = (long)((g.w + 3) & ~3) * g.h;
        cudaError_t e = buf.ensure((boff + 4 * (size_t)bplane) * sizeof(float), &held);
        if (e != cudaSuccess) return ctx->cuda(e, "autotune buffers");
        float* p = buf.as<float>();
        float *A = p, *Bp = p + n0, *gx = p + 2 * n0, *gy = p + 3 * n0, *a0 = p + 4 * n0, *a1 = p + 5 * n0,
              *a2 = p + 6 * n0, *fu = p + 7 * n0, *fv = p + 8 * n0, *nu = p + 9 * n0, *nv = p + 10 * n0,
              *AT = p + 11 * n0, *BT = p + 12 * n0, *uT = p + 13 * n0, *vT = p + 14 * n0, *fsave = p + 15 * n0;
        const float amps[15] = {40.f, 40.f, 8.f, 8.f, 60.f, 20.f, 60.f, 3.f, 3.f, 0.f, 0.f, 40.f, 40.f, 0.f, 0.f};
        for (int i = 0; i < 15; i++) {
            k_tune_fill<<<grid1((long)n0), TB, 0, ctx->stream>>>(p + i * n0, (long)n0, 0x9e3779b9u * (i + 1), amps[i]);
            ctx->launches++;
        }
        float* bin = p + boff;
        float* bout = bin + 2 * bplane;
        k_tune_fill<<<grid1(2 * bplane), TB, 0, ctx->stream>>>(bin, 2 * bplane, 0x85ebca6bu, 50.f);
        ctx->launches++;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        auto timed = [&](auto&& run) -> float {  // the best of three after a warm-up launch
            run();
            float best = 1e30f;
            for (int r = 0; r < 3; r++) {
                cudaEventRecord(e0, ctx->stream);
                run();
                cudaEventRecord(e1, ctx->stream);
                cudaEventSynchronize(e1);
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                best = std::min(best, ms);
            }
            return best;
        };
        bool af = s->taps_above_first != 0;
        for (int l : todo) {
            int w = g.sizes[l][0], h = g.sizes[l][1];
            LevelTune best = default_tune(w, h);
            // the solver iteration: every tile shape with 256 and 512 threads (64 x 64 with 512)
            const LevelTune iter_cands[5] = {{LEVEL_TILE_32x32, 256, 0, 0}, {LEVEL_TILE_32x32, 512, 0, 0},
                                             {LEVEL_TILE_64x32, 256, 0, 0}, {LEVEL_TILE_64x32, 512, 0, 0},
                                             {LEVEL_TILE_64x64, 512, 0, 0}};
            float bt = 1e30f;
            for (const LevelTune& c : iter_cands) {
                float ms = timed([&] { level_iter(ctx, c, A, Bp, gx, gy, a0, a1, a2, fu, fv, w, h, af, nu, nv, nullptr, false, bin, bout,
                                                  (w + 3) & ~3, bplane); });
                if (ms < bt) {
                    bt = ms;
                    best.iter_tile = c.iter_tile;
                    best.iter_threads = c.iter_threads;
                }
            }
            // block matching: the row and the column kernel, 128 to 512 threads per line (each one's
            // input field restored before every launch)
            if (w >= 3 && h >= 3) {
                cudaMemcpyAsync(fsave, fu, (size_t)w * h * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream);
                float br = 1e30f, bc = 1e30f;
                for (int th : {128, 256, 512}) {
                    float ms = timed([&] {
                        cudaMemcpyAsync(fu, fsave, (size_t)w * h * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream);
                        LAUNCH(ctx, k_bm_rows, h - 2, th, bm_smem_bytes(w), A, Bp, fu, fv, w, h, uT, vT);
                    });
                    if (ms < br) { br = ms; best.bm_rows_threads = th; }
                    ms = timed([&] {
                        cudaMemcpyAsync(uT, fsave, (size_t)w * h * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream);
                        LAUNCH(ctx, k_bm_cols, w - 2, th, bm_smem_bytes(h), AT, BT, uT, vT, w, h, fu, fv);
                    });
                    if (ms < bc) { bc = ms; best.bm_cols_threads = th; }
                }
            }
            ctx->tune_table[key(w, h)] = best;
            if (measured) (*measured)++;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        e = cudaStreamSynchronize(ctx->stream);
        if (e == cudaSuccess) e = cudaGetLastError();
        buf.release(&held);
        if (e != cudaSuccess) return ctx->cuda(e, "autotune");
    }
    if (path) {
        FILE* f = fopen(path, "w");
        if (!f) return ctx->fail(TW_ERR_BAD_PARAM, "autotune: cannot write %s", path);
        std::string js = table_json(ctx);
        fwrite(js.data(), 1, js.size(), f);
        fclose(f);
    }
    return TW_OK;
}

size_t tw_tuning_table(tw_ctx* ctx, char* buf, size_t cap) {
    if (!ctx) return 0;
    std::lock_guard<std::mutex> lk(ctx->mu);
    std::string js = table_json(ctx);
    if (buf && cap) {
        size_t m = std::min(js.size(), cap - 1);
        std::memcpy(buf, js.data(), m);
        buf[m] = 0;
    }
    return js.size();
}

int tw_tuning_clear(tw_ctx* ctx) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tune_table.clear();
    return TW_OK;
}

}  // extern "C"

extern "C" int tw_tuning_set(tw_ctx* ctx, int32_t width, int32_t height, int32_t iter_tile, int32_t iter_threads,
                             int32_t bm_rows_threads, int32_t bm_cols_threads) {
    if (!ctx) return TW_ERR_BAD_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (width <= 0 || height <= 0 || iter_tile < 0 || iter_tile >= LEVEL_TILE_COUNT ||
        !tw::valid_threads(iter_threads, LEVEL_ITER_MAX_THREADS) || !tw::valid_threads(bm_rows_threads, 1024) ||
        !tw::valid_threads(bm_cols_threads, 1024))
        return ctx->fail(TW_ERR_BAD_PARAM, "tuning entry: tile %d, threads %d / %d / %d", iter_tile, iter_threads,
                         bm_rows_threads, bm_cols_threads);
    ctx->tune_table[tw::key(width, height)] = LevelTune{iter_tile, iter_threads, bm_rows_threads, bm_cols_threads};
    return TW_OK;
}
