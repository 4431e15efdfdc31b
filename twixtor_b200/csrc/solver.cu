// Pyramid filters and the optical flow solver, strict mode. Each kernel cites the reference
// function (plugins/retime-engine/src/...) whose per-element arithmetic it repeats.
#include "kernels.cuh"
#include "level.cuh"

namespace tw {
TW_VARIANT_BEGIN

// flow/conv.rs:101-137 (border_value_ordered): one border element of a line whose element t is
// line[t * stride]. `multi` selects the 2- and 3-channel rule (the -1.0 sentinel decides whether a
// tap exists, so a real sample of exactly -1.0 is dropped too); LEFT_FIRST adds the tap at i - j
// before the tap at i + j.
template <bool LEFT_FIRST, class T>
__device__ __forceinline__ float border_value(const float* __restrict__ line, long stride, int len, int i,
                                              const T& t, bool multi) {
    float centre = (i >= 0 && i < len) ? line[(long)i * stride] : 0.0f;
    float num = t.k[0] * centre;
    float den = t.k[0];
#pragma unroll 1
    for (int j = t.n - 1; j >= 1; j--) {
        float kj = t.k[j];
#pragma unroll
        for (int side = 0; side < 2; side++) {
            bool right = (side == 0) != LEFT_FIRST;
            int tt = right ? i + j : i - j;
            bool inside = tt >= 0 && tt < len;
            float xv, wv;
            if (!multi) {
                xv = inside ? line[(long)tt * stride] : 0.0f;
                wv = inside ? kj : 0.0f;
            } else {
                float v = inside ? line[(long)tt * stride] : -1.0f;
                float mask = (v != -1.0f) ? 1.0f : 0.0f;
                xv = v;
                wv = mask * kj;
            }
            den = den + wv;
            num = num + xv * wv;
        }
    }
    return num / den;
}

// conv.rs:141-190 (hrow + interior_run), one output sample per thread
template <class T>
__device__ __forceinline__ void conv_h_px(const float* __restrict__ src, float* __restrict__ dst, int w, int h,
                                          const T& t, bool multi) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const float* row = src + (long)y * w;
    int n = t.n;
    int head = min(n, w);
    int interior = max(w - 2 * n, 0);
    float r;
    if (x >= head && x < head + interior) {
        r = row[x] * t.k[0];
#pragma unroll 1
        for (int j = n - 1; j >= 1; j--) r = r + (row[x + j] + row[x - j]) * t.k[j];
    } else {
        r = border_value<false>(row, 1, w, x, t, multi);
    }
    dst[(long)y * w + x] = r;
}

// conv.rs:268-301 (vrow_ordered); the optional band output is flow.rs:266-267 (band = orig - blur)
template <class T>
__device__ __forceinline__ void conv_v_px(const float* __restrict__ src, float* __restrict__ dst, int w, int h,
                                          const T& t, bool multi, bool above_first, const float* __restrict__ orig,
                                          float* __restrict__ band) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    int n = t.n;
    int head = min(n, h);
    int interior = max(h - 2 * n, 0);
    float r;
    if (y >= head && y < head + interior) {
        r = src[(long)y * w + x] * t.k[0];
#pragma unroll 1
        for (int j = n - 1; j >= 1; j--) r = r + (src[(long)(y + j) * w + x] + src[(long)(y - j) * w + x]) * t.k[j];
    } else if (above_first) {
        r = border_value<true>(src + x, w, h, y, t, multi);
    } else {
        r = border_value<false>(src + x, w, h, y, t, multi);
    }
    long i = (long)y * w + x;
    dst[i] = r;
    if (band) band[i] = orig[i] - r;
}

__global__ void k_conv_h(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t, bool multi) {
    conv_h_px(src, dst, w, h, t, multi);
}

__global__ void k_conv_v(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t, bool multi,
                         bool above_first, const float* __restrict__ orig, float* __restrict__ band) {
    conv_v_px(src, dst, w, h, t, multi, above_first, orig, band);
}

// the same passes with the wide half kernels of the matte choke (one channel)
__global__ void k_conv_h_wide(const float* __restrict__ src, float* __restrict__ dst, int w, int h, WideTaps t) {
    conv_h_px(src, dst, w, h, t, false);
}

__global__ void k_conv_v_wide(const float* __restrict__ src, float* __restrict__ dst, int w, int h, WideTaps t,
                              bool above_first) {
    conv_v_px(src, dst, w, h, t, false, above_first, (const float*)nullptr, (float*)nullptr);
}

// ---- the 360 mode of the pyramid's filters (prep.rs:261-299, conv.rs:192-400, sample.rs:196-286) ------

// conv.rs:192-244 (hrow_wrapx): s = x[i] k0, then s = s + (x[(i+j) mod w] + x[(i-j) mod w]) k[j] for
// j = n-1 down to 1; the interior run is the same chain without a wrap
__global__ void k_conv_h_wrap(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const float* row = src + (long)y * w;
    float r = row[x] * t.k[0];
#pragma unroll 1
    for (int j = t.n - 1; j >= 1; j--) {
        int rr = (x + j) % w;
        int l = ((x - j) % w + w) % w;
        r = r + (row[rr] + row[l]) * t.k[j];
    }
    dst[(long)y * w + x] = r;
}

// conv.rs:326-400 (vpass_sphere): the element of column x at row yy, outside 0..h-1 found by the
// equirectangular walk from the edge row (reflect, and half a turn in x at every reflection)
__device__ __forceinline__ float sphere_at(const float* __restrict__ src, int w, int h, int x, int yy) {
    if (yy >= 0 && yy < h) return src[(long)yy * w + x];
    int half = w / 2;
    int c = x, r, d, steps;
    if (yy < 0) { r = 0; d = -1; steps = -yy; }
    else { r = h - 1; d = 1; steps = yy - h + 1; }
#pragma unroll 1
    for (int m = 0; m < steps; m++) {
        r += d;
        if (r < 0) { r = 0; d = -d; c = (half + c) % w; }
        else if (r >= h) { r = h - 1; d = -d; c = (half + c) % w; }
    }
    return src[(long)r * w + c];
}

// the column pass of the 360 mode: s = g[y] k0, s = s + (g[y+j] + g[y-j]) k[j]; with `band`, the band
// orig - s and its transpose (element (x, y) at [x * h + y]) for the column sweeps (flow.rs:264-267)
__global__ void k_conv_v_sphere(const float* __restrict__ src, float* __restrict__ dst, int w, int h, Taps t,
                                const float* __restrict__ orig, float* __restrict__ band, float* __restrict__ band_t) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    float r = src[(long)y * w + x] * t.k[0];
#pragma unroll 1
    for (int j = t.n - 1; j >= 1; j--) r = r + (sphere_at(src, w, h, x, y + j) + sphere_at(src, w, h, x, y - j)) * t.k[j];
    long i = (long)y * w + x;
    dst[i] = r;
    if (band) {
        float b = orig[i] - r;
        band[i] = b;
        if (band_t) band_t[(long)x * h + y] = b;
    }
}

// sample.rs:255-286 (bilinear1_sphere)
__device__ __forceinline__ float bilinear1_sphere(const float* __restrict__ img, int w, int h, float x, float y) {
    int w1 = w - 1, h1 = h - 1;
    int tx = cvtt32(x), ty = cvtt32(y);
    int ix = min(max(tx, 0), w1), iy = min(max(ty, 0), h1);
    float fx = x - (float)tx, fy = y - (float)ty;
    int x1 = ix + 1 > w1 ? 0 : ix + 1;
    int xc = ix, xd = x1, yc = iy + 1;
    if (iy + 1 > h1) {
        int half = w / 2;
        xc = (half + ix) % w;
        xd = (half + x1) % w;
        yc = h1;
    }
    float p00 = img[(long)iy * w + ix], p10 = img[(long)iy * w + x1];
    float p01 = img[(long)yc * w + xc], p11 = img[(long)yc * w + xd];
    float top = (p10 - p00) * fx + p00;
    float bot = (p11 - p01) * fx + p01;
    return (bot - top) * fy + top;
}

// sample.rs:205-230 (resample1_wrapx): the steps sw / dw and sh / dh, the equirectangular sampler
__global__ void k_resample_sphere(const float* __restrict__ src, int sw, int sh, float* __restrict__ dst, int dw, int dh) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    float sx = (float)sw / (float)dw, sy = (float)sh / (float)dh;
    dst[(long)y * dw + x] = bilinear1_sphere(src, sw, sh, (float)x * sx, (float)y * sy);
}

// flow/sample.rs:91-112 (resample1): corner aligned bilinear
__global__ void k_resample(const float* __restrict__ src, int sw, int sh, float* __restrict__ dst, int dw, int dh) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    float sx = ((float)sw - 1.0f) / (float)(dw - 1);
    float sy = ((float)sh - 1.0f) / (float)(dh - 1);
    dst[(long)y * dw + x] = bilinear1(src, sw, sh, (float)x * sx, (float)y * sy);
}

// flow.rs:283-328 (calc_grad, calc_a)
__global__ void k_grad_tensor(const float* __restrict__ img, int w, int h, float* __restrict__ gxo,
                              float* __restrict__ gyo, float* __restrict__ a0, float* __restrict__ a1,
                              float* __restrict__ a2) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    long i = (long)y * w + x;
    float c = img[i];
    float nx = 0.0f, dx = 0.0f, ny = 0.0f, dy = 0.0f;
    if (x >= 1) { nx = (c - img[i - 1]) + 0.0f; dx = 1.0f; }
    if (y >= 1) { ny = (c - img[i - w]) + 0.0f; dy = 1.0f; }
    if (x + 1 <= w - 1) { nx = nx + (img[i + 1] - c); dx = dx + 1.0f; }
    if (y + 1 <= h - 1) { ny = ny + (img[i + w] - c); dy = dy + 1.0f; }
    float gx = nx / dx, gy = ny / dy;
    gxo[i] = gx;
    gyo[i] = gy;
    a0[i] = gx * gx;
    a1[i] = gx * gy;
    a2[i] = gy * gy;
}

// flow.rs:334-357 (calc_b): i1 = imgA, i0 = imgB
__global__ void k_calc_b(const float* __restrict__ i1, const float* __restrict__ i0, const float* __restrict__ gx,
                         const float* __restrict__ gy, const float* __restrict__ fu, const float* __restrict__ fv,
                         int w, int h, float* __restrict__ bx, float* __restrict__ by) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    long i = (long)y * w + x;
    float fw = (float)w, fh = (float)h;
    float sx = (float)x - fu[i];
    float sy = (float)y - fv[i];
    if (sx < 0.0f || fw - 1.0f < sx || sy < 0.0f || fh - 1.0f < sy) {
        bx[i] = 0.0f;
        by[i] = 0.0f;
    } else {
        float s = bilinear1(i0, w, h, sx, sy);
        float r = s - i1[i];
        bx[i] = r * gx[i];
        by[i] = r * gy[i];
    }
}

// flow.rs:361-371 (new_disp)
__global__ void k_new_disp(float* __restrict__ fu, float* __restrict__ fv, const float* __restrict__ a0,
                           const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ bx,
                           const float* __restrict__ by, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float aa = a0[i], ab = a1[i], ad = a2[i];
    float b0 = bx[i], b1 = by[i];
    float t = ab * ab - ad * aa;
    if (fabsf(t) > 40.0f) {
        fu[i] = (ab * b1 - ad * b0) / t + fu[i];
        fv[i] = (ab * b0 - aa * b1) / t + fv[i];
    }
}

// flow.rs:430-442 (all_flow_out_of_range), as "some pixel is in range"
__global__ void k_range_any(const float* __restrict__ fu, const float* __restrict__ fv, int w, int h,
                            int* __restrict__ any_in_range) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    bool in = false;
    if (x < w && y < h) {
        long i = (long)y * w + x;
        float px = (float)x + fu[i];
        float py = (float)y + fv[i];
        float fw = (float)(w - 1), fh = (float)(h - 1);
        in = 0.0f <= px && px <= fw && 0.0f <= py && py <= fh;
    }
    if (__syncthreads_or(in) && threadIdx.x == 0) atomicOr(any_in_range, 1);
}

// flow.rs:1292-1300: state[0] = check (still live), state[1] = some pixel in range at this level
__global__ void k_range_apply(float* __restrict__ fu, float* __restrict__ fv, long n, int* __restrict__ state,
                              bool damp_now, float damp) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool zero = state[0] != 0 && state[1] == 0;
    float u = zero ? 0.0f : fu[i];
    float v = zero ? 0.0f : fv[i];
    if (damp_now) {  // scale_values (flow.rs:422-427): f * p, untouched for f == 1
        u = damp * u;
        v = damp * v;
    }
    fu[i] = u;
    fv[i] = v;
}

// the check state of a solve: check live, nothing in range yet (flow.rs:1270)
__global__ void k_range_init(int* __restrict__ state) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        state[0] = 1;
        state[1] = 0;
    }
}

// the check state after a level: check = check && nothing was in range; clears the flag for the next level
__global__ void k_range_next(int* __restrict__ state) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        state[0] = (state[0] != 0 && state[1] == 0) ? 1 : 0;
        state[1] = 0;
    }
}

// flow.rs:376-391 (upsample_flow) with sample.rs:69-86 (bilinear2) on the planar field
__global__ void k_upsample_flow(const float* __restrict__ su, const float* __restrict__ sv, int sw, int sh,
                                float* __restrict__ du, float* __restrict__ dv, int dw, int dh) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    float sx = ((float)dw - 1.0f) / (float)(sw - 1);
    float sy = ((float)dh - 1.0f) / (float)(sh - 1);
    float rx = (float)(1.0 / (double)sx);
    float ry = (float)(1.0 / (double)sy);
    int ix, iy;
    float fx, fy;
    cell((float)x * rx, sw, ix, fx);
    cell((float)y * ry, sh, iy, fy);
    long i = (long)iy * sw + ix;
    float r[2];
    const float* planes[2] = {su, sv};
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const float* p = planes[c];
        float p00 = p[i], p10 = p[i + 1], p01 = p[i + sw], p11 = p[i + sw + 1];
        float top = (p10 - p00) * fx + p00;
        float bot = (p11 - p01) * fx + p01;
        r[c] = (bot - top) * fy + top;
    }
    long o = (long)y * dw + x;
    du[o] = r[0] * sx;
    dv[o] = r[1] * sy;
}

// flow.rs:1305: scale_values(flow, -1.0), written interleaved; flags a NaN
__global__ void k_negate_interleave(const float* __restrict__ fu, const float* __restrict__ fv, long n,
                                    float* __restrict__ out, int* __restrict__ nan_flag) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float u = -1.0f * fu[i], v = -1.0f * fv[i];
    out[2 * i] = u;
    out[2 * i + 1] = v;
    if (isnan(u) || isnan(v)) atomicOr(nan_flag, 1);
}

__global__ void k_deinterleave(const float* __restrict__ in, long n, float* __restrict__ fu, float* __restrict__ fv) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fu[i] = in[2 * i];
    fv[i] = in[2 * i + 1];
}

__global__ void k_interleave(const float* __restrict__ fu, const float* __restrict__ fv, long n, float* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[2 * i] = fu[i];
    out[2 * i + 1] = fv[i];
}

__global__ void k_fill(float* __restrict__ p, long n, float v) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// =====================================================================================================
// Block matching (flow.rs:447-622).
//
// A sweep is an in-place, loop-carried recurrence along a row (or a column): with v the vectors
// before the sweep, v'[x] = accept(x, v'[x-1]) ? v'[x-1] : v[x], where accept(x, n) holds when the
// target of v[x] lies in the level, its block cost c0 exists, the cost c1 at the target of n
// exists and c1 < c0 (Block::step, flow.rs:529-546). Every v'[x] is therefore the ORIGINAL vector
// of the start s <= x of its run, and a run started at j continues while accept(x, v[j]) holds.
// The kernel evaluates that exactly, in parallel:
//   1. c0[x] and the validity of v[x] for every x of the line;
//   2. end[j] = the first x past j where accept(x, v[j]) fails, for every candidate start j;
//   3. the run starts: 0, end[0], end[end[0]], ... (a chain walked in shared memory);
//   4. v'[x] = v[start of x's run].
// Each cost evaluation is Block::cost bit for bit, so the result equals the sequential sweep.

// Shared memory of one line of length len: u, v, c0 (floats), the three rows of A along the line
// (floats), end and two queues (ints), then 8 counters and two ints per 32-position chunk.
size_t bm_smem_bytes(int len) { return (size_t)len * 4 * (3 + 3 + 3) + (size_t)(8 + 2 * ((len + 31) / 32)) * 4; }

constexpr int BM_STAGES = 3;      // run extension tests made one per queued candidate before the lane groups
constexpr int BM_GROUP = 8;       // lanes per queued candidate after the stages (positions tested per round)
static_assert(BM_GROUP >= 2 && BM_GROUP < 32 && 32 % BM_GROUP == 0, "groups tile a warp");
constexpr int BM_TERM = 1 << 30;  // "past the line" in the chain tables

// The 3x3 patch of A around line position i (flow.rs:454-469) from the three lines of A in shared
// memory (rows y-1..y+1 for a row sweep, columns x-1..x+1 for a column sweep).
template <bool COLS>
__device__ __forceinline__ void bm_patch(const float* s_a, int len, int i, float p[9]) {
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) p[r * 3 + c] = COLS ? s_a[c * len + (i - 1 + r)] : s_a[r * len + (i - 1 + c)];
}

// accept(i, n) of the sweep at line position i with its patch p (Block::step, flow.rs:529-546): ci is
// the cost of the current vector (NaN when the step cannot happen at i: no target or no cost).
template <bool COLS>
__device__ __forceinline__ bool bm_accept_p(const float p[9], const float* __restrict__ B, int w, int h, int fixed,
                                            int i, float nu, float nv, float ci) {
    if (isnan(ci)) return false;  // None, or a NaN cost that nothing compares below
    int x = COLS ? fixed : i, y = COLS ? i : fixed;
    float c1;
    if (!bm_cost<COLS>(B, w, h, p, (float)x - nu, (float)y - nv, c1)) return false;
    return c1 < ci;
}

template <bool COLS>
__device__ __forceinline__ bool bm_accept(const float* s_a, int len, const float* __restrict__ B, int w, int h,
                                          int fixed, int i, float nu, float nv, float ci) {
    float p[9];
    bm_patch<COLS>(s_a, len, i, p);
    return bm_accept_p<COLS>(p, B, w, h, fixed, i, nu, nv, ci);
}

// The cost of the vector (u, v) at line position i (flow.rs:529-536): NaN when its target leaves the
// level or the block has no cost.
template <bool COLS>
__device__ __forceinline__ float bm_own_cost(const float p[9], const float* __restrict__ B, int w, int h, int fixed,
                                             int i, float u, float v) {
    float c = __int_as_float(0x7fc00000);
    int x = COLS ? fixed : i, y = COLS ? i : fixed;
    float tx = (float)x - u;
    float ty = (float)y - v;
    if (0.0f <= tx && tx <= (float)(w - 1) && 0.0f <= ty && ty <= (float)(h - 1)) {
        float cost;
        if (bm_cost<COLS>(B, w, h, p, tx, ty, cost)) c = cost;
    }
    return c;
}

// Appends val to q (counter *n) for the lanes of the warp with `want`: one atomic per warp. Every lane
// of the warp calls it.
__device__ __forceinline__ void bm_push(int* q, int* n, bool want, int val) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (m) {
        const int lane = threadIdx.x & 31, lead = __ffs(m) - 1;
        int base = 0;
        if (lane == lead) base = atomicAdd(n, __popc(m));
        base = __shfl_sync(0xffffffffu, base, lead);
        if (want) q[base + __popc(m & ((1u << lane) - 1u))] = val;
    }
}

// One sweep over a line held in shared memory (su, sv: the field along the line, updated in place;
// s_a: the three lines of A across it). The line is the row y (COLS false: pixel (i, y)) or the
// column x (COLS true: pixel (x, i)); len is its length. Forward sweeps run i = 1..len-2 with the
// neighbour i - 1, reverse sweeps i = len-2..1 with the neighbour i + 1. In "sweep order" position
// q (q = i forward, q = len-1-i reverse) both are the same forward recurrence
// v'[q] = accept(q, v'[q-1]) ? v'[q-1] : v[q], so every v'[q] is the vector of its run's start, and
// a run started at j ends at end[j], the first position past j that refuses v[j]. The sweep:
//   1. c0[i], the cost of the current vector (the reverse sweep recomputes it only where the forward
//      sweep replaced the vector, those positions listed by the forward sweep), and the test of
//      v[q-1] at every q: end[q-1] = q where it refuses, the others queued;
//   2. the queued candidates extended one position per stage (BM_STAGES stages, the survivors
//      compacted after each), then the rest by groups of BM_GROUP lanes testing as many positions at once;
//   3. the chain of run starts 0, end[0], end[end[0]], ... in 32-position chunks, one warp per
//      chunk: the successor tables doubled by shuffles give every position's first chain element
//      past the chunk; one thread walks the chunks from position 0 (their entries and the last start
//      before each);
//   4. the owner of every position (the last start at or before it, by binary lifting over the
//      doubled tables from the chunk's entry), and v[owner] into the line.
// Every cost is Block::cost bit for bit, so the result equals the sequential sweep. The in place
// update is safe: step 4 reads only run starts, which keep their own vectors.
template <bool COLS>
__device__ void bm_sweep(float* su, float* sv, float* c0, const float* s_a, int* endp, int* qa, int* qb, int* ctl,
                         int* entry, int* prevl, const float* __restrict__ B, int w, int h, int fixed, int len,
                         bool reverse) {
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    auto line_of = [&](int q) -> int { return reverse ? len - 1 - q : q; };  // sweep position -> line index
    // 1. the reverse sweep's costs of the replaced vectors (qa holds their line indices, ctl[3] their count)
    if (reverse) {
        const int n = ctl[3];
        for (int k = tid; k < n; k += nt) {
            const int i = qa[k];
            float p[9];
            bm_patch<COLS>(s_a, len, i, p);
            c0[i] = bm_own_cost<COLS>(p, B, w, h, fixed, i, su[i], sv[i]);
        }
        __syncthreads();
    }
    //    the test of v[q-1] at q (candidate j = q - 1), the forward sweep computing c0 on the way
    for (int qb0 = 0; qb0 < len; qb0 += nt) {
        const int q = qb0 + tid, j = q - 1;
        bool more = false;
        if (q >= 1 && q < len) {
            if (q <= len - 2) {
                const int i = line_of(q), jl = line_of(j);
                float p[9];
                bm_patch<COLS>(s_a, len, i, p);
                float ci;
                if (!reverse) {
                    ci = bm_own_cost<COLS>(p, B, w, h, fixed, i, su[i], sv[i]);
                    c0[i] = ci;
                } else {
                    ci = c0[i];
                }
                if (!bm_accept_p<COLS>(p, B, w, h, fixed, i, su[jl], sv[jl], ci)) endp[j] = q;
                else if (q + 1 <= len - 2) more = true;
                else endp[j] = len - 1;
            } else {
                endp[j] = len - 1;  // j = len - 2: no position left to test
            }
        }
        bm_push(qa, ctl + 0, more, j);
    }
    __syncthreads();
    // 2. stage t tests position j + t + 2 of every queued candidate j (counters rotate over ctl[0..2]:
    //    stage t reads ctl[t % 3], appends to ctl[(t + 1) % 3] and clears ctl[(t + 2) % 3], whose last
    //    reader passed the barrier before this stage)
    int nq = ctl[0];
    int* cur = qa;
    int* nxt = qb;
    int t = 0;
    for (; t < BM_STAGES && nq > 0; t++) {
        if (tid == 0) ctl[(t + 2) % 3] = 0;
        const int step = t + 2;
        for (int kb = 0; kb < nq; kb += nt) {
            const int k = kb + tid;
            bool more = false;
            int j = 0;
            if (k < nq) {
                j = cur[k];
                const int qq = j + step;  // <= len - 2: a candidate is queued only with a position left
                const int jl = line_of(j), il = line_of(qq);
                if (!bm_accept<COLS>(s_a, len, B, w, h, fixed, il, su[jl], sv[jl], c0[il])) endp[j] = qq;
                else if (qq + 1 > len - 2) endp[j] = len - 1;
                else more = true;
            }
            bm_push(nxt, ctl + (t + 1) % 3, more, j);
        }
        __syncthreads();
        nq = ctl[(t + 1) % 3];
        int* sw = cur;
        cur = nxt;
        nxt = sw;
    }
    //    the long runs: a group of BM_GROUP lanes per candidate, BM_GROUP positions per test round
    if (nq > 0) {
        constexpr int GPW = 32 / BM_GROUP;  // groups per warp
        const int g = lane / BM_GROUP, sub = lane % BM_GROUP, step = BM_STAGES + 2;
        for (int kb = warp * GPW; kb < nq; kb += nw * GPW) {
            const int k = kb + g;
            bool live = k < nq;
            const int j = live ? cur[k] : 0;
            const int jl = line_of(j);
            const float nu = live ? su[jl] : 0.0f, nv = live ? sv[jl] : 0.0f;
            int pos = j + step;
            for (int guard = 0; guard <= len && __any_sync(FULL, live); guard += BM_GROUP) {
                const int qq = pos + sub;
                bool refuse = false;
                if (live && qq <= len - 2) {
                    const int il = line_of(qq);
                    refuse = !bm_accept<COLS>(s_a, len, B, w, h, fixed, il, nu, nv, c0[il]);
                }
                const unsigned gm = (__ballot_sync(FULL, refuse) >> (g * BM_GROUP)) & ((1u << BM_GROUP) - 1u);
                if (live) {
                    if (gm) {
                        if (sub == 0) endp[j] = pos + __ffs(gm) - 1;
                        live = false;
                    } else if (pos + BM_GROUP > len - 2) {
                        if (sub == 0) endp[j] = len - 1;
                        live = false;
                    } else {
                        pos += BM_GROUP;
                    }
                }
            }
        }
    }
    __syncthreads();
    // 3. per chunk: J = the successor (end) doubled five times, L = the last start inside the chunk on
    //    the way; the queues are free now and take the two tables
    const int nch = (len + 31) >> 5;
    int* exitq = qa;
    int* lastq = qb;
    for (int c = warp; c < nch; c += nw) {
        const int base = c << 5, q = base + lane;
        int J = q <= len - 2 ? endp[q] : BM_TERM;
        int L = q;
#pragma unroll
        for (int r = 0; r < 5; r++) {
            const int src = J - base;  // > 0: a successor lies past its position
            const int tJ = __shfl_sync(FULL, J, src & 31);
            const int tL = __shfl_sync(FULL, L, src & 31);
            if (src < 32) {
                J = tJ;
                L = tL;
            }
        }
        if (q < len) {
            exitq[q] = J;
            lastq[q] = L;
        }
    }
    __syncthreads();
    //    the walk over the chunks from position 0: entry[c] = the first start in chunk c (-1: none),
    //    prevl[c] = the last start before it
    if (tid == 0) {
        int E = 0, Lp = -1, k = 0;
        for (int guard = 0; guard < len; guard++) {
            const int kE = E >> 5;
            for (; k < kE; k++) {
                entry[k] = -1;
                prevl[k] = Lp;
            }
            entry[kE] = E;
            prevl[kE] = Lp;
            k = kE + 1;
            Lp = lastq[E];
            const int F = exitq[E];
            if (F >= len - 1) break;  // the line's last position, or past it: no start to follow
            E = F;
        }
        for (; k < nch; k++) {
            entry[k] = -1;
            prevl[k] = Lp;
        }
        ctl[0] = ctl[1] = ctl[2] = ctl[3] = 0;  // the next sweep's counters and the list of replaced positions
    }
    __syncthreads();
    // 4. owners by binary lifting from the chunk's entry over the doubled tables Jr[r] (2^r successors,
    //    saturated at the chunk's end), then the scatter; the forward sweep lists the replaced
    //    positions for the reverse sweep's costs
    for (int c = warp; c < nch; c += nw) {
        const int base = c << 5, q = base + lane;
        int Jr[5];
        Jr[0] = q <= len - 2 ? endp[q] : BM_TERM;
#pragma unroll
        for (int r = 1; r < 5; r++) {
            const int src = Jr[r - 1] - base;
            const int tv = __shfl_sync(FULL, Jr[r - 1], src & 31);
            Jr[r] = src < 32 ? tv : Jr[r - 1];
        }
        const int e = entry[c];
        int own = prevl[c];
        if (e >= 0) {  // the same for the whole warp
            int x = e;
#pragma unroll
            for (int r = 4; r >= 0; r--) {
                const int y = __shfl_sync(FULL, Jr[r], (x - base) & 31);
                if (y <= q) x = y;
            }
            if (q >= e) own = x;
        }
        const bool moved = q >= 1 && q <= len - 2 && own != q;
        const int i = line_of(q);
        if (moved) {
            const int o = line_of(own);
            su[i] = su[o];
            sv[i] = sv[o];
        }
        if (!reverse) bm_push(qa, ctl + 3, moved, i);
    }
    __syncthreads();
}

// The two sweeps of a line (flow.rs:551-622: left to right then right to left, or top to bottom
// then bottom to top), with the field, A's three lines and the tables in shared memory. The line is
// read contiguously from src (row y of the row-major field, or column x of the transposed one; a
// column's two end elements, which no sweep changes, from the row-major field ends) and its swept
// interior written across: element i of line `fixed` to dst[i * other + fixed], other = h for a row
// (into the transposed field the column sweeps read) and w for a column (back into the row-major
// field). So no transpose of the field runs between the row and the column sweeps; the reference
// transposes its field for the column sweeps (flow.rs:583-621). A and B of a column sweep are the
// transposed planes (element (x, y) at [x * h + y]) so that the line's patches stay contiguous.
template <bool COLS>
__device__ void bm_line(const float* __restrict__ A, const float* __restrict__ B, const float* src_u,
                        const float* src_v, const float* ends_u, const float* ends_v, float* dst_u, float* dst_v, int w,
                        int h, int fixed) {
    extern __shared__ float sm[];
    const int len = COLS ? h : w, other = COLS ? w : h;
    if (len < 3) return;  // no interior position
    const int nch = (len + 31) >> 5;
    float* su = sm;
    float* sv = su + len;
    float* c0 = sv + len;
    float* s_a = c0 + len;  // 3 * len
    int* endp = (int*)(s_a + 3 * len);
    int* qa = endp + len;
    int* qb = qa + len;
    int* ctl = qb + len;  // 8 counters
    int* entry = ctl + 8;
    int* prevl = entry + nch;
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
        if (COLS && (i == 0 || i == len - 1)) {
            su[i] = ends_u[(long)i * w + fixed];
            sv[i] = ends_v[(long)i * w + fixed];
        } else {
            su[i] = src_u[(long)fixed * len + i];
            sv[i] = src_v[(long)fixed * len + i];
        }
#pragma unroll
        for (int o = 0; o < 3; o++)  // A at offset o-1 across the line: rows y-1..y+1, or columns x-1..x+1
            s_a[o * len + i] = __ldg(A + (long)(fixed - 1 + o) * len + i);
    }
    if (threadIdx.x < 8) ctl[threadIdx.x] = 0;
    __syncthreads();
    bm_sweep<COLS>(su, sv, c0, s_a, endp, qa, qb, ctl, entry, prevl, B, w, h, fixed, len, false);
    bm_sweep<COLS>(su, sv, c0, s_a, endp, qa, qb, ctl, entry, prevl, B, w, h, fixed, len, true);
    for (int i = threadIdx.x + 1; i <= len - 2; i += blockDim.x) {
        dst_u[(long)i * other + fixed] = su[i];
        dst_v[(long)i * other + fixed] = sv[i];
    }
}

// Two planes of w x h (row major) into their transposes (h x w), through a padded shared tile.
__global__ void k_transpose2(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ at,
                             float* __restrict__ bt, int w, int h) {
    __shared__ float ta[32][33], tb[32][33];
    int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int x = x0 + threadIdx.x, y = y0 + r;
        if (x < w && y < h) {
            ta[r][threadIdx.x] = a[(long)y * w + x];
            tb[r][threadIdx.x] = b[(long)y * w + x];
        }
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int y = y0 + threadIdx.x, x = x0 + r;
        if (x < w && y < h) {
            at[(long)x * h + y] = ta[threadIdx.x][r];
            bt[(long)x * h + y] = tb[threadIdx.x][r];
        }
    }
}

// The row sweeps of rows 1..h-2 of the field (fu, fv), the result into the transposed planes
// (uT, vT; element (x, y) at [x * h + y]) at the interior of those rows
__global__ void k_bm_rows(const float* __restrict__ A, const float* __restrict__ B, const float* __restrict__ fu,
                          const float* __restrict__ fv, int w, int h, float* __restrict__ uT, float* __restrict__ vT) {
    int y = blockIdx.x + 1;  // rows 1..h-2
    if (y > h - 2) return;
    bm_line<false>(A, B, fu, fv, nullptr, nullptr, uT, vT, w, h, y);
}

// The column sweeps of columns 1..w-2 from the transposed planes (uT, vT) that k_bm_rows wrote, the
// end rows 0 and h-1 from (fu, fv); the result into (fu, fv) at rows 1..h-2 of those columns
__global__ void k_bm_cols(const float* __restrict__ AT, const float* __restrict__ BT, const float* __restrict__ uT,
                          const float* __restrict__ vT, int w, int h, float* fu, float* fv) {
    int x = blockIdx.x + 1;  // columns 1..w-2
    if (x > w - 2) return;
    bm_line<true>(AT, BT, uT, vT, fu, fv, fu, fv, w, h, x);
}

TW_VARIANT_END
}  // namespace tw
