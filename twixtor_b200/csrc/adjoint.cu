// The adjoint of warp + blend (the differentiable twin of compose_vectors' Blend with warping code
// 0): out = ta + (tb - ta) * w with ta = warp(A, F_BA, 1 - wa), tb = warp(B, F_AB, wa), w = 1 - wa,
// where warp(S, F, s)(p) samples S bilinearly at p + F(p r) (s / r) (the flow sampled bilinearly at
// p r, r = (flow size - 1) / (image size - 1) per axis, the step s / r formed once per side as
// warp.rs:636-651 forms sx, sy), the position clamped
// to the image rectangle. One fused kernel per pixel recomputes the forward sample (nothing of the
// forward pass is stored), takes the output gradient (given, or the sign of out - target for the
// photometric L1 loss) and scatters:
//   dA, dB     the bilinear weights times (1 - w) g and w g, accumulated per CTA in a shared tile
//              of the box the CTA's samples reach, then added to global memory once per pixel
//              (vector atomics; straight to global memory when the box does not fit);
//   dF_BA, dF_AB  the image gradient at the sample point times s / r, through the flow's bilinear
//              weights: accumulated per CTA in shared memory (a tile of flow texels), then added
//              to global memory once per texel.
// Frames are float RGBA (4 channels, any premultiplication), batch items back to back.
#include "kernels.cuh"
#include <climits>

namespace tw {

namespace {

constexpr int FT_X = ADJ_TX + 2, FT_Y = ADJ_TY + 2;  // the flow texel tile when r <= 1 per axis

__device__ __forceinline__ float4 ld4(const float* p, long i) { return reinterpret_cast<const float4*>(p)[i]; }

struct Sample {
    int ix, iy;      // top left corner
    float fx, fy;    // fractions
    bool cx, cy;     // position clamped (no positional gradient on that axis)
};

// the bilinear footprint of (x, y) in a w x h grid, the last column / row folded as warp.rs does
__device__ __forceinline__ void footprint(float x, float y, int w, int h, int& ix, int& iy, float& fx, float& fy) {
    ix = (int)floorf(x);
    iy = (int)floorf(y);
    fx = x - (float)ix;
    fy = y - (float)iy;
    if (ix >= w - 1) { ix = w - 2; fx = 1.0f; }
    if (iy >= h - 1) { iy = h - 2; fy = 1.0f; }
    if (ix < 0) { ix = 0; fx = 0.0f; }
    if (iy < 0) { iy = 0; fy = 0.0f; }
}

__device__ __forceinline__ Sample sample_at(float px, float py, int w, int h) {
    Sample s;
    s.cx = !(px >= 0.0f && px <= (float)(w - 1));
    s.cy = !(py >= 0.0f && py <= (float)(h - 1));
    px = fminf(fmaxf(px, 0.0f), (float)(w - 1));
    py = fminf(fmaxf(py, 0.0f), (float)(h - 1));
    footprint(px, py, w, h, s.ix, s.iy, s.fx, s.fy);
    return s;
}

__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t, a.w + (b.w - a.w) * t);
}

__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

__device__ __forceinline__ float4 scale4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }

// One side: the sample of S (and its four corners) at p + F(p r) (s / r); sx, sy = s / r
struct Side {
    Sample smp;
    float4 val;
    int fix, fiy;    // the flow footprint
    float ffx, ffy;
};

__device__ __forceinline__ Side side_at(const float* S, const float* F, const AdjParams& P, int x, int y, float sx,
                                        float sy) {
    Side d;
    float qx = (float)x * P.rx, qy = (float)y * P.ry;
    footprint(qx, qy, P.fw, P.fh, d.fix, d.fiy, d.ffx, d.ffy);
    long f00 = ((long)d.fiy * P.fw + d.fix) * 2, f01 = f00 + (long)P.fw * 2;
    float2 a = *reinterpret_cast<const float2*>(F + f00), b = *reinterpret_cast<const float2*>(F + f00 + 2);
    float2 c = *reinterpret_cast<const float2*>(F + f01), e = *reinterpret_cast<const float2*>(F + f01 + 2);
    float u = (a.x + (b.x - a.x) * d.ffx) * (1.0f - d.ffy) + (c.x + (e.x - c.x) * d.ffx) * d.ffy;
    float v = (a.y + (b.y - a.y) * d.ffx) * (1.0f - d.ffy) + (c.y + (e.y - c.y) * d.ffx) * d.ffy;
    float px = (float)x + u * sx, py = (float)y + v * sy;
    d.smp = sample_at(px, py, P.w, P.h);
    long i00 = (long)d.smp.iy * P.w + d.smp.ix, i01 = i00 + P.w;
    d.val = lerp4(lerp4(ld4(S, i00), ld4(S, i00 + 1), d.smp.fx), lerp4(ld4(S, i01), ld4(S, i01 + 1), d.smp.fx), d.smp.fy);
    return d;
}

// where a side's image gradient goes: a shared tile of the CTA's box (tile != nullptr) or the
// global gradient (vector atomics)
struct Acc {
    float* tile;     // four planes of ADJ_BOX_PX floats (a warp's adjacent pixels on adjacent banks)
    int bx, by, bw, bh;
    float* global;   // a cell outside the box (a NaN flow) goes here too
};

__device__ __forceinline__ void acc_add(const Acc& c, const AdjParams& P, int px, int py, float4 v) {
    int lx = px - c.bx, ly = py - c.by;
    if (c.tile && lx >= 0 && lx < c.bw && ly >= 0 && ly < c.bh) {
        float* t = c.tile + (ly * c.bw + lx);
        atomicAdd(t, v.x);
        atomicAdd(t + ADJ_BOX_PX, v.y);
        atomicAdd(t + 2 * ADJ_BOX_PX, v.z);
        atomicAdd(t + 3 * ADJ_BOX_PX, v.w);
    } else if (c.global) {
        atomicAdd(reinterpret_cast<float4*>(c.global) + ((long)py * P.w + px), v);
    }
}

// the gradient of one side: dS at the four corners, the positional gradient into the flow tile
// (shared) or straight to global memory
__device__ __forceinline__ void side_back(const float* S, const Side& d, float4 g, const AdjParams& P, const Acc& acc,
                                          float* sflow, int tx0, int ty0, bool tiled, float* dF, float sx, float sy) {
    const Sample& s = d.smp;
    float w00 = (1.0f - s.fx) * (1.0f - s.fy), w10 = s.fx * (1.0f - s.fy), w01 = (1.0f - s.fx) * s.fy, w11 = s.fx * s.fy;
    acc_add(acc, P, s.ix, s.iy, scale4(g, w00));
    acc_add(acc, P, s.ix + 1, s.iy, scale4(g, w10));
    acc_add(acc, P, s.ix, s.iy + 1, scale4(g, w01));
    acc_add(acc, P, s.ix + 1, s.iy + 1, scale4(g, w11));
    if (!dF) return;
    // d val / d px and d val / d py of the bilinear sample, per channel (the corners read again: the
    // forward kept only the value)
    long i00 = (long)s.iy * P.w + s.ix, i01 = i00 + P.w;
    float4 c00 = ld4(S, i00), c10 = ld4(S, i00 + 1), c01 = ld4(S, i01), c11 = ld4(S, i01 + 1);
    float4 dx = lerp4(make_float4(c10.x - c00.x, c10.y - c00.y, c10.z - c00.z, c10.w - c00.w),
                      make_float4(c11.x - c01.x, c11.y - c01.y, c11.z - c01.z, c11.w - c01.w), s.fy);
    float4 dy = lerp4(make_float4(c01.x - c00.x, c01.y - c00.y, c01.z - c00.z, c01.w - c00.w),
                      make_float4(c11.x - c10.x, c11.y - c10.y, c11.z - c10.z, c11.w - c10.w), s.fx);
    float gu = s.cx ? 0.0f : dot4(g, dx) * sx;
    float gv = s.cy ? 0.0f : dot4(g, dy) * sy;
    float fw00 = (1.0f - d.ffx) * (1.0f - d.ffy), fw10 = d.ffx * (1.0f - d.ffy), fw01 = (1.0f - d.ffx) * d.ffy,
          fw11 = d.ffx * d.ffy;
    const int cx[4] = {0, 1, 0, 1}, cy[4] = {0, 0, 1, 1};
    const float wt[4] = {fw00, fw10, fw01, fw11};
    if (tiled) {
        // adjacent lanes whose samples share the flow cell (a flow at half the image size pairs
        // them) add their contributions first: one shared atomic for the pair
        // (lanes past the image's right edge are inactive: only the active ones exchange)
        int lane = threadIdx.x & 31;
        unsigned mask = __activemask();
        int key = d.fiy * P.fw + d.fix;
        int okey = __shfl_xor_sync(mask, key, 1);
        bool pair = (mask >> (lane ^ 1) & 1u) && okey == key;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float u = gu * wt[k], v = gv * wt[k];
            float ou = __shfl_xor_sync(mask, u, 1), ov = __shfl_xor_sync(mask, v, 1);
            if (pair) {
                if (lane & 1) continue;
                u += ou;
                v += ov;
            }
            if (u == 0.0f && v == 0.0f) continue;
            int lx = d.fix + cx[k] - tx0, ly = d.fiy + cy[k] - ty0;
            atomicAdd(sflow + (ly * FT_X + lx) * 2, u);
            atomicAdd(sflow + (ly * FT_X + lx) * 2 + 1, v);
        }
        return;
    }
    if (gu == 0.0f && gv == 0.0f) return;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int fx = d.fix + cx[k], fy = d.fiy + cy[k];
        atomicAdd(reinterpret_cast<float2*>(dF) + ((long)fy * P.fw + fx), make_float2(gu * wt[k], gv * wt[k]));
    }
}

}  // namespace

// One CTA per 32 x 32 output tile of a batch item, 256 threads, 4 pixels a thread (the columns of a
// warp adjacent). Three passes: (1) the bounding box of each side's sample cells, from the extremes
// of the flow texels the tile reads;
// (2) the forward recomputed, the loss and the backward, the image gradients added into a shared
// tile of each box (when it fits, else straight to global memory with vector atomics) and the flow
// gradients into the shared flow tile; (3) the shared tiles added to global memory, one coalesced
// vector atomic per touched pixel. Smooth flows shift a tile nearly rigidly, so a box holds about
// one tile: the global atomics drop from 8 to about 2.5 per output pixel.
__global__ void __launch_bounds__(ADJ_THREADS, 3) k_warp_blend_adjoint(AdjParams P) {
    extern __shared__ float4 adj_smem[];
    float* sacc0 = reinterpret_cast<float*>(adj_smem);  // four planes of ADJ_BOX_PX floats per side
    float* sacc1 = sacc0 + 4 * ADJ_BOX_PX;
    float* sflow0 = sacc1 + 4 * ADJ_BOX_PX;
    float* sflow1 = sflow0 + FT_X * FT_Y * 2;
    __shared__ int box[2][4];                       // min x, min y, max x, max y of the cells
    int b = blockIdx.z;
    long img = (long)P.w * P.h * 4 * b, flo = (long)P.fw * P.fh * 2 * b;
    const float* A = P.a + img;
    const float* B = P.b + img;
    const float* Fba = P.f_ba + flo;
    const float* Fab = P.f_ab + flo;
    float frac = 1.0f - P.wa;
    // the steps per flow unit of the two sides (A by F_BA at 1 - wa, B by F_AB at wa)
    const float sxa = frac / P.rx, sya = frac / P.ry, sxb = P.wa / P.rx, syb = P.wa / P.ry;
    int x0 = blockIdx.x * ADJ_TX, y0 = blockIdx.y * ADJ_TY;
    int x = x0 + (int)(threadIdx.x % ADJ_TX);
    int yb = y0 + (int)(threadIdx.x / ADJ_TX);
    const int ROWS = ADJ_THREADS / ADJ_TX;  // 8 rows a pass
    int tx0 = min((int)floorf((float)x0 * P.rx), max(P.fw - 2, 0));
    int ty0 = min((int)floorf((float)y0 * P.ry), max(P.fh - 2, 0));
    bool tiled = P.tiled;
    bool backward = P.grad_out || P.target;
    if (threadIdx.x < 2) {
        box[threadIdx.x][0] = INT_MAX;
        box[threadIdx.x][1] = INT_MAX;
        box[threadIdx.x][2] = INT_MIN;
        box[threadIdx.x][3] = INT_MIN;
    }
    if (tiled)
        for (int i = threadIdx.x; i < FT_X * FT_Y * 2; i += blockDim.x) sflow0[i] = sflow1[i] = 0.0f;
    __syncthreads();
    // pass 1: the boxes the samples reach, from the flow texels the tile's pixels read: the flow at
    // a pixel is a convex combination of its footprint's texels, and every step from the flow to
    // the sample cell is monotone, so the extremes of the texels bound the cells
    __shared__ float ext[ADJ_THREADS / 32][2][4];  // per warp and side: min u, max u, min v, max v
    if (backward) {
        int xe = min(x0 + ADJ_TX - 1, P.w - 1), ye = min(y0 + ADJ_TY - 1, P.h - 1);
        int fx0, fy0, fx1, fy1;
        float t0, t1;
        footprint((float)x0 * P.rx, (float)y0 * P.ry, P.fw, P.fh, fx0, fy0, t0, t1);
        footprint((float)xe * P.rx, (float)ye * P.ry, P.fw, P.fh, fx1, fy1, t0, t1);
        int tw = fx1 + 2 - fx0, th = fy1 + 2 - fy0;
        float e[2][4];
#pragma unroll
        for (int s = 0; s < 2; s++) e[s][0] = e[s][2] = INFINITY, e[s][1] = e[s][3] = -INFINITY;
        for (int ty = threadIdx.x >> 5; ty < th; ty += blockDim.x >> 5) {  // a warp per texel row
            for (int tx = threadIdx.x & 31; tx < tw; tx += 32) {
                long k = ((long)(fy0 + ty) * P.fw + fx0 + tx) * 2;
                float2 f0 = *reinterpret_cast<const float2*>(Fba + k), f1 = *reinterpret_cast<const float2*>(Fab + k);
                e[0][0] = fminf(e[0][0], f0.x); e[0][1] = fmaxf(e[0][1], f0.x);
                e[0][2] = fminf(e[0][2], f0.y); e[0][3] = fmaxf(e[0][3], f0.y);
                e[1][0] = fminf(e[1][0], f1.x); e[1][1] = fmaxf(e[1][1], f1.x);
                e[1][2] = fminf(e[1][2], f1.y); e[1][3] = fmaxf(e[1][3], f1.y);
            }
        }
#pragma unroll
        for (int s = 0; s < 2; s++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                e[s][0] = fminf(e[s][0], __shfl_xor_sync(0xffffffffu, e[s][0], o));
                e[s][1] = fmaxf(e[s][1], __shfl_xor_sync(0xffffffffu, e[s][1], o));
                e[s][2] = fminf(e[s][2], __shfl_xor_sync(0xffffffffu, e[s][2], o));
                e[s][3] = fmaxf(e[s][3], __shfl_xor_sync(0xffffffffu, e[s][3], o));
            }
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int s = 0; s < 2; s++)
#pragma unroll
                for (int k = 0; k < 4; k++) ext[threadIdx.x >> 5][s][k] = e[s][k];
        __syncthreads();
        if (threadIdx.x < 2) {
            int s = threadIdx.x;
            float m[4] = {INFINITY, -INFINITY, INFINITY, -INFINITY};
            for (int wi = 0; wi < ADJ_THREADS / 32; wi++) {
                m[0] = fminf(m[0], ext[wi][s][0]);
                m[1] = fmaxf(m[1], ext[wi][s][1]);
                m[2] = fminf(m[2], ext[wi][s][2]);
                m[3] = fmaxf(m[3], ext[wi][s][3]);
            }
            const float sx = s == 0 ? sxa : sxb, sy = s == 0 ? sya : syb;
            // the extremes of u * sx and of v * sy, as side_at forms them
            float ua = m[0] * sx, ub = m[1] * sx;
            float va = m[2] * sy, vb = m[3] * sy;
            float lo_x = (float)x0 + fminf(ua, ub), hi_x = (float)xe + fmaxf(ua, ub);
            float lo_y = (float)y0 + fminf(va, vb), hi_y = (float)ye + fmaxf(va, vb);
            Sample a = sample_at(lo_x, lo_y, P.w, P.h), c = sample_at(hi_x, hi_y, P.w, P.h);
            bool finite = m[0] <= m[1] && m[2] <= m[3];
            box[s][0] = a.ix;
            box[s][1] = a.iy;
            box[s][2] = finite ? c.ix : a.ix - 1;  // no finite texel: an empty box, the global path
            box[s][3] = c.iy;
        }
    }
    __syncthreads();
    int bw[2], bh[2];
    bool shared_box[2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
        bw[s] = box[s][2] - box[s][0] + 2;
        bh[s] = box[s][3] - box[s][1] + 2;
        shared_box[s] = backward && box[s][2] >= box[s][0] && (long)bw[s] * bh[s] <= ADJ_BOX_PX;
    }
#pragma unroll
    for (int s = 0; s < 2; s++) {
        if (!shared_box[s]) continue;
        float* t = s == 0 ? sacc0 : sacc1;
        for (int i = threadIdx.x; i < bw[s] * bh[s]; i += blockDim.x)
            t[i] = t[i + ADJ_BOX_PX] = t[i + 2 * ADJ_BOX_PX] = t[i + 3 * ADJ_BOX_PX] = 0.0f;
    }
    __syncthreads();
    // pass 2: forward, loss, backward
    float loss = 0.0f;
    for (int j = 0; j < ADJ_TY / ROWS; j++) {
        int y = yb + j * ROWS;
        if (x >= P.w || y >= P.h) continue;
        Side sa = side_at(A, Fba, P, x, y, sxa, sya);
        Side sb = side_at(B, Fab, P, x, y, sxb, syb);
        float4 out = lerp4(sa.val, sb.val, frac);
        long i = (long)y * P.w + x;
        if (P.out) reinterpret_cast<float4*>(P.out + img)[i] = out;
        if (!backward) continue;
        float4 g;
        if (P.target) {  // the photometric L1 loss: d|out - t| / d out = sign(out - t)
            float4 t = ld4(P.target + img, i);
            float4 r = make_float4(out.x - t.x, out.y - t.y, out.z - t.z, out.w - t.w);
            loss += fabsf(r.x) + fabsf(r.y) + fabsf(r.z) + fabsf(r.w);
            g = make_float4((r.x > 0.0f) - (r.x < 0.0f), (r.y > 0.0f) - (r.y < 0.0f), (r.z > 0.0f) - (r.z < 0.0f),
                            (r.w > 0.0f) - (r.w < 0.0f));
        } else {
            g = ld4(P.grad_out + img, i);
        }
        Acc ca{shared_box[0] ? sacc0 : nullptr, box[0][0], box[0][1], bw[0], bh[0], P.da ? P.da + img : nullptr};
        Acc cb{shared_box[1] ? sacc1 : nullptr, box[1][0], box[1][1], bw[1], bh[1], P.db ? P.db + img : nullptr};
        side_back(A, sa, scale4(g, 1.0f - frac), P, ca, sflow0, tx0, ty0, tiled, P.df_ba ? P.df_ba + flo : nullptr, sxa, sya);
        side_back(B, sb, scale4(g, frac), P, cb, sflow1, tx0, ty0, tiled, P.df_ab ? P.df_ab + flo : nullptr, sxb, syb);
    }
    if (P.loss) {  // the loss of the batch item: a warp shuffle sum, one atomic per warp
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, o);
        if ((threadIdx.x & 31) == 0 && loss != 0.0f) atomicAdd(P.loss + b, loss);
    }
    __syncthreads();
    // pass 3: the shared tiles into global memory
#pragma unroll
    for (int s = 0; s < 2; s++) {
        float* dS = s == 0 ? P.da : P.db;
        if (!shared_box[s] || !dS) continue;
        float* acc = s == 0 ? sacc0 : sacc1;
        float4* g4 = reinterpret_cast<float4*>(dS + img);
        // a warp per box row, its lanes along the row (no division by the box width)
        for (int ry = threadIdx.x >> 5; ry < bh[s]; ry += blockDim.x >> 5) {
            const int py = box[s][1] + ry;
            for (int rx = threadIdx.x & 31; rx < bw[s]; rx += 32) {
                const int i = ry * bw[s] + rx;
                float4 v = make_float4(acc[i], acc[i + ADJ_BOX_PX], acc[i + 2 * ADJ_BOX_PX], acc[i + 3 * ADJ_BOX_PX]);
                if (v.x == 0.0f && v.y == 0.0f && v.z == 0.0f && v.w == 0.0f) continue;
                const int px = box[s][0] + rx;
                if (px < P.w && py < P.h) atomicAdd(g4 + ((long)py * P.w + px), v);
            }
        }
    }
    if (tiled) {
        for (int i = threadIdx.x; i < FT_X * FT_Y; i += blockDim.x) {
            int lx = i % FT_X, ly = i / FT_X;
            int fx = tx0 + lx, fy = ty0 + ly;
            if (fx >= P.fw || fy >= P.fh) continue;
            long k = (long)fy * P.fw + fx;
            float2 ga = make_float2(sflow0[i * 2], sflow0[i * 2 + 1]);
            float2 gb = make_float2(sflow1[i * 2], sflow1[i * 2 + 1]);
            if (P.df_ba && (ga.x != 0.0f || ga.y != 0.0f)) atomicAdd(reinterpret_cast<float2*>(P.df_ba + flo) + k, ga);
            if (P.df_ab && (gb.x != 0.0f || gb.y != 0.0f)) atomicAdd(reinterpret_cast<float2*>(P.df_ab + flo) + k, gb);
        }
    }
}

}  // namespace tw
