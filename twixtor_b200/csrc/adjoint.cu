// The adjoint of warp + blend (the differentiable twin of compose_vectors' Blend with warping code
// 0): out = ta + (tb - ta) * w with ta = warp(A, F_BA, 1 - wa), tb = warp(B, F_AB, wa), w = 1 - wa,
// where warp(S, F, s)(p) samples S bilinearly at p + F(p r) s / r (the flow sampled bilinearly at
// p r, r = (flow size - 1) / (image size - 1) per axis, as warp.rs:693-786), the position clamped
// to the image rectangle. One fused kernel per pixel recomputes the forward sample (nothing of the
// forward pass is stored), takes the output gradient (given, or the sign of out - target for the
// photometric L1 loss) and scatters:
//   dA, dB     the bilinear weights times (1 - w) g and w g (vector atomics, 16 bytes per corner);
//   dF_BA, dF_AB  the image gradient at the sample point times s / r, through the flow's bilinear
//              weights: accumulated per CTA in shared memory (a tile of flow texels), then added
//              to global memory once per texel.
// Frames are float RGBA (4 channels, any premultiplication), batch items back to back.
#include "kernels.cuh"

namespace tw {

namespace {

constexpr int AT_X = 32, AT_Y = 8;               // pixels per CTA
constexpr int FT_X = AT_X + 2, FT_Y = AT_Y + 2;  // the flow texel tile when r <= 1 per axis

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

// One side: the sample of S (and its four corners) at p + F(p r) s / r
struct Side {
    Sample smp;
    float4 c00, c10, c01, c11, val;
    int fix, fiy;    // the flow footprint
    float ffx, ffy;
};

__device__ __forceinline__ Side side_at(const float* S, const float* F, const AdjParams& P, int x, int y, float amount) {
    Side d;
    float qx = (float)x * P.rx, qy = (float)y * P.ry;
    footprint(qx, qy, P.fw, P.fh, d.fix, d.fiy, d.ffx, d.ffy);
    long f00 = ((long)d.fiy * P.fw + d.fix) * 2, f01 = f00 + (long)P.fw * 2;
    float2 a = *reinterpret_cast<const float2*>(F + f00), b = *reinterpret_cast<const float2*>(F + f00 + 2);
    float2 c = *reinterpret_cast<const float2*>(F + f01), e = *reinterpret_cast<const float2*>(F + f01 + 2);
    float u = (a.x + (b.x - a.x) * d.ffx) * (1.0f - d.ffy) + (c.x + (e.x - c.x) * d.ffx) * d.ffy;
    float v = (a.y + (b.y - a.y) * d.ffx) * (1.0f - d.ffy) + (c.y + (e.y - c.y) * d.ffx) * d.ffy;
    float px = (float)x + u * amount / P.rx, py = (float)y + v * amount / P.ry;
    d.smp = sample_at(px, py, P.w, P.h);
    long i00 = (long)d.smp.iy * P.w + d.smp.ix, i01 = i00 + P.w;
    d.c00 = ld4(S, i00);
    d.c10 = ld4(S, i00 + 1);
    d.c01 = ld4(S, i01);
    d.c11 = ld4(S, i01 + 1);
    d.val = lerp4(lerp4(d.c00, d.c10, d.smp.fx), lerp4(d.c01, d.c11, d.smp.fx), d.smp.fy);
    return d;
}

// the gradient of one side: dS at the four corners (vector atomics), the positional gradient into
// the flow tile (shared) or straight to global memory
__device__ __forceinline__ void side_back(const Side& d, float4 g, const AdjParams& P, float* dS, float* sflow, int tx0,
                                          int ty0, bool tiled, float* dF, float amount) {
    const Sample& s = d.smp;
    long i00 = (long)s.iy * P.w + s.ix, i01 = i00 + P.w;
    float w00 = (1.0f - s.fx) * (1.0f - s.fy), w10 = s.fx * (1.0f - s.fy), w01 = (1.0f - s.fx) * s.fy, w11 = s.fx * s.fy;
    if (dS) {
        atomicAdd(reinterpret_cast<float4*>(dS) + i00, scale4(g, w00));
        atomicAdd(reinterpret_cast<float4*>(dS) + i00 + 1, scale4(g, w10));
        atomicAdd(reinterpret_cast<float4*>(dS) + i01, scale4(g, w01));
        atomicAdd(reinterpret_cast<float4*>(dS) + i01 + 1, scale4(g, w11));
    }
    if (!dF) return;
    // d val / d px and d val / d py of the bilinear sample, per channel
    float4 dx = lerp4(make_float4(d.c10.x - d.c00.x, d.c10.y - d.c00.y, d.c10.z - d.c00.z, d.c10.w - d.c00.w),
                      make_float4(d.c11.x - d.c01.x, d.c11.y - d.c01.y, d.c11.z - d.c01.z, d.c11.w - d.c01.w), s.fy);
    float4 dy = lerp4(make_float4(d.c01.x - d.c00.x, d.c01.y - d.c00.y, d.c01.z - d.c00.z, d.c01.w - d.c00.w),
                      make_float4(d.c11.x - d.c10.x, d.c11.y - d.c10.y, d.c11.z - d.c10.z, d.c11.w - d.c10.w), s.fx);
    float gu = s.cx ? 0.0f : dot4(g, dx) * amount / P.rx;
    float gv = s.cy ? 0.0f : dot4(g, dy) * amount / P.ry;
    if (gu == 0.0f && gv == 0.0f) return;
    float fw00 = (1.0f - d.ffx) * (1.0f - d.ffy), fw10 = d.ffx * (1.0f - d.ffy), fw01 = (1.0f - d.ffx) * d.ffy,
          fw11 = d.ffx * d.ffy;
    const int cx[4] = {0, 1, 0, 1}, cy[4] = {0, 0, 1, 1};
    const float wt[4] = {fw00, fw10, fw01, fw11};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int fx = d.fix + cx[k], fy = d.fiy + cy[k];
        if (tiled) {
            int lx = fx - tx0, ly = fy - ty0;
            atomicAdd(sflow + (ly * FT_X + lx) * 2, gu * wt[k]);
            atomicAdd(sflow + (ly * FT_X + lx) * 2 + 1, gv * wt[k]);
        } else {
            atomicAdd(reinterpret_cast<float2*>(dF) + ((long)fy * P.fw + fx), make_float2(gu * wt[k], gv * wt[k]));
        }
    }
}

}  // namespace

// grid: (ceil(w / 32), ceil(h / 8), batch), 256 threads
__global__ void __launch_bounds__(AT_X * AT_Y) k_warp_blend_adjoint(AdjParams P) {
    __shared__ float sflow[2][FT_X * FT_Y * 2];
    int b = blockIdx.z;
    long img = (long)P.w * P.h * 4 * b, flo = (long)P.fw * P.fh * 2 * b;
    int x0 = blockIdx.x * AT_X, y0 = blockIdx.y * AT_Y;
    int x = x0 + (int)(threadIdx.x % AT_X), y = y0 + (int)(threadIdx.x / AT_X);
    // the flow texels this tile's footprints reach, when they fit the shared tile
    int tx0 = (int)floorf((float)x0 * P.rx), ty0 = (int)floorf((float)y0 * P.ry);
    tx0 = min(tx0, max(P.fw - 2, 0));
    ty0 = min(ty0, max(P.fh - 2, 0));
    bool tiled = P.tiled;
    if (tiled) {
        for (int i = threadIdx.x; i < FT_X * FT_Y * 2; i += blockDim.x) {
            sflow[0][i] = 0.0f;
            sflow[1][i] = 0.0f;
        }
        __syncthreads();
    }
    bool live = x < P.w && y < P.h;
    float loss = 0.0f;
    if (live) {
        const float* A = P.a + img;
        const float* B = P.b + img;
        float frac = 1.0f - P.wa;
        Side sa = side_at(A, P.f_ba + flo, P, x, y, frac);
        Side sb = side_at(B, P.f_ab + flo, P, x, y, P.wa);
        float4 out = lerp4(sa.val, sb.val, frac);
        long i = (long)y * P.w + x;
        if (P.out) reinterpret_cast<float4*>(P.out + img)[i] = out;
        float4 g;
        if (P.target) {  // the photometric L1 loss: d|out - t| / d out = sign(out - t)
            float4 t = ld4(P.target + img, i);
            float4 r = make_float4(out.x - t.x, out.y - t.y, out.z - t.z, out.w - t.w);
            loss = fabsf(r.x) + fabsf(r.y) + fabsf(r.z) + fabsf(r.w);
            g = make_float4((r.x > 0.0f) - (r.x < 0.0f), (r.y > 0.0f) - (r.y < 0.0f), (r.z > 0.0f) - (r.z < 0.0f),
                            (r.w > 0.0f) - (r.w < 0.0f));
        } else {
            g = P.grad_out ? ld4(P.grad_out + img, i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (P.grad_out || P.target) {
            side_back(sa, scale4(g, 1.0f - frac), P, P.da ? P.da + img : nullptr, sflow[0], tx0, ty0, tiled,
                      P.df_ba ? P.df_ba + flo : nullptr, frac);
            side_back(sb, scale4(g, frac), P, P.db ? P.db + img : nullptr, sflow[1], tx0, ty0, tiled,
                      P.df_ab ? P.df_ab + flo : nullptr, P.wa);
        }
    }
    if (P.loss) {  // the loss of the batch item: a warp shuffle sum, one atomic per warp
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, o);
        if ((threadIdx.x & 31) == 0 && loss != 0.0f) atomicAdd(P.loss + b, loss);
    }
    if (tiled) {
        __syncthreads();
        for (int i = threadIdx.x; i < FT_X * FT_Y; i += blockDim.x) {
            int lx = i % FT_X, ly = i / FT_X;
            int fx = tx0 + lx, fy = ty0 + ly;
            if (fx >= P.fw || fy >= P.fh) continue;
            long k = (long)fy * P.fw + fx;
            float2 ga = make_float2(sflow[0][i * 2], sflow[0][i * 2 + 1]);
            float2 gb = make_float2(sflow[1][i * 2], sflow[1][i * 2 + 1]);
            if (P.df_ba && (ga.x != 0.0f || ga.y != 0.0f)) atomicAdd(reinterpret_cast<float2*>(P.df_ba + flo) + k, ga);
            if (P.df_ab && (gb.x != 0.0f || gb.y != 0.0f)) atomicAdd(reinterpret_cast<float2*>(P.df_ab + flo) + k, gb);
        }
    }
}

}  // namespace tw
