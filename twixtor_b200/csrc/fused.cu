// Fused, shared-memory tiled kernels of the pyramid and of one solver level (strict mode).
//
// Each kernel computes a TX x TY tile of its outputs. Intermediate planes live only in shared
// memory, over the tile plus the halo the later stages need, and are recomputed in the halo rather
// than exchanged between CTAs. Every element still takes the reference's own operation order
// (flow/conv.rs for the separable passes, flow.rs for the solver steps), so the results are bit
// identical to the unfused kernels and to the reference CPU path.
#include "kernels.cuh"
#include "level.cuh"
#include "luma.cuh"

namespace tw {
TW_VARIANT_BEGIN

constexpr int FT_X = 32;  // tile width (outputs)
constexpr int FT_Y = 32;  // tile height
constexpr int FT_THREADS = 1024;  // the launch bound; each launch picks 256 to 1024 threads

// A separable pass over a shared-memory region, both directions:
//   src: RH x RW region whose (0,0) is global (gx0, gy0); dst: OH x OW region at global (ox0, oy0).
// Horizontal: dst(r, c) = pass along row gy0 + r (OH == RH, oy0 == gy0) at global column ox0 + c.
// Vertical:   dst(r, c) = pass along column ox0 + c (OW == RW, ox0 == gx0) at global row oy0 + r.
// Elements whose output position lies outside the image are left undefined (never read).
template <int N, bool MULTI, bool VERT, bool ABOVE_FIRST>
__device__ __forceinline__ void region_pass(const float* src, int RW, int gx0, int gy0, float* dst, int OW, int OH,
                                            int ox0, int oy0, int w, int h, const float* k) {
    for (int e = threadIdx.x; e < OW * OH; e += blockDim.x) {
        int r = e / OW, c = e - r * OW;
        int X = ox0 + c, Y = oy0 + r;
        if (X < 0 || X >= w || Y < 0 || Y >= h) continue;
        float v;
        if (!VERT) {
            const float* line = src + (Y - gy0) * RW;
            v = pass_elem<N, MULTI, false>(line, gx0, 1, w, X, k);
        } else {
            const float* line = src + (X - gx0);
            v = pass_elem<N, MULTI, ABOVE_FIRST>(line, gy0, RW, h, Y, k);
        }
        dst[e] = v;
    }
}

template <int N, bool MULTI>
__device__ __forceinline__ void vpass(const float* src, int RW, int gx0, int gy0, float* dst, int OW, int OH, int ox0,
                                      int oy0, int w, int h, const float* k, bool above_first) {
    if (above_first) region_pass<N, MULTI, true, true>(src, RW, gx0, gy0, dst, OW, OH, ox0, oy0, w, h, k);
    else region_pass<N, MULTI, true, false>(src, RW, gx0, gy0, dst, OW, OH, ox0, oy0, w, h, k);
}

// ---- pyramid: blur5 + band (flow.rs:261-268) and the first reduction step --------------------------

// tmp = blur5(orig) and band = orig - tmp over one tile; orig is a plane, or (luma_src != nullptr)
// the luma of an engine image computed on the fly (prep.rs:168-235; luma_mode: the LUMA_* bits).
__global__ void __launch_bounds__(FT_THREADS) k_blur5_band(const float* __restrict__ orig, const void* __restrict__ luma_src,
                                                           int fmt, int luma_mode, int w, int h, bool above_first,
                                                           float* __restrict__ tmp_out, float* __restrict__ band_out,
                                                           float* __restrict__ band_t_out) {
    constexpr int N = 3, HALO = N - 1;
    constexpr int RW = FT_X + 2 * HALO, RH = FT_Y + 2 * HALO;
    __shared__ float s_in[RH * RW];
    __shared__ float s_h[RH * FT_X];
    __shared__ float s_t[FT_Y][FT_X + 1];  // the band tile, for the transposed copy
    const float k[3] = {0.375f, 0.25f, 0.0625f};  // flow/conv.rs:48
    int X0 = blockIdx.x * FT_X, Y0 = blockIdx.y * FT_Y;
    int gx0 = X0 - HALO, gy0 = Y0 - HALO;
    for (int e = threadIdx.x; e < RW * RH; e += blockDim.x) {
        int r = e / RW, c = e - r * RW;
        int X = gx0 + c, Y = gy0 + r;
        float v = 0.0f;
        if (X >= 0 && X < w && Y >= 0 && Y < h) {
            long i = (long)Y * w + X;
            v = luma_src ? luma_px(luma_src, fmt, i, luma_mode) : orig[i];
        }
        s_in[e] = v;
    }
    __syncthreads();
    region_pass<N, false, false, false>(s_in, RW, gx0, gy0, s_h, FT_X, RH, X0, gy0, w, h, k);
    __syncthreads();
    for (int e = threadIdx.x; e < FT_X * FT_Y; e += blockDim.x) {
        int r = e / FT_X, c = e - r * FT_X;
        int X = X0 + c, Y = Y0 + r;
        if (X >= w || Y >= h) continue;
        const float* line = s_h + c;
        float v = above_first ? pass_elem<N, false, true>(line, gy0, FT_X, h, Y, k)
                              : pass_elem<N, false, false>(line, gy0, FT_X, h, Y, k);
        long i = (long)Y * w + X;
        tmp_out[i] = v;
        if (band_out) {
            float bv = s_in[(Y - gy0) * RW + (X - gx0)] - v;
            band_out[i] = bv;
            s_t[r][c] = bv;
        }
    }
    if (band_t_out) {  // the band transposed (element (x, y) at [x * h + y]) for the column sweeps
        __syncthreads();
        for (int e = threadIdx.x; e < FT_X * FT_Y; e += blockDim.x) {
            int c = e / FT_Y, r = e - c * FT_Y;
            int X = X0 + c, Y = Y0 + r;
            if (X < w && Y < h) band_t_out[(long)X * h + Y] = s_t[r][c];
        }
    }
}

// R outputs of a pass along one line at line indices i0 .. i0 + R - 1 (global), written to
// out[r * ostride] for r < nvalid where the index lies in [0, len). The line's element t (global
// index) is line[(t - origin) * stride]; the region holds indices [origin, origin + rlen). The
// register path runs only when every output is interior and every input lies in the region.
template <int N, int R, bool MULTI, bool LEFT_FIRST>
__device__ __forceinline__ void pass_run(const float* line, int origin, int rlen, int stride, int len, int i0,
                                         const float* k, float* out, int ostride, int nvalid) {
    constexpr int NV = R + 2 * N - 2;
    bool interior = nvalid == R && len >= 2 * N && i0 >= N && i0 + R - 1 < len - N && i0 - (N - 1) >= origin &&
                    i0 + R - 1 + (N - 1) < origin + rlen;
    if (interior) {
        float v[NV];
        const float* base = line + (i0 - (N - 1) - origin) * stride;
#pragma unroll
        for (int j = 0; j < NV; j++) v[j] = base[j * stride];
#pragma unroll
        for (int r = 0; r < R; r++) {
            float s = v[r + N - 1] * k[0];
#pragma unroll
            for (int j = N - 1; j >= 1; j--) s = s + (v[r + N - 1 + j] + v[r + N - 1 - j]) * k[j];
            out[r * ostride] = s;
        }
    } else {
        for (int r = 0; r < nvalid; r++) {
            int i = i0 + r;
            if (i < 0 || i >= len) continue;
            out[r * ostride] = pass_elem<N, MULTI, LEFT_FIRST>(line, origin, stride, len, i, k);
        }
    }
}

// ---- one solver level: gradient, tensor and its blur (flow.rs:1275-1277) ---------------------------

// mask (may be null): the level mask of X of a layered solve; the gradient is zero where the mask
// is below 0.95 at the pixel or at one of its four neighbours that exist (flow.rs:743-761).
// b_out (may be null): calc_b of the first iteration from the level's flow fu, fv, the image i0 and
// the mask of Y (flow.rs:334-357), into two planes of pitch bp (plane stride bplane).
__global__ void __launch_bounds__(FT_THREADS) k_level_init(const float* __restrict__ img, int w, int h, Taps g7,
                                                           bool above_first, float* __restrict__ gxo,
                                                           float* __restrict__ gyo, float* __restrict__ a0o,
                                                           float* __restrict__ a1o, float* __restrict__ a2o,
                                                           const float* __restrict__ mask,
                                                           const float* __restrict__ fu, const float* __restrict__ fv,
                                                           const float* __restrict__ i0,
                                                           const float* __restrict__ mask_y, float* __restrict__ b_out,
                                                           int bp, long bplane) {
    constexpr int N = 8, HALO = N - 1;
    constexpr int RW = FT_X + 2 * HALO, RH = FT_Y + 2 * HALO;
    constexpr int RS = RW | 1, HS = FT_X | 1;  // row strides (odd: a warp's lanes on distinct rows hit distinct banks)
    constexpr int R = 8;                        // outputs per thread of the register blocked passes
    extern __shared__ float sm[];
    float* s_t = sm;                  // 3 x RH x RS tensor
    float* s_h = s_t + 3 * RH * RS;   // 3 x RH x HS
    int X0 = blockIdx.x * FT_X, Y0 = blockIdx.y * FT_Y;
    int gx0 = X0 - HALO, gy0 = Y0 - HALO;
    for (int e = threadIdx.x; e < RW * RH; e += blockDim.x) {
        int r = e / RW, c = e - r * RW;
        int x = gx0 + c, y = gy0 + r;
        float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
        if (x >= 0 && x < w && y >= 0 && y < h) {
            long i = (long)y * w + x;
            float cc = __ldg(img + i);  // flow.rs:283-316
            float nx = 0.0f, dx = 0.0f, ny = 0.0f, dy = 0.0f;
            if (x >= 1) { nx = (cc - __ldg(img + i - 1)) + 0.0f; dx = 1.0f; }
            if (y >= 1) { ny = (cc - __ldg(img + i - w)) + 0.0f; dy = 1.0f; }
            if (x + 1 <= w - 1) { nx = nx + (__ldg(img + i + 1) - cc); dx = dx + 1.0f; }
            if (y + 1 <= h - 1) { ny = ny + (__ldg(img + i + w) - cc); dy = dy + 1.0f; }
            float gx = nx / dx, gy = ny / dy;
            if (mask) {
                auto off = [&](long j) { return __ldg(mask + j) < 0.95f; };
                if (off(i) || (y >= 1 && off(i - w)) || (y + 1 < h && off(i + w)) || (x >= 1 && off(i - 1)) ||
                    (x + 1 < w && off(i + 1))) {
                    gx = 0.0f;
                    gy = 0.0f;
                }
            }
            t0 = gx * gx;  // flow.rs:319-328
            t1 = gx * gy;
            t2 = gy * gy;
            if (x >= X0 && x < X0 + FT_X && y >= Y0 && y < Y0 + FT_Y) {
                gxo[i] = gx;
                gyo[i] = gy;
                if (b_out) {  // calc_b of the level's first iteration
                    float b0, b1;
                    calc_b_at(i0, mask_y, w, h, x, y, __ldg(fu + i), __ldg(fv + i), cc, gx, gy, b0, b1);
                    b_out[(long)y * bp + x] = b0;
                    b_out[bplane + (long)y * bp + x] = b1;
                }
            }
        }
        const int se = r * RS + c;
        s_t[se] = t0;
        s_t[RH * RS + se] = t1;
        s_t[2 * RH * RS + se] = t2;
    }
    __syncthreads();
    // blur7 of the tensor, register blocked (pass_run: R outputs from R + 14 inputs held in
    // registers, each output with the interior chain, or the border rule near the image's edges):
    // horizontal along the region's rows at the tile's columns, a lane per row
    {
        constexpr int NSEG = FT_X / R;
        for (int e = threadIdx.x; e < 3 * RH * NSEG; e += blockDim.x) {
            const int r = e % RH, rest = e / RH;
            const int seg = rest % NSEG, ch = rest / NSEG;
            const int Y = gy0 + r;
            if (Y < 0 || Y >= h) continue;
            const int c0 = seg * R;
            pass_run<N, R, true, false>(s_t + ch * RH * RS + r * RS, gx0, RW, 1, w, X0 + c0, g7.k,
                                        s_h + ch * RH * HS + r * HS + c0, 1, R);
        }
    }
    __syncthreads();
    //    vertical at the tile's rows, a lane per column, into the tensor planes
    {
        constexpr int NSEG = FT_Y / R;
        float* outs[3] = {a0o, a1o, a2o};
        for (int e = threadIdx.x; e < 3 * FT_X * NSEG; e += blockDim.x) {
            const int c = e % FT_X, rest = e / FT_X;
            const int seg = rest % NSEG, ch = rest / NSEG;
            const int X = X0 + c;
            if (X >= w) continue;
            const int r0 = seg * R;
            const float* line = s_h + ch * RH * HS + c;
            float* dst = (ch == 0 ? outs[0] : ch == 1 ? outs[1] : outs[2]) + (long)(Y0 + r0) * w + X;  // rows past h are never written
            if (above_first) pass_run<N, R, true, true>(line, gy0, RH, HS, h, Y0 + r0, g7.k, dst, w, R);
            else pass_run<N, R, true, false>(line, gy0, RH, HS, h, Y0 + r0, g7.k, dst, w, R);
        }
    }
}

size_t level_init_smem() {
    constexpr int RW = FT_X + 14, RH = FT_Y + 14;
    return sizeof(float) * (3 * RH * (RW | 1) + 3 * RH * (FT_X | 1));
}

// ---- one solver iteration (flow.rs:1278-1282): calc_b, blur7 of B, new_disp, blur5 of the flow -----
// mask_y (may be null): the level mask of Y of a layered solve
//
// calc_b depends only on the flow at its own pixel, so it is computed once per pixel where the flow
// is made: k_level_init for the level's first iteration, each iteration's epilogue for the next one
// (k_calc_b_pitched after the level's block matching). B lives in two planes with a pitch of a
// multiple of 4 floats, so that an iteration loads its B region with 128-bit loads.
//
// Halos: the flow's blur5 needs new_disp on the tile + 5; new_disp needs blurred B there, which
// needs B on the tile + 12. The tile is TX x TY outputs (a template: the host picks the shape per
// level size from its tuning table). The separable passes are register blocked: a thread computes R
// consecutive outputs along the pass from R + 2N - 2 inputs held in registers (each input read once
// from shared memory instead of once per tap), each output with the reference's interior chain;
// outputs near the image border, or at the ragged end of a region, take the element rule (interior
// chain or border renormalisation) one by one. Horizontal passes give each lane of a warp its own
// row (row strides are odd, so the lanes hit distinct banks), vertical passes its own column.

template <int TX, int TY>
struct IterGeom {
    static constexpr int HB = 12, HD = 5;
    static constexpr int BW = TX + 2 * HB, BH = TY + 2 * HB;  // B region
    static constexpr int DW = TX + 2 * HD, DH = TY + 2 * HD;  // new_disp region
    static constexpr int BS = BW | 1;                          // row strides (odd)
    static constexpr int HS = DW | 1;
    static constexpr int DS = DW | 1;
    static constexpr int FS = TX | 1;
    // buffer 1: B (2 planes BH x BS), later the blurred B / new flow (2 planes DH x DS), last the
    // tile's new flow (2 planes TY x TX)
    // buffer 2: the horizontal pass of B (2 planes BH x HS), later of the flow (2 planes DH x FS)
    static constexpr int BUF1 = 2 * BH * BS;
    static constexpr int BUF2 = 2 * BH * HS;
    static constexpr size_t SMEM = sizeof(float) * (BUF1 + BUF2);
    static_assert(2 * DH * DS <= BUF1 && 2 * DH * FS <= BUF2 && 2 * TX * TY <= BUF1, "the reused buffers must fit");
};

template <int TX, int TY>
__device__ __forceinline__ void level_iter_body(const float* __restrict__ b_in, int bp, long bplane,
                                                const float* __restrict__ i1, const float* __restrict__ i0,
                                                const float* __restrict__ gx, const float* __restrict__ gy,
                                                const float* __restrict__ a0, const float* __restrict__ a1,
                                                const float* __restrict__ a2, const float* __restrict__ fu,
                                                const float* __restrict__ fv, int w, int h, const Taps& g7,
                                                const Taps& g5, bool above_first, float* __restrict__ fu_out,
                                                float* __restrict__ fv_out, const float* __restrict__ mask_y,
                                                float* __restrict__ b_out) {
    using G = IterGeom<TX, TY>;
    constexpr int R7 = 6, R5 = 8;  // outputs per thread of the blur7 and blur5 passes
    extern __shared__ float sm[];
    float* s_b = sm;            // 2 x BH x BS
    float* s_h = sm + G::BUF1;  // 2 x BH x HS
    float* s_d = s_b;           // reuse: 2 x DH x DS (blurred B -> new flow)
    float* s_f = s_h;           // reuse: 2 x DH x FS
    const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY;
    const int bx0 = X0 - G::HB, by0 = Y0 - G::HB;
    const int dx0 = X0 - G::HD, dy0 = Y0 - G::HD;
    const int nt = blockDim.x;
    // 1. B over the B region, from the planes b_in (calc_b of flow.rs:334-357, computed once per pixel
    //    by the kernel that produced the flow): 128-bit loads of 4 columns (bx0 and the pitch are
    //    multiples of 4, the planes 16-byte aligned), zero outside the level as calc_b gives there;
    //    four loads per thread in flight before their stores
    {
        constexpr int Q = G::BW / 4;  // 128-bit groups per region row
        constexpr int NQ = 2 * G::BH * Q;
        static_assert(G::BW % 4 == 0 && G::HB % 4 == 0, "the B region must start and end on 4-column groups");
        for (int e0 = threadIdx.x; e0 < NQ; e0 += 4 * nt) {
            float4 v[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int e = e0 + k * nt;
                const int q = e % Q, rest = e / Q;
                const int r = rest % G::BH, ch = rest / G::BH;
                const int x = bx0 + 4 * q, y = by0 + r;
                v[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (e < NQ && x >= 0 && x < w && y >= 0 && y < h) {
                    v[k] = __ldg(reinterpret_cast<const float4*>(b_in + ch * bplane + (long)y * bp + x));
                    if (x + 1 >= w) v[k].y = 0.0f;  // the pitch's padding columns
                    if (x + 2 >= w) v[k].z = 0.0f;
                    if (x + 3 >= w) v[k].w = 0.0f;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int e = e0 + k * nt;
                if (e >= NQ) break;
                const int q = e % Q, rest = e / Q;
                const int r = rest % G::BH, ch = rest / G::BH;
                float* d = s_b + ch * G::BH * G::BS + r * G::BS + 4 * q;
                d[0] = v[k].x;
                d[1] = v[k].y;
                d[2] = v[k].z;
                d[3] = v[k].w;
            }
        }
    }
    __syncthreads();
    // 2. blur7 of B (2 channels): horizontal along the B rows, outputs at the new_disp columns
    {
        constexpr int NSEG = (G::DW + R7 - 1) / R7;
        for (int e = threadIdx.x; e < 2 * G::BH * NSEG; e += nt) {
            int r = e % G::BH, rest = e / G::BH;
            int seg = rest % NSEG, ch = rest / NSEG;
            int Y = by0 + r;
            if (Y < 0 || Y >= h) continue;
            int c0 = seg * R7;
            const float* line = s_b + ch * G::BH * G::BS + r * G::BS;
            pass_run<8, R7, true, false>(line, bx0, G::BW, 1, w, dx0 + c0, g7.k,
                                         s_h + ch * G::BH * G::HS + r * G::HS + c0, 1, min(R7, G::DW - c0));
        }
    }
    __syncthreads();
    //    vertical, outputs at the new_disp rows (into buffer 1, whose B is no longer needed)
    {
        constexpr int NSEG = (G::DH + R7 - 1) / R7;
        for (int e = threadIdx.x; e < 2 * G::DW * NSEG; e += nt) {
            int c = e % G::DW, rest = e / G::DW;
            int seg = rest % NSEG, ch = rest / NSEG;
            int X = dx0 + c;
            if (X < 0 || X >= w) continue;
            int r0 = seg * R7;
            const float* line = s_h + ch * G::BH * G::HS + c;
            float* o = s_d + ch * G::DH * G::DS + r0 * G::DS + c;
            int nv = min(R7, G::DH - r0);
            if (above_first) pass_run<8, R7, true, true>(line, by0, G::BH, G::HS, h, dy0 + r0, g7.k, o, G::DS, nv);
            else pass_run<8, R7, true, false>(line, by0, G::BH, G::HS, h, dy0 + r0, g7.k, o, G::DS, nv);
        }
    }
    __syncthreads();
    // 3. new_disp over the new_disp region (flow.rs:361-371), in place on the blurred B (one element
    //    per thread and round: batching more raises the registers past three blocks per SM, which
    //    costs more when several solves share the GPU than the batching gains)
    for (int e = threadIdx.x; e < G::DW * G::DH; e += nt) {
        int r = e / G::DW, c = e - r * G::DW;
        int x = dx0 + c, y = dy0 + r;
        if (x < 0 || x >= w || y < 0 || y >= h) continue;
        int i = y * w + x;
        float aa = __ldg(a0 + i), ab = __ldg(a1 + i), ad = __ldg(a2 + i);
        int si = r * G::DS + c;
        float b0 = s_d[si], b1 = s_d[G::DH * G::DS + si];
        float u = __ldg(fu + i), v = __ldg(fv + i);
        float t = ab * ab - ad * aa;
        if (fabsf(t) > 40.0f) {
            u = (ab * b1 - ad * b0) / t + u;
            v = (ab * b0 - aa * b1) / t + v;
        }
        s_d[si] = u;
        s_d[G::DH * G::DS + si] = v;
    }
    __syncthreads();
    // 4. blur5 of the flow: horizontal at the tile columns, then vertical at the tile rows
    {
        constexpr int NSEG = (TX + R5 - 1) / R5;
        for (int e = threadIdx.x; e < 2 * G::DH * NSEG; e += nt) {
            int r = e % G::DH, rest = e / G::DH;
            int seg = rest % NSEG, ch = rest / NSEG;
            int Y = dy0 + r;
            if (Y < 0 || Y >= h) continue;
            int c0 = seg * R5;
            const float* line = s_d + ch * G::DH * G::DS + r * G::DS;
            pass_run<6, R5, true, false>(line, dx0, G::DW, 1, w, X0 + c0, g5.k,
                                         s_f + ch * G::DH * G::FS + r * G::FS + c0, 1, min(R5, TX - c0));
        }
    }
    __syncthreads();
    //    vertical at the tile rows, into the tile buffer (buffer 1: its new_disp region was read by the
    //    horizontal pass)
    float* s_o = s_b;  // 2 x TY x TX
    {
        constexpr int NSEG = (TY + R5 - 1) / R5;
        for (int e = threadIdx.x; e < 2 * TX * NSEG; e += nt) {
            int c = e % TX, rest = e / TX;
            int seg = rest % NSEG, ch = rest / NSEG;
            int X = X0 + c;
            if (X >= w) continue;
            int r0 = seg * R5;
            const float* line = s_f + ch * G::DH * G::FS + c;
            int nv = min(R5, TY - r0);
            float* dst = s_o + ch * TY * TX + r0 * TX + c;  // rows past h are never written
            if (above_first) pass_run<6, R5, true, true>(line, dy0, G::DH, G::FS, h, Y0 + r0, g5.k, dst, TX, nv);
            else pass_run<6, R5, true, false>(line, dy0, G::DH, G::FS, h, Y0 + r0, g5.k, dst, TX, nv);
        }
    }
    __syncthreads();
    // 5. the new flow to the planes; with b_out also calc_b of the next iteration at every pixel of the
    //    tile (flow.rs:334-357), two pixels per thread and round with their loads in flight together
    {
        constexpr int K = 2;
        for (int e0 = threadIdx.x; e0 < TX * TY; e0 += K * nt) {
            float u[K], v[K], i1v[K], gxv[K], gyv[K];
            bool in[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                const int e = e0 + k * nt;
                const int r = e / TX, c = e - r * TX;
                const int x = X0 + c, y = Y0 + r;
                in[k] = e < TX * TY && x < w && y < h;
                u[k] = v[k] = i1v[k] = gxv[k] = gyv[k] = 0.0f;
                if (in[k]) {
                    const int i = y * w + x;
                    u[k] = s_o[e];
                    v[k] = s_o[TY * TX + e];
                    fu_out[i] = u[k];
                    fv_out[i] = v[k];
                    if (b_out) {
                        i1v[k] = __ldg(i1 + i);
                        gxv[k] = __ldg(gx + i);
                        gyv[k] = __ldg(gy + i);
                    }
                }
            }
            if (b_out) {
#pragma unroll
                for (int k = 0; k < K; k++) {
                    if (!in[k]) continue;
                    const int e = e0 + k * nt;
                    const int r = e / TX, c = e - r * TX;
                    const int x = X0 + c, y = Y0 + r;
                    float b0, b1;
                    calc_b_at(i0, mask_y, w, h, x, y, u[k], v[k], i1v[k], gxv[k], gyv[k], b0, b1);
                    b_out[(long)y * bp + x] = b0;
                    b_out[bplane + (long)y * bp + x] = b1;
                }
            }
        }
    }
}

// The iteration reads B from b_in and, with b_out (same pitch bp and plane stride bplane), writes the
// next iteration's B; b_in and b_out are different buffers (other tiles still read b_in's halo).
#define TW_LEVEL_ITER(TX, TY)                                                                                         \
    __global__ void __launch_bounds__(LEVEL_ITER_MAX_THREADS) k_level_iter_##TX##x##TY(                              \
        const float* __restrict__ b_in, int bp, long bplane, const float* __restrict__ i1,                          \
        const float* __restrict__ i0, const float* __restrict__ gx, const float* __restrict__ gy,                    \
        const float* __restrict__ a0, const float* __restrict__ a1, const float* __restrict__ a2,                    \
        const float* __restrict__ fu, const float* __restrict__ fv, int w, int h, Taps g7, Taps g5,                  \
        bool above_first, float* __restrict__ fu_out, float* __restrict__ fv_out, const float* __restrict__ mask_y,  \
        float* __restrict__ b_out) {                                                                                 \
        level_iter_body<TX, TY>(b_in, bp, bplane, i1, i0, gx, gy, a0, a1, a2, fu, fv, w, h, g7, g5, above_first,    \
                                fu_out, fv_out, mask_y, b_out);                                                      \
    }
TW_LEVEL_ITER(32, 32)
TW_LEVEL_ITER(64, 32)
TW_LEVEL_ITER(64, 64)
#undef TW_LEVEL_ITER

size_t level_iter_smem(int tile) {
    switch (tile) {
        case LEVEL_TILE_64x32: return IterGeom<64, 32>::SMEM;
        case LEVEL_TILE_64x64: return IterGeom<64, 64>::SMEM;
        default: return IterGeom<32, 32>::SMEM;
    }
}

// calc_b (flow.rs:334-357) of the next iteration where the flow changed outside an iteration (after
// the block matching and the user displacement of the finest level): one thread per pixel, into two
// planes of pitch bp (plane stride bplane).
__global__ void k_calc_b_pitched(const float* __restrict__ i1, const float* __restrict__ i0,
                                 const float* __restrict__ gx, const float* __restrict__ gy,
                                 const float* __restrict__ fu, const float* __restrict__ fv, int w, int h,
                                 const float* __restrict__ mask_y, float* __restrict__ b_out, int bp, long bplane) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    const int i = y * w + x;
    float b0, b1;
    calc_b_at(i0, mask_y, w, h, x, y, __ldg(fu + i), __ldg(fv + i), __ldg(i1 + i), __ldg(gx + i), __ldg(gy + i), b0, b1);
    b_out[(long)y * bp + x] = b0;
    b_out[bplane + (long)y * bp + x] = b1;
}

// ---- the end of a level (flow.rs:1292-1303): range reset, damping, then the upsample ---------------

// The coarse field (with the reset and damping of its level applied on the fly) upsampled to the
// next finer level (flow.rs:376-391, bilinear2 of sample.rs:69-86). Applying the elementwise reset
// and damping to the four gathered samples is the same as applying them to the whole field first.
__global__ void k_apply_upsample(const float* __restrict__ su, const float* __restrict__ sv, int sw, int sh,
                                 const int* __restrict__ any, int l, int start, bool damp_now, float damp,
                                 float* __restrict__ du, float* __restrict__ dv, int dw, int dh) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    float u, v;
    upsample_at(su, sv, sw, sh, zero_at_level(any, l, start), damp_now, damp, x, y, dw, dh, &u, &v);
    long o = (long)y * dw + x;
    du[o] = u;
    dv[o] = v;
}

// The finest level: reset and damping, then the final negation (flow.rs:1305) into the
// interleaved FlowField; flags a NaN.
__global__ void k_apply_negate(const float* __restrict__ fu, const float* __restrict__ fv, long n,
                              const int* __restrict__ any, int start, bool damp_now, float damp,
                              float* __restrict__ out, int* __restrict__ nan_flag) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool zero = zero_at_level(any, 0, start);
    float u = zero ? 0.0f : fu[i];
    float v = zero ? 0.0f : fv[i];
    if (damp_now) {
        u = damp * u;
        v = damp * v;
    }
    u = -1.0f * u;
    v = -1.0f * v;
    out[2 * i] = u;
    out[2 * i + 1] = v;
    if (isnan(u) || isnan(v)) atomicOr(nan_flag, 1);
}

TW_VARIANT_END
}  // namespace tw

namespace tw {
TW_VARIANT_BEGIN
// flow/extras.rs:64-72: v >= 0.95 gives 1, else 0 (a NaN gives 0), in place
__global__ void k_binarize(float* __restrict__ p, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = p[i] >= 0.95f ? 1.0f : 0.0f;
}
TW_VARIANT_END
}  // namespace tw
