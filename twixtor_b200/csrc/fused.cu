// Fused, shared-memory tiled kernels of the pyramid and of one solver level (strict mode).
//
// Each kernel computes a TX x TY tile of its outputs. Intermediate planes live only in shared
// memory, over the tile plus the halo the later stages need, and are recomputed in the halo rather
// than exchanged between CTAs. Every element still takes the reference's own operation order
// (flow/conv.rs for the separable passes, flow.rs for the solver steps), so the results are bit
// identical to the unfused kernels and to the reference CPU path.
#include "kernels.cuh"
#include "luma.cuh"

namespace tw {

constexpr int FT_X = 32;  // tile width (outputs)
constexpr int FT_Y = 32;  // tile height
constexpr int FT_THREADS = 1024;  // the launch bound; each launch picks 256 to 1024 threads

// ---- separable pass elements ---------------------------------------------------------------------

// flow/conv.rs:101-137 on a line held in shared memory: element t of the line (global index, inside
// [0, len)) lives at line[(t - origin) * stride].
template <int N, bool MULTI, bool LEFT_FIRST>
__device__ __forceinline__ float border_sm(const float* line, int origin, int stride, int len, int i, const float* k) {
    float centre = line[(i - origin) * stride];
    float num = k[0] * centre;
    float den = k[0];
#pragma unroll
    for (int j = N - 1; j >= 1; j--) {
        float kj = k[j];
#pragma unroll
        for (int side = 0; side < 2; side++) {
            bool right = (side == 0) != LEFT_FIRST;
            int t = right ? i + j : i - j;
            bool inside = t >= 0 && t < len;
            float xv, wv;
            if (!MULTI) {
                xv = inside ? line[(t - origin) * stride] : 0.0f;
                wv = inside ? kj : 0.0f;
            } else {
                float v = inside ? line[(t - origin) * stride] : -1.0f;
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

// One output of a pass along a line (conv.rs:141-190 horizontally, :268-301 vertically): the
// interior chain for elements whose taps all lie inside [n, len - n), the border rule otherwise.
template <int N, bool MULTI, bool LEFT_FIRST>
__device__ __forceinline__ float pass_elem(const float* line, int origin, int stride, int len, int i, const float* k) {
    if (len >= 2 * N && i >= N && i < len - N) {
        const float* c = line + (i - origin) * stride;
        float s = c[0] * k[0];
#pragma unroll
        for (int j = N - 1; j >= 1; j--) s = s + (c[j * stride] + c[-j * stride]) * k[j];
        return s;
    }
    return border_sm<N, MULTI, LEFT_FIRST>(line, origin, stride, len, i, k);
}

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

// ---- one solver level: gradient, tensor and its blur (flow.rs:1275-1277) ---------------------------

// mask (may be null): the level mask of X of a layered solve; the gradient is zero where the mask
// is below 0.95 at the pixel or at one of its four neighbours that exist (flow.rs:743-761)
__global__ void __launch_bounds__(FT_THREADS) k_level_init(const float* __restrict__ img, int w, int h, Taps g7,
                                                           bool above_first, float* __restrict__ gxo,
                                                           float* __restrict__ gyo, float* __restrict__ a0o,
                                                           float* __restrict__ a1o, float* __restrict__ a2o,
                                                           const float* __restrict__ mask) {
    constexpr int N = 8, HALO = N - 1;
    constexpr int RW = FT_X + 2 * HALO, RH = FT_Y + 2 * HALO;
    extern __shared__ float sm[];
    float* s_t = sm;                  // 3 x RH x RW tensor
    float* s_h = s_t + 3 * RH * RW;   // 3 x RH x FT_X
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
            }
        }
        s_t[e] = t0;
        s_t[RH * RW + e] = t1;
        s_t[2 * RH * RW + e] = t2;
    }
    __syncthreads();
    for (int ch = 0; ch < 3; ch++)
        region_pass<N, true, false, false>(s_t + ch * RH * RW, RW, gx0, gy0, s_h + ch * RH * FT_X, FT_X, RH, X0, gy0, w,
                                           h, g7.k);
    __syncthreads();
    float* outs[3] = {a0o, a1o, a2o};
    for (int e = threadIdx.x; e < 3 * FT_X * FT_Y; e += blockDim.x) {
        int ch = e / (FT_X * FT_Y);
        int q = e - ch * FT_X * FT_Y;
        int r = q / FT_X, c = q - r * FT_X;
        int X = X0 + c, Y = Y0 + r;
        if (X >= w || Y >= h) continue;
        const float* line = s_h + ch * RH * FT_X + c;
        float v = above_first ? pass_elem<N, true, true>(line, gy0, FT_X, h, Y, g7.k)
                              : pass_elem<N, true, false>(line, gy0, FT_X, h, Y, g7.k);
        outs[ch][(long)Y * w + X] = v;
    }
}

size_t level_init_smem() {
    constexpr int RW = FT_X + 14, RH = FT_Y + 14;
    return sizeof(float) * (3 * RH * RW + 3 * RH * FT_X);
}

// ---- one solver iteration (flow.rs:1278-1282): calc_b, blur7 of B, new_disp, blur5 of the flow -----
// mask_y (may be null): the level mask of Y of a layered solve

// Halos: the flow's blur5 needs new_disp on the tile + 5; new_disp needs blurred B there, which
// needs B on the tile + 12.
constexpr int IT_HB = 12;                 // B region halo
constexpr int IT_HD = 5;                  // new_disp region halo
constexpr int IT_BW = FT_X + 2 * IT_HB;   // 56
constexpr int IT_BH = FT_Y + 2 * IT_HB;
constexpr int IT_DW = FT_X + 2 * IT_HD;   // 42
constexpr int IT_DH = FT_Y + 2 * IT_HD;

size_t level_iter_smem() {
    // buffer 1: B (2 planes IT_BH x IT_BW), later the blurred B / new flow (2 x IT_DH x IT_DW)
    // buffer 2: horizontal pass of B (2 x IT_BH x IT_DW), later of the flow (2 x IT_DH x FT_X)
    return sizeof(float) * (2 * IT_BH * IT_BW + 2 * IT_BH * IT_DW);
}

__global__ void __launch_bounds__(FT_THREADS) k_level_iter(const float* __restrict__ i1, const float* __restrict__ i0,
                                                           const float* __restrict__ gx, const float* __restrict__ gy,
                                                           const float* __restrict__ a0, const float* __restrict__ a1,
                                                           const float* __restrict__ a2, const float* __restrict__ fu,
                                                           const float* __restrict__ fv, int w, int h, Taps g7, Taps g5,
                                                           bool above_first, float* __restrict__ fu_out,
                                                           float* __restrict__ fv_out,
                                                           const float* __restrict__ mask_y) {
    extern __shared__ float sm[];
    float* s_b = sm;                                  // 2 x IT_BH x IT_BW
    float* s_h = s_b + 2 * IT_BH * IT_BW;             // 2 x IT_BH x IT_DW
    float* s_d = s_b;                                 // reuse: 2 x IT_DH x IT_DW (blurred B -> new flow)
    float* s_f = s_h;                                 // reuse: 2 x IT_DH x FT_X
    int X0 = blockIdx.x * FT_X, Y0 = blockIdx.y * FT_Y;
    int bx0 = X0 - IT_HB, by0 = Y0 - IT_HB;
    int dx0 = X0 - IT_HD, dy0 = Y0 - IT_HD;
    const float fw = (float)w, fh = (float)h;
    // 1. B = calc_b over the B region (flow.rs:334-357)
    for (int e = threadIdx.x; e < IT_BW * IT_BH; e += blockDim.x) {
        int r = e / IT_BW, c = e - r * IT_BW;
        int x = bx0 + c, y = by0 + r;
        float b0 = 0.0f, b1 = 0.0f;
        if (x >= 0 && x < w && y >= 0 && y < h) {
            long i = (long)y * w + x;
            float sx = (float)x - __ldg(fu + i);
            float sy = (float)y - __ldg(fv + i);
            // flow.rs:777-845: in a layered solve the warped mask of Y must be at least 0.999
            if (!(sx < 0.0f || fw - 1.0f < sx || sy < 0.0f || fh - 1.0f < sy) &&
                (!mask_y || bilinear1(mask_y, w, h, sx, sy) >= 0.999f)) {
                float s = bilinear1(i0, w, h, sx, sy);
                float rr = s - __ldg(i1 + i);
                b0 = rr * __ldg(gx + i);
                b1 = rr * __ldg(gy + i);
            }
        }
        s_b[e] = b0;
        s_b[IT_BH * IT_BW + e] = b1;
    }
    __syncthreads();
    // 2. blur7 of B (2 channels): horizontal over the B rows, at the new_disp columns
    for (int ch = 0; ch < 2; ch++)
        region_pass<8, true, false, false>(s_b + ch * IT_BH * IT_BW, IT_BW, bx0, by0, s_h + ch * IT_BH * IT_DW, IT_DW,
                                           IT_BH, dx0, by0, w, h, g7.k);
    __syncthreads();
    //    vertical, at the new_disp rows (into buffer 1, whose B is no longer needed)
    for (int ch = 0; ch < 2; ch++)
        vpass<8, true>(s_h + ch * IT_BH * IT_DW, IT_DW, dx0, by0, s_d + ch * IT_DH * IT_DW, IT_DW, IT_DH, dx0, dy0, w, h,
                       g7.k, above_first);
    __syncthreads();
    // 3. new_disp over the new_disp region (flow.rs:361-371), in place on the blurred B
    for (int e = threadIdx.x; e < IT_DW * IT_DH; e += blockDim.x) {
        int r = e / IT_DW, c = e - r * IT_DW;
        int x = dx0 + c, y = dy0 + r;
        if (x < 0 || x >= w || y < 0 || y >= h) continue;
        long i = (long)y * w + x;
        float aa = __ldg(a0 + i), ab = __ldg(a1 + i), ad = __ldg(a2 + i);
        float b0 = s_d[e], b1 = s_d[IT_DH * IT_DW + e];
        float u = __ldg(fu + i), v = __ldg(fv + i);
        float t = ab * ab - ad * aa;
        if (fabsf(t) > 40.0f) {
            u = (ab * b1 - ad * b0) / t + u;
            v = (ab * b0 - aa * b1) / t + v;
        }
        s_d[e] = u;
        s_d[IT_DH * IT_DW + e] = v;
    }
    __syncthreads();
    // 4. blur5 of the flow: horizontal at the tile columns, then vertical at the tile rows
    for (int ch = 0; ch < 2; ch++)
        region_pass<6, true, false, false>(s_d + ch * IT_DH * IT_DW, IT_DW, dx0, dy0, s_f + ch * IT_DH * FT_X, FT_X,
                                           IT_DH, X0, dy0, w, h, g5.k);
    __syncthreads();
    for (int e = threadIdx.x; e < 2 * FT_X * FT_Y; e += blockDim.x) {
        int ch = e / (FT_X * FT_Y);
        int q = e - ch * FT_X * FT_Y;
        int r = q / FT_X, c = q - r * FT_X;
        int X = X0 + c, Y = Y0 + r;
        if (X >= w || Y >= h) continue;
        const float* line = s_f + ch * IT_DH * FT_X + c;
        float v = above_first ? pass_elem<6, true, true>(line, dy0, FT_X, h, Y, g5.k)
                              : pass_elem<6, true, false>(line, dy0, FT_X, h, Y, g5.k);
        (ch == 0 ? fu_out : fv_out)[(long)Y * w + X] = v;
    }
}

// ---- the end of a level (flow.rs:1292-1303): range reset, damping, then the upsample ---------------

// any[k] (k = level) is set when some pixel of level k is in range after its refinement.
// check at level l = no level processed before (start .. l+1) had a pixel in range.
__device__ __forceinline__ bool zero_at_level(const int* any, int l, int start) {
    bool check = true;
    for (int k = start; k > l; k--) check = check && any[k] == 0;
    return check && any[l] == 0;
}

// The coarse field (with the reset and damping of its level applied on the fly) upsampled to the
// next finer level (flow.rs:376-391, bilinear2 of sample.rs:69-86). Applying the elementwise reset
// and damping to the four gathered samples is the same as applying them to the whole field first.
__global__ void k_apply_upsample(const float* __restrict__ su, const float* __restrict__ sv, int sw, int sh,
                                 const int* __restrict__ any, int l, int start, bool damp_now, float damp,
                                 float* __restrict__ du, float* __restrict__ dv, int dw, int dh) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    bool zero = zero_at_level(any, l, start);
    float sx = ((float)dw - 1.0f) / (float)(sw - 1);
    float sy = ((float)dh - 1.0f) / (float)(sh - 1);
    float rx = (float)(1.0 / (double)sx);
    float ry = (float)(1.0 / (double)sy);
    int ix, iy;
    float fx, fy;
    cell((float)x * rx, sw, ix, fx);
    cell((float)y * ry, sh, iy, fy);
    long i = (long)iy * sw + ix;
    const float* planes[2] = {su, sv};
    float r[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const float* p = planes[c];
        float q[4] = {p[i], p[i + 1], p[i + sw], p[i + sw + 1]};
#pragma unroll
        for (int m = 0; m < 4; m++) {
            float v = zero ? 0.0f : q[m];
            if (damp_now) v = damp * v;
            q[m] = v;
        }
        float top = (q[1] - q[0]) * fx + q[0];
        float bot = (q[3] - q[2]) * fx + q[2];
        r[c] = (bot - top) * fy + top;
    }
    long o = (long)y * dw + x;
    du[o] = r[0] * sx;
    dv[o] = r[1] * sy;
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

}  // namespace tw

namespace tw {
// flow/extras.rs:64-72: v >= 0.95 gives 1, else 0 (a NaN gives 0), in place
__global__ void k_binarize(float* __restrict__ p, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = p[i] >= 0.95f ? 1.0f : 0.0f;
}
}  // namespace tw
