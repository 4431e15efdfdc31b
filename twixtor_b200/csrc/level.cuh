// Per element rules shared by the solver's kernels (the tiled level kernels, block matching and the
// persistent coarse-level solve): the separable filter element with its border rule
// (flow/conv.rs), Block::cost of block matching (flow.rs:474-523) and the range state of a level
// (flow.rs:1292-1300). Each repeats the reference's operation order, so every kernel that calls
// them computes the same bits.
#pragma once
#include "kernels.cuh"

namespace tw {

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

// flow.rs:474-523 (Block::cost). B(X, Y) is B[Y * w + X] for a row-major plane (COLS false) and
// B[X * h + Y] for its transpose (COLS true); the arithmetic does not depend on the layout. Indices
// are 32-bit (a level plane holds at most 6144 x 6144 elements).
template <bool COLS, bool LDG = true>
__device__ __forceinline__ bool bm_cost(const float* __restrict__ B, int w, int h, const float p[9], float x2, float y2,
                                        float& out) {
    float wm2 = (float)(w - 2), hm2 = (float)(h - 2);
    if (x2 > wm2 || y2 > hm2) return false;
    int ix, iy;
    float fx, fy;
    if (x2 == wm2) { ix = cvtt32(wm2 - 1.0f); fx = 1.0f; }
    else { ix = cvtt32(x2); fx = x2 - (float)ix; }
    if (y2 == hm2) { iy = cvtt32(hm2 - 1.0f); fy = 1.0f; }
    else { iy = cvtt32(y2); fy = y2 - (float)iy; }
    if (ix < 1 || iy < 1) return false;
    float w11 = fy * fx;
    float w10 = fx - w11;
    float w01 = fy - w11;
    float w00 = ((1.0f - fx) - fy) + w11;
    float t[4][4];
    if (!COLS) {
        const float* base = B + (iy - 1) * w + (ix - 1);
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) t[r][c] = LDG ? __ldg(base + r * w + c) : base[r * w + c];
    } else {
        const float* base = B + (ix - 1) * h + (iy - 1);
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
            for (int r = 0; r < 4; r++) t[r][c] = LDG ? __ldg(base + c * h + r) : base[c * h + r];
    }
    float sq[9];
#pragma unroll
    for (int b = 0; b < 3; b++) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            float q = ((w00 * t[b][a] + w10 * t[b][a + 1]) + w01 * t[b + 1][a]) + w11 * t[b + 1][a + 1];
            float d = p[b * 3 + a] - q;
            sq[b * 3 + a] = d * d;
        }
    }
    float s = sq[0] + sq[1];
#pragma unroll
    for (int k = 2; k < 8; k++) s = s + sq[k];
    out = sq[8] + s;
    return true;
}

// flow.rs:334-357 (calc_b) at pixel (x, y) whose flow is (u, v): B = (I0(x - u, y - v) - I1) * grad,
// zero where the source point leaves the level, and in a layered solve (mask_y) where the warped
// mask of Y is below 0.999 (flow.rs:777-845). i1v, gxv, gyv: I1 and the gradient at the pixel.
__device__ __forceinline__ void calc_b_at(const float* __restrict__ i0, const float* __restrict__ mask_y, int w, int h,
                                          int x, int y, float u, float v, float i1v, float gxv, float gyv, float& b0,
                                          float& b1) {
    const float sx = (float)x - u, sy = (float)y - v;
    b0 = 0.0f;
    b1 = 0.0f;
    if (!(sx < 0.0f || (float)w - 1.0f < sx || sy < 0.0f || (float)h - 1.0f < sy) &&
        (!mask_y || bilinear1(mask_y, w, h, sx, sy) >= 0.999f)) {
        const float rr = bilinear1(i0, w, h, sx, sy) - i1v;
        b0 = rr * gxv;
        b1 = rr * gyv;
    }
}

// any[k] (k = level) is set when some pixel of level k is in range after its refinement.
// check at level l = no level processed before (start .. l+1) had a pixel in range.
__device__ __forceinline__ bool zero_at_level(const int* any, int l, int start) {
    bool check = true;
    for (int k = start; k > l; k--) check = check && any[k] == 0;
    return check && any[l] == 0;
}

// flow.rs:376-391 (upsample_flow, bilinear2 of sample.rs:69-86) at output pixel (x, y) of dw x dh:
// the coarse field su / sv of sw x sh with the reset (zero) and the damping of its level applied to
// the four gathered samples, which is the same as applying them to the whole field first.
__device__ __forceinline__ void upsample_at(const float* su, const float* sv, int sw, int sh, bool zero,
                                            bool damp_now, float damp, int x, int y, int dw, int dh, float* u,
                                            float* v) {
    float sx = ((float)dw - 1.0f) / (float)(sw - 1);
    float sy = ((float)dh - 1.0f) / (float)(sh - 1);
    float rx = (float)(1.0 / (double)sx);
    float ry = (float)(1.0 / (double)sy);
    int ix, iy;
    float fx, fy;
    cell((float)x * rx, sw, ix, fx);
    cell((float)y * ry, sh, iy, fy);
    int i = iy * sw + ix;
    const float* planes[2] = {su, sv};
    float r[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const float* p = planes[c];
        float q[4] = {p[i], p[i + 1], p[i + sw], p[i + sw + 1]};
#pragma unroll
        for (int m = 0; m < 4; m++) {
            float t = zero ? 0.0f : q[m];
            if (damp_now) t = damp * t;
            q[m] = t;
        }
        float top = (q[1] - q[0]) * fx + q[0];
        float bot = (q[3] - q[2]) * fx + q[2];
        r[c] = (bot - top) * fy + top;
    }
    *u = r[0] * sx;
    *v = r[1] * sy;
}

}  // namespace tw
