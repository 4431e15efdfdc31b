// The persistent coarse-level solve: one CTA walks every coarse level of a solve (flow.rs:1258-1307)
// in a single launch.
//
// The coarse levels of a pyramid are tiny (15 x 8 to 60 x 33 at 1080p) and, launched kernel by
// kernel, they cost about eleven launches each whose time is all latency. Here one block of 1024
// threads keeps both bands and every solver plane of a level in shared memory and runs, level after
// level with block barriers between the stages: the gradient and the blurred tensor, the three
// iterations (calc_b, blur7, new_disp, blur5), the four block matching sweeps, the range check and
// the upsample (with the reset and the damping of the level) into the next level; the last one
// writes the flow of the first level the tiled kernels take over. Every element follows the same
// rules as those kernels (level.cuh), so the flow is bit identical. No block waits on another.
//
// Block matching here gives each line to a group of 8 lanes (4 lines per warp, 128 in flight): the
// sweep's recurrence v'[q] = accept(q, v'[q-1]) ? v'[q-1] : v[q] is walked run by run.
// S[q] = accept(q, v[q-1]) (the test when q-1 kept its own vector) is evaluated for every position
// up front; a stretch of positions that start their own runs is skipped with ballots over S, and a
// run that goes on tests its vector at the next 8 positions at once (one lane each), the first
// refusal ending it (most runs end within a few positions).
#include "kernels.cuh"
#include "level.cuh"

namespace tw {
TW_VARIANT_BEGIN

namespace {

constexpr int NT = COARSE_THREADS;
constexpr int GL = 8;        // lanes per line of block matching
constexpr int NG = NT / GL;  // lines in flight

// sample.rs:47-64 on a plane in shared memory (bilinear1 reads global memory through __ldg)
__device__ __forceinline__ float bilinear_s(const float* img, int w, int h, float x, float y) {
    int ix, iy;
    float fx, fy;
    cell(x, w, ix, fx);
    cell(y, h, iy, fy);
    int i = iy * w + ix;
    float p00 = img[i], p10 = img[i + 1], p01 = img[i + w], p11 = img[i + w + 1];
    float top = (p10 - p00) * fx + p00;
    float bot = (p11 - p01) * fx + p01;
    return (bot - top) * fy + top;
}

// One separable pass of the multi channel rule over a plane (src -> dst, both w x h in shared
// memory): along the rows (VERT false) or the columns.
template <int N, bool VERT>
__device__ __forceinline__ void plane_pass(const float* src, float* dst, int w, int h, const float* k, bool af) {
    for (int e = threadIdx.x; e < w * h; e += NT) {
        int y = e / w, x = e - y * w;
        float v;
        if (!VERT) v = pass_elem<N, true, false>(src + y * w, 0, 1, w, x, k);
        else if (af) v = pass_elem<N, true, true>(src + x, 0, w, h, y, k);
        else v = pass_elem<N, true, false>(src + x, 0, w, h, y, k);
        dst[e] = v;
    }
}

// Block::step's test at pixel (x, y) for the neighbour's vector (nu, nv) against c0, the cost of
// the pixel's own vector (NaN when no step can happen there).
__device__ __forceinline__ bool accept_at(const float* A, const float* B, int w, int h, int x, int y, float nu, float nv,
                                          float c0) {
    if (isnan(c0)) return false;
    float p[9];
    const float* a = A + (y - 1) * w + (x - 1);
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) p[r * 3 + c] = a[r * w + c];
    float c1;
    if (!bm_cost<false, false>(B, w, h, p, (float)x - nu, (float)y - nv, c1)) return false;
    return c1 < c0;
}

// One sweep of one line by one group of GL lanes (the group's lanes call it together; gmask names
// them), in place on the field (fu, fv row-major w x h): the row y (COLS false) or the column x;
// reverse: from the far end. c0w / sw: the group's scratch.
template <bool COLS>
__device__ void sweep_line(const float* A, const float* B, float* fu, float* fv, int w, int h, int fixed, bool reverse,
                           float* c0w, unsigned char* sw, int gl, unsigned gmask, int gshift) {
    const int len = COLS ? h : w;
    const float w1 = (float)(w - 1), h1 = (float)(h - 1);
    auto line_of = [&](int q) { return reverse ? len - 1 - q : q; };
    auto elem = [&](int i) { return COLS ? i * w + fixed : fixed * w + i; };
    auto xy = [&](int i, int* x, int* y) {
        *x = COLS ? fixed : i;
        *y = COLS ? i : fixed;
    };
    auto group_ballot = [&](bool p) { return (__ballot_sync(gmask, p) >> gshift) & ((1u << GL) - 1u); };
    // c0 of every interior position, then S
    for (int q = 1 + gl; q <= len - 2; q += GL) {
        int i = line_of(q), e = elem(i), x, y;
        xy(i, &x, &y);
        float c = __int_as_float(0x7fc00000);
        float tx = (float)x - fu[e], ty = (float)y - fv[e];
        if (0.0f <= tx && tx <= w1 && 0.0f <= ty && ty <= h1) {
            float p[9];
            const float* a = A + (y - 1) * w + (x - 1);
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int cc = 0; cc < 3; cc++) p[r * 3 + cc] = a[r * w + cc];
            float cost;
            if (bm_cost<false, false>(B, w, h, p, tx, ty, cost)) c = cost;
        }
        c0w[q] = c;
    }
    __syncwarp(gmask);
    for (int q = 1 + gl; q <= len - 2; q += GL) {
        int i = line_of(q), x, y;
        xy(i, &x, &y);
        int ep = elem(line_of(q - 1));
        sw[q] = accept_at(A, B, w, h, x, y, fu[ep], fv[ep], c0w[q]) ? 1 : 0;
    }
    __syncwarp(gmask);
    float ou = 0.0f, ov = 0.0f;  // the vector of the run in progress (uniform over the group)
    bool own = true;             // position q - 1 kept its own vector
    int q = 1;
    while (q <= len - 2) {
        if (own) {
            // the first r >= q that takes the vector of r - 1: positions q .. r - 1 start runs
            int r = -1;
            for (int qb = q; qb <= len - 2 && r < 0; qb += GL) {
                int qq = qb + gl;
                unsigned m = group_ballot(qq <= len - 2 && sw[qq]);
                if (m) r = qb + __ffs(m) - 1;
            }
            if (r < 0) break;
            int ep = elem(line_of(r - 1));
            ou = fu[ep];
            ov = fv[ep];
            if (gl == 0) {
                int e = elem(line_of(r));
                fu[e] = ou;
                fv[e] = ov;
            }
            q = r + 1;
            own = false;
        } else {
            // the run of (ou, ov) goes on while the next positions accept it
            int qq = q + gl;
            bool valid = qq <= len - 2;
            bool acc = false;
            if (valid) {
                int x, y;
                xy(line_of(qq), &x, &y);
                acc = accept_at(A, B, w, h, x, y, ou, ov, c0w[qq]);
            }
            unsigned va = group_ballot(valid);
            unsigned am = group_ballot(acc);
            unsigned fails = va & ~am;
            int f = fails ? __ffs(fails) - 1 : __popc(va);
            if (valid && gl < f) {
                int e = elem(line_of(qq));
                fu[e] = ou;
                fv[e] = ov;
            }
            if (!fails) {
                q += __popc(va);
            } else {
                q += f + 1;  // position q + f starts its own run
                own = true;
            }
        }
    }
    __syncwarp(gmask);
}

}  // namespace

__global__ void __launch_bounds__(COARSE_THREADS) k_solve_coarse(CoarseJob J) {
    extern __shared__ float sm[];
    constexpr int M = COARSE_MAX_PIXELS;
    float* A = sm;  // the bands of X and Y at the level
    float* B = A + M;
    float *gx = B + M, *gy = gx + M, *a0 = gy + M, *a1 = a0 + M, *a2 = a1 + M;
    float *fu = a2 + M, *fv = fu + M, *nu = fv + M, *nv = nu + M;
    float *t0 = nv + M, *t1 = t0 + M, *t2 = t1 + M, *t3 = t2 + M;
    float* c0_all = t3 + M;                                   // NG x COARSE_MAX_LINE
    unsigned char* s_all = (unsigned char*)(c0_all + NG * COARSE_MAX_LINE);
    __shared__ int s_any[32];
    const int tid = threadIdx.x;
    const int grp = tid / GL, gl = tid % GL, gshift = (tid & 31) & ~(GL - 1);
    const unsigned gmask = ((1u << GL) - 1u) << gshift;
    float* c0w = c0_all + grp * COARSE_MAX_LINE;
    unsigned char* sw = s_all + grp * COARSE_MAX_LINE;
    if (tid < 32) s_any[tid] = 0;
    for (int l = J.start; l >= J.last; l--) {
        const int w = J.sizes[l][0], h = J.sizes[l][1], n = w * h;
        const float fw = (float)w, fh = (float)h;
        for (int i = tid; i < n; i += NT) {
            A[i] = __ldg(J.x + J.offs[l] + i);
            B[i] = __ldg(J.y + J.offs[l] + i);
            if (l == J.start) fu[i] = fv[i] = 0.0f;
        }
        __syncthreads();
        // gradient and tensor (flow.rs:283-328), then blur7 of the tensor
        for (int i = tid; i < n; i += NT) {
            int y = i / w, x = i - y * w;
            float cc = A[i];
            float nx = 0.0f, dx = 0.0f, ny = 0.0f, dy = 0.0f;
            if (x >= 1) { nx = (cc - A[i - 1]) + 0.0f; dx = 1.0f; }
            if (y >= 1) { ny = (cc - A[i - w]) + 0.0f; dy = 1.0f; }
            if (x + 1 <= w - 1) { nx = nx + (A[i + 1] - cc); dx = dx + 1.0f; }
            if (y + 1 <= h - 1) { ny = ny + (A[i + w] - cc); dy = dy + 1.0f; }
            float g0 = nx / dx, g1 = ny / dy;
            gx[i] = g0;
            gy[i] = g1;
            a0[i] = g0 * g0;
            a1[i] = g0 * g1;
            a2[i] = g1 * g1;
        }
        __syncthreads();
        plane_pass<8, false>(a0, t0, w, h, J.g7.k, J.af);
        plane_pass<8, false>(a1, t1, w, h, J.g7.k, J.af);
        plane_pass<8, false>(a2, t2, w, h, J.g7.k, J.af);
        __syncthreads();
        plane_pass<8, true>(t0, a0, w, h, J.g7.k, J.af);
        plane_pass<8, true>(t1, a1, w, h, J.g7.k, J.af);
        plane_pass<8, true>(t2, a2, w, h, J.g7.k, J.af);
        __syncthreads();
        for (int it = 0; it < 3; it++) {
            // calc_b (flow.rs:334-357): B of the iteration into t0 / t1
            for (int i = tid; i < n; i += NT) {
                int y = i / w, x = i - y * w;
                float b0 = 0.0f, b1 = 0.0f;
                float sx = (float)x - fu[i], sy = (float)y - fv[i];
                if (!(sx < 0.0f || fw - 1.0f < sx || sy < 0.0f || fh - 1.0f < sy)) {
                    float rr = bilinear_s(B, w, h, sx, sy) - A[i];
                    b0 = rr * gx[i];
                    b1 = rr * gy[i];
                }
                t0[i] = b0;
                t1[i] = b1;
            }
            __syncthreads();
            plane_pass<8, false>(t0, t2, w, h, J.g7.k, J.af);
            plane_pass<8, false>(t1, t3, w, h, J.g7.k, J.af);
            __syncthreads();
            plane_pass<8, true>(t2, t0, w, h, J.g7.k, J.af);
            plane_pass<8, true>(t3, t1, w, h, J.g7.k, J.af);
            __syncthreads();
            // new_disp (flow.rs:361-371) into nu / nv
            for (int i = tid; i < n; i += NT) {
                float aa = a0[i], ab = a1[i], ad = a2[i];
                float b0 = t0[i], b1 = t1[i];
                float u = fu[i], v = fv[i];
                float t = ab * ab - ad * aa;
                if (fabsf(t) > 40.0f) {
                    u = (ab * b1 - ad * b0) / t + u;
                    v = (ab * b0 - aa * b1) / t + v;
                }
                nu[i] = u;
                nv[i] = v;
            }
            __syncthreads();
            // blur5 of the flow back into fu / fv
            plane_pass<6, false>(nu, t2, w, h, J.g5.k, J.af);
            plane_pass<6, false>(nv, t3, w, h, J.g5.k, J.af);
            __syncthreads();
            plane_pass<6, true>(t2, fu, w, h, J.g5.k, J.af);
            plane_pass<6, true>(t3, fv, w, h, J.g5.k, J.af);
            __syncthreads();
        }
        // block matching (flow.rs:551-622): the row sweeps, then the column sweeps
        if (J.refine && w >= 3 && h >= 3) {
            for (int y = 1 + grp; y <= h - 2; y += NG) {
                sweep_line<false>(A, B, fu, fv, w, h, y, false, c0w, sw, gl, gmask, gshift);
                sweep_line<false>(A, B, fu, fv, w, h, y, true, c0w, sw, gl, gmask, gshift);
            }
            __syncthreads();
            for (int x = 1 + grp; x <= w - 2; x += NG) {
                sweep_line<true>(A, B, fu, fv, w, h, x, false, c0w, sw, gl, gmask, gshift);
                sweep_line<true>(A, B, fu, fv, w, h, x, true, c0w, sw, gl, gmask, gshift);
            }
            __syncthreads();
        }
        // the range check (flow.rs:430-442)
        int in = 0;
        for (int i = tid; i < n; i += NT) {
            int y = i / w, x = i - y * w;
            float px = (float)x + fu[i], py = (float)y + fv[i];
            if (0.0f <= px && px <= fw - 1.0f && 0.0f <= py && py <= fh - 1.0f) in = 1;
        }
        if (__syncthreads_or(in) && tid == 0) {
            s_any[l] = 1;
            J.any[l] = 1;
        }
        __syncthreads();
        // the reset and the damping of the level, then the upsample into the next level
        const int dw = J.sizes[l - 1][0], dh = J.sizes[l - 1][1];
        const bool zero = zero_at_level(s_any, l, J.start);
        const bool damp_now = l == J.start && J.damp_any;
        float* ou = l == J.last ? J.fu_out : nu;
        float* ov = l == J.last ? J.fv_out : nv;
        for (int i = tid; i < dw * dh; i += NT) {
            int y = i / dw, x = i - y * dw;
            float u, v;
            upsample_at(fu, fv, w, h, zero, damp_now, J.damp, x, y, dw, dh, &u, &v);
            ou[i] = u;
            ov[i] = v;
        }
        __syncthreads();
        float* t = fu;
        fu = nu;
        nu = t;
        t = fv;
        fv = nv;
        nv = t;
    }
}

size_t coarse_smem_bytes() {
    return sizeof(float) * (15 * (size_t)COARSE_MAX_PIXELS + (size_t)NG * COARSE_MAX_LINE) + (size_t)NG * COARSE_MAX_LINE;
}

TW_VARIANT_END
}  // namespace tw
