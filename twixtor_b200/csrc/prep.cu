// The image prep of the optical flow (plugins/retime-engine/src/prep.rs:296-340): Delinearize with
// the plugin runtime's single precision powf (crt_powf.cuh), and the per pixel map of the
// Contrast / Edge Enhance step after its Gaussian blur.
#include "crt_powf.cuh"
#include "kernels.cuh"

namespace tw {

__constant__ unsigned long long c_pow_rcp[257] = TW_POW_RCP_INIT;
__constant__ unsigned long long c_pow_log[257] = TW_POW_LOG_INIT;
__constant__ unsigned long long c_pow_exp2[64] = TW_POW_EXP2_INIT;

static const unsigned long long h_pow_rcp[257] = TW_POW_RCP_INIT;
static const unsigned long long h_pow_log[257] = TW_POW_LOG_INIT;
static const unsigned long long h_pow_exp2[64] = TW_POW_EXP2_INIT;

__device__ float crt_powf(float x, float y) { return crt_powf_with(x, y, PowTables{c_pow_rcp, c_pow_log, c_pow_exp2}); }

float crt_powf_host(float x, float y) { return crt_powf_with(x, y, PowTables{h_pow_rcp, h_pow_log, h_pow_exp2}); }

// prep.rs:296-307 (delinearize): p = powf(max(p, 0) / 255, 1 / 2.2) * 255 (-0.0 stays -0.0)
__global__ void k_delinearize(float* __restrict__ p, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float inv = 1.0f / 2.2f;
    float v = p[i];
    if (v <= 0.0f && v != 0.0f) v = 0.0f;
    float base = v / 255.0f;
    p[i] = crt_powf(base, inv) * 255.0f;
}

// prep.rs:326-340 after the blur: the solver's one sided gradient (flow.rs:283-316) of the blurred
// plane, m = sqrt(gx^2 + gy^2), f = m <= 20 ? m * 0.05 : 1, p = (f * 255 + p) * 0.5
__global__ void k_edge_map(const float* __restrict__ src, float* __restrict__ dst, int w, int h) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)w * h) return;
    int y = (int)(i / w), x = (int)(i - (long)y * w);
    float c = src[i];
    float nx = 0.0f, dx = 0.0f, ny = 0.0f, dy = 0.0f;
    if (x >= 1) { nx = (c - src[i - 1]) + 0.0f; dx = 1.0f; }
    if (y >= 1) { ny = (c - src[i - w]) + 0.0f; dy = 1.0f; }
    if (x + 1 <= w - 1) { nx = nx + (src[i + 1] - c); dx = dx + 1.0f; }
    if (y + 1 <= h - 1) { ny = ny + (src[i + w] - c); dy = dy + 1.0f; }
    float gx = nx / dx, gy = ny / dy;
    float m = sqrtf(gx * gx + gy * gy);
    float f = m <= 20.0f ? m * 0.05f : 1.0f;
    dst[i] = (f * 255.0f + c) * 0.5f;
}

// the powf above over arrays, for the checks against the runtime's traced values
__global__ void k_check_powf(const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ out, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = crt_powf(x[i], y[i]);
}

}  // namespace tw
