// Block matching for callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc at all: a plugin running inside an application that owns the
// device memory pool (a video host that hands out only its own frame buffers), or code on a
// real-time render thread where a driver allocation can stall or is forbidden. They can still pass
// their own device buffers for the inputs and the output. This entry point runs the four block
// matching sweeps (flow.rs:551-622) on such buffers without allocating anything: its only scratch
// (the field split into two float planes, the transposes of the two images and of the field for
// the column sweeps) lives in the file-scope device array below, which every GPU that loads the
// library holds until the process exits.
#include <cuda_runtime.h>

#include "../../include/twixtor_b200.h"
#include "kernels.cuh"

namespace {

// Scratch of the allocation-free block matching: the u and v planes of the field, the transposes
// of A and B, and the transposed field of the column sweeps (6 planes).
constexpr long NOALLOC_MAX_PIXELS = TW_NOALLOC_MAX_PIXELS;
static __device__ __align__(256) float g_noalloc_planes[6 * NOALLOC_MAX_PIXELS];

// The set-up of every call, in the CUDA context current on the calling thread: the device address of
// the scratch array there (the host side name g_noalloc_planes is only a stand-in, not a device
// pointer) and the shared memory limit of the sweep kernels. Both belong to the context, not to the
// device ordinal (a host may bind its own driver context, or reset the device between calls), so
// nothing is cached across calls; neither allocates.
int setup(float** planes) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_planes) != cudaSuccess || !p) return TW_ERR_CUDA;
    int smem = (int)tw::bm_smem_bytes(tw::BM_MAX_LINE);
    if (cudaFuncSetAttribute(tw::k_bm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return TW_ERR_CUDA;
    if (cudaFuncSetAttribute(tw::k_bm_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return TW_ERR_CUDA;
    *planes = (float*)p;
    return TW_OK;
}

// One launch through cudaLaunchKernel, whose return code is this launch's own: an error that the
// host's earlier launches left pending is neither reported as this call's nor cleared.
template <typename... Args>
cudaError_t launch(void (*kernel)(Args...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    void* argv[] = {(void*)&args...};
    return cudaLaunchKernel((const void*)kernel, grid, block, argv, smem, s);
}

}  // namespace

extern "C" int tw_block_match_noalloc(const float* a, const float* b, float* flow, int32_t width, int32_t height,
                                      void* stream) {
    if (!a || !b || !flow || width <= 0 || height <= 0) return TW_ERR_BAD_PARAM;
    if ((long)width * height > NOALLOC_MAX_PIXELS || width > tw::BM_MAX_LINE || height > tw::BM_MAX_LINE)
        return TW_ERR_TOO_LARGE;
    float* planes = nullptr;
    int rc = setup(&planes);
    if (rc != TW_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    long n = (long)width * height;
    float* fu = planes;
    float* fv = fu + n;
    float *at = fv + n, *bt = at + n, *ut = bt + n, *vt = ut + n;
    const int tb = 256;
    dim3 g1((unsigned)((n + tb - 1) / tb));
    dim3 tt(32, 8), ga((width + 31) / 32, (height + 31) / 32);
    const float* cfu = fu;
    const float* cfv = fv;
    const float* cut = ut;
    const float* cvt = vt;
    // every element of the planes this call reads is written first, so the previous call's
    // contents never reach the result
    cudaError_t e = launch(tw::k_deinterleave, g1, dim3(tb), 0, s, (const float*)flow, n, fu, fv);
    if (e == cudaSuccess && width >= 3 && height >= 3) {
        // the row sweeps write the transposed field (ut, vt), the column sweeps read it with the
        // transposes of A and B and write the result back into (fu, fv)
        e = launch(tw::k_bm_rows, dim3(height - 2), dim3(tb), tw::bm_smem_bytes(width), s, a, b, cfu, cfv, (int)width,
                   (int)height, ut, vt);
        if (e == cudaSuccess) e = launch(tw::k_transpose2, ga, tt, 0, s, a, b, at, bt, (int)width, (int)height);
        if (e == cudaSuccess)
            e = launch(tw::k_bm_cols, dim3(width - 2), dim3(tb), tw::bm_smem_bytes(height), s, (const float*)at,
                       (const float*)bt, cut, cvt, (int)width, (int)height, fu, fv);
    }
    if (e == cudaSuccess) e = launch(tw::k_interleave, g1, dim3(tb), 0, s, cfu, cfv, n, flow);
    if (e != cudaSuccess) return TW_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return TW_ERR_CUDA;
    return TW_OK;
}
