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

#include <mutex>

#include "../../include/twixtor_b200.h"
#include "kernels.cuh"

namespace {

// Scratch of the allocation-free block matching: the u and v planes of the field, the transposes
// of A and B, and the transposed field of the column sweeps (6 planes).
constexpr long NOALLOC_MAX_PIXELS = TW_NOALLOC_MAX_PIXELS;
static __device__ __align__(256) float g_noalloc_planes[6 * NOALLOC_MAX_PIXELS];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
float* g_planes_addr[MAX_DEVICES] = {};  // device address of g_noalloc_planes, per device

// Once per device, with that device current: the device address of the scratch array (the host
// side name g_noalloc_planes is only a stand-in, not a device pointer) and the shared memory limit
// of the sweep kernels. Neither allocates.
int setup(int device, float** planes) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (device < 0 || device >= MAX_DEVICES) return TW_ERR_UNSUPPORTED;
    if (!g_planes_addr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_planes) != cudaSuccess || !p) return TW_ERR_CUDA;
        if (cudaFuncSetAttribute(tw::k_bm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tw::bm_smem_bytes(tw::BM_MAX_LINE)) != cudaSuccess)
            return TW_ERR_CUDA;
        if (cudaFuncSetAttribute(tw::k_bm_cols, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tw::bm_smem_bytes(tw::BM_MAX_LINE)) != cudaSuccess)
            return TW_ERR_CUDA;
        g_planes_addr[device] = (float*)p;
    }
    *planes = g_planes_addr[device];
    return TW_OK;
}

}  // namespace

extern "C" int tw_block_match_noalloc(const float* a, const float* b, float* flow, int32_t width, int32_t height,
                                      void* stream) {
    if (!a || !b || !flow || width <= 0 || height <= 0) return TW_ERR_BAD_PARAM;
    if ((long)width * height > NOALLOC_MAX_PIXELS || width > tw::BM_MAX_LINE || height > tw::BM_MAX_LINE)
        return TW_ERR_TOO_LARGE;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return TW_ERR_CUDA;
    float* planes = nullptr;
    int rc = setup(device, &planes);
    if (rc != TW_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    long n = (long)width * height;
    float* fu = planes;
    float* fv = fu + n;
    float *at = fv + n, *bt = at + n, *ut = bt + n, *vt = ut + n;
    const int tb = 256;
    unsigned g1 = (unsigned)((n + tb - 1) / tb);
    dim3 tt(32, 8), ga((width + 31) / 32, (height + 31) / 32), gb((height + 31) / 32, (width + 31) / 32);
    // every element of the planes this call reads is written first, so the previous call's
    // contents never reach the result
    tw::k_deinterleave<<<g1, tb, 0, s>>>(flow, n, fu, fv);
    if (width >= 3 && height >= 3) {
        tw::k_bm_rows<<<height - 2, tb, tw::bm_smem_bytes(width), s>>>(a, b, fu, fv, width, height);
        tw::k_transpose2<<<ga, tt, 0, s>>>(a, b, at, bt, width, height);
        tw::k_transpose2<<<ga, tt, 0, s>>>(fu, fv, ut, vt, width, height);
        tw::k_bm_cols<<<width - 2, tb, tw::bm_smem_bytes(height), s>>>(at, bt, ut, vt, width, height);
        tw::k_transpose2<<<gb, tt, 0, s>>>(ut, vt, fu, fv, height, width);
    }
    tw::k_interleave<<<g1, tb, 0, s>>>(fu, fv, n, flow);
    if (cudaGetLastError() != cudaSuccess) return TW_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return TW_ERR_CUDA;
    return TW_OK;
}
