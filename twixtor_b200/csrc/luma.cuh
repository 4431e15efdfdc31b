// The luma of an engine pixel (prep.rs:168-235): Rec.601-like weights over R, G, B, optionally
// plus 0.3 * alpha (Track RGB+A), or the video range conversion of the red channel (the
// "Video Range" luma: (R - 16) * 255 / 219 on the 8 bit scale). Engine pixels are A, R, G, B.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace tw {

enum : int { LUMA_TRACK_ALPHA = 1, LUMA_VIDEO_RANGE = 2 };

__device__ __forceinline__ float luma_px(const void* eng, int fmt, long i, int mode) {
    bool track_alpha = mode & LUMA_TRACK_ALPHA, video_range = mode & LUMA_VIDEO_RANGE;
    if (fmt == 0) {
        uchar4 p = reinterpret_cast<const uchar4*>(eng)[i];
        float a = (float)p.x, r = (float)p.y, g = (float)p.z, b = (float)p.w;
        if (video_range) return ((r - 16.0f) * 255.0f) / 219.0f;
        float sum = (r * 0.3f + g * 0.59f) + b * 0.11f;
        return track_alpha ? (float)((double)sum + (double)a * 0.3) : sum;
    }
    if (fmt == 1) {
        ushort4 p = reinterpret_cast<const ushort4*>(eng)[i];
        if (video_range) return (((float)p.y / 257.0f - 16.0f) * 255.0f) / 219.0f;
        double sum = ((double)p.z * 0.59 + (double)p.y * 0.3) + (double)p.w * 0.11;
        if (track_alpha) sum += (double)p.x * 0.3;
        return (float)(sum / 257.0);
    }
    float4 p = reinterpret_cast<const float4*>(eng)[i];
    if (video_range) return ((p.y * 255.0f - 16.0f) * 255.0f) / 219.0f;
    double sum = ((double)p.z * 0.59 + (double)p.y * 0.3) + (double)p.w * 0.11;
    if (track_alpha) sum += (double)p.x * 0.3;
    return (float)(sum * 255.0);
}

}  // namespace tw
