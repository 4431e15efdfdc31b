// Test infrastructure: the CPU oracle's restatement of the compositor's tails in the reference: the
// Weighted Blend filters (plugins/retime-engine/src/filters.rs: the separable blur of the
// sharpening step, the difference mask and its clean-up, the masked composite, one half of Weighted
// Blend) and Blur Compensation (warp/blurcomp.rs: the flow directed motion blur and its amount).
// Only the tests, the smoke check and the benchmark's CPU legs load it.
#pragma once
#include "oracle_core.h"

namespace orc {

struct Mask {  // filters.rs:16-49: one byte per pixel, top row first
    int w = 0, h = 0;
    std::vector<uint8_t> d;
    Mask() {}
    Mask(int w_, int h_, uint8_t v = 0) : w(w_), h(h_), d((size_t)w_ * h_, v) {}
};

std::vector<float> wb_blur_taps(float radius);                                   // filters.rs:75-93
void wb_blur(Image& img, float radius, bool above_first);                        // filters.rs:254-280
float wb_mask_limit(Fmt fmt, float threshold);                                   // filters.rs:293-295
Mask difference_mask(const Image& warped, const Image& original, float threshold);  // filters.rs:301-334
void mask_prune(Mask& m, int limit);                                             // filters.rs:360-375
void mask_dilate_rows(Mask& m);                                                  // filters.rs:406-418
void mask_fill(Mask& m, int limit, uint8_t value);                               // filters.rs:387-400
void mask_replicate_border(Mask& m);                                             // filters.rs:425-496
void clean_mask(Mask& m);                                                        // filters.rs:507-520
Mask change_mask(const Image& warped, const Image& original);                    // filters.rs:525-529
void composite_masked(Image& dest, const Image& src, const Mask& m);             // filters.rs:543-603
float sharpen_weight(float t);                                                   // filters.rs:627-631
void sharpen_step(Image& frame, const Image& original, float t, bool above_first);  // filters.rs:649-657

// warp/blurcomp.rs:176-559 (motion_blur): returns 0, 1 (mismatch) or 2 (a NaN tap, a vector of more
// than 65536 taps, or with is360 a tap that the wrap loops cannot bring into the frame)
int motion_blur(Image& dest, const Image& src, const FlowField& flow, float amount, bool hiq, float shutter,
                std::string* err, bool is360 = false);
// warp/blurcomp.rs:42-130 (blur_compensation; with is360 blur_compensation_wrap, :73-87): in place on
// the composed image
int blur_compensation(Image& img, const FlowField& flow, float s0, float s1, float blur, bool hiq, std::string* err,
                      bool is360 = false);

}  // namespace orc
