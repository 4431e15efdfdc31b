// CPU oracle of the forward warp (forward.rs, forward/mesh.rs, forward/raster.rs,
// forward/pyramid.rs). TEST INFRASTRUCTURE ONLY (see oracle_core.h).
#pragma once
#include "oracle_core.h"

namespace orc {

struct FwVtx {  // forward/raster.rs:13-22: position and the payload (u, v, d)
    float x, y, u, v, d;
};

// The receiver of the covered pixels of one scan conversion, in order.
struct FwHit {
    int x, y;
    float u, v, d;
};
struct FwHits {
    std::vector<FwHit> hits;
    bool outside = false;
};

int fw_level_count(int w, int h);                                               // forward/pyramid.rs:20-36
void fw_positions(int w, int h, const FlowField& flow, float amount, std::vector<float>* xy);  // mesh.rs:21-46
float fw_mip_level(int w, int h, const FlowField& flow, float amount, int c, int r);          // mesh.rs:63-91
void fw_triangle(const FwVtx tri[3], int w1, int h1, FwHits* sink);              // raster.rs:171-300
// forward.rs:229-320 (textured, pyramid = true) and :327-373 (Gouraud, pyramid = false).
// Returns 0, 1 (mismatch) or 2 (unsupported: the degenerate pass would write outside).
int forward_warp(Image& out, const Image& src, const FlowField& flow, float amount, bool pyramid, Coverage* cov,
                 std::string* err);
// compose/vector.rs:117-147 (compose_forward) with forward.rs:384-496: warping codes 2 (coverage,
// Smart Blend or its binary variant, combine, invert, hole fill) and 3 (no coverage), Nearest and
// Blend and Weighted Blend; the textured forward warp, or the Gouraud variant with cs.gouraud.
int compose_forward(const ComposeSettings& cs, const Selection& sel, const Image& a, const Image& b,
                    const FlowField* f_ab, const FlowField* f_ba, Image* out, std::string* err);

}  // namespace orc
