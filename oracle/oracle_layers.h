// CPU oracle of the layered composition with plates (layers/plates.rs, matte.rs). TEST
// INFRASTRUCTURE ONLY (see oracle_core.h).
#pragma once
#include "oracle_core.h"

namespace orc {

struct LPlane {  // plates.rs:33-37: a matte plane in the units of the depth
    float white = 1.0f;
    std::vector<float> v;
};

// One layered frame: FG mattes (raw, w*h values, FG1 first) at A and at B, the per layer
// sensitivities (FG1 .. FGn, Main_BG last), the solve and compose settings and the selection.
struct LayerJob {
    ComposeSettings cs;
    FlowSettings fs;
    Selection sel;
    std::vector<std::vector<float>> mattes_a, mattes_b;
    std::vector<float> sensitivity;
};

LPlane raw_plane(const float* m, size_t n, Fmt fmt);
LPlane comp_plane(const std::vector<LPlane>& raws, int k, Fmt fmt, size_t n);
Image layer_times(const Image& src, const LPlane& p);
bool solver_mask(const std::vector<LPlane>& raws, const LPlane& comp, int k, size_t n, std::vector<float>* out);
void over_pl(Image& dest, const Image& src);
// layers/plates.rs:330-412 (solve_and_compose_plates) with the tracking frames equal to A and B
int compose_layers_plates(const LayerJob& job, const Image& a, const Image& b, Image* out, std::string* err);

}  // namespace orc
