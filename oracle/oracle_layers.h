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
    std::vector<float> shrink;  // the inverse matte shrink of every FG layer (empty: all zero)
    int first = 0, last = -1;   // the displayed group first..=last (last -1: the full group 0..=nfg)
    // the tracking points of every layer (nfg + 1 lists, Main_BG last; empty: none): (x, y at A, x, y
    // at B) in output pixels, in the row order of the images
    std::vector<std::vector<std::array<float, 4>>> points;
};

// layers.rs:120-129 (LayerJob::display_group): the group of the Display popup
void display_group(int display, int nfg, int* first, int* last);
// matte.rs:280-310 (choke_pl), the plugin's matte choke of a w x h float plane
void choke_pl(std::vector<float>& m, int w, int h, float amount);
// layers.rs:497-528 (rebuilt_plate): the single group display of an unwarped frame; mattes raw (0..1)
// in host rows; the fill runs on bottom-up rows when `reversed`
int rebuilt_plate(const Image& frame, const std::vector<std::vector<float>>& mattes, const std::vector<float>& shrink,
                  int k, bool reversed, bool above_first, Image* out, std::string* err,
                  bool is360 = false);

LPlane raw_plane(const float* m, size_t n, Fmt fmt);
LPlane comp_plane(const std::vector<LPlane>& raws, const std::vector<float>& shrink, int k, Fmt fmt, int w, int h);
Image layer_times(const Image& src, const LPlane& p);
bool solver_mask(const std::vector<LPlane>& raws, const LPlane& comp, int k, size_t n, std::vector<float>* out);
void over_pl(Image& dest, const Image& src);
// layers/plates.rs:330-412 (solve_and_compose_plates) with the tracking frames equal to A and B
int compose_layers_plates(const LayerJob& job, const Image& a, const Image& b, Image* out, std::string* err);

}  // namespace orc
