// CPU oracle: Smart Blend and the hole fill (warping code 1). TEST INFRASTRUCTURE ONLY.
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "oracle_core.h"

namespace orc {

struct FillGeometry {  // holefill.rs:133-171
    std::vector<std::pair<int, int>> dims;
    int top = 0;
};
FillGeometry fill_geometry(int w, int h);

// smartblend.rs:268-298: smart_blend (binary false) / smart_blend_binary (binary true)
void smart_blend(Image& out, const Image& p1, const Image& p2, float w, bool binary);

// holefill.rs:452-491; mask_kind 1 u8, 2 u16, 3 f32 (w*h entries); wrap: the is360 passes
// (holefill.rs:34-40: the circular horizontal pass, the equirectangular column walk, the period
// keeping resample)
int fill_holes(Image& img, const void* mask, int mask_kind, bool above_first, std::string* err, bool wrap = false);
// holefill.rs:497-518 (fill_flow_holes_with): the two components of a flow
int fill_flow_holes(FlowField& flow, const void* mask, int mask_kind, bool above_first, std::string* err,
                    bool wrap = false);

// warping code 1 compositions (smartblend.rs:350-393): Nearest and Blend
int compose_smart(const ComposeSettings& cs, const Selection& sel, const Image& a, const Image& b, const FlowField* f_ab,
                  const FlowField* f_ba, bool taps_above_first, Image* out, std::string* err);

// smartblend.rs:427-456 (weighted_tail): the sharpening of both warped frames against the unwarped
// ones, then with coverage (c1 != null) Smart Blend, the combined and inverted coverage and the
// fill, else the plain blend. c1 is left holding the holes.
int weighted_tail(Image& out, Image& ta, const Image& a, Image& tb, const Image& b, float wa, Coverage* c1,
                  const Coverage* c2, bool taps_above_first, std::string* err);

}  // namespace orc
