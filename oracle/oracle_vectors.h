// CPU oracle of the vector encoder and the single layer Create Vectors pass (vectors.rs,
// create_vectors.rs). TEST INFRASTRUCTURE ONLY (see oracle_core.h).
#pragma once
#include "oracle_core.h"

namespace orc {

// vectors.rs:57-130: flow -> encoded vector image of dst's size and format
int encode_vectors(Image& dst, const FlowField& flow, float scale, std::string* err);
// vectors.rs:148-156
Image zero_vectors_image(int w, int h, Fmt fmt);

struct CreateVectorsSettings {  // create_vectors.rs:97-135
    int quality = 4;           // 4 Normal (half res), 5 Full res
    bool hiq = true;
    float sensitivity = 0.7f;
    bool track_rgb_a = false;
    float max_displace = 2048.0f;
    bool taps_above_first = true;  // the solver's vertical border taps (flow/conv.rs:598-615)
    bool prep_contrast_edge = false, prep_delinearize = false;  // plugins/create-vectors/src/glue.rs:138-139
};
// create_vectors.rs:162-183 (one layer)
int create_vectors(const Image& x, const Image& y, const CreateVectorsSettings& s, Image* out, std::string* err);

// ---- Vectors In (compose/vector.rs:323-397, vectors.rs:474-583) ----
// vectors.rs:474-522: the encoded image -> the flow of its size (alpha 0 the zero vector)
FlowField decode_vectors(const Image& vec, float max_displace);
// vectors.rs:555-561: 255 - A, 65535 - A or 1 - A as raw mask bytes of kind 1, 2 or 3
void vector_hole_mask(const Image& vec, std::vector<uint8_t>* bytes, int* kind);
// vectors.rs:573-578
void apply_vec_scale(FlowField& flow, float sx, float sy);
// compose/vector.rs:335-345: decode, flow hole fill (the tap order), Vec Scale
int flow_from_vector_image(const Image& vec, float max_displace, float sx, float sy, bool above_first, FlowField* out,
                           std::string* err);
// compose/vector.rs:370-397: the inversion of a flow (textured forward warp, or Gouraud with !pyramid)
int invert_flow(const FlowField& flow, bool pyramid, bool above_first, FlowField* out, std::string* err);
// plugins/vectors-in/src/vectorin.rs:125-155: the vector image's alpha capped by a layer matte
void matte_step(Image& img, const std::vector<float>& m);

// ---- the Debug views of Create Vectors (debug.rs) ----
// debug.rs:155-171: view code 0 Blend, 1 Diff, 2 Detail Compare, else Edge Compare, of W' against y
Image debug_views_of(const Image& wp, const Image& y, int code);
// debug.rs:104-152: code 4 is the Warp view
int debug_view(const Image& x, const Image& y, const FlowField& flow, int code, bool gouraud, Image* out,
               std::string* err);

}  // namespace orc
