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

}  // namespace orc
