// Test infrastructure: the oracle's restatement of the reference CPU path evaluated in double
// precision, the FP64 yardstick of the fast mode (its flow error in pixels and its frame PSNR).
// Every source of the oracle is compiled here with `float` spelled `double`, so each step keeps the
// reference's order of operations (flow.rs, flow/conv.rs, prep.rs, ...) with 53-bit arithmetic;
// only the plain solve (or_solve_pair) and the compositions are meant to be called from this
// build (the paths that reinterpret float bit patterns, the Delinearize powf and the NaN rule, are
// meaningless in it). Built as its own library, liboracle64.so, beside liboracle.so.
#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#define float double
#include "oracle_core.cpp"
#include "oracle_api.cpp"
#include "oracle_smart.cpp"
#include "oracle_forward.cpp"
#include "oracle_vectors.cpp"
#include "oracle_layers.cpp"
#include "oracle_filters.cpp"
#undef float
