// Build step: the table of positive finite floats x where glibc's logf(x) differs from
// tw_log_base(x) (twlog.h). Writes little-endian pairs (uint32 input bits, uint32 glibc result
// bits), sorted by input, to the file named by argv[1].
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "twlog.h"

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    const uint32_t first = 1, end = 0x7f800000u;  // every positive subnormal and normal float
    int nt = omp_get_max_threads();
    uint32_t** lists = calloc((size_t)nt, sizeof(uint32_t*));
    size_t* counts = calloc((size_t)nt, sizeof(size_t));
    size_t* caps = calloc((size_t)nt, sizeof(size_t));
#pragma omp parallel
    {
        int t = omp_get_thread_num();
        uint64_t span = (end - first + (uint64_t)nt - 1) / nt;
        uint64_t lo = first + span * t, hi = lo + span;
        if (hi > end) hi = end;
        for (uint64_t b = lo; b < hi; b++) {
            uint32_t u = (uint32_t)b;
            float x;
            memcpy(&x, &u, 4);
            float g = logf(x);
            float m = tw_log_base((double)x);
            uint32_t gb, mb;
            memcpy(&gb, &g, 4);
            memcpy(&mb, &m, 4);
            if (gb != mb) {
                if (counts[t] == caps[t]) {
                    caps[t] = caps[t] ? caps[t] * 2 : 4096;
                    lists[t] = realloc(lists[t], caps[t] * 2 * sizeof(uint32_t));
                }
                lists[t][counts[t] * 2] = u;
                lists[t][counts[t] * 2 + 1] = gb;
                counts[t]++;
            }
        }
    }
    FILE* f = fopen(argv[1], "wb");
    if (!f) return 1;
    size_t total = 0;
    for (int t = 0; t < nt; t++) {
        if (counts[t] && fwrite(lists[t], 8, counts[t], f) != counts[t]) return 1;
        total += counts[t];
    }
    fclose(f);
    printf("%zu\n", total);
    return 0;
}
