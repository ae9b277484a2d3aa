/* Build step: the C library's logf is not correctly rounded. The reference computes the
 * opacity cutoff of its tight tile bounds with it (src/splat/tile_coverage.cpp:36,
 * qmax = 2 * std::log(255 * opacity)), so the tile ids depend on its exact results. The
 * kernels compute the correctly rounded log instead and apply this table of the inputs
 * where the C library's result differs (always by one ulp).
 *
 * This program enumerates every float x in [1, 255] (the range of 255 * o for
 * o in [1/255, 1]), compares logf(x) with the correctly rounded (float)log((double)x), and
 * writes a C source with:
 *   gsr_logf_fixups[]        sorted entries ((x_bits - base) << 1) | up, up = the C
 *                            library's result is one ulp above the correctly rounded one
 *   gsr_logf_bucket_start[]  for bucket b = (x_bits - base) >> 10, the first entry index
 * A CPU test re-runs the comparison against the running C library.
 *
 * Usage: gen_logf_fixups <out.c> */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    const float lo = 1.0f, hi = 255.0f;
    uint32_t lob, hib;
    memcpy(&lob, &lo, 4);
    memcpy(&hib, &hi, 4);
    const uint32_t span = hib - lob + 1;
    const uint32_t buckets = (span >> 10) + 2;
    uint32_t cap = 1u << 18, n = 0;
    uint32_t* fix = (uint32_t*)malloc(sizeof(uint32_t) * cap);
    uint32_t* start = (uint32_t*)calloc(buckets, sizeof(uint32_t));
    for (uint32_t u = lob; u <= hib; ++u) {
        float x, f, g;
        memcpy(&x, &u, 4);
        f = logf(x);
        g = (float)log((double)x);
        uint32_t fb, gb;
        memcpy(&fb, &f, 4);
        memcpy(&gb, &g, 4);
        if (fb == gb) continue;
        if (fb != gb + 1u && gb != fb + 1u) {
            fprintf(stderr, "logf differs by more than one ulp at %a\n", x);
            return 1;
        }
        if (n == cap) {
            cap *= 2;
            fix = (uint32_t*)realloc(fix, sizeof(uint32_t) * cap);
        }
        fix[n++] = ((u - lob) << 1) | (fb > gb ? 1u : 0u);
    }
    /* bucket starts: start[b] = first entry whose offset >> 10 >= b */
    uint32_t e = 0;
    for (uint32_t b = 0; b < buckets; ++b) {
        while (e < n && ((fix[e] >> 1) >> 10) < b) ++e;
        start[b] = e;
    }
    FILE* out = fopen(argv[1], "w");
    if (!out) return 1;
    fprintf(out, "/* generated by gen_logf_fixups.c from this machine's C library; do not edit */\n");
    fprintf(out, "#include <stdint.h>\n");
    fprintf(out, "const uint32_t gsr_logf_fixup_base = 0x%08xu;\n", lob);
    fprintf(out, "const uint32_t gsr_logf_fixup_last = 0x%08xu;\n", hib);
    fprintf(out, "const uint32_t gsr_logf_fixup_count = %uu;\n", n);
    fprintf(out, "const uint32_t gsr_logf_bucket_count = %uu;\n", buckets);
    fprintf(out, "const uint32_t gsr_logf_fixups[%u] = {", n ? n : 1);
    for (uint32_t i = 0; i < n; ++i) fprintf(out, "%s%u", i == 0 ? "\n" : ((i % 12) ? "," : ",\n"), fix[i]);
    if (!n) fprintf(out, "0");
    fprintf(out, "};\nconst uint32_t gsr_logf_bucket_start[%u] = {", buckets);
    for (uint32_t b = 0; b < buckets; ++b) fprintf(out, "%s%u", b == 0 ? "\n" : ((b % 12) ? "," : ",\n"), start[b]);
    fprintf(out, "};\n");
    fclose(out);
    printf("logf fixups: %u of %u inputs\n", n, span);
    free(fix);
    free(start);
    return 0;
}
