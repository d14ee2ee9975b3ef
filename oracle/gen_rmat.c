/*
 * gen_rmat -- write the benchmark's seeded RMAT edge list as a reference
 * binary edge file.  TEST INFRASTRUCTURE ONLY: bench.py's reference arm runs
 * it as a separate process, so that the process timing the reference loads
 * nothing but the reference's own build.  The edges are orc_generate_rmat's
 * (og_oracle.c), equal to the product's generator bit for bit.
 *
 * usage: gen_rmat SCALE EDGE_FACTOR SEED WEIGHTED OUT
 *   WEIGHTED 1: {u32 src, u32 dst, f32 w} records (.wbin), 0: {u32 src, u32 dst} (.bin)
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "og_oracle.h"

int main(int argc, char **argv)
{
    if (argc != 6)
    {
        fprintf(stderr, "usage: %s SCALE EDGE_FACTOR SEED WEIGHTED OUT\n", argv[0]);
        return 2;
    }
    const uint32_t scale = (uint32_t)strtoul(argv[1], NULL, 10), ef = (uint32_t)strtoul(argv[2], NULL, 10);
    const uint64_t seed = strtoull(argv[3], NULL, 10);
    const int weighted = atoi(argv[4]);
    if (scale == 0 || scale > 30 || ef == 0)
    {
        fprintf(stderr, "gen_rmat: bad sizes\n");
        return 2;
    }
    const uint64_t E = ((uint64_t)1 << scale) * ef;
    uint32_t *src = malloc(E * 4), *dst = malloc(E * 4);
    float *w = weighted ? malloc(E * 4) : NULL;
    if (!src || !dst || (weighted && !w) || orc_generate_rmat(scale, ef, seed, 0.57, 0.19, 0.19, 1, src, dst, w))
    {
        fprintf(stderr, "gen_rmat: allocation or size error\n");
        return 1;
    }
    FILE *f = fopen(argv[5], "wb");
    if (!f)
    {
        perror(argv[5]);
        return 1;
    }
    const size_t rec = weighted ? 3 : 2, chunk = (size_t)1 << 20;
    uint32_t *buf = malloc(chunk * rec * 4);
    for (uint64_t i = 0; i < E; i += chunk)
    {
        const size_t n = (size_t)((E - i) < chunk ? (E - i) : chunk);
        for (size_t j = 0; j < n; j++)
        {
            buf[j * rec] = src[i + j];
            buf[j * rec + 1] = dst[i + j];
            if (weighted)
            {
                union { float f; uint32_t u; } x;
                x.f = w[i + j];
                buf[j * rec + 2] = x.u;
            }
        }
        if (fwrite(buf, rec * 4, n, f) != n)
        {
            perror("fwrite");
            return 1;
        }
    }
    fclose(f);
    free(buf);
    free(src);
    free(dst);
    free(w);
    return 0;
}
