/* Oracle (test infrastructure only): CPU restatement of the reference's Gaussian sketch.
 *
 * tensorsvm-train.cu:2621-2643 (gaussrand) draws standard normals with the Marsaglia polar
 * method over glibc rand(), in float arithmetic, with static state; srand() is never called,
 * so the stream is glibc's default seed 1.  LRA fills Q (n x k, row-major) in i-then-j order
 * (tensorsvm-train.cu:1966-1974), so the sketch is simply the first n*k values of the stream.
 *
 * This file is compiled with -ffp-contract=off so that the float expressions are evaluated
 * exactly as the reference's x86-64 host code evaluates them (no fused multiply-add).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

/* Fill out[0..count) with the reference's gaussrand() stream, starting from a freshly
 * seeded glibc generator (srand(1) is glibc's default state). Returns the number of
 * rand() calls consumed. */
long oracle_polar_sketch(float *out, long count)
{
    srand(1);
    long produced = 0, draws = 0;
    while (produced < count) {
        float v1, v2, s;
        do {
            float u1 = (float)rand() / RAND_MAX;
            float u2 = (float)rand() / RAND_MAX;
            draws += 2;
            v1 = 2 * u1 - 1;
            v2 = 2 * u2 - 1;
            s = v1 * v1 + v2 * v2;
        } while (s >= 1 || s == 0);
        /* tensorsvm-train.cu:2637/2639: X = V * sqrt(-2 * log(S) / S), float overloads. */
        float f = sqrtf(-2 * logf(s) / s);
        out[produced++] = v1 * f;
        if (produced < count) out[produced++] = v2 * f;
    }
    return draws;
}

/* The raw glibc rand() stream from seed 1 (used to pin the GPU generator's recurrence). */
void oracle_rand_stream(uint32_t *out, long count)
{
    srand(1);
    for (long i = 0; i < count; ++i) out[i] = (uint32_t)rand();
}
