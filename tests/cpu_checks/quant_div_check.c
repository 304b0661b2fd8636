/* Exhaustive check that dividing by a dequantisation weight w through its
 * rounded reciprocal y = RN(1/w) (Markstein's method: q0 = RN(a*y),
 * r = fma(-q0, w, a) exact, q = RN(q0 + r*y)) gives the IEEE quotient RN(a/w)
 * for every float a, for every weight of the DCT8/16/32 tables of all three
 * channels. The sequence and the quotient both scale exactly with a's
 * exponent (no intermediate leaves the normal range for the quotients the
 * quantisers form), and both are odd in a, so checking every significand of
 * a in [1, 2) covers every a. Prints the number of (weight, a) pairs that
 * differ and exits non-zero if there are any. */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../cujpegxl_b200/csrc/jxl_dequant_tables.inc"

static float weights[3 * (64 + 256 + 1024)];
static int nweights;
static int next_w;
static long long mismatches;
static pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;

static float from_bits(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static long long check_weight(float w) {
    const float y = 1.0f / w;
    long long bad = 0;
    for (uint32_t m = 0; m < (1u << 23); ++m) {
        const float a = from_bits(0x3f800000u | m);
        const float q0 = a * y;
        const float r = fmaf(-q0, w, a);
        const float q = fmaf(r, y, q0);
        bad += q != a / w;
    }
    return bad;
}

static void* worker(void* arg) {
    (void)arg;
    for (;;) {
        pthread_mutex_lock(&mu);
        const int i = next_w++;
        pthread_mutex_unlock(&mu);
        if (i >= nweights) return NULL;
        const long long bad = check_weight(weights[i]);
        if (bad) {
            pthread_mutex_lock(&mu);
            mismatches += bad;
            fprintf(stderr, "weight %a: %lld quotients differ\n", weights[i], bad);
            pthread_mutex_unlock(&mu);
        }
    }
}

static void add(float w) {
    for (int i = 0; i < nweights; ++i) {
        if (weights[i] == w) return;
    }
    weights[nweights++] = w;
}

int main(int argc, char** argv) {
    const int threads = argc > 1 ? atoi(argv[1]) : 8;
    for (int c = 0; c < 3; ++c) {
        for (int i = 0; i < 64; ++i) add(from_bits(kDequantBits8[c][i]));
        for (int i = 0; i < 256; ++i) add(from_bits(kDequantBits16[c][i]));
        for (int i = 0; i < 1024; ++i) add(from_bits(kDequantBits32[c][i]));
    }
    pthread_t t[256];
    const int n = threads < 1 ? 1 : (threads > 256 ? 256 : threads);
    for (int i = 0; i < n; ++i) pthread_create(&t[i], NULL, worker, NULL);
    for (int i = 0; i < n; ++i) pthread_join(t[i], NULL);
    printf("%d distinct weights, %lld mismatching quotients\n", nweights, mismatches);
    return mismatches != 0;
}
