/*
 * Oracle: CPU restatement of the reference's random numbers and sample seeding.
 * TEST INFRASTRUCTURE ONLY.
 *
 *   MWC64X generator       src/imbatracer/render/random.h:15-47 (multiplier 4294883355,
 *                          random_float = x / (float)0xFFFFFFFF, random_int = x % (max-min) + min)
 *   per-sample seeding     render/ray_gen/ray_gen.h:49-72 (camera samples) and :128-141 (light
 *                          samples): seed = (int)seed_base, four rounds of seed = 33*seed ^ i
 *                          with int wrap-around, RNG(seed) sign-extends into the 64-bit state,
 *                          then discard((seed % 5) + 16 + idx % 5) with C remainder semantics
 */
#include <stdint.h>

uint32_t oracle_mwc64x(uint64_t* state) {
    const uint32_t c = (uint32_t)(*state >> 32);
    const uint32_t x = (uint32_t)(*state & 0xFFFFFFFFu);
    *state = (uint64_t)x * 4294883355ULL + c;
    return x ^ c;
}

float oracle_random_float(uint64_t* state) {
    return (float)oracle_mwc64x(state) / (float)0xFFFFFFFFu;
}

int oracle_random_int(uint64_t* state, int min, int max) {
    return max == min ? min : (int)(oracle_mwc64x(state) % (uint32_t)(max - min) + (uint32_t)min);
}

/* Seeds the RNG of sample i. `idx` is pixel_idx for camera samples (ray_gen.h:70) or the
 * ray index i itself for light samples (ray_gen.h:139). */
uint64_t oracle_seed_state(uint64_t seed_base, int i, int idx) {
    int32_t seed = (int32_t)(uint32_t)seed_base;
    for (int r = 0; r < 4; ++r) seed = (int32_t)((uint32_t)33 * (uint32_t)seed ^ (uint32_t)i);
    uint64_t state = (uint64_t)(int64_t)seed;
    const int n = (seed % 5) + 16 + idx % 5;
    for (int k = 0; k < n; ++k) oracle_mwc64x(&state);
    return state;
}

/* Seeds `count` camera samples starting at sample index `first` with `spp` samples per pixel. */
void oracle_seed_camera(uint64_t seed_base, int first, int count, int spp, uint64_t* states) {
    for (int j = 0; j < count; ++j) {
        const int i = first + j;
        states[j] = oracle_seed_state(seed_base, i, i / spp);
    }
}

/* Draws n floats from each of `count` generators (row-major out[count][n]). */
void oracle_draw_floats(uint64_t* states, int count, int n, float* out) {
    for (int j = 0; j < count; ++j)
        for (int k = 0; k < n; ++k) out[(int64_t)j * n + k] = oracle_random_float(states + j);
}
