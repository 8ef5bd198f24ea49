// Device restatement of the reference's random numbers (src/imbatracer/render/random.h) and
// of the per-sample seeding of its ray generators (render/ray_gen/ray_gen.h:49-72, 128-141).
// Bit-exact with the reference: integer arithmetic, and the float conversion of a 32-bit
// draw divided by 2^32 (the float value of 0xFFFFFFFF).
#pragma once

#include <stdint.h>

namespace imbart {

struct Rng {
    uint64_t state;

    __host__ __device__ __forceinline__ uint32_t mwc64x() {
        const uint32_t c = (uint32_t)(state >> 32);
        const uint32_t x = (uint32_t)(state & 0xFFFFFFFFu);
        state = (uint64_t)x * 4294883355ULL + c;
        return x ^ c;
    }
    // random_float(): MWC64X() / (float)0xFFFFFFFF, i.e. rounded x scaled by 2^-32 exactly.
    __host__ __device__ __forceinline__ float next_float() {
        return (float)mwc64x() * 2.3283064365386963e-10f;
    }
    // random_int(min, max): min + MWC64X() % (max - min), max exclusive.
    __host__ __device__ __forceinline__ int next_int(int lo, int hi) {
        return hi == lo ? lo : (int)(mwc64x() % (uint32_t)(hi - lo) + (uint32_t)lo);
    }
    __host__ __device__ __forceinline__ void discard(int n) {
        for (int i = 0; i < n; ++i) mwc64x();
    }
};

// Seeds sample i: seed = (int)seed_base, four rounds of Bernstein's hash seed = 33*seed ^ i
// with int wrap-around, the state is the sign-extended seed, then (seed % 5) + 16 + idx % 5
// draws are discarded (idx = pixel index for camera samples, the ray index for light samples).
__host__ __device__ __forceinline__ Rng seed_sample(uint64_t seed_base, int i, int idx) {
    int32_t seed = (int32_t)(uint32_t)seed_base;
    for (int r = 0; r < 4; ++r) seed = (int32_t)((uint32_t)33 * (uint32_t)seed ^ (uint32_t)i);
    Rng rng{(uint64_t)(int64_t)seed};
    rng.discard((seed % 5) + 16 + idx % 5);
    return rng;
}

}  // namespace imbart
