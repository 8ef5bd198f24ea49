/* Force-included before every reference source compiled into oracle/_ref. The reference
 * seeds each queue fill from std::random_device (ray_gen.h:49-50,128-129,
 * light_vertices.cpp:34-35), which makes its images non-deterministic. This prelude routes
 * those draws to a value the harness sets (imbart_ref_set_seed), without editing the
 * reference sources. TEST INFRASTRUCTURE ONLY. */
#ifndef IMBART_REF_PRELUDE_H
#define IMBART_REF_PRELUDE_H
#include <random>
#include <cstdint>

extern uint64_t imbart_ref_seed_value;
extern uint64_t imbart_ref_seed_step;

namespace std {
struct imbart_fixed_random_device {
    typedef unsigned int result_type;
    imbart_fixed_random_device() {}
    unsigned int operator()() {
        const uint64_t v = imbart_ref_seed_value;
        imbart_ref_seed_value += imbart_ref_seed_step;
        return (unsigned int)v;
    }
};
}  // namespace std
#define random_device imbart_fixed_random_device
#endif
