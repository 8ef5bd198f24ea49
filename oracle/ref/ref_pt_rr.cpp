// The reference's PathTracer (render/integrators/pt.cpp, compiled here from the reference tree
// a second time) with its Russian roulette deferred to bounce `rr_start`: the one call to
// russian_roulette in PathTracer::bounce (pt.cpp:53-57) is routed through a wrapper that, for
// paths with fewer than rr_start bounces, neither draws the random number nor kills the path
// (pdf 1), and otherwise runs the reference's russian_roulette unchanged. Everything else is
// the reference's code. rr_start 0 is the reference's own behaviour. The class is renamed
// (PathTracerRRStart) so that it links beside the unmodified PathTracer of pt.cpp.
// TEST INFRASTRUCTURE ONLY: the oracle for the GPU path tracer's rr_start parameter.
#include "imbatracer/render/random.h"

namespace imba {
int imbart_rr_start = 0;

template <typename State, typename Draw>
inline bool imbart_rr_deferred(const State& state, const rgb& throughput, Draw draw, float& pdf) {
    if (state.bounces < imbart_rr_start) {
        pdf = 1.0f;
        return true;
    }
    return russian_roulette(throughput, draw(), pdf);
}
}  // namespace imba

#define russian_roulette(thr, rnd, pdf) imbart_rr_deferred(state_out, thr, [&]() { return (rnd); }, pdf)
#define PathTracer PathTracerRRStart
#include "imbatracer/render/integrators/pt.cpp"
#undef PathTracer
#undef russian_roulette

// Factory for the harness (ref_harness.cpp), which only sees the Integrator interface.
extern "C" imba::Integrator* imbart_make_pt_rr(imba::Scene& scene, imba::PerspectiveCamera& cam,
                                              imba::RayScheduler<imba::PTState, imba::ShadowState>& sched,
                                              int max_path_len, int rr_start) {
    imba::imbart_rr_start = rr_start;
    return new imba::PathTracerRRStart(scene, cam, sched, max_path_len);
}
