// The reference's LightVertices (render/integrators/light_vertices.h) compiled with this
// repository's include/shadow ahead of the reference's src/, so that the HashGrid it holds is
// libimbart's GPU grid (include/imbart_hashgrid.hpp) — the drop-in path for the photon grid.
// Built by oracle/ref/build_ref.py into oracle/_ref/libref_gpu_grid.so, linked to libimbart.
// TEST INFRASTRUCTURE ONLY: the test compares its merges with the reference's own HashGrid.
#include <cstdint>
#include <vector>

#define private public
#include "imbatracer/render/integrators/light_vertices.h"
#undef private

// The harness globals the force-included prelude and the TBB shim refer to (this library is
// loaded on its own, without libref.so).
uint64_t imbart_ref_seed_value = 0;
uint64_t imbart_ref_seed_step = 0;
int imbart_ref_tbb_threads = 1;

extern "C" {

// n vertices at pos (xyz packed) go into a LightVertices cache (add_vertex_to_cache), which
// builds its grid with `radius` (LightVertices::build, light_vertices.h:70-75); then one
// get_merge (light_vertices.h:95-100) per query. out_ids (nq*k) receives cache indices.
int refgpu_light_vertices_merge(const float* pos, int n, float radius, const float* queries, int nq, int k,
                                int* out_ids, int* out_counts) {
    using namespace imba;
    LightVertices lv(n);
    lv.cache_.resize((size_t)n);
    lv.clear();
    for (int i = 0; i < n; ++i) {
        LightPathVertex v;
        v.isect.pos = float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        v.throughput = rgb(0.0f);
        v.path_length = 2;
        v.dVC = v.dVCM = v.dVM = 0.0f;
        lv.add_vertex_to_cache(v);
    }
    lv.build(radius, true);
    if (lv.accel_.size() != (size_t)n) return -1;
    std::vector<const VCMPhoton*> out((size_t)k);
    const VCMPhoton* base = lv.accel_.photons();
    for (int q = 0; q < nq; ++q) {
        const int c = lv.get_merge(float3(queries[3 * q], queries[3 * q + 1], queries[3 * q + 2]), out, k);
        out_counts[q] = c;
        for (int j = 0; j < k; ++j) out_ids[(size_t)q * k + j] = j < c ? (int)(out[j] - base) : -1;
    }
    return 0;
}

}  // extern "C"
