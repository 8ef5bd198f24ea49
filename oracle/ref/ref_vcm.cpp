// Harness around the reference's VCM family (render/integrators/vcm.cpp, light_vertices.cpp),
// compiled in place into oracle/_ref/libref.so. TEST INFRASTRUCTURE ONLY.
//
// The reference runs an iteration as render() = light pass + camera pass with seeds drawn from
// std::random_device (routed to the harness's fixed seed by ref_prelude.h). To compare the
// GPU passes one at a time, the harness drives the integrator's own private passes
// (trace_light_paths, trace_camera_paths) and reads its light-vertex cache; access to the
// private members is granted by compiling the reference headers with `private` and
// `protected` defined as `public` in this translation unit only (the class layouts do not
// change). The iteration preamble (radius shrinking, MIS eta values; vcm.cpp:25-46) is set
// through ref_vcm_begin_iteration before each light pass.
#include <algorithm>
#include <atomic>
#include <cassert>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#define private public
#define protected public
#include "imbatracer/render/integrators/vcm.h"
#include "imbatracer/render/scheduling/tile_scheduler.h"
#include "imbatracer/render/ray_gen/tile_gen.h"
#undef private
#undef protected

extern "C" void imbart_ref_set_seed(uint64_t value, uint64_t step);
imba::Scene* ref_scene_of(void* h);

using namespace imba;

namespace {

struct RefVcmBase {
    virtual ~RefVcmBase() {}
    virtual float pixel_size() = 0;
    virtual float base_radius() = 0;
    virtual int cache_capacity() = 0;
    virtual float begin_iteration(int iteration) = 0;
    virtual void light_pass(AtomicImage& img) = 0;
    virtual void camera_pass(AtomicImage& img) = 0;
    virtual int vertices(float* out, int cap) = 0;
    virtual void mis_eta(float* out2) = 0;
    virtual void time_grid(int reps, int threads, double* out3) = 0;
};

template <VCMSubAlgorithm algo>
struct RefVcm : RefVcmBase {
    Scene& scene;
    UserSettings settings;
    PerspectiveCamera cam;
    DefaultTileGen<VCMState> gen;
    TileScheduler<VCMState, VCMShadowState, false> sched;
    VCMIntegrator<algo> integ;

    RefVcm(Scene& s, const UserSettings& st, const PerspectiveCamera& c)
        : scene(s), settings(st), cam(c),
          gen(st.width, st.height, st.concurrent_spp, st.tile_size),
          sched(gen, s, st.num_connections + 1, 1, st.tile_size * st.tile_size * st.concurrent_spp, true),
          integ(s, cam, sched, st) {
        integ.preprocess();
    }

    float pixel_size() override { return integ.pixel_size(); }
    float base_radius() override { return integ.base_radius_; }
    int cache_capacity() override { return (int)integ.light_vertices_.cache_.size(); }

    // vcm.cpp:25-46, without tracing.
    float begin_iteration(int iteration) override {
        const float radius_alpha = 0.75f;
        integ.light_vertices_.clear();
        integ.cur_iteration_ = iteration;
        integ.pm_radius_ = integ.base_radius_ / powf(static_cast<float>(iteration), 0.5f * (1.0f - radius_alpha));
        integ.pm_radius_ = std::max(integ.pm_radius_, 1e-7f);
        const float eta_vcm = pi * sqr(integ.pm_radius_) * settings.light_path_count;
        integ.mis_eta_vc_ = integ.mis_pow(1.0f / eta_vcm);
        integ.mis_eta_vm_ = algo == ALGO_BPT ? 0.0f : integ.mis_pow(eta_vcm);
        return integ.pm_radius_;
    }

    void light_pass(AtomicImage& img) override {
        if (algo != ALGO_PT) integ.trace_light_paths(img);
    }

    void camera_pass(AtomicImage& img) override {
        if (algo != ALGO_LT) integ.trace_camera_paths(img);
    }

    void mis_eta(float* out2) override {
        out2[0] = integ.mis_eta_vc_;
        out2[1] = integ.mis_eta_vm_;
    }

    // The reference's photon grid over the current cache, timed on its own: `reps` rebuilds
    // (LightVertices::build -> HashGrid::build, light_vertices.h:70-75) and one k-nearest
    // query (LightVertices::get_merge, as vertex_merging calls it, vcm.cpp:571-576) at every
    // cached vertex, spread over `threads` OpenMP threads. out: seconds per build, seconds
    // for all queries, queries.
    void time_grid(int reps, int threads, double* out3) override {
        LightVertices& lv = integ.light_vertices_;
        const auto t0 = std::chrono::steady_clock::now();
        for (int r = 0; r < reps; ++r) lv.build(integ.pm_radius_, true);
        const auto t1 = std::chrono::steady_clock::now();
        const int n = lv.count();
        const int k = settings.num_knn;
        long long found = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads) reduction(+ : found)
        for (int i = 0; i < n; ++i) {
            std::vector<const VCMPhoton*> out(k);
            found += lv.get_merge(lv.cache_[i].isect.pos, out, k);
        }
        const auto t2 = std::chrono::steady_clock::now();
        out3[0] = std::chrono::duration<double>(t1 - t0).count() / std::max(reps, 1);
        out3[1] = std::chrono::duration<double>(t2 - t1).count();
        out3[2] = (double)n;
        (void)found;
    }

    // 28 floats per vertex: pos, mat | out_dir, path_length | normal, dVC | geom_normal, dVCM |
    // u_tangent, dVM | v_tangent, uv.x | throughput, uv.y.
    int vertices(float* out, int cap) override {
        if (algo == ALGO_LT || algo == ALGO_PT) return 0;   // these never build the cache
        const LightVertices& lv = integ.light_vertices_;
        const int n = std::min(lv.count(), cap);
        for (int i = 0; i < n; ++i) {
            const LightPathVertex& v = lv.cache_[i];
            const Intersection& is = v.isect;
            int mat = -1;
            for (int m = 0; m < (int)scene.materials().size(); ++m)
                if (scene.materials()[m].get() == is.mat) mat = m;
            float* o = out + 28 * (size_t)i;
            auto put3 = [&](int at, const float3& a) { o[at] = a.x; o[at + 1] = a.y; o[at + 2] = a.z; };
            put3(0, is.pos);
            std::memcpy(o + 3, &mat, 4);
            put3(4, is.out_dir);
            std::memcpy(o + 7, &v.path_length, 4);
            put3(8, is.normal);
            o[11] = v.dVC;
            put3(12, is.geom_normal);
            o[15] = v.dVCM;
            put3(16, is.u_tangent);
            o[19] = v.dVM;
            put3(20, is.v_tangent);
            o[23] = is.uv.x;
            o[24] = v.throughput.x; o[25] = v.throughput.y; o[26] = v.throughput.z;
            o[27] = is.uv.y;
        }
        return lv.count();
    }
};

void copy_image(AtomicImage& img, int w, int h, float* out) {
    for (int i = 0; i < w * h; ++i)
        for (int k = 0; k < 3; ++k) out[3 * i + k] = img.pixels()[i][k];
}

struct Handle {
    std::unique_ptr<RefVcmBase> vcm;
    int w, h;
};

}  // namespace

extern "C" {

// algo: 0 VCM, 1 BPT, 2 PPM, 3 LT, 4 PT (the VCMSubAlgorithm order, vcm.h:37-43).
// One camera tile of tile_size^2 pixels (tile_size >= width, height makes sample indices
// global); the light tile generator splits each light's paths into tiles of tile_size^2.
void* ref_vcm_create(void* scene_h, int algo, int w, int h, const float* pos, const float* dir, const float* up,
                     float fov, int spp, int max_path_len, int light_path_count, int num_connections, int num_knn,
                     float radius_factor, int tile_size, uint64_t preprocess_seed) {
    Scene& scene = *ref_scene_of(scene_h);
    UserSettings st;
    st.width = w; st.height = h; st.fov = fov;
    st.concurrent_spp = spp; st.max_path_len = max_path_len; st.light_path_count = light_path_count;
    st.num_connections = num_connections; st.num_knn = num_knn; st.radius_factor = radius_factor;
    st.tile_size = tile_size; st.thread_count = 1;
    st.traversal_platform = UserSettings::gpu;
    PerspectiveCamera cam((float)w, (float)h, fov);
    cam.move(float3(pos[0], pos[1], pos[2]), float3(dir[0], dir[1], dir[2]), float3(up[0], up[1], up[2]));
    imbart_ref_set_seed(preprocess_seed, 1);   // cache-size probe paths draw one seed each
    auto* hd = new Handle{nullptr, w, h};
    switch (algo) {
        case 0: hd->vcm.reset(new RefVcm<ALGO_VCM>(scene, st, cam)); break;
        case 1: hd->vcm.reset(new RefVcm<ALGO_BPT>(scene, st, cam)); break;
        case 2: hd->vcm.reset(new RefVcm<ALGO_PPM>(scene, st, cam)); break;
        case 3: hd->vcm.reset(new RefVcm<ALGO_LT>(scene, st, cam)); break;
        default: hd->vcm.reset(new RefVcm<ALGO_PT>(scene, st, cam)); break;
    }
    return hd;
}

void ref_vcm_destroy(void* h) { delete static_cast<Handle*>(h); }

// out: pixel size, base radius, cache capacity.
void ref_vcm_info(void* h, float* out3) {
    RefVcmBase& v = *static_cast<Handle*>(h)->vcm;
    out3[0] = v.pixel_size();
    out3[1] = v.base_radius();
    out3[2] = (float)v.cache_capacity();
}

// Sets the iteration's radius and MIS constants; returns the photon radius. out2: eta_vc, eta_vm.
float ref_vcm_begin_iteration(void* h, int iteration, float* out2) {
    RefVcmBase& v = *static_cast<Handle*>(h)->vcm;
    const float r = v.begin_iteration(iteration);
    if (out2) v.mis_eta(out2);
    return r;
}

// Light pass: light tile t (all lights in order) fills its queue with seed_base = seed + t * step.
void ref_vcm_light_pass(void* h, uint64_t seed, uint64_t step, float* image_out) {
    Handle* hd = static_cast<Handle*>(h);
    AtomicImage img(hd->w, hd->h);
    img.clear();
    imbart_ref_set_seed(seed, step);
    hd->vcm->light_pass(img);
    copy_image(img, hd->w, hd->h, image_out);
}

int ref_vcm_light_vertices(void* h, float* out, int cap) {
    return static_cast<Handle*>(h)->vcm->vertices(out, cap);
}

void ref_vcm_time_grid(void* h, int reps, int threads, double* out3) {
    static_cast<Handle*>(h)->vcm->time_grid(reps, threads, out3);
}

void ref_vcm_camera_pass(void* h, uint64_t seed, float* image_out) {
    Handle* hd = static_cast<Handle*>(h);
    AtomicImage img(hd->w, hd->h);
    img.clear();
    imbart_ref_set_seed(seed, 0);
    hd->vcm->camera_pass(img);
    copy_image(img, hd->w, hd->h, image_out);
}

}  // extern "C"
