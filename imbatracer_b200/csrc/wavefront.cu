// Wavefront path tracing on the GPU: sample generation, per-bounce shading and shadow-ray
// resolution around the traversal kernels — the device form of the reference's
// TileScheduler loop (src/imbatracer/render/scheduling/tile_scheduler.h:100-144) driving
// PathTracer (src/imbatracer/render/integrators/pt.cpp) with PixelRayGen samples
// (render/ray_gen/ray_gen.h:36-112).
//
// One frame: camera samples fill the path queue; per bounce the closest-hit kernel traces
// the queue, the shading kernel resolves misses (environment), emitter hits and surface
// hits (next-event estimation into the shadow queue, BSDF continuation into the next path
// queue, both appended with warp-aggregated atomics), the any-hit kernel traces the shadow
// queue and unoccluded contributions are added to the image. Each path carries its own
// MWC64X state, consumed in the reference's order, so the image is independent of queue
// order; samples are indexed globally (one tile covering the image), as in the reference
// run with a tile at least as large as the image.
//
// This file is compiled with -fmad=false (see build.py): the shading arithmetic rounds like
// the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "imbart_internal.h"
#include "rng.cuh"
#include "shade.cuh"

using imbart::Rng;
using namespace imbart::sh;

struct imbart_shading {
    int device = 0;
    ShadingScene s{};
    std::vector<void*> allocations;
};

struct imbart_pt_context {
    int device = 0;
    long long cap = 0;       // paths per queue
    float4* rays[2] = {nullptr, nullptr};
    int4* hits = nullptr;
    int* pixel[2] = {nullptr, nullptr};
    unsigned long long* rng[2] = {nullptr, nullptr};
    float4* thr[2] = {nullptr, nullptr};     // throughput xyz, last_pdf in w
    int* bounces[2] = {nullptr, nullptr};    // bounces | last_specular << 31
    float4* srays = nullptr;                 // shadow rays
    int4* shits = nullptr;
    int* spixel = nullptr;
    float4* scontrib = nullptr;
    int* counts = nullptr;                   // [0] next path queue size, [1] shadow queue size
    int* host_counts = nullptr;              // pinned
    imbart_pt_profile* profile = nullptr;    // measurement of the traversal launches
    cudaEvent_t ev[2] = {nullptr, nullptr};
    unsigned long long* work = nullptr;      // device: closest nodes/tris/insts, shadow nodes/tris/insts
};

namespace imbart {
namespace {

bool ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? IMBART_ERR_OUT_OF_MEMORY : IMBART_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// Appends `pred` lanes of the warp to a queue: one atomic per warp, slots in lane order.
__device__ __forceinline__ int warp_append(int* counter, bool pred) {
    const unsigned active = __activemask();
    const unsigned m = __ballot_sync(active, pred);
    if (m == 0u) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(active, base, leader);
    return pred ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

// Triangle-light frames and emitter areas, computed on the device with the reference's
// formulas (TriangleLight ctor, light.h:99-108; Tri::area, tri.h:21).
__global__ void setup_lights_kernel(TriLight* lights, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    TriLight& L = lights[i];
    const V3 p0(L.v[0][0], L.v[0][1], L.v[0][2]), p1(L.v[1][0], L.v[1][1], L.v[1][2]), p2(L.v[2][0], L.v[2][1], L.v[2][2]);
    V3 n = cross(p1 - p0, p2 - p0);
    L.area = length(n) * 0.5f;
    n = normalize(n);
    V3 t, b;
    local_coordinates(n, t, b);
    L.normal[0] = n.x; L.normal[1] = n.y; L.normal[2] = n.z;
    L.tangent[0] = t.x; L.tangent[1] = t.y; L.tangent[2] = t.z;
    L.binormal[0] = b.x; L.binormal[1] = b.y; L.binormal[2] = b.z;
}

__global__ void emitter_area_kernel(const float* vertices, const int4* tris, int n_tris, Material* mats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_tris) return;
    const int4 t = tris[i];
    if (mats[t.w].kind != kEmissive) return;
    const V3 v0 = load3(vertices, t.x), v1 = load3(vertices, t.y), v2 = load3(vertices, t.z);
    mats[t.w].area = length(cross(v1 - v0, v2 - v0)) / 2;
}

struct CameraParams {
    float r2w[16];
    float pos[3];
    int width, height, spp;
    int tile_left, tile_top, tile_w, full_w;
    unsigned long long seed_base;
};

// PixelRayGen::fill_queue + the path tracer's sample function (pt.cpp:168-177) +
// PerspectiveCamera::generate_ray (camera.h:57-65, 77-80).
__global__ void camera_kernel(CameraParams c, long long first, int n, float4* rays, int* pixel,
                              unsigned long long* rng_out, float4* thr, int* bounces, int* sample_out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int i = (int)(first + j);
    const int pixel_idx = i / c.spp;
    const int y = pixel_idx / c.tile_w;
    const int x = pixel_idx % c.tile_w;
    Rng rng = seed_sample(c.seed_base, i, pixel_idx);
    const float sx = static_cast<float>(x + c.tile_left) + rng.next_float();
    const float sy = static_cast<float>(y + c.tile_top) + rng.next_float();
    const float* m = c.r2w;
    const float t0 = m[0] * sy + m[1] * sx + m[2] * 0.0f + m[3] * 1.0f;
    const float t1 = m[4] * sy + m[5] * sx + m[6] * 0.0f + m[7] * 1.0f;
    const float t2 = m[8] * sy + m[9] * sx + m[10] * 0.0f + m[11] * 1.0f;
    const float t3 = m[12] * sy + m[13] * sx + m[14] * 0.0f + m[15] * 1.0f;
    const V3 w(t0 / t3, t1 / t3, t2 / t3);
    const V3 d = normalize(w - V3(c.pos[0], c.pos[1], c.pos[2]));
    rays[2 * j + 0] = make_float4(c.pos[0], c.pos[1], c.pos[2], 0.0f);
    rays[2 * j + 1] = make_float4(d.x, d.y, d.z, FLT_MAX);
    pixel[j] = (y + c.tile_top) * c.full_w + (x + c.tile_left);
    rng_out[j] = rng.state;
    if (thr) thr[j] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    if (bounces) bounces[j] = 0;
    if (sample_out) sample_out[j] = i % c.spp;
}

struct ShadeParams {
    ShadingScene s;
    int n;                   // paths in the input queue
    int max_path_len;
    int rr_start;            // Russian roulette from this bounce on (0: the reference's behaviour)
    const float4* rays; const int4* hits; const int* pixel; const unsigned long long* rng;
    const float4* thr; const int* bounces;
    float4* o_rays; int* o_pixel; unsigned long long* o_rng; float4* o_thr; int* o_bounces;
    float4* s_rays; int* s_pixel; float4* s_contrib;
    int* counts;             // [0] out paths, [1] shadow rays
    float* image;
};

__device__ __forceinline__ void add_image(float* img, int pixel, V3 c) {
    atomicAdd(img + 3 * pixel + 0, c.x);
    atomicAdd(img + 3 * pixel + 1, c.y);
    atomicAdd(img + 3 * pixel + 2, c.z);
}

// PathTracer::process_primary_rays for one wavefront (pt.cpp:82-160, 17-80).
__global__ void __launch_bounds__(128) pt_shade_kernel(ShadeParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool alive = false, shadow = false;
    float4 o_org = make_float4(0, 0, 0, 0), o_dir = o_org, s_org = o_org, s_dir = o_org;
    V3 s_c(0.0f);
    Rng rng{0};
    V3 thr(0.0f);
    float last_pdf = 0.0f;
    int bounces = 0, pixel = 0;
    bool last_spec = false;
    if (i < p.n) {
        const ShadingScene& s = p.s;
        const float4 ro = p.rays[2 * i], rd = p.rays[2 * i + 1];
        const int4 h = p.hits[i];
        pixel = p.pixel[i];
        rng.state = p.rng[i];
        const float4 t4 = p.thr[i];
        thr = V3(t4.x, t4.y, t4.z);
        last_pdf = t4.w;
        const int bf = p.bounces[i];
        bounces = bf & 0x7fffffff;
        last_spec = (bf >> 31) & 1;
        if (h.x < 0) {
            // Miss: environment with MIS (pt.cpp:95-116).
            if (s.has_env) {
                const V3 out_dir = normalize(V3(rd.x, rd.y, rd.z));
                float pdf_direct_w;
                const V3 li = env_radiance(s, out_dir, &pdf_direct_w);
                const float pdf_lightpick = 1.0f / (float)s.light_count;
                const float pdf_di = pdf_direct_w * pdf_lightpick;
                const float pdf_hit = last_pdf;
                const float mis = (bounces == 0 || last_spec) ? 1.0f : (pdf_hit / (pdf_hit + pdf_di));
                add_image(p.image, pixel, thr * li * mis);
            }
        } else {
            const float tmax = __int_as_float(h.z);
            const Isect is = calculate_intersection(s, h.x, h.y, tmax, __int_as_float(h.w), V3(ro.x, ro.y, ro.z),
                                                    V3(rd.x, rd.y, rd.z));
            const float offset = 1e-3f * tmax;
            const Material& mat = s.materials[is.mat];
            if (mat.kind == kEmissive) {
                // Emitter hit (pt.cpp:133-151), AreaEmitter::radiance (light.h:22-43).
                float pdf_direct_a = 1.0f;
                V3 li(0.0f);
                if (dot(is.geom_normal, is.out_dir) > 0.0f) {
                    pdf_direct_a = 1.0f / mat.area;
                    li = V3(mat.emission[0], mat.emission[1], mat.emission[2]);
                }
                float pdf_di = pdf_direct_a / (float)s.light_count;
                const float d_sqr = tmax * tmax;
                const float cos_light = dot(is.normal, is.out_dir);
                pdf_di *= d_sqr / cos_light;
                const float mis = (bounces == 0 || last_spec) ? 1.0f : last_pdf / (last_pdf + pdf_di);
                add_image(p.image, pixel, thr * li * mis);
            } else {
                const Bsdf bsdf{&mat, is.normal, is.u_tangent, is.v_tangent, is.geom_normal};
                // Next-event estimation (pt.cpp:17-44).
                const int l = rng.next_int(0, s.light_count);
                const float pdf_lightpick = 1.0f / (float)s.light_count;
                const DirectSample ds = (s.has_env && l == 0) ? env_light_sample(s, rng)
                                                              : tri_light_sample(s.lights[l - s.has_env], is.pos, rng);
                const V3 bsdf_value = bsdf.eval(is.out_dir, ds.dir);
                const float pdf_hit = bsdf.pdf(is.out_dir, ds.dir);
                const float pdf_di = pdf_lightpick * ds.pdf_direct_w;
                const float mis = ds.delta ? 1.0f : pdf_di / (pdf_di + pdf_hit);
                if (!(pdf_hit == 0.0f || pdf_di == 0.0f)) {
                    s_c = thr * bsdf_value * fabsf(dot(is.normal, ds.dir)) * ds.radiance * mis / pdf_lightpick;
                    const float off = 1e-3f * (ds.distance == FLT_MAX ? 1.0f : ds.distance);
                    s_org = make_float4(is.pos.x, is.pos.y, is.pos.z, off);
                    s_dir = make_float4(ds.dir.x, ds.dir.y, ds.dir.z, ds.distance - off);
                    shadow = true;
                }
                // Continuation (pt.cpp:46-80).
                if (bounces + 1 < p.max_path_len) {
                    float rr_pdf = 1.0f;
                    bool go = true;
                    if (bounces >= p.rr_start) go = russian_roulette(thr, rng.next_float(), rr_pdf);
                    if (go) {
                        V3 dir;
                        int flags;
                        float pdf;
                        const V3 value = bsdf.sample(is.out_dir, dir, rng, flags, pdf);
                        if (!(pdf == 0.0f || flags == kNone || is_black(value))) {
                            const float cos_term = fabsf(dot(is.normal, dir));
                            thr = thr * (value * cos_term / (pdf * rr_pdf));
                            bounces += 1;
                            last_spec = (flags & kSpecular) != 0;
                            last_pdf = pdf;
                            o_org = make_float4(is.pos.x, is.pos.y, is.pos.z, offset);
                            o_dir = make_float4(dir.x, dir.y, dir.z, FLT_MAX);
                            alive = true;
                        }
                    }
                }
            }
        }
    }
    const int slot = warp_append(p.counts + 0, alive);
    if (alive) {
        p.o_rays[2 * slot] = o_org;
        p.o_rays[2 * slot + 1] = o_dir;
        p.o_pixel[slot] = pixel;
        p.o_rng[slot] = rng.state;
        p.o_thr[slot] = make_float4(thr.x, thr.y, thr.z, last_pdf);
        p.o_bounces[slot] = bounces | (last_spec ? (int)0x80000000 : 0);
    }
    const int sslot = warp_append(p.counts + 1, shadow);
    if (shadow) {
        p.s_rays[2 * sslot] = s_org;
        p.s_rays[2 * sslot + 1] = s_dir;
        p.s_pixel[sslot] = pixel;
        p.s_contrib[sslot] = make_float4(s_c.x, s_c.y, s_c.z, 0.0f);
    }
}

// Integrator::process_shadow_rays (integrator.h:49-63): unoccluded shadow rays add their
// contribution to the image.
__global__ void shadow_accumulate_kernel(int n, const int4* hits, const int* pixel, const float4* contrib,
                                         float* image) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (hits[i].x >= 0) return;
    const float4 c = contrib[i];
    add_image(image, pixel[i], V3(c.x, c.y, c.z));
}

template <typename T>
bool dev_alloc(T** p, size_t n, std::vector<void*>* track = nullptr) {
    *p = nullptr;
    if (!ok(cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(n, 1)), "cudaMalloc")) return false;
    if (track) track->push_back(*p);
    return true;
}

void free_ctx_buffers(imbart_pt_context* c) {
    for (int k = 0; k < 2; ++k) {
        cudaFree(c->rays[k]); cudaFree(c->pixel[k]); cudaFree(c->rng[k]); cudaFree(c->thr[k]); cudaFree(c->bounces[k]);
        c->rays[k] = nullptr; c->pixel[k] = nullptr; c->rng[k] = nullptr; c->thr[k] = nullptr; c->bounces[k] = nullptr;
    }
    cudaFree(c->hits); cudaFree(c->srays); cudaFree(c->shits); cudaFree(c->spixel); cudaFree(c->scontrib);
    c->hits = nullptr; c->srays = nullptr; c->shits = nullptr; c->spixel = nullptr; c->scontrib = nullptr;
    c->cap = 0;
}

bool ensure_capacity(imbart_pt_context* c, long long n) {
    if (c->cap >= n) return true;
    free_ctx_buffers(c);
    bool good = true;
    for (int k = 0; k < 2 && good; ++k)
        good = dev_alloc(&c->rays[k], 2 * n) && dev_alloc(&c->pixel[k], n) && dev_alloc(&c->rng[k], n) &&
               dev_alloc(&c->thr[k], n) && dev_alloc(&c->bounces[k], n);
    good = good && dev_alloc(&c->hits, n) && dev_alloc(&c->srays, 2 * n) && dev_alloc(&c->shits, n) &&
           dev_alloc(&c->spixel, n) && dev_alloc(&c->scontrib, n);
    if (!good) { free_ctx_buffers(c); return false; }
    c->cap = n;
    return true;
}

}  // namespace
}  // namespace imbart

using namespace imbart;

extern "C" {

imbart_shading* imbart_shading_create(int device, const float* vertices, int n_vertices, const float* normals,
                                      const float* texcoords, const int* tris, const float* geom_normals, int n_tris,
                                      const float* inst_inv, int n_inst, const int* mat_kind,
                                      const float* mat_params, int n_mats, const float* tri_lights,
                                      int n_tri_lights, const float* env_color, const float* bsphere) {
    if (!vertices || !normals || !texcoords || !tris || !geom_normals || !inst_inv || !mat_kind || !mat_params ||
        n_vertices <= 0 || n_tris <= 0 || n_inst <= 0 || n_mats <= 0 || n_tri_lights < 0 ||
        (n_tri_lights > 0 && !tri_lights) || (n_tri_lights == 0 && !env_color)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_shading_create: invalid argument");
        return nullptr;
    }
    int prev = 0;
    cudaGetDevice(&prev);
    if (!ok(cudaSetDevice(device), "cudaSetDevice")) return nullptr;
    imbart_shading* h = new imbart_shading;
    h->device = device;
    ShadingScene& s = h->s;
    std::vector<Material> mats(n_mats);
    for (int m = 0; m < n_mats; ++m) {
        const float* q = mat_params + 16 * m;
        Material& M = mats[m];
        M.kind = mat_kind[m];
        for (int k = 0; k < 3; ++k) { M.color[k] = q[k]; M.spec[k] = q[3 + k]; M.emission[k] = q[9 + k]; }
        M.exponent = q[6]; M.eta = q[7]; M.kappa = q[8]; M.area = 1.0f;
    }
    std::vector<TriLight> lights(std::max(n_tri_lights, 1));
    for (int l = 0; l < n_tri_lights; ++l) {
        const float* q = tri_lights + 12 * l;
        TriLight& L = lights[l];
        std::memset(&L, 0, sizeof(L));
        for (int v = 0; v < 3; ++v) for (int a = 0; a < 3; ++a) L.v[v][a] = q[3 * v + a];
        for (int a = 0; a < 3; ++a) L.intensity[a] = q[9 + a];
    }
    auto upl = [&](const void* src, size_t bytes) -> void* {
        void* d = nullptr;
        if (!ok(cudaMalloc(&d, std::max<size_t>(bytes, 4)), "cudaMalloc")) return nullptr;
        h->allocations.push_back(d);
        if (!ok(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy")) return nullptr;
        return d;
    };
    s.vertices = (const float*)upl(vertices, sizeof(float) * 3 * (size_t)n_vertices);
    s.normals = (const float*)upl(normals, sizeof(float) * 3 * (size_t)n_vertices);
    s.texcoords = (const float*)upl(texcoords, sizeof(float) * 2 * (size_t)n_vertices);
    s.tris = (const int4*)upl(tris, sizeof(int4) * (size_t)n_tris);
    s.geom_normals = (const float*)upl(geom_normals, sizeof(float) * 3 * (size_t)n_tris);
    s.inst_inv = (const float*)upl(inst_inv, sizeof(float) * 12 * (size_t)n_inst);
    Material* dmats = (Material*)upl(mats.data(), sizeof(Material) * mats.size());
    TriLight* dlights = (TriLight*)upl(lights.data(), sizeof(TriLight) * lights.size());
    s.materials = dmats;
    s.lights = dlights;
    s.n_tri_lights = n_tri_lights;
    s.has_env = env_color ? 1 : 0;
    s.light_count = n_tri_lights + s.has_env;
    for (int k = 0; k < 3; ++k) s.env_color[k] = env_color ? env_color[k] : 0.0f;
    for (int k = 0; k < 5; ++k) s.bsphere[k] = bsphere ? bsphere[k] : 0.0f;
    const bool good = s.vertices && s.normals && s.texcoords && s.tris && s.geom_normals && s.inst_inv && dmats && dlights;
    if (good) {
        if (n_tri_lights > 0) setup_lights_kernel<<<(n_tri_lights + 127) / 128, 128>>>(dlights, n_tri_lights);
        emitter_area_kernel<<<(n_tris + 127) / 128, 128>>>(s.vertices, s.tris, n_tris, dmats);
    }
    const bool synced = good && ok(cudaDeviceSynchronize(), "shading setup");
    cudaSetDevice(prev);
    if (!synced) {
        for (void* a : h->allocations) cudaFree(a);
        delete h;
        return nullptr;
    }
    return h;
}

void imbart_shading_destroy(imbart_shading* h) {
    if (!h) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    for (void* a : h->allocations) cudaFree(a);
    cudaSetDevice(prev);
    delete h;
}

imbart_pt_context* imbart_pt_create(int device) {
    imbart_pt_context* c = new imbart_pt_context;
    c->device = device;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    const bool good = ok(cudaMalloc((void**)&c->counts, sizeof(int) * 4), "cudaMalloc") &&
                      ok(cudaMallocHost((void**)&c->host_counts, sizeof(int) * 4), "cudaMallocHost");
    cudaSetDevice(prev);
    if (!good) { delete c; return nullptr; }
    return c;
}

void imbart_pt_destroy(imbart_pt_context* c) {
    if (!c) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    free_ctx_buffers(c);
    cudaFree(c->counts);
    cudaFreeHost(c->host_counts);
    cudaFree(c->work);
    if (c->ev[0]) { cudaEventDestroy(c->ev[0]); cudaEventDestroy(c->ev[1]); }
    cudaSetDevice(prev);
    delete c;
}

int imbart_camera_rays(const float* raster_to_world, const float* cam_pos, int width, int height, int spp,
                       unsigned long long seed_base, long long first, int count, imbart_ray* rays, int* pixel_ids,
                       int* sample_ids, unsigned long long* rng_states, void* stream) {
    if (!raster_to_world || !cam_pos || width <= 0 || height <= 0 || spp <= 0 || count < 0 || first < 0 ||
        (count > 0 && (!rays || !pixel_ids || !rng_states))) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_camera_rays: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (count == 0) return 0;
    CameraParams c;
    std::memcpy(c.r2w, raster_to_world, sizeof(c.r2w));
    std::memcpy(c.pos, cam_pos, sizeof(c.pos));
    c.width = width; c.height = height; c.spp = spp;
    c.tile_left = 0; c.tile_top = 0; c.tile_w = width; c.full_w = width;
    c.seed_base = seed_base;
    camera_kernel<<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        c, first, count, reinterpret_cast<float4*>(rays), pixel_ids, rng_states, nullptr, nullptr, sample_ids);
    note_launches(1);
    return ok(cudaGetLastError(), "camera kernel") ? 0 : IMBART_ERR_CUDA;
}

int imbart_pt_render(imbart_pt_context* ctx, const imbart_scene* scene, const imbart_shading* sh,
                     const float* raster_to_world, const float* cam_pos, int width, int height, int spp,
                     int max_path_len, int rr_start, unsigned long long seed_base, float* image,
                     long long max_paths_in_flight, long long* stats, void* stream) {
    if (!ctx || !scene || !sh || !raster_to_world || !cam_pos || !image || width <= 0 || height <= 0 || spp <= 0 ||
        max_path_len < 1) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_pt_render: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const long long total = (long long)width * height * spp;
    long long chunk = max_paths_in_flight > 0 ? max_paths_in_flight : (16ll << 20);
    chunk = std::min(chunk, total);
    chunk = std::min(chunk, (long long)(1 << 30));
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(ctx->device);
    if (!ensure_capacity(ctx, chunk)) { cudaSetDevice(prev); return IMBART_ERR_OUT_OF_MEMORY; }
    CameraParams c;
    std::memcpy(c.r2w, raster_to_world, sizeof(c.r2w));
    std::memcpy(c.pos, cam_pos, sizeof(c.pos));
    c.width = width; c.height = height; c.spp = spp;
    c.tile_left = 0; c.tile_top = 0; c.tile_w = width; c.full_w = width;
    c.seed_base = seed_base;
    long long n_closest = 0, n_shadow = 0, n_waves = 0;
    int rc = 0;
    imbart_pt_profile* prof = ctx->profile;
    if (prof) {
        if (!ctx->ev[0]) { cudaEventCreate(&ctx->ev[0]); cudaEventCreate(&ctx->ev[1]); }
        if (prof->work && !ctx->work && !ok(cudaMalloc((void**)&ctx->work, sizeof(unsigned long long) * 6), "cudaMalloc")) {
            cudaSetDevice(prev);
            return IMBART_ERR_OUT_OF_MEMORY;
        }
        if (prof->work) cudaMemsetAsync(ctx->work, 0, sizeof(unsigned long long) * 6, st);
    }
    // One traversal launch, timed / counted when profiling.
    auto trace = [&](const void* rays, void* hits, int count, int flags) -> int {
        const bool any = flags == IMBART_TRACE_ANY;
        unsigned long long* work = (prof && prof->work) ? ctx->work + (any ? 3 : 0) : nullptr;
        if (prof && prof->events) cudaEventRecord(ctx->ev[0], st);
        const int r = launch_trace_internal(scene, rays, hits, nullptr, count, flags, st, work);
        if (prof && prof->events) {
            cudaEventRecord(ctx->ev[1], st);
            cudaEventSynchronize(ctx->ev[1]);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
            (any ? prof->shadow_ms : prof->closest_ms) += ms;
        }
        if (prof) {
            (any ? prof->shadow_launches : prof->closest_launches) += 1;
            (any ? prof->shadow_rays : prof->closest_rays) += count;
        }
        return r;
    };
    for (long long first = 0; first < total && !rc; first += chunk) {
        int n = (int)std::min(chunk, total - first);
        int cur = 0;
        camera_kernel<<<(n + 127) / 128, 128, 0, st>>>(c, first, n, ctx->rays[cur], ctx->pixel[cur], ctx->rng[cur],
                                                       ctx->thr[cur], ctx->bounces[cur], nullptr);
        note_launches(1);
        while (n > 0) {
            rc = trace(ctx->rays[cur], ctx->hits, n, IMBART_TRACE_CLOSEST);
            if (rc) break;
            n_closest += n;
            ++n_waves;
            if (!ok(cudaMemsetAsync(ctx->counts, 0, sizeof(int) * 2, st), "cudaMemsetAsync")) { rc = IMBART_ERR_CUDA; break; }
            ShadeParams p;
            p.s = sh->s;
            p.n = n;
            p.max_path_len = max_path_len;
            p.rr_start = rr_start;
            p.rays = ctx->rays[cur]; p.hits = ctx->hits; p.pixel = ctx->pixel[cur]; p.rng = ctx->rng[cur];
            p.thr = ctx->thr[cur]; p.bounces = ctx->bounces[cur];
            const int nxt = 1 - cur;
            p.o_rays = ctx->rays[nxt]; p.o_pixel = ctx->pixel[nxt]; p.o_rng = ctx->rng[nxt];
            p.o_thr = ctx->thr[nxt]; p.o_bounces = ctx->bounces[nxt];
            p.s_rays = ctx->srays; p.s_pixel = ctx->spixel; p.s_contrib = ctx->scontrib;
            p.counts = ctx->counts;
            p.image = image;
            pt_shade_kernel<<<(n + 127) / 128, 128, 0, st>>>(p);
            note_launches(1);
            if (!ok(cudaGetLastError(), "shade kernel") ||
                !ok(cudaMemcpyAsync(ctx->host_counts, ctx->counts, sizeof(int) * 2, cudaMemcpyDeviceToHost, st),
                    "cudaMemcpyAsync") ||
                !ok(cudaStreamSynchronize(st), "cudaStreamSynchronize")) {
                rc = IMBART_ERR_CUDA;
                break;
            }
            const int n_next = ctx->host_counts[0];
            const int n_sh = ctx->host_counts[1];
            if (n_sh > 0) {
                rc = trace(ctx->srays, ctx->shits, n_sh, IMBART_TRACE_ANY);
                if (rc) break;
                n_shadow += n_sh;
                shadow_accumulate_kernel<<<(n_sh + 127) / 128, 128, 0, st>>>(n_sh, ctx->shits, ctx->spixel,
                                                                             ctx->scontrib, image);
                note_launches(1);
                if (!ok(cudaGetLastError(), "shadow kernel")) { rc = IMBART_ERR_CUDA; break; }
            }
            n = n_next;
            cur = nxt;
        }
    }
    if (stats) { stats[0] = n_closest; stats[1] = n_shadow; stats[2] = n_waves; }
    if (!rc && prof && prof->work) {
        unsigned long long w[6];
        if (ok(cudaMemcpyAsync(w, ctx->work, sizeof(w), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync") &&
            ok(cudaStreamSynchronize(st), "cudaStreamSynchronize")) {
            for (int k = 0; k < 3; ++k) { prof->closest_work[k] += w[k]; prof->shadow_work[k] += w[3 + k]; }
        } else {
            rc = IMBART_ERR_CUDA;
        }
    }
    cudaSetDevice(prev);
    return rc;
}

int imbart_pt_set_profile(imbart_pt_context* ctx, imbart_pt_profile* profile) {
    if (!ctx) { set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_pt_set_profile"); return IMBART_ERR_INVALID_ARGUMENT; }
    ctx->profile = profile;
    return 0;
}

}  // extern "C"
