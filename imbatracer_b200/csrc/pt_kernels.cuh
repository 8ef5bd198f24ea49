// Path-tracing kernels of the wavefront loop, shared by the single-frame renderer
// (wavefront.cu) and the request server (server.cu). Both translation units are compiled with
// -fmad=false so that the shading arithmetic rounds like the reference's.
//
// Every kernel comes in two forms. The single-request form reads the scene, the image and
// the path parameters from its launch parameters. The merged form (kMulti) serves a queue that
// mixes paths of many render requests over several scenes: each path carries the slot of its
// request, whose table entry (ReqDev) names the scene's shading data, its image and its path
// parameters, and the root of its scene in the shared node pool for the traversal kernel.
// A path's arithmetic is the same in both forms, so a request renders the same image alone
// and in a mix (up to the order of the float additions into its image).
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "imbart_internal.h"
#include "rng.cuh"
#include "shade.cuh"

// Shading data of one scene on one GPU (imbart_shading_create).
struct imbart_shading {
    int device = 0;
    imbart::sh::ShadingScene s{};
    std::vector<void*> allocations;
    unsigned kind_mask = 0;     // bit k: some material has kind k (grouping pays only for several)
};

namespace imbart {
namespace pt {
namespace {   // every including translation unit gets its own copy of the kernels

using imbart::Rng;
using namespace imbart::sh;

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

// Light frames and emitter areas, computed on the device with the reference's formulas
// (TriangleLight ctor, light.h:99-108: normal, area, frame; DirectionalLight and SpotLight
// ctors, :195-199 and :294-302: frame of the direction; Tri::area, tri.h:21).
__global__ void setup_lights_kernel(LightSrc* lights, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    LightSrc& L = lights[i];
    if (L.kind == kLightDirectional || L.kind == kLightSpot) {
        V3 t, b;
        local_coordinates(V3(L.normal[0], L.normal[1], L.normal[2]), t, b);
        L.tangent[0] = t.x; L.tangent[1] = t.y; L.tangent[2] = t.z;
        L.binormal[0] = b.x; L.binormal[1] = b.y; L.binormal[2] = b.z;
        return;
    }
    if (L.kind != kLightTri) return;
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

// Host-side decoding of the material / light arrays of imbart_shading_create(_ex). With
// textures, params[12] / params[13] are the diffuse-texture / bump-map indices (< 0: none).
// Bit k set when some material has kind k. Emitters are left out: a path that hits one
// ends after a few instructions, so they add no divergence worth grouping for.
inline unsigned material_kind_mask(const std::vector<Material>& mats) {
    unsigned m = 0;
    for (const Material& x : mats)
        if (x.kind != kEmissive) m |= 1u << (x.kind & 7);
    return m;
}

inline std::vector<Material> decode_materials(const int* kind, const float* params, int n, bool textured) {
    std::vector<Material> mats(n);
    for (int m = 0; m < n; ++m) {
        const float* q = params + 16 * m;
        Material& M = mats[m];
        M.kind = kind[m];
        for (int k = 0; k < 3; ++k) { M.color[k] = q[k]; M.spec[k] = q[3 + k]; M.emission[k] = q[9 + k]; }
        M.exponent = q[6]; M.eta = q[7]; M.kappa = q[8]; M.area = 1.0f;
        M.tex = textured && q[12] >= 0.0f ? (int)q[12] : -1;
        M.bump = textured && q[13] >= 0.0f ? (int)q[13] : -1;
    }
    return mats;
}

// Lights of 12 floats each; kinds (NULL: all triangles): triangle p0, p1, p2, intensity;
// directional: direction (travel), 6 unused, intensity; point: position, 6 unused, intensity;
// spot: position, axis, half-angle in radians, 2 unused, intensity.
inline std::vector<LightSrc> decode_lights(const int* kinds, const float* params, int n) {
    std::vector<LightSrc> lights(n > 1 ? n : 1);
    for (int l = 0; l < n; ++l) {
        const float* q = params + 12 * l;
        LightSrc& L = lights[l];
        std::memset(&L, 0, sizeof(L));
        L.kind = kinds ? kinds[l] : kLightTri;
        for (int a = 0; a < 3; ++a) L.intensity[a] = q[9 + a];
        if (L.kind == kLightTri) {
            for (int v = 0; v < 3; ++v) for (int a = 0; a < 3; ++a) L.v[v][a] = q[3 * v + a];
        } else if (L.kind == kLightDirectional) {
            for (int a = 0; a < 3; ++a) L.normal[a] = q[a];
        } else {
            for (int a = 0; a < 3; ++a) L.v[0][a] = q[a];
            if (L.kind == kLightSpot) {
                for (int a = 0; a < 3; ++a) L.normal[a] = q[3 + a];
                L.cos_angle = std::cos(q[6]);   // SpotLight ctor: cosf(angle) (light.h:298)
            }
        }
    }
    return lights;
}

inline bool valid_light_kinds(const int* kinds, int n) {
    for (int l = 0; kinds && l < n; ++l)
        if (kinds[l] < kLightTri || kinds[l] > kLightSpot) return false;
    return true;
}

struct CameraParams {
    float r2w[16];
    float pos[3];
    int width, height, spp;
    int tile_left, tile_top, tile_w, full_w;
    unsigned long long seed_base;
};

// One render request of a merged queue (device table entry, indexed by request slot).
struct ReqDev {
    float r2w[16];
    float pos[3];
    int width, height, spp;
    int max_path_len, rr_start;
    int scene_slot;           // entry of the shading-scene table
    int root;                 // top-level root of the scene in the node pool
    unsigned long long seed_base;
    float* image;             // width * height * 3 floats
};

// A run of consecutive camera samples of one request appended to a merged queue.
struct GenChunk {
    long long first_sample;   // sample index within the request
    int req;                  // request slot
    int count;
    int out_begin;            // first queue position (relative to the append offset)
    int pad;
};

// PixelRayGen::fill_queue + the path tracer's sample function (pt.cpp:168-177) +
// PerspectiveCamera::generate_ray (camera.h:57-65, 77-80) for global sample index i.
__device__ __forceinline__ void camera_sample(const float* m, const float* pos, int spp, int tile_left, int tile_top,
                                              int tile_w, int full_w, unsigned long long seed_base, int i,
                                              float4* ray_out, int* pixel_out, unsigned long long* rng_out) {
    const int pixel_idx = i / spp;
    const int y = pixel_idx / tile_w;
    const int x = pixel_idx % tile_w;
    Rng rng = seed_sample(seed_base, i, pixel_idx);
    const float sx = static_cast<float>(x + tile_left) + rng.next_float();
    const float sy = static_cast<float>(y + tile_top) + rng.next_float();
    const float t0 = m[0] * sy + m[1] * sx + m[2] * 0.0f + m[3] * 1.0f;
    const float t1 = m[4] * sy + m[5] * sx + m[6] * 0.0f + m[7] * 1.0f;
    const float t2 = m[8] * sy + m[9] * sx + m[10] * 0.0f + m[11] * 1.0f;
    const float t3 = m[12] * sy + m[13] * sx + m[14] * 0.0f + m[15] * 1.0f;
    const V3 w(t0 / t3, t1 / t3, t2 / t3);
    const V3 d = normalize(w - V3(pos[0], pos[1], pos[2]));
    ray_out[0] = make_float4(pos[0], pos[1], pos[2], 0.0f);
    ray_out[1] = make_float4(d.x, d.y, d.z, FLT_MAX);
    *pixel_out = (y + tile_top) * full_w + (x + tile_left);
    *rng_out = rng.state;
}

__global__ void camera_kernel(CameraParams c, long long first, int n, float4* rays, int* pixel,
                              unsigned long long* rng_out, float4* thr, int* bounces, int* sample_out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int i = (int)(first + j);
    camera_sample(c.r2w, c.pos, c.spp, c.tile_left, c.tile_top, c.tile_w, c.full_w, c.seed_base, i, rays + 2 * j,
                  pixel + j, rng_out + j);
    if (thr) thr[j] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    if (bounces) bounces[j] = 0;
    if (sample_out) sample_out[j] = i % c.spp;
}

// camera_kernel with the camera and the sample range read on the device (`*cam`, `*first`,
// `*n`: the state of a frame captured as a CUDA graph), walked with a grid stride.
__global__ void camera_range_kernel(const CameraParams* cam, const long long* first, const int* n_ptr, float4* rays,
                                    int* pixel, unsigned long long* rng_out, float4* thr, int* bounces) {
    const CameraParams& c = *cam;
    const long long f = *first;
    const int n = *n_ptr;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        camera_sample(c.r2w, c.pos, c.spp, c.tile_left, c.tile_top, c.tile_w, c.full_w, c.seed_base, (int)(f + j),
                      rays + 2 * j, pixel + j, rng_out + j);
        thr[j] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        bounces[j] = 0;
    }
}

// Camera samples of several requests, appended at queue position `offset`: thread j finds its
// chunk by binary search over the chunks' out_begin.
__global__ void camera_multi_kernel(const ReqDev* reqs, const GenChunk* chunks, int n_chunks, int n, int offset,
                                    float4* rays, int* pixel, unsigned long long* rng_out, float4* thr, int* bounces,
                                    int* req_out, int* root_out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int lo = 0, hi = n_chunks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (chunks[mid].out_begin <= j) lo = mid;
        else hi = mid - 1;
    }
    const GenChunk ch = chunks[lo];
    const ReqDev& R = reqs[ch.req];
    const int i = (int)(ch.first_sample + (j - ch.out_begin));
    const int q = offset + j;
    camera_sample(R.r2w, R.pos, R.spp, 0, 0, R.width, R.width, R.seed_base, i, rays + 2 * q, pixel + q, rng_out + q);
    thr[q] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    bounces[q] = 0;
    req_out[q] = ch.req;
    root_out[q] = R.root;
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
    // merged queues only
    const ReqDev* reqs; const ShadingScene* scenes;
    const int* req; const int* root;
    int* o_req; int* o_root; int* s_req; int* s_root;
    int* terminated;         // per request slot: paths that ended
    const int* perm;         // optional: shade path perm[i] in thread i (paths grouped by material)
    const int* n_ptr;        // optional: queue size read on the device (`n` is then its bound)
};

__device__ __forceinline__ void add_image(float* img, int pixel, V3 c) {
    atomicAdd(img + 3 * pixel + 0, c.x);
    atomicAdd(img + 3 * pixel + 1, c.y);
    atomicAdd(img + 3 * pixel + 2, c.z);
}

// The state a shaded path leaves behind: an optional continuation and an optional shadow ray.
struct ShadeOut {
    bool alive = false, shadow = false;
    float4 o_org, o_dir, s_org, s_dir;
    V3 s_c{0.0f};
    V3 thr{0.0f};
    float last_pdf = 0.0f;
    int bounces = 0;
    bool last_spec = false;
    Rng rng{0};
};

// PathTracer::process_primary_rays for one path (pt.cpp:82-160, 17-80).
__device__ __forceinline__ void shade_path(const ShadingScene& s, int max_path_len, int rr_start, float* image,
                                           float4 ro, float4 rd, int4 h, int pixel, unsigned long long rng_state,
                                           float4 t4, int bf, ShadeOut& o) {
    o.rng.state = rng_state;
    V3 thr(t4.x, t4.y, t4.z);
    float last_pdf = t4.w;
    int bounces = bf & 0x7fffffff;
    bool last_spec = (bf >> 31) & 1;
    Rng& rng = o.rng;
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
            add_image(image, pixel, thr * li * mis);
        }
        return;
    }
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
        add_image(image, pixel, thr * li * mis);
        return;
    }
    const Bsdf bsdf = surface_bsdf(s, mat, is.normal, is.u_tangent, is.v_tangent, is.geom_normal, is.uv[0], is.uv[1],
                                   false);
    // Next-event estimation (pt.cpp:17-44).
    const int l = rng.next_int(0, s.light_count);
    const float pdf_lightpick = 1.0f / (float)s.light_count;
    const DirectSample ds = light_sample_direct(s, l, is.pos, rng);
    const V3 bsdf_value = bsdf.eval(is.out_dir, ds.dir);
    const float pdf_hit = bsdf.pdf(is.out_dir, ds.dir);
    const float pdf_di = pdf_lightpick * ds.pdf_direct_w;
    const float mis = ds.delta ? 1.0f : pdf_di / (pdf_di + pdf_hit);
    if (!(pdf_hit == 0.0f || pdf_di == 0.0f)) {
        o.s_c = thr * bsdf_value * fabsf(dot(is.normal, ds.dir)) * ds.radiance * mis / pdf_lightpick;
        const float off = 1e-3f * (ds.distance == FLT_MAX ? 1.0f : ds.distance);
        o.s_org = make_float4(is.pos.x, is.pos.y, is.pos.z, off);
        o.s_dir = make_float4(ds.dir.x, ds.dir.y, ds.dir.z, ds.distance - off);
        o.shadow = true;
    }
    // Continuation (pt.cpp:46-80).
    if (bounces + 1 < max_path_len) {
        float rr_pdf = 1.0f;
        bool go = true;
        if (bounces >= rr_start) go = russian_roulette(thr, rng.next_float(), rr_pdf);
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
                o.o_org = make_float4(is.pos.x, is.pos.y, is.pos.z, offset);
                o.o_dir = make_float4(dir.x, dir.y, dir.z, FLT_MAX);
                o.thr = thr;
                o.last_pdf = last_pdf;
                o.bounces = bounces;
                o.last_spec = last_spec;
                o.alive = true;
            }
        }
    }
}

// RayQueue::sort_by_material (ray_queue.h:211-244) for the device queue: the paths of a
// wavefront grouped by what shading will run for them (material kind of the hit, or a miss),
// so that the warps of the shading kernel follow one code path each. The reference sorts the
// queue itself with a two-pass counting sort; here a permutation is built and the shading
// kernel reads through it. The sort is a stable counting sort over tiles of kGroupTile
// entries: per-tile key counts, one scan (key-major, tile-minor), then each tile places its
// entries in index order. Stable, so paths that were neighbours in the queue (neighbouring
// samples) stay neighbours within their group, and the permutation is deterministic. Results
// per path do not depend on the order.
constexpr int kShadeKeys = 8;   // material kinds 0..5, 6: miss (7: a finished light-path slot)
constexpr int kGroupTile = 8192;

inline int group_tiles(long long n) { return (int)((n + kGroupTile - 1) / kGroupTile); }

__device__ __forceinline__ int shade_key(const ShadingScene& s, int4 h) {
    if (h.x < 0) return 6;
    return s.materials[s.tris[h.x].w].kind & 7;
}

// The grouping kernels take the queue size from `n`, or with `n_ptr` set read it on the
// device (`n` then bounds it), so a launch sized for the bound can sit in a CUDA graph.
__device__ __forceinline__ int queue_size(const int* n_ptr, int n) { return n_ptr ? min(*n_ptr, n) : n; }

__global__ void __launch_bounds__(256) shade_key_kernel(ShadingScene s, const int4* __restrict__ hits, int n,
                                                        const int* n_ptr, uint8_t* keys) {
    n = queue_size(n_ptr, n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        keys[i] = (uint8_t)shade_key(s, hits[i]);
}

// The same keys for a merged wavefront: each path's hit is looked up in its request's scene.
__global__ void __launch_bounds__(256) shade_key_multi_kernel(const ReqDev* __restrict__ reqs,
                                                              const ShadingScene* __restrict__ scenes,
                                                              const int* __restrict__ req, const int4* __restrict__ hits,
                                                              int n, const int* n_ptr, uint8_t* keys) {
    n = queue_size(n_ptr, n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        keys[i] = (uint8_t)shade_key(scenes[reqs[req[i]].scene_slot], hits[i]);
}

// Keys of tile blockIdx.x (8 rounds of 256 entries): tile_counts[8 * tile + k] = entries with
// key k.
__global__ void __launch_bounds__(256) group_count_kernel(const uint8_t* __restrict__ keys, int n, const int* n_ptr,
                                                          int* __restrict__ tile_counts) {
    n = queue_size(n_ptr, n);
    const int base = blockIdx.x * kGroupTile;
    if (base >= n) return;
    __shared__ int warp_counts[8][kShadeKeys];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int mine = 0;   // lane k < 8: this warp's entries with key k
    for (int r = 0; r < kGroupTile / 256; ++r) {
        const int i = base + r * 256 + threadIdx.x;
        const int k = i < n ? min((int)keys[i], kShadeKeys - 1) : kShadeKeys;   // keys above 7 group as 7
        for (int kk = 0; kk < kShadeKeys; ++kk) {
            const int c = __popc(__ballot_sync(0xffffffffu, k == kk));
            if (lane == kk) mine += c;
        }
    }
    if (lane < kShadeKeys) warp_counts[warp][lane] = mine;
    __syncthreads();
    if (threadIdx.x < kShadeKeys) {
        int total = 0;
        for (int w = 0; w < 8; ++w) total += warp_counts[w][threadIdx.x];
        tile_counts[kShadeKeys * blockIdx.x + threadIdx.x] = total;
    }
}

// Exclusive scan of the tile counts in key-major order, in place: tile_counts[8 * t + k]
// becomes the first position of tile t's key-k entries in the permutation. One block.
__global__ void __launch_bounds__(1024) group_scan_kernel(int* tile_counts, int n, const int* n_ptr) {
    n = queue_size(n_ptr, n);
    const int tiles = (n + kGroupTile - 1) / kGroupTile;
    const int per = (tiles + 1023) / 1024;
    const int t0 = min((int)threadIdx.x * per, tiles), t1 = min(t0 + per, tiles);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int k = 0; k < kShadeKeys; ++k) {
        int local = 0;
        for (int t = t0; t < t1; ++t) local += tile_counts[kShadeKeys * t + k];
        int incl = local;
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int w = warp_sums[lane];
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, w, d);
                if (lane >= d) w += v;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        int run = carry + (warp > 0 ? warp_sums[warp - 1] : 0) + incl - local;
        for (int t = t0; t < t1; ++t) {
            const int c = tile_counts[kShadeKeys * t + k];
            tile_counts[kShadeKeys * t + k] = run;
            run += c;
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_sums[31];
        __syncthreads();
    }
}

// Places the entries of tile blockIdx.x at their scanned offsets, in index order within each
// key (round by round, warp by warp, lane by lane).
__global__ void __launch_bounds__(256) group_scatter_kernel(const uint8_t* __restrict__ keys, int n, const int* n_ptr,
                                                            const int* __restrict__ tile_offsets, int* __restrict__ perm) {
    n = queue_size(n_ptr, n);
    const int base = blockIdx.x * kGroupTile;
    if (base >= n) return;
    __shared__ int run[kShadeKeys];                 // entries of each key placed so far (+ tile offset)
    __shared__ int warp_counts[8][kShadeKeys];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    if (threadIdx.x < kShadeKeys) run[threadIdx.x] = tile_offsets[kShadeKeys * blockIdx.x + threadIdx.x];
    for (int r = 0; r < kGroupTile / 256; ++r) {
        const int i = base + r * 256 + threadIdx.x;
        const bool valid = i < n;
        const int k = valid ? min((int)keys[i], kShadeKeys - 1) : kShadeKeys;
        unsigned same = 0;
        for (int kk = 0; kk < kShadeKeys; ++kk) {
            const unsigned m = __ballot_sync(0xffffffffu, k == kk);
            if (lane == kk) warp_counts[warp][kk] = __popc(m);
            if (k == kk) same = m;
        }
        __syncthreads();
        if (valid) {
            int off = run[k] + __popc(same & lt_mask);
            for (int w = 0; w < warp; ++w) off += warp_counts[w][k];
            perm[off] = i;
        }
        int total = 0;
        if (threadIdx.x < kShadeKeys)
            for (int w = 0; w < 8; ++w) total += warp_counts[w][threadIdx.x];
        __syncthreads();
        if (threadIdx.x < kShadeKeys) run[threadIdx.x] += total;
    }
}

// The permutation of a queue of n entries (n_ptr: size read on the device, n its bound) from
// its keys; tile_counts holds 8 ints per tile (group_tiles(n) tiles).
inline void launch_grouping(const uint8_t* keys, int n, const int* n_ptr, int* tile_counts, int* perm,
                            cudaStream_t st) {
    const int tiles = group_tiles(n);
    group_count_kernel<<<tiles, 256, 0, st>>>(keys, n, n_ptr, tile_counts);
    group_scan_kernel<<<1, 1024, 0, st>>>(tile_counts, n, n_ptr);
    group_scatter_kernel<<<tiles, 256, 0, st>>>(keys, n, n_ptr, tile_counts, perm);
    note_launches(3);
}

// One wavefront of shading: continuations go to the next path queue, shadow rays to the
// shadow queue (both appended in warp order). In the merged form every path that ends adds
// one to its request's `terminated` counter.
template <bool kMulti>
__device__ __forceinline__ void shade_queue_entry(const ShadeParams& p, int t, int n) {
    ShadeOut o;
    int pixel = 0, req = 0, root = 0;
    if (t < n) {
        const int i = p.perm ? p.perm[t] : t;
        pixel = p.pixel[i];
        const float4 ro = p.rays[2 * i], rd = p.rays[2 * i + 1];
        const int4 h = p.hits[i];
        const unsigned long long rs = p.rng[i];
        const float4 t4 = p.thr[i];
        const int bf = p.bounces[i];
        if (kMulti) {
            req = p.req[i];
            root = p.root[i];
            const ReqDev& R = p.reqs[req];
            shade_path(p.scenes[R.scene_slot], R.max_path_len, R.rr_start, R.image, ro, rd, h, pixel, rs, t4, bf, o);
        } else {
            shade_path(p.s, p.max_path_len, p.rr_start, p.image, ro, rd, h, pixel, rs, t4, bf, o);
        }
    }
    const int slot = warp_append(p.counts + 0, o.alive);
    if (o.alive) {
        p.o_rays[2 * slot] = o.o_org;
        p.o_rays[2 * slot + 1] = o.o_dir;
        p.o_pixel[slot] = pixel;
        p.o_rng[slot] = o.rng.state;
        p.o_thr[slot] = make_float4(o.thr.x, o.thr.y, o.thr.z, o.last_pdf);
        p.o_bounces[slot] = o.bounces | (o.last_spec ? (int)0x80000000 : 0);
        if (kMulti) { p.o_req[slot] = req; p.o_root[slot] = root; }
    }
    const int sslot = warp_append(p.counts + 1, o.shadow);
    if (o.shadow) {
        p.s_rays[2 * sslot] = o.s_org;
        p.s_rays[2 * sslot + 1] = o.s_dir;
        p.s_pixel[sslot] = pixel;
        p.s_contrib[sslot] = make_float4(o.s_c.x, o.s_c.y, o.s_c.z, 0.0f);
        if (kMulti) { p.s_req[sslot] = req; p.s_root[sslot] = root; }
    }
    if (kMulti) {
        const bool ended = t < n && !o.alive;
        const unsigned m = __ballot_sync(__activemask(), ended);
        if (ended) {
            const unsigned peers = __match_any_sync(m, req);
            if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(p.terminated + req, __popc(peers));
        }
    }
}

// One queue entry per thread: the launch covers the queue (or its bound, when the size is read
// on the device; threads past the size only take part in the warp-wide appends).
template <bool kMulti>
__global__ void __launch_bounds__(128) pt_shade_kernel(ShadeParams p) {
    shade_queue_entry<kMulti>(p, blockIdx.x * blockDim.x + threadIdx.x, queue_size(p.n_ptr, p.n));
}

// Integrator::process_shadow_rays (integrator.h:49-63): unoccluded shadow rays add their
// contribution to the image. The ray count is read from the device (`count`), `bound` sizes
// the launch.
template <bool kMulti>
__global__ void shadow_accumulate_kernel(const int* count, const int4* hits, const int* pixel, const float4* contrib,
                                         float* image, const int* sreq, const ReqDev* reqs) {
    const int n = *count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (hits[i].x >= 0) continue;
        const float4 c = contrib[i];
        float* img = kMulti ? reqs[sreq[i]].image : image;
        add_image(img, pixel[i], V3(c.x, c.y, c.z));
    }
}

}  // namespace
}  // namespace pt
}  // namespace imbart
