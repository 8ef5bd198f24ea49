// The VCM family on the GPU: vertex connection and merging, bidirectional path tracing,
// progressive photon mapping, light tracing and the VCM-weighted path tracer — the device form
// of the reference's VCMIntegrator<algo> (src/imbatracer/render/integrators/vcm.cpp, vcm.h)
// with its light-vertex cache (light_vertices.h/.cpp) and photon grid (rangesearch.h).
//
// An iteration is a light pass followed by a camera pass (vcm.cpp:25-55).
//  * Light pass (vcm.cpp:64-104, 192-320): light paths are generated per light tile with the
//    reference's seeding (UniformLightTileGen / LightRayGen, tile_gen.h:101-177,
//    ray_gen.h:115-166) and kept in fixed slots (path p stays in slot p); every wavefront
//    traces all slots (finished paths carry an empty ray interval and cost one ray fetch).
//    Each non-specular hit stores a light vertex and (except for PPM) connects to the camera
//    through a shadow ray. Vertices are appended in (wavefront, path) order with a scan, so
//    the cache is the same on every run.
//  * Camera pass (vcm.cpp:106-130, 322-611): camera samples with the path tracer's seeding;
//    per hit: environment / emitter contributions with MIS, next-event estimation, connections
//    to cached light vertices chosen by the path's RNG, merging with the k nearest photons of
//    the grid (inline, no shadow ray), and a Russian-roulette bounce.
// Shadow rays of both passes are resolved by the any-hit kernel and accumulated into the
// image (process_shadow_rays_dbg, vcm.cpp:613-632). The MIS partial weights dVC / dVCM / dVM
// follow the reference's formulas with its association order (mis_pow is the identity: the
// reference's power is 1). Compiled with -fmad=false, like the rest of the shading code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>
#include <vector>

#include "hashgrid_query.cuh"
#include "imbart_internal.h"
#include "pt_kernels.cuh"

using namespace imbart;
using namespace imbart::sh;
using imbart::pt::warp_append;
using imbart::pt::add_image;

namespace imbart {
namespace {

constexpr int kAlgoBpt = IMBART_BPT, kAlgoPpm = IMBART_PPM, kAlgoLt = IMBART_LT, kAlgoPt = IMBART_VCM_PT;

bool ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? IMBART_ERR_OUT_OF_MEMORY : IMBART_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// A light tile: `count` consecutive light paths of one light, seeded from one queue fill.
struct LightTile {
    int first;            // first path slot
    int count;
    int light;
    unsigned int seed;    // the fill's seed_base (32 bits: std::random_device draws)
};

struct VcmParams {
    ShadingScene s;
    int algo, width, height, max_path_len, num_connections, num_knn, light_path_count;
    float eta_vc, eta_vm, pm_radius, base_radius, vc_weight;
    float w2r[16], r2w[16], cam_pos[3], cam_dir[3], img_plane_dist;
    // light vertices and their grid
    const float4* cache;
    int cache_count;
    const float4* grid_sorted;
    const int* grid_ends;
    const float* grid_params;
    unsigned int grid_table;
    int merging;
    float* image;
    int* counts;          // [0] next camera queue, [1] shadow rays, [2] live light paths, [3] merges
};

__device__ __forceinline__ V3 v3(float4 a) { return V3(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// VCMIntegrator::shading_normal_adjoint (vcm.h:125-127)
__device__ __forceinline__ float shading_normal_adjoint(V3 normal, V3 geom_normal, V3 out_dir, V3 in_dir) {
    return dot(out_dir, normal) * dot(in_dir, geom_normal) / dot(out_dir, geom_normal);
}


// VCMIntegrator::bounce (vcm.cpp:132-190). Returns false when the path ends.
__device__ __forceinline__ bool vcm_bounce(const VcmParams& p, Rng& rng, V3& thr, int& path_length, float& dVC,
                                           float& dVCM, float& dVM, const Isect& is, const Bsdf& bsdf, bool adjoint,
                                           float offset, float4& org, float4& dir_out) {
    float rr_pdf;
    if (!russian_roulette(thr, rng.next_float(), rr_pdf)) return false;
    int allowed = kAllFlags;
    if (p.algo == kAlgoPpm && !adjoint) allowed = kSpecular | kRefl | kTrans;
    float pdf_dir_w;
    V3 sample_dir;
    int sampled;
    const V3 bsdf_value = bsdf.sample(is.out_dir, sample_dir, rng, sampled, pdf_dir_w, allowed);
    const bool is_specular = (sampled & kSpecular) != 0;
    if (sampled == 0 || pdf_dir_w == 0.0f || is_black(bsdf_value)) return false;
    float pdf_rev_w = pdf_dir_w;
    if (!is_specular) pdf_rev_w = bsdf.pdf(sample_dir, is.out_dir);
    const float cos_theta_i = adjoint ? fabsf(shading_normal_adjoint(is.normal, is.geom_normal, is.out_dir, sample_dir))
                                      : fabsf(dot(sample_dir, is.normal));
    if (is_specular) {
        dVCM = 0.0f;
        dVC *= cos_theta_i;
        dVM *= cos_theta_i;
    } else {
        dVC = (cos_theta_i / pdf_dir_w) * (dVC * pdf_rev_w + dVCM + p.eta_vm);
        dVM = (cos_theta_i / pdf_dir_w) * (dVM * pdf_rev_w + dVCM * p.eta_vc + 1.0f);
        dVCM = 1.0f / pdf_dir_w;
    }
    thr = thr * (bsdf_value * cos_theta_i / (rr_pdf * pdf_dir_w));
    path_length++;
    org = make_float4(is.pos.x, is.pos.y, is.pos.z, offset);
    dir_out = make_float4(sample_dir.x, sample_dir.y, sample_dir.z, FLT_MAX);
    return true;
}

// ---------------------------------------------------------------------------------------
// Light pass
// ---------------------------------------------------------------------------------------

// The light-sample function of trace_light_paths (vcm.cpp:64-101) for LightRayGen sample i of
// a tile: RNG seeded as in ray_gen.h:128-141 (the tile-local index scrambles the seed and
// sets the discard).
// Light paths first + j for the n slots j (a rank of a multi-GPU iteration traces a range of
// the iteration's paths; every path is seeded by its global index).
__global__ void light_gen_kernel(VcmParams p, const LightTile* tiles, int n_tiles, int first, int n, float4* rays,
                                 unsigned long long* rng_out, float4* thr, float4* w) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int g = first + j;
    int lo = 0, hi = n_tiles - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tiles[mid].first <= g) lo = mid;
        else hi = mid - 1;
    }
    const LightTile t = tiles[lo];
    const int i = g - t.first;
    Rng rng = seed_sample(t.seed, i, i);
    const ShadingScene& s = p.s;
    const float pdf_lightpick = 1.0f / (float)s.light_count;
    const EmitSample e = light_emit(s, t.light, rng);
    rays[2 * j + 0] = make_float4(e.pos.x, e.pos.y, e.pos.z, 1e-3f);
    rays[2 * j + 1] = make_float4(e.dir.x, e.dir.y, e.dir.z, FLT_MAX);
    const V3 tp = e.radiance / pdf_lightpick;
    thr[j] = f4(tp, __int_as_float(1));
    const float dVCM = e.pdf_direct_a / e.pdf_emit_w;
    const float dVC = light_is_delta(s, t.light) ? 0.0f : e.cos_out / (e.pdf_emit_w * pdf_lightpick);
    const float dVM = dVC * p.eta_vc;
    w[j] = make_float4(dVC, dVCM, dVM, light_is_finite(s, t.light) ? 1.0f : 0.0f);   // w: finite light
    rng_out[j] = rng.state;
}

// Material grouping keys of light-path slots (pt::shade_key; finished slots get key 7).
__global__ void __launch_bounds__(256) light_key_kernel(ShadingScene s, const int4* __restrict__ hits,
                                                        const float4* __restrict__ thrs, int n, uint8_t* keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = (uint8_t)(__float_as_int(thrs[i].w) < 0 ? 7 : pt::shade_key(s, hits[i]));
}

// connect_to_camera (vcm.cpp:260-320): a shadow ray towards the camera. Returns false when the
// vertex does not project into the image or the BSDF cannot reach the camera.
__device__ __forceinline__ bool camera_connection(const VcmParams& p, V3 thr, float dVC, float dVCM, const Isect& is,
                                                  const Bsdf& bsdf, float4& org, float4& dir, int& pixel, V3& contrib) {
    const V3 cam_pos(p.cam_pos[0], p.cam_pos[1], p.cam_pos[2]);
    const V3 cam_dir(p.cam_dir[0], p.cam_dir[1], p.cam_dir[2]);
    V3 dir_to_cam = cam_pos - is.pos;
    if (dot(-dir_to_cam, cam_dir) < 0.0f) return false;
    // PerspectiveCamera::world_to_raster / raster_to_id (camera.h:67-86).
    const float* m = p.w2r;
    const V3 x = is.pos;
    const float t0 = m[0] * x.x + m[1] * x.y + m[2] * x.z + m[3] * 1.0f;
    const float t1 = m[4] * x.x + m[5] * x.y + m[6] * x.z + m[7] * 1.0f;
    const float t3 = m[12] * x.x + m[13] * x.y + m[14] * x.z + m[15] * 1.0f;
    const float rx = t1 / t3, ry = t0 / t3;
    const float fx = floorf(rx), fy = floorf(ry);
    if (!(fx >= 0.0f && fx < (float)p.width && fy >= 0.0f && fy < (float)p.height)) return false;
    pixel = (int)((float)(int)fy * (float)p.width + (float)(int)fx);
    if (pixel < 0 || pixel >= p.width * p.height) return false;
    const float dist_sqr = dot(dir_to_cam, dir_to_cam);
    const float dist = sqrtf(dist_sqr);
    dir_to_cam = dir_to_cam / dist;
    const float cos_theta_cam = fabsf(dot(cam_dir, -dir_to_cam));
    const float cos_theta_surf = fabsf(shading_normal_adjoint(is.normal, is.geom_normal, is.out_dir, dir_to_cam));
    const V3 bsdf_value = bsdf.eval(is.out_dir, dir_to_cam);
    const float pdf_rev_w = bsdf.pdf(dir_to_cam, is.out_dir);
    if (pdf_rev_w == 0.0f) return false;
    const float img_to_surf = (sqr(p.img_plane_dist) * cos_theta_surf) /
                              (dist_sqr * cos_theta_cam * sqr(cos_theta_cam));
    const float pdf_cam = img_to_surf;
    const float P = (float)p.light_path_count;
    const float mis_weight_light = (pdf_cam / P) * (p.eta_vm + dVCM + dVC * pdf_rev_w);
    const float mis_weight = p.algo == kAlgoLt ? 1.0f : (1.0f / (mis_weight_light + 1.0f));
    contrib = thr * (mis_weight * bsdf_value * img_to_surf / P);
    const float offset = dist * 1e-3f;
    org = make_float4(is.pos.x, is.pos.y, is.pos.z, offset);
    dir = make_float4(dir_to_cam.x, dir_to_cam.y, dir_to_cam.z, dist - offset);
    return true;
}

// process_light_rays for every light-path slot (vcm.cpp:192-258). A finished slot holds
// path_length -1 and an empty ray interval.
__global__ void __launch_bounds__(128) light_shade_kernel(VcmParams p, int n, float4* rays, const int4* hits,
                                                          unsigned long long* rngs, float4* thrs, float4* ws,
                                                          float4* stage, int* vflags, float4* s_rays, int* s_pixel,
                                                          float4* s_contrib, const int* perm) {
    // Thread t shades slot perm[t] (slots grouped by material); every write goes to the slot.
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (perm && t < n) ? perm[t] : t;
    bool alive = false, vertex = false, shadow = false;
    float4 s_org = make_float4(0, 0, 0, 0), s_dir = s_org;
    int s_pix = 0;
    V3 s_c(0.0f);
    if (i < n) {
        const float4 t4 = thrs[i];
        int pl = __float_as_int(t4.w);
        if (pl >= 0) {
            const int4 h = hits[i];
            if (h.x >= 0) {
                const ShadingScene& s = p.s;
                const float4 ro = rays[2 * i], rd = rays[2 * i + 1];
                const float tmax = __int_as_float(h.z);
                const Isect is = calculate_intersection(s, h.x, h.y, tmax, __int_as_float(h.w), V3(ro.x, ro.y, ro.z),
                                                        V3(rd.x, rd.y, rd.z));
                const float cos_theta_o = fabsf(dot(is.out_dir, is.normal));
                if (cos_theta_o != 0.0f) {
                    const float4 w4 = ws[i];
                    float dVC = w4.x, dVCM = w4.y, dVM = w4.z;
                    const bool finite = w4.w != 0.0f;
                    if (pl > 1 || finite) dVCM *= sqr(tmax);
                    dVCM *= 1.0f / cos_theta_o;
                    dVC *= 1.0f / cos_theta_o;
                    dVM *= 1.0f / cos_theta_o;
                    V3 thr = v3(t4);
                    const Material& mat = s.materials[is.mat];
                    const Bsdf bsdf = surface_bsdf(s, mat, is.normal, is.u_tangent, is.v_tangent, is.geom_normal,
                                                   is.uv[0], is.uv[1], true);
                    if (!is_specular_material(mat)) {
                        if (p.algo != kAlgoLt) {
                            float4* v = stage + 7 * (size_t)i;
                            v[0] = f4(is.pos, __int_as_float(is.mat));
                            v[1] = f4(is.out_dir, __int_as_float(pl + 1));
                            v[2] = f4(is.normal, dVC);
                            v[3] = f4(is.geom_normal, dVCM);
                            v[4] = f4(is.u_tangent, dVM);
                            v[5] = f4(is.v_tangent, is.uv[0]);
                            v[6] = f4(thr, is.uv[1]);
                            vertex = true;
                        }
                        if (p.algo != kAlgoPpm)
                            shadow = camera_connection(p, thr, dVC, dVCM, is, bsdf, s_org, s_dir, s_pix, s_c);
                    }
                    Rng rng{rngs[i]};
                    float4 org, dir;
                    const float offset = tmax * 1e-4f;
                    alive = vcm_bounce(p, rng, thr, pl, dVC, dVCM, dVM, is, bsdf, true, offset, org, dir);
                    if (alive) {
                        rays[2 * i] = org;
                        rays[2 * i + 1] = dir;
                        thrs[i] = f4(thr, __int_as_float(pl));
                        ws[i] = make_float4(dVC, dVCM, dVM, w4.w);
                        rngs[i] = rng.state;
                    }
                }
            }
            if (!alive) {
                thrs[i] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
                rays[2 * i + 1].w = -1.0f;   // empty interval: later wavefronts skip the slot
            }
        }
        vflags[i] = vertex ? 1 : 0;
    }
    const unsigned live = __ballot_sync(0xffffffffu, alive);
    if ((threadIdx.x & 31) == 0 && live) atomicAdd(p.counts + 2, __popc(live));
    const int slot = warp_append(p.counts + 1, shadow);
    if (shadow) {
        s_rays[2 * slot] = s_org;
        s_rays[2 * slot + 1] = s_dir;
        s_pixel[slot] = s_pix;
        s_contrib[slot] = f4(s_c, 0.0f);
    }
}

// Stable compaction of the live light-path slots (path length >= 0): flags, then the same
// block-count / scan as the vertex append, then a scatter of the path states to the second
// buffers in slot order, so paths keep their relative order and the vertex cache its
// (wavefront, path) order.
__global__ void live_flags_kernel(const float4* __restrict__ thrs, int n, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = __float_as_int(thrs[i].w) >= 0 ? 1 : 0;
}

// Deterministic append of the staged vertices: exclusive scan of the per-slot flags in slot
// order (block counts, one scan of the block counts, per-block ranks).
constexpr int kScanBlock = 256;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanBlock * kScanPer;

__global__ void flag_count_kernel(const int* flags, int n, int* block_sums) {
    __shared__ int warp_sums[kScanBlock / 32];
    const int base = blockIdx.x * kScanTile;
    int c = 0;
    for (int k = 0; k < kScanPer; ++k) {
        const int i = base + k * kScanBlock + threadIdx.x;
        if (i < n) c += flags[i];
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < kScanBlock / 32; ++k) t += warp_sums[k];
        block_sums[blockIdx.x] = t;
    }
}

// Single-block exclusive scan of the block sums (any count); total in block_sums[n_blocks].
__global__ void block_scan_kernel(int* block_sums, int n_blocks) {
    __shared__ int carry;
    __shared__ int warp_sums[kScanBlock / 32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n_blocks; base += kScanBlock) {
        const int i = base + threadIdx.x;
        const int v = i < n_blocks ? block_sums[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if ((threadIdx.x & 31) >= o) incl += u;
        }
        if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = incl;
        __syncthreads();
        int before = 0;
        for (int k = 0; k < (int)(threadIdx.x >> 5); ++k) before += warp_sums[k];
        const int excl = carry + before + incl - v;
        __syncthreads();
        if (i < n_blocks) block_sums[i] = excl;
        if (threadIdx.x == kScanBlock - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sums[n_blocks] = carry;
}

__global__ void vertex_scatter_kernel(const int* flags, int n, const int* block_offsets, const float4* stage,
                                      float4* cache, int cache_base) {
    __shared__ int warp_sums[kScanBlock / 32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = block_offsets[blockIdx.x];
    __syncthreads();
    const int base = blockIdx.x * kScanTile;
    for (int k = 0; k < kScanPer; ++k) {
        const int i = base + k * kScanBlock + threadIdx.x;
        const int f = i < n ? flags[i] : 0;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        const int lane = threadIdx.x & 31;
        if (lane == 0) warp_sums[threadIdx.x >> 5] = __popc(m);
        __syncthreads();
        int before = 0;
        for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) before += warp_sums[w];
        if (f) {
            const int dst = cache_base + carry + before + __popc(m & ((1u << lane) - 1u));
            for (int q = 0; q < 7; ++q) cache[7 * (size_t)dst + q] = stage[7 * (size_t)i + q];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < kScanBlock / 32; ++w) t += warp_sums[w];
            carry += t;
        }
        __syncthreads();
    }
}

__global__ void compact_paths_kernel(const int* flags, int n, const int* block_offsets, const float4* rays,
                                     const unsigned long long* rngs, const float4* thrs, const float4* ws,
                                     float4* rays2, unsigned long long* rngs2, float4* thrs2, float4* ws2) {
    __shared__ int warp_sums[kScanBlock / 32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = block_offsets[blockIdx.x];
    __syncthreads();
    const int base = blockIdx.x * kScanTile;
    for (int k = 0; k < kScanPer; ++k) {
        const int i = base + k * kScanBlock + threadIdx.x;
        const int f = i < n ? flags[i] : 0;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        const int lane = threadIdx.x & 31;
        if (lane == 0) warp_sums[threadIdx.x >> 5] = __popc(m);
        __syncthreads();
        int before = 0;
        for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) before += warp_sums[w];
        if (f) {
            const int dst = carry + before + __popc(m & ((1u << lane) - 1u));
            rays2[2 * (size_t)dst] = rays[2 * (size_t)i];
            rays2[2 * (size_t)dst + 1] = rays[2 * (size_t)i + 1];
            rngs2[dst] = rngs[i];
            thrs2[dst] = thrs[i];
            ws2[dst] = ws[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < kScanBlock / 32; ++w) t += warp_sums[w];
            carry += t;
        }
        __syncthreads();
    }
}

// process_shadow_rays_dbg (vcm.cpp:613-632); the ray count is read on the device.
__global__ void vcm_shadow_kernel(const int* count, const int4* hits, const int* pixel, const float4* contrib,
                                  float* image) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count) return;
    if (hits[i].x >= 0) return;
    const float4 c = contrib[i];
    add_image(image, pixel[i], V3(c.x, c.y, c.z));
}

// ---------------------------------------------------------------------------------------
// Camera pass
// ---------------------------------------------------------------------------------------

// The camera-sample function of trace_camera_paths (vcm.cpp:106-130) with PixelRayGen seeding.
__global__ void vcm_camera_kernel(VcmParams p, unsigned long long seed_base, int spp, long long first, int n,
                                  float4* rays, int* pixel, unsigned long long* rng_out, float4* thr, float4* w) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int i = (int)(first + j);
    pt::camera_sample(p.r2w, p.cam_pos, spp, 0, 0, p.width, p.width, seed_base, i, rays + 2 * j, pixel + j,
                      rng_out + j);
    const float4 rd = rays[2 * j + 1];
    const V3 dir(rd.x, rd.y, rd.z);
    const float cos_theta_o = dot(dir, V3(p.cam_dir[0], p.cam_dir[1], p.cam_dir[2]));
    const float pdf_cam_w = sqr(p.img_plane_dist / cos_theta_o) / cos_theta_o;
    thr[j] = make_float4(1.0f, 1.0f, 1.0f, __int_as_float(1));
    w[j] = make_float4(0.0f, (float)p.light_path_count / pdf_cam_w, 0.0f, 0.0f);
}

struct CamShadow {
    float4 org, dir;
    V3 c;
};

// VCMIntegrator::direct_illum (vcm.cpp:441-486).
__device__ __forceinline__ bool vcm_direct_illum(const VcmParams& p, Rng& rng, V3 thr, float dVC, float dVCM,
                                                 const Isect& is, const Bsdf& bsdf, CamShadow& out) {
    const ShadingScene& s = p.s;
    const int l = rng.next_int(0, s.light_count);
    const float pdf_lightpick_inv = (float)s.light_count;
    const DirectSample sample = light_sample_direct(s, l, is.pos, rng);
    const float cos_theta_o = sample.cos_out;
    const float offset = 1e-3f * (sample.distance == FLT_MAX ? 1.0f : sample.distance);
    out.org = make_float4(is.pos.x, is.pos.y, is.pos.z, offset);
    out.dir = make_float4(sample.dir.x, sample.dir.y, sample.dir.z, sample.distance - offset);
    const float cos_theta_i = fabsf(dot(is.normal, sample.dir));
    const V3 bsdf_value = bsdf.eval(is.out_dir, sample.dir);
    const float pdf_dir_w = bsdf.pdf(is.out_dir, sample.dir);
    const float pdf_rev_w = bsdf.pdf(sample.dir, is.out_dir);
    if (pdf_dir_w == 0.0f || pdf_rev_w == 0.0f) return false;
    const float pdf_forward = sample.delta ? 0.0f : pdf_dir_w;
    const float mis_weight_light = pdf_forward * pdf_lightpick_inv / sample.pdf_direct_w;
    const float mis_weight_camera = (sample.pdf_emit_w * cos_theta_i / (sample.pdf_direct_w * cos_theta_o)) *
                                    (p.eta_vm + dVCM + dVC * pdf_rev_w);
    const float mis_weight = p.algo == kAlgoPt ? 1.0f : (1.0f / (mis_weight_camera + 1.0f + mis_weight_light));
    out.c = thr * mis_weight * bsdf_value * cos_theta_i * sample.radiance * pdf_lightpick_inv;
    return true;
}

// One connection of VCMIntegrator::connect (vcm.cpp:488-569) to cache vertex `idx`.
__device__ __forceinline__ bool vcm_connect_one(const VcmParams& p, int cam_path_length, V3 thr, float dVC,
                                                float dVCM, const Isect& is, const Bsdf& bsdf_cam, int idx,
                                                CamShadow& out) {
    const float4* v = p.cache + 7 * (size_t)idx;
    const float4 q0 = __ldg(v), q1 = __ldg(v + 1);
    const int light_path_length = __float_as_int(q1.w);
    if (light_path_length + cam_path_length > p.max_path_len) return false;
    const int mi = __float_as_int(q0.w);
    if (mi < 0 || mi >= p.s.n_materials) return false;   // a loaded cache with a bad material index
    const float4 q2 = __ldg(v + 2), q3 = __ldg(v + 3), q4 = __ldg(v + 4), q5 = __ldg(v + 5), q6 = __ldg(v + 6);
    const V3 lpos = v3(q0), lout = v3(q1), lnormal = v3(q2), lgn = v3(q3);
    const Material& lmat = p.s.materials[mi];
    const Bsdf light_bsdf = surface_bsdf(p.s, lmat, lnormal, v3(q4), v3(q5), lgn, q5.w, q6.w, true);
    V3 connect_dir = lpos - is.pos;
    const float connect_dist_sq = dot(connect_dir, connect_dir);
    const float connect_dist = sqrtf(connect_dist_sq);
    connect_dir = connect_dir * (1.0f / connect_dist);
    if (connect_dist < p.base_radius) return false;
    const V3 bsdf_value_cam = bsdf_cam.eval(is.out_dir, connect_dir);
    const float pdf_dir_cam_w = bsdf_cam.pdf(is.out_dir, connect_dir);
    const float pdf_rev_cam_w = bsdf_cam.pdf(connect_dir, is.out_dir);
    const V3 neg_dir = -connect_dir;
    const V3 bsdf_value_light = light_bsdf.eval(lout, neg_dir);
    const float pdf_dir_light_w = light_bsdf.pdf(lout, neg_dir);
    const float pdf_rev_light_w = light_bsdf.pdf(neg_dir, lout);
    if (pdf_dir_cam_w == 0.0f || pdf_dir_light_w == 0.0f || pdf_rev_cam_w == 0.0f || pdf_rev_light_w == 0.0f)
        return false;
    const float cos_theta_cam = fabsf(dot(is.normal, connect_dir));
    const float cos_theta_light = fabsf(shading_normal_adjoint(lnormal, lgn, lout, neg_dir));
    const float geom_term = cos_theta_cam * cos_theta_light / connect_dist_sq;
    if (geom_term <= 0.0f) return false;
    const float pdf_cam_a = pdf_dir_cam_w * cos_theta_light / connect_dist_sq;
    const float pdf_light_a = pdf_dir_light_w * cos_theta_cam / connect_dist_sq;
    const float mis_weight_light = pdf_cam_a * (p.eta_vm + q3.w + q2.w * pdf_rev_light_w);
    const float mis_weight_camera = pdf_light_a * (p.eta_vm + dVCM + dVC * pdf_rev_cam_w);
    const float mis_weight = 1.0f / (mis_weight_camera + 1.0f + mis_weight_light);
    out.c = thr * p.vc_weight * mis_weight * geom_term * bsdf_value_cam * bsdf_value_light * v3(q6);
    const float offset = 1e-3f * connect_dist;
    out.org = make_float4(is.pos.x, is.pos.y, is.pos.z, offset);
    out.dir = make_float4(connect_dir.x, connect_dir.y, connect_dir.z, connect_dist - offset);
    return true;
}

// VCMIntegrator::vertex_merging (vcm.cpp:571-611): the k nearest photons of the grid, one
// thread per query (the path for k > 32; vcm_merge_warp_kernel serves k <= 32).
__device__ __forceinline__ V3 vcm_merge(const VcmParams& p, V3 thr, float dVCM, float dVM, const Isect& is,
                                        const Bsdf& bsdf) {
    float dist[kGridMaxK];
    int ids[kGridMaxK];
    float prm[10];
    for (int k = 0; k < 10; ++k) prm[k] = __ldg(p.grid_params + k);
    const int k = p.num_knn;
    const int count = grid_query_knn(p.grid_sorted, p.grid_ends, prm, p.grid_table, is.pos.x, is.pos.y, is.pos.z, k,
                                     dist, ids);
    float radius_sqr = p.pm_radius * p.pm_radius;
    if (count == k) {
        const float4 q = __ldg(p.cache + 7 * (size_t)ids[k - 1]);
        const V3 d = v3(q) - is.pos;
        radius_sqr = dot(d, d);
    }
    V3 contrib(0.0f);
    for (int i = 0; i < count; ++i) {
        const float4* v = p.cache + 7 * (size_t)ids[i];
        const float4 q0 = __ldg(v), q1 = __ldg(v + 1), q3 = __ldg(v + 3), q4 = __ldg(v + 4), q6 = __ldg(v + 6);
        const V3 photon_in_dir = v3(q1);
        const V3 bsdf_value = bsdf.eval(is.out_dir, photon_in_dir);
        const float pdf_dir_w = bsdf.pdf(is.out_dir, photon_in_dir);
        const float pdf_rev_w = bsdf.pdf(photon_in_dir, is.out_dir);
        if (pdf_dir_w == 0.0f || pdf_rev_w == 0.0f || is_black(bsdf_value)) continue;
        const float mis_weight_light = q3.w * p.eta_vc + q4.w * pdf_dir_w;
        const float mis_weight_camera = dVCM * p.eta_vc + dVM * pdf_rev_w;
        const float mis_weight = p.algo == kAlgoPpm ? 1.0f : (1.0f / (mis_weight_light + 1.0f + mis_weight_camera));
        const V3 dp = v3(q0) - is.pos;
        const float d = dot(dp, dp);
        const float kernel = 1.0f - d / radius_sqr;
        contrib = contrib + mis_weight * bsdf_value * kernel * v3(q6);
    }
    contrib = contrib * (2.0f / (kPi * radius_sqr * (float)p.light_path_count));
    return thr * contrib;
}

// A camera vertex waiting for merging (7 float4): pos + pixel, out_dir + material, normal +
// dVCM, geometric normal + dVM, u tangent + uv.x, v tangent + uv.y, throughput.
constexpr int kMergeRec = 7;

// Vertex merging for the camera vertices queued by the shading kernel (count on the device).
__global__ void __launch_bounds__(128) vcm_merge_kernel(VcmParams p, const int* count, const float4* recs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count) return;
    const float4* r = recs + kMergeRec * (size_t)i;
    const float4 m0 = r[0], m1 = r[1], m2 = r[2], m3 = r[3], m4 = r[4], m5 = r[5], m6 = r[6];
    Isect is;
    is.pos = v3(m0);
    is.out_dir = v3(m1);
    is.normal = v3(m2);
    is.geom_normal = v3(m3);
    is.u_tangent = v3(m4);
    is.v_tangent = v3(m5);
    is.mat = __float_as_int(m1.w);
    const Bsdf bsdf = surface_bsdf(p.s, p.s.materials[is.mat], is.normal, is.u_tangent, is.v_tangent, is.geom_normal,
                                   m4.w, m5.w, false);
    add_image(p.image, __float_as_int(m0.w), vcm_merge(p, v3(m6), m2.w, m3.w, is, bsdf));
}

// Vertex merging with one warp per queued camera vertex (k <= 32): the warp's k-nearest
// search (grid_query_knn_warp, one list entry per lane), the found photons evaluated one per
// lane, and their contributions summed in list order, so the result equals the per-thread
// query's.
__global__ void __launch_bounds__(128) vcm_merge_warp_kernel(VcmParams p, const int* count_ptr, const float4* recs) {
    const int lane = threadIdx.x & 31;
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (q >= *count_ptr) return;   // uniform across the warp
    const float4* r = recs + kMergeRec * (size_t)q;
    const float4 m0 = r[0], m1 = r[1], m2 = r[2], m3 = r[3], m4 = r[4], m5 = r[5], m6 = r[6];
    const float qx = m0.x, qy = m0.y, qz = m0.z;
    float prm[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) prm[k] = __ldg(p.grid_params + k);
    const int k = p.num_knn;
    float my_d;               // list entry `lane`
    int my_id;
    const int count = grid_query_knn_warp(p.grid_sorted, p.grid_ends, prm, p.grid_table, qx, qy, qz, k, my_d, my_id);
    if (count == 0) return;
    // Evaluate the found photons, one per lane.
    const V3 pos(qx, qy, qz), out_dir = v3(m1), thr = v3(m6);
    const float dVCM = m2.w, dVM = m3.w;
    float radius_sqr = p.pm_radius * p.pm_radius;
    V3 c(0.0f);
    float4 lq0 = make_float4(0, 0, 0, 0);
    if (lane < count) lq0 = __ldg(p.cache + 7 * (size_t)my_id);
    if (count == k) {
        const V3 d = V3(__shfl_sync(0xffffffffu, lq0.x, k - 1), __shfl_sync(0xffffffffu, lq0.y, k - 1),
                        __shfl_sync(0xffffffffu, lq0.z, k - 1)) - pos;
        radius_sqr = dot(d, d);
    }
    if (lane < count) {
        const Material& mat = p.s.materials[__float_as_int(m1.w)];
        const Bsdf bsdf = surface_bsdf(p.s, mat, v3(m2), v3(m4), v3(m5), v3(m3), m4.w, m5.w, false);
        const float4* v = p.cache + 7 * (size_t)my_id;
        const float4 q1 = __ldg(v + 1), q3 = __ldg(v + 3), q4 = __ldg(v + 4), q6 = __ldg(v + 6);
        const V3 photon_in_dir = v3(q1);
        const V3 bsdf_value = bsdf.eval(out_dir, photon_in_dir);
        const float pdf_dir_w = bsdf.pdf(out_dir, photon_in_dir);
        const float pdf_rev_w = bsdf.pdf(photon_in_dir, out_dir);
        if (!(pdf_dir_w == 0.0f || pdf_rev_w == 0.0f || is_black(bsdf_value))) {
            const float mis_weight_light = q3.w * p.eta_vc + q4.w * pdf_dir_w;
            const float mis_weight_camera = dVCM * p.eta_vc + dVM * pdf_rev_w;
            const float mis_weight = p.algo == kAlgoPpm ? 1.0f : (1.0f / (mis_weight_light + 1.0f + mis_weight_camera));
            const V3 dp = v3(lq0) - pos;
            const float d = dot(dp, dp);
            const float kernel = 1.0f - d / radius_sqr;
            c = mis_weight * bsdf_value * kernel * v3(q6);
        }
    }
    // Sum in list order, as the reference accumulates.
    V3 contrib(0.0f);
    for (int l = 0; l < count; ++l)
        contrib = contrib + V3(__shfl_sync(0xffffffffu, c.x, l), __shfl_sync(0xffffffffu, c.y, l),
                               __shfl_sync(0xffffffffu, c.z, l));
    if (lane == 0) {
        contrib = contrib * (2.0f / (kPi * radius_sqr * (float)p.light_path_count));
        add_image(p.image, __float_as_int(m0.w), thr * contrib);
    }
}

// process_camera_rays (vcm.cpp:322-439) for one wavefront of camera paths. Shadow rays (next
// event + connections, at most 1 + num_connections per path) go to the shadow queue, each kind
// appended by the whole warp so that the warp stays converged.
__global__ void __launch_bounds__(128) vcm_camera_shade_kernel(
    VcmParams p, int n, const float4* rays, const int4* hits, const int* pixels, const unsigned long long* rngs,
    const float4* thrs, const float4* ws, float4* o_rays, int* o_pixel, unsigned long long* o_rng, float4* o_thr,
    float4* o_w, float4* s_rays, int* s_pixel, float4* s_contrib, float4* merge_recs, const int* perm) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (perm && t < n) ? perm[t] : t;
    bool alive = false;
    float4 o_org = make_float4(0, 0, 0, 0), o_dir = o_org;
    Rng rng{0};
    V3 thr(0.0f);
    float dVC = 0.0f, dVCM = 0.0f, dVM = 0.0f;
    int pl = 0, pixel = 0;
    const ShadingScene& s = p.s;
    Isect is;
    Bsdf bsdf{nullptr, V3(0.0f), V3(0.0f), V3(0.0f), V3(0.0f)};
    bool surface = false;      // a non-emissive hit that shades further
    float tmax = 0.0f;
    if (i < n) {
        pixel = pixels[i];
        const float4 ro = rays[2 * i], rd = rays[2 * i + 1];
        const int4 h = hits[i];
        rng.state = rngs[i];
        const float4 t4 = thrs[i];
        thr = v3(t4);
        pl = __float_as_int(t4.w);
        const float4 w4 = ws[i];
        dVC = w4.x; dVCM = w4.y; dVM = w4.z;
        if (h.x < 0) {
            if (s.has_env && p.algo != kAlgoPt) {
                const V3 out_dir = normalize(V3(rd.x, rd.y, rd.z));
                float pdf_direct_w, pdf_emit_w;
                const V3 li = env_radiance_emit(s, out_dir, &pdf_direct_w, &pdf_emit_w);
                const float pdf_lightpick = 1.0f / (float)s.light_count;
                const float pdf_di = pdf_direct_w * pdf_lightpick;
                const float pdf_e = pdf_emit_w * pdf_lightpick;
                const float mis_weight_camera = pdf_di * dVCM + pdf_e * dVC;
                const float mis_weight = p.algo == kAlgoPpm ? 1.0f : (1.0f / (mis_weight_camera + 1.0f));
                add_image(p.image, pixel, thr * li * mis_weight);
            }
        } else {
            tmax = __int_as_float(h.z);
            is = calculate_intersection(s, h.x, h.y, tmax, __int_as_float(h.w), V3(ro.x, ro.y, ro.z),
                                        V3(rd.x, rd.y, rd.z));
            const float cos_theta_o = fabsf(dot(is.out_dir, is.normal));
            const Material& mat = s.materials[is.mat];
            bsdf = surface_bsdf(s, mat, is.normal, is.u_tangent, is.v_tangent, is.geom_normal, is.uv[0], is.uv[1],
                                false);
            dVCM *= sqr(tmax) / cos_theta_o;
            dVC *= 1.0f / cos_theta_o;
            dVM *= 1.0f / cos_theta_o;
            if (cos_theta_o != 0.0f) {
                if (mat.kind == kEmissive) {
                    const float pdf_lightpick = 1.0f / (float)s.light_count;
                    float pdf_direct_a, pdf_emit_w;
                    const V3 radiance = area_emitter_radiance(mat, is.out_dir, is.geom_normal, &pdf_direct_a,
                                                              &pdf_emit_w);
                    const float pdf_di = pdf_direct_a * pdf_lightpick;
                    const float pdf_e = pdf_emit_w * pdf_lightpick;
                    const float mis_weight_camera = pdf_di * dVCM + pdf_e * dVC;
                    const float mis_weight = (p.algo == kAlgoPpm || pl == 1) ? 1.0f
                                                                             : (1.0f / (mis_weight_camera + 1.0f));
                    add_image(p.image, pixel, thr * radiance * mis_weight);
                } else if (pl < p.max_path_len) {
                    surface = true;
                }
            }
        }
    }
    // Next-event estimation.
    {
        CamShadow sh;
        bool push = false;
        if (surface && p.algo != kAlgoPpm) push = vcm_direct_illum(p, rng, thr, dVC, dVCM, is, bsdf, sh);
        const int slot = warp_append(p.counts + 1, push);
        if (push) {
            s_rays[2 * slot] = sh.org;
            s_rays[2 * slot + 1] = sh.dir;
            s_pixel[slot] = pixel;
            s_contrib[slot] = f4(sh.c, 0.0f);
        }
    }
    // Connections to light vertices.
    const bool nonspec = surface && !is_specular_material(*bsdf.m);
    if (p.algo != kAlgoPt && p.algo != kAlgoPpm) {
        for (int c = 0; c < p.num_connections; ++c) {
            CamShadow sh;
            bool push = false;
            if (nonspec && p.cache_count > 0) {
                const int idx = rng.next_int(0, p.cache_count);
                push = vcm_connect_one(p, pl, thr, dVC, dVCM, is, bsdf, idx, sh);
            }
            const int slot = warp_append(p.counts + 1, push);
            if (push) {
                s_rays[2 * slot] = sh.org;
                s_rays[2 * slot + 1] = sh.dir;
                s_pixel[slot] = pixel;
                s_contrib[slot] = f4(sh.c, 0.0f);
            }
        }
    }
    // Vertex merging runs in vcm_merge_kernel over the queued camera vertices.
    const bool merge = surface && p.algo != kAlgoBpt && p.algo != kAlgoPt && nonspec && p.merging;
    const int mslot = warp_append(p.counts + 3, merge);
    if (merge) {
        float4* r = merge_recs + kMergeRec * (size_t)mslot;
        r[0] = f4(is.pos, __int_as_float(pixel));
        r[1] = f4(is.out_dir, __int_as_float(is.mat));
        r[2] = f4(is.normal, dVCM);
        r[3] = f4(is.geom_normal, dVM);
        r[4] = f4(is.u_tangent, is.uv[0]);
        r[5] = f4(is.v_tangent, is.uv[1]);
        r[6] = f4(thr, 0.0f);
    }
    if (surface) {
        const float offset = tmax * 1e-4f;
        alive = vcm_bounce(p, rng, thr, pl, dVC, dVCM, dVM, is, bsdf, false, offset, o_org, o_dir);
    }
    const int slot = warp_append(p.counts + 0, alive);
    if (alive) {
        o_rays[2 * slot] = o_org;
        o_rays[2 * slot + 1] = o_dir;
        o_pixel[slot] = pixel;
        o_rng[slot] = rng.state;
        o_thr[slot] = f4(thr, __int_as_float(pl));
        o_w[slot] = make_float4(dVC, dVCM, dVM, 0.0f);
    }
}

// Integrator::estimate_pixel_size (integrator.cpp:14-70): for every 8th pixel in x and y, rays
// through the raster points (x, y), (x+1, y), (x, y+1), (x+1, y+1) (x outer, y inner).
__global__ void pixel_probe_rays_kernel(const float* r2w, const float* cam_pos, int nx, int ny, float4* rays) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nx * ny) return;
    const int x = (q / ny) * 8, y = (q % ny) * 8;
    for (int c = 0; c < 4; ++c) {
        const float sx = (float)(x + (c & 1)), sy = (float)(y + (c >> 1));
        const float* m = r2w;
        const float t0 = m[0] * sy + m[1] * sx + m[2] * 0.0f + m[3] * 1.0f;
        const float t1 = m[4] * sy + m[5] * sx + m[6] * 0.0f + m[7] * 1.0f;
        const float t2 = m[8] * sy + m[9] * sx + m[10] * 0.0f + m[11] * 1.0f;
        const float t3 = m[12] * sy + m[13] * sx + m[14] * 0.0f + m[15] * 1.0f;
        const V3 w(t0 / t3, t1 / t3, t2 / t3);
        const V3 d = normalize(w - V3(cam_pos[0], cam_pos[1], cam_pos[2]));
        rays[2 * (4 * q + c) + 0] = make_float4(cam_pos[0], cam_pos[1], cam_pos[2], 0.0f);
        rays[2 * (4 * q + c) + 1] = make_float4(d.x, d.y, d.z, FLT_MAX);
    }
}

// The four distances between the hit points of a probe quad (p0-p1, p1-p3, p3-p2, p2-p0), or
// a negative first entry when a ray missed.
__global__ void pixel_probe_dist_kernel(const float4* rays, const int4* hits, int n_quads, float4* out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_quads) return;
    V3 p[4];
    bool all = true;
    for (int c = 0; c < 4; ++c) {
        const int4 h = hits[4 * q + c];
        all = all && h.x >= 0;
        const float4 o = rays[2 * (4 * q + c)], d = rays[2 * (4 * q + c) + 1];
        p[c] = __int_as_float(h.z) * V3(d.x, d.y, d.z) + V3(o.x, o.y, o.z);
    }
    if (!all) { out[q] = make_float4(-1.0f, 0.0f, 0.0f, 0.0f); return; }
    out[q] = make_float4(length(p[0] - p[1]), length(p[1] - p[3]), length(p[3] - p[2]), length(p[2] - p[0]));
}

template <typename T>
bool grow(T** p, long long* cap, long long need, long long keep = 0) {
    if (*cap >= need) return true;
    const long long n = std::max(need, *cap * 3 / 2);
    T* q = nullptr;
    if (!ok(cudaMalloc((void**)&q, sizeof(T) * (size_t)std::max(n, 1ll)), "cudaMalloc")) return false;
    if (keep > 0 && *p && !ok(cudaMemcpy(q, *p, sizeof(T) * (size_t)keep, cudaMemcpyDeviceToDevice), "cudaMemcpy")) {
        cudaFree(q);
        return false;
    }
    cudaFree(*p);
    *p = q;
    *cap = n;
    return true;
}

template <typename T>
bool realloc_exact(T** ptr, size_t elems) {
    cudaFree(*ptr);
    *ptr = nullptr;
    return ok(cudaMalloc((void**)ptr, std::max<size_t>(elems, 1) * sizeof(T)), "cudaMalloc");
}

}  // namespace
}  // namespace imbart

namespace imbart {
namespace {
// Scratch of the pixel-size estimate: camera, probe rays and hits, per-query distances.
struct PixelProbe {
    float* cam = nullptr;
    float4* rays = nullptr;
    int4* hits = nullptr;
    float4* dist = nullptr;
    long long cap = 0;
    std::vector<float4> host;
    void release() {
        cudaFree(cam); cudaFree(rays); cudaFree(hits); cudaFree(dist);
        cam = nullptr; rays = nullptr; hits = nullptr; dist = nullptr; cap = 0;
    }
};
}  // namespace
}  // namespace imbart

struct imbart_vcm {
    imbart::PixelProbe probe;
    int device = 0;
    // light-path slots
    long long l_cap = 0;
    float4* l_rays = nullptr;
    int4* l_hits = nullptr;
    unsigned long long* l_rng = nullptr;
    float4* l_thr = nullptr;
    float4* l_w = nullptr;
    // second set of path states, for the stable compaction of the live slots
    float4* l_rays2 = nullptr;
    unsigned long long* l_rng2 = nullptr;
    float4* l_thr2 = nullptr;
    float4* l_w2 = nullptr;
    float4* stage = nullptr;
    int* vflags = nullptr;
    int* bsums = nullptr;
    imbart::LightTile* d_tiles = nullptr;
    long long tiles_cap = 0;
    // vertex cache (7 float4 per vertex) and its photon grid
    float4* cache = nullptr;
    long long cache_cap = 0;        // float4s
    int cache_count = 0;
    imbart_hashgrid* grid = nullptr;
    bool grid_built = false;
    // camera queues
    long long c_cap = 0;
    float4* c_rays[2] = {nullptr, nullptr};
    int* c_pixel[2] = {nullptr, nullptr};
    unsigned long long* c_rng[2] = {nullptr, nullptr};
    float4* c_thr[2] = {nullptr, nullptr};
    float4* c_w[2] = {nullptr, nullptr};
    int4* c_hits = nullptr;
    float4* c_merge = nullptr;      // queued camera vertices for merging (7 float4 each)
    // Material grouping of a wavefront (keys, shading order, 8 counts then offsets per tile).
    long long sort_cap = 0;
    bool use_perm = false;
    uint8_t* keys = nullptr;
    int* perm = nullptr;
    int* tile_counts = nullptr;
    // shadow queue
    long long s_cap = 0;
    float4* s_rays = nullptr;
    int4* s_hits = nullptr;
    int* s_pixel = nullptr;
    float4* s_contrib = nullptr;
    int* counts = nullptr;
    int* host_counts = nullptr;     // pinned
    // iteration state
    int iteration = 0;
    float pm_radius = 0.0f, eta_vc = 0.0f, eta_vm = 0.0f;
};

namespace imbart {
namespace {

void free_vcm(imbart_vcm* v) {
    void* ptrs[] = {v->keys, v->perm, v->tile_counts,
                    v->l_rays, v->l_hits, v->l_rng, v->l_thr, v->l_w, v->l_rays2, v->l_rng2, v->l_thr2, v->l_w2,
                    v->stage, v->vflags, v->bsums, v->d_tiles,
                    v->cache, v->c_hits, v->c_merge, v->s_rays, v->s_hits, v->s_pixel, v->s_contrib, v->counts};
    for (void* p : ptrs) cudaFree(p);
    for (int k = 0; k < 2; ++k) {
        void* q[] = {v->c_rays[k], v->c_pixel[k], v->c_rng[k], v->c_thr[k], v->c_w[k]};
        for (void* p : q) cudaFree(p);
    }
    cudaFreeHost(v->host_counts);
    if (v->grid) imbart_hashgrid_destroy(v->grid);
    v->probe.release();
}

bool valid_settings(const imbart_vcm_settings* st) {
    return st && st->algorithm >= IMBART_VCM && st->algorithm <= IMBART_VCM_PT && st->spp > 0 &&
           st->max_path_len >= 1 && st->light_path_count > 0 && st->num_connections >= 0 && st->num_knn >= 1 &&
           st->num_knn <= kGridMaxK && st->light_tile_size >= 0 && st->base_radius > 0.0f &&
           st->radius_exponent >= 0.0f && (st->grid_cell_factor == 0.0f || st->grid_cell_factor >= 1.0f) &&
           st->grid_table_size >= 0;
}

bool ensure_shadow(imbart_vcm* v, long long need) {
    if (v->s_cap >= need) return true;
    need = std::max(need, v->s_cap * 3 / 2);   // geometric growth: reallocation synchronizes the device
    const bool good = realloc_exact(&v->s_rays, 2 * (size_t)need) && realloc_exact(&v->s_hits, (size_t)need) &&
                      realloc_exact(&v->s_pixel, (size_t)need) && realloc_exact(&v->s_contrib, (size_t)need);
    v->s_cap = good ? need : 0;
    return good;
}

// The shading order of a wavefront of n paths: keys from `key_launch(keys)`, then the stable
// counting sort into v->perm (pt::launch_grouping).
template <typename KeyLaunch>
bool group_paths(imbart_vcm* v, const imbart_shading* sh, int n, cudaStream_t s, KeyLaunch key_launch) {
    v->use_perm = __builtin_popcount(sh->kind_mask) > 1;    // one kind: nothing to group
    if (!v->use_perm) return true;
    if (v->sort_cap < n) {
        const long long c = std::max<long long>(n, v->sort_cap * 3 / 2);
        const bool good = realloc_exact(&v->keys, (size_t)c) && realloc_exact(&v->perm, (size_t)c) &&
                          realloc_exact(&v->tile_counts, (size_t)pt::kShadeKeys * pt::group_tiles(c));
        v->sort_cap = good ? c : 0;
        if (!good) return false;
    }
    key_launch(v->keys);
    pt::launch_grouping(v->keys, n, nullptr, v->tile_counts, v->perm, s);
    note_launches(1);
    return ok(cudaGetLastError(), "grouping kernels");
}

VcmParams make_params(const imbart_vcm* v, const imbart_shading* sh, const imbart_camera* cam,
                      const imbart_vcm_settings* st, float* image) {
    VcmParams p{};
    p.s = sh->s;
    p.algo = st->algorithm;
    p.width = cam->width;
    p.height = cam->height;
    p.max_path_len = st->max_path_len;
    p.num_connections = st->num_connections;
    p.num_knn = st->num_knn;
    p.light_path_count = st->light_path_count;
    p.eta_vc = v->eta_vc;
    p.eta_vm = v->eta_vm;
    p.pm_radius = v->pm_radius;
    p.base_radius = st->base_radius;
    std::memcpy(p.w2r, cam->world_to_raster, sizeof(p.w2r));
    std::memcpy(p.r2w, cam->raster_to_world, sizeof(p.r2w));
    std::memcpy(p.cam_pos, cam->pos, sizeof(p.cam_pos));
    std::memcpy(p.cam_dir, cam->dir, sizeof(p.cam_dir));
    p.img_plane_dist = cam->img_plane_dist;
    p.cache = v->cache;
    p.cache_count = v->cache_count;
    // LightVertices::count() / (light_path_count * num_connections) (vcm.cpp:491)
    p.vc_weight = st->num_connections > 0
                      ? (float)v->cache_count / (float(st->light_path_count) * float(st->num_connections))
                      : 0.0f;
    p.image = image;
    p.counts = v->counts;
    if (v->grid_built) {
        const void* sorted = nullptr;
        int table = 0, n = 0;
        if (hashgrid_device_view(v->grid, &sorted, &p.grid_ends, &p.grid_params, &table, &n)) {
            p.grid_sorted = static_cast<const float4*>(sorted);
            p.grid_table = (unsigned)table;
            p.merging = n > 0 ? 1 : 0;
        }
    }
    return p;
}

// UniformLightTileGen (tile_gen.h:101-177): paths per light (the remainder to light 0) split
// into tiles of `desired` paths; a last partial tile exists when it exceeds desired / 2 or is
// the light's only tile, and takes all remaining paths. Tile t's queue fill draws seed
// seed + t * step.
std::vector<LightTile> light_tiles(int light_count, int path_count, int desired, unsigned long long seed,
                                   unsigned long long step) {
    std::vector<int> rays(light_count, path_count / light_count);
    rays[0] += path_count % light_count;
    std::vector<LightTile> out;
    int first = 0, t = 0;
    for (int l = 0; l < light_count; ++l) {
        int tiles = rays[l] / desired;
        if ((rays[l] % desired) > desired / 2 || tiles == 0) tiles++;
        for (int k = 0; k < tiles; ++k) {
            const int count = (k == tiles - 1) ? rays[l] - k * desired : desired;
            out.push_back(LightTile{first, count, l, (unsigned int)(seed + (unsigned long long)t * step)});
            first += count;
            ++t;
        }
    }
    return out;
}

int build_grid(imbart_vcm* v, const imbart_vcm_settings* st, cudaStream_t s) {
    v->grid_built = false;
    if ((st->algorithm != IMBART_VCM && st->algorithm != IMBART_PPM) || v->cache_count == 0) return 0;
    // LightVertices::build (light_vertices.h:70-75): HashGrid::build(radius) over the cache.
    // The reference's cell of 2r and 2n buckets unless the settings choose others.
    const float cell_factor = st->grid_cell_factor > 0.0f ? st->grid_cell_factor : 2.0f;
    const int rc = imbart_hashgrid_build(v->grid, reinterpret_cast<const float*>(v->cache), 28, v->cache_count,
                                         v->pm_radius, cell_factor, st->grid_table_size, s);
    v->grid_built = rc == 0;
    return rc;
}

// Integrator::estimate_pixel_size (integrator.cpp:14-70) with caller-owned scratch buffers.
int estimate_pixel_size(const imbart_scene* scene, const imbart_camera* cam, float* pixel_size, cudaStream_t s,
                        PixelProbe& pb) {
    if (!scene || !cam || !pixel_size || cam->width <= 0 || cam->height <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_estimate_pixel_size: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    const int nx = (cam->width + 7) / 8, ny = (cam->height + 7) / 8, nq = nx * ny;
    bool good = true;
    if (!pb.cam) good = ok(cudaMalloc((void**)&pb.cam, sizeof(float) * 19), "cudaMalloc");
    if (good && pb.cap < nq) {
        const long long c = std::max<long long>(nq, pb.cap * 3 / 2);
        good = realloc_exact(&pb.rays, 8 * (size_t)c) && realloc_exact(&pb.hits, 4 * (size_t)c) &&
               realloc_exact(&pb.dist, (size_t)c);
        pb.cap = good ? c : 0;
    }
    pb.host.resize(nq);
    float hcam[19];
    std::memcpy(hcam, cam->raster_to_world, sizeof(float) * 16);
    std::memcpy(hcam + 16, cam->pos, sizeof(float) * 3);
    good = good && ok(cudaMemcpyAsync(pb.cam, hcam, sizeof(hcam), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    if (good) {
        pixel_probe_rays_kernel<<<(nq + 127) / 128, 128, 0, s>>>(pb.cam, pb.cam + 16, nx, ny, pb.rays);
        note_launches(1);
        good = launch_trace_internal(scene, pb.rays, pb.hits, nullptr, 4 * nq, IMBART_TRACE_CLOSEST, s, nullptr) == 0;
    }
    if (good) {
        pixel_probe_dist_kernel<<<(nq + 127) / 128, 128, 0, s>>>(pb.rays, pb.hits, nq, pb.dist);
        note_launches(1);
        good = ok(cudaMemcpyAsync(pb.host.data(), pb.dist, sizeof(float4) * (size_t)nq, cudaMemcpyDeviceToHost, s),
                  "cudaMemcpyAsync") &&
               ok(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    }
    if (!good) return IMBART_ERR_CUDA;
    // The reference's reduction, in its order (one serial range, integrator.cpp:37-59).
    float total = 0.0f;
    int count = 0;
    for (int q = 0; q < nq; ++q) {
        if (pb.host[q].x < 0.0f) continue;
        total += pb.host[q].x;
        total += pb.host[q].y;
        total += pb.host[q].z;
        total += pb.host[q].w;
        count += 4;
    }
    *pixel_size = count == 0 ? 1.0f : total / count;
    return 0;
}

}  // namespace

int vcm_estimate_pixel_size(imbart_vcm* v, const imbart_scene* scene, const imbart_camera* cam, float* pixel_size,
                            void* stream) {
    if (!v) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_estimate_pixel_size: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    return estimate_pixel_size(scene, cam, pixel_size, (cudaStream_t)stream, v->probe);
}

}  // namespace imbart

using namespace imbart;

extern "C" {

imbart_vcm* imbart_vcm_create(int device) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (!ok(cudaSetDevice(device), "cudaSetDevice")) return nullptr;
    imbart_vcm* v = new imbart_vcm;
    v->device = device;
    const bool good = ok(cudaMalloc((void**)&v->counts, sizeof(int) * 4), "cudaMalloc") &&
                      ok(cudaMallocHost((void**)&v->host_counts, sizeof(int) * 4), "cudaMallocHost") &&
                      (v->grid = imbart_hashgrid_create(device)) != nullptr;
    cudaSetDevice(prev);
    if (!good) {
        free_vcm(v);
        delete v;
        return nullptr;
    }
    return v;
}

void imbart_vcm_destroy(imbart_vcm* v) {
    if (!v) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(v->device);
    free_vcm(v);
    cudaSetDevice(prev);
    delete v;
}

int imbart_vcm_begin_iteration(imbart_vcm* v, const imbart_vcm_settings* st, int iteration, float* out3) {
    if (!v || !valid_settings(st) || iteration < 1) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_vcm_begin_iteration: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    // vcm.cpp:27-46
    const float radius_alpha = 0.75f;
    v->iteration = iteration;
    const float exponent = st->radius_exponent > 0.0f ? st->radius_exponent : 0.5f * (1.0f - radius_alpha);
    v->pm_radius = st->base_radius / powf(static_cast<float>(iteration), exponent);
    v->pm_radius = std::max(v->pm_radius, 1e-7f);
    const float pi = 3.14159265359f;
    const float eta_vcm = pi * (v->pm_radius * v->pm_radius) * (float)st->light_path_count;
    v->eta_vc = 1.0f / eta_vcm;
    v->eta_vm = st->algorithm == IMBART_BPT ? 0.0f : eta_vcm;
    v->cache_count = 0;
    v->grid_built = false;
    if (out3) { out3[0] = v->pm_radius; out3[1] = v->eta_vc; out3[2] = v->eta_vm; }
    return 0;
}

int imbart_vcm_light_pass(imbart_vcm* v, const imbart_scene* scene, const imbart_shading* sh,
                          const imbart_camera* cam, const imbart_vcm_settings* st, float* image, long long* stats,
                          void* stream) {
    return imbart_vcm_light_pass_range(v, scene, sh, cam, st, 0, st ? st->light_path_count : 0, image, nullptr, 0,
                                       stats, stream);
}

int imbart_vcm_light_pass_range(imbart_vcm* v, const imbart_scene* scene, const imbart_shading* sh,
                                const imbart_camera* cam, const imbart_vcm_settings* st, int first_path, int n_paths,
                                float* image, int* wave_counts, int wave_cap, long long* stats, void* stream) {
    if (!v || !scene || !sh || !cam || !image || !valid_settings(st) || cam->width <= 0 || cam->height <= 0 ||
        v->iteration < 1 || sh->s.light_count <= 0 || first_path < 0 || n_paths < 0 ||
        (long long)first_path + n_paths > st->light_path_count || wave_cap < 0 || (wave_cap > 0 && !wave_counts)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_vcm_light_pass: invalid argument (begin the iteration first)");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (stats) { stats[0] = 0; stats[1] = 0; stats[2] = 0; }
    for (int k = 0; k < wave_cap; ++k) wave_counts[k] = 0;
    v->cache_count = 0;
    v->grid_built = false;
    if (st->algorithm == IMBART_VCM_PT || n_paths == 0) return 0;   // the VCM path tracer traces no light paths
    cudaStream_t s = (cudaStream_t)stream;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(v->device);
    const int P_total = st->light_path_count;
    const int P = n_paths;        // slots of this call: paths first_path + slot
    const int desired = st->light_tile_size > 0 ? st->light_tile_size : P_total;
    const std::vector<LightTile> tiles =
        light_tiles(sh->s.light_count, P_total, desired, st->light_seed, st->light_seed_step);
    bool good = true;
    if (v->l_cap < P) {
        const long long c = std::max<long long>(P, v->l_cap * 3 / 2);
        const long long cb = (c + kScanTile - 1) / kScanTile;
        good = realloc_exact(&v->l_rays, 2 * (size_t)c) && realloc_exact(&v->l_hits, (size_t)c) &&
               realloc_exact(&v->l_rng, (size_t)c) && realloc_exact(&v->l_thr, (size_t)c) &&
               realloc_exact(&v->l_w, (size_t)c) && realloc_exact(&v->l_rays2, 2 * (size_t)c) &&
               realloc_exact(&v->l_rng2, (size_t)c) && realloc_exact(&v->l_thr2, (size_t)c) &&
               realloc_exact(&v->l_w2, (size_t)c) && realloc_exact(&v->stage, 7 * (size_t)c) &&
               realloc_exact(&v->vflags, (size_t)c) && realloc_exact(&v->bsums, (size_t)cb + 1);
        v->l_cap = good ? c : 0;
    }
    if (good && v->tiles_cap < (long long)tiles.size()) {
        good = realloc_exact(&v->d_tiles, tiles.size());
        v->tiles_cap = good ? (long long)tiles.size() : 0;
    }
    good = good && ensure_shadow(v, P);
    if (!good) { cudaSetDevice(prev); return IMBART_ERR_OUT_OF_MEMORY; }
    if (!ok(cudaMemcpyAsync(v->d_tiles, tiles.data(), sizeof(LightTile) * tiles.size(), cudaMemcpyHostToDevice, s),
            "cudaMemcpyAsync")) {
        cudaSetDevice(prev);
        return IMBART_ERR_CUDA;
    }
    VcmParams p = make_params(v, sh, cam, st, image);
    const int grid = (P + 127) / 128;
    light_gen_kernel<<<grid, 128, 0, s>>>(p, v->d_tiles, (int)tiles.size(), first_path, P, v->l_rays, v->l_rng,
                                          v->l_thr, v->l_w);
    note_launches(1);
    int rc = 0;
    long long n_closest = 0, n_shadow = 0, n_waves = 0;
    int live = P;
    int n = P;   // slots in use: the live paths after the last compaction, in path order
    while (live > 0 && !rc) {
        if (live <= n / 2) {
            // At most half the slots are live: compact them (stable) so that this and later
            // wavefronts launch over the live paths only.
            const int nb = (n + kScanTile - 1) / kScanTile;
            live_flags_kernel<<<(n + 255) / 256, 256, 0, s>>>(v->l_thr, n, v->vflags);
            flag_count_kernel<<<nb, kScanBlock, 0, s>>>(v->vflags, n, v->bsums);
            block_scan_kernel<<<1, kScanBlock, 0, s>>>(v->bsums, nb);
            compact_paths_kernel<<<nb, kScanBlock, 0, s>>>(v->vflags, n, v->bsums, v->l_rays, v->l_rng, v->l_thr,
                                                           v->l_w, v->l_rays2, v->l_rng2, v->l_thr2, v->l_w2);
            note_launches(4);
            std::swap(v->l_rays, v->l_rays2);
            std::swap(v->l_rng, v->l_rng2);
            std::swap(v->l_thr, v->l_thr2);
            std::swap(v->l_w, v->l_w2);
            n = live;
        }
        const int grid_n = (n + 127) / 128;
        const int n_blocks_n = (n + kScanTile - 1) / kScanTile;
        rc = launch_trace_internal(scene, v->l_rays, v->l_hits, nullptr, n, IMBART_TRACE_CLOSEST, s, nullptr);
        if (rc) break;
        n_closest += live;
        ++n_waves;
        // Room for up to n new vertices before the wavefront appends.
        if (!grow(&v->cache, &v->cache_cap, 7ll * (v->cache_count + (long long)n), 7ll * v->cache_count)) {
            rc = IMBART_ERR_OUT_OF_MEMORY;
            break;
        }
        p.cache = v->cache;
        if (!ok(cudaMemsetAsync(v->counts, 0, sizeof(int) * 4, s), "cudaMemsetAsync")) { rc = IMBART_ERR_CUDA; break; }
        if (!group_paths(v, sh, n, s, [&](uint8_t* keys) {
                light_key_kernel<<<(n + 255) / 256, 256, 0, s>>>(p.s, v->l_hits, v->l_thr, n, keys);
            })) {
            rc = IMBART_ERR_CUDA;
            break;
        }
        light_shade_kernel<<<grid_n, 128, 0, s>>>(p, n, v->l_rays, v->l_hits, v->l_rng, v->l_thr, v->l_w, v->stage,
                                                  v->vflags, v->s_rays, v->s_pixel, v->s_contrib,
                                                  v->use_perm ? v->perm : nullptr);
        flag_count_kernel<<<n_blocks_n, kScanBlock, 0, s>>>(v->vflags, n, v->bsums);
        block_scan_kernel<<<1, kScanBlock, 0, s>>>(v->bsums, n_blocks_n);
        vertex_scatter_kernel<<<n_blocks_n, kScanBlock, 0, s>>>(v->vflags, n, v->bsums, v->stage, v->cache,
                                                                v->cache_count);
        note_launches(4);
        rc = launch_trace_internal(scene, v->s_rays, v->s_hits, nullptr, n, IMBART_TRACE_ANY, s, nullptr, nullptr,
                                   v->counts + 1);
        if (rc) break;
        vcm_shadow_kernel<<<grid_n, 128, 0, s>>>(v->counts + 1, v->s_hits, v->s_pixel, v->s_contrib, image);
        note_launches(1);
        if (!ok(cudaGetLastError(), "light pass kernels") ||
            !ok(cudaMemcpyAsync(v->host_counts, v->counts, sizeof(int) * 3, cudaMemcpyDeviceToHost, s),
                "cudaMemcpyAsync") ||
            !ok(cudaMemcpyAsync(v->host_counts + 3, v->bsums + n_blocks_n, sizeof(int), cudaMemcpyDeviceToHost, s),
                "cudaMemcpyAsync") ||
            !ok(cudaStreamSynchronize(s), "cudaStreamSynchronize")) {
            rc = IMBART_ERR_CUDA;
            break;
        }
        n_shadow += v->host_counts[1];
        v->cache_count += v->host_counts[3];
        if (n_waves <= wave_cap) wave_counts[n_waves - 1] = v->host_counts[3];
        live = v->host_counts[2];
    }
    if (!rc) rc = build_grid(v, st, s);
    if (stats) { stats[0] = n_closest; stats[1] = n_shadow; stats[2] = n_waves; }
    cudaSetDevice(prev);
    return rc;
}

int imbart_vcm_light_vertices(imbart_vcm* v, const float** vertices, int* count) {
    if (!v || !vertices || !count) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_vcm_light_vertices: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    *vertices = reinterpret_cast<const float*>(v->cache);
    *count = v->cache_count;
    return 0;
}

int imbart_vcm_copy_light_vertices(imbart_vcm* v, float* host_out, int capacity) {
    if (!v || capacity < 0 || (capacity > 0 && !host_out)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_vcm_copy_light_vertices: invalid argument");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    const int n = std::min(capacity, v->cache_count);
    if (n > 0) {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(v->device);
        const bool good = ok(cudaMemcpy(host_out, v->cache, sizeof(float) * 28 * (size_t)n, cudaMemcpyDeviceToHost),
                             "cudaMemcpy");
        cudaSetDevice(prev);
        if (!good) return -IMBART_ERR_CUDA;
    }
    return capacity == 0 ? v->cache_count : n;
}

int imbart_vcm_load_light_vertices(imbart_vcm* v, const imbart_vcm_settings* st, const float* vertices, int count,
                                   void* stream) {
    if (!v || !valid_settings(st) || count < 0 || (count > 0 && !vertices) || v->iteration < 1) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_vcm_load_light_vertices: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(v->device);
    int rc = 0;
    if (!grow(&v->cache, &v->cache_cap, 7ll * std::max(count, 1))) rc = IMBART_ERR_OUT_OF_MEMORY;
    if (!rc && count > 0 &&
        !ok(cudaMemcpyAsync(v->cache, vertices, sizeof(float) * 28 * (size_t)count, cudaMemcpyDefault, s),
            "cudaMemcpyAsync"))
        rc = IMBART_ERR_CUDA;
    v->cache_count = rc ? 0 : count;
    if (!rc) rc = build_grid(v, st, s);
    cudaSetDevice(prev);
    return rc;
}

int imbart_vcm_camera_pass(imbart_vcm* v, const imbart_scene* scene, const imbart_shading* sh,
                           const imbart_camera* cam, const imbart_vcm_settings* st, float* image,
                           long long max_paths_in_flight, long long* stats, void* stream) {
    const long long total = cam && st ? (long long)cam->width * cam->height * st->spp : 0;
    return imbart_vcm_camera_pass_range(v, scene, sh, cam, st, 0, total, image, max_paths_in_flight, stats, stream);
}

int imbart_vcm_camera_pass_range(imbart_vcm* v, const imbart_scene* scene, const imbart_shading* sh,
                                 const imbart_camera* cam, const imbart_vcm_settings* st, long long first_sample,
                                 long long n_samples, float* image, long long max_paths_in_flight, long long* stats,
                                 void* stream) {
    if (!v || !scene || !sh || !cam || !image || !valid_settings(st) || cam->width <= 0 || cam->height <= 0 ||
        v->iteration < 1 || first_sample < 0 || n_samples < 0 ||
        first_sample + n_samples > (long long)cam->width * cam->height * st->spp) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_vcm_camera_pass: invalid argument (begin the iteration first)");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (stats) { stats[0] = 0; stats[1] = 0; stats[2] = 0; }
    if (st->algorithm == IMBART_LT) return 0;   // light tracing has no camera paths
    cudaStream_t s = (cudaStream_t)stream;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(v->device);
    const long long total = n_samples;
    const int per = 1 + st->num_connections;
    long long chunk = max_paths_in_flight > 0 ? max_paths_in_flight : (8ll << 20);
    chunk = std::min(chunk, total);
    chunk = std::min(chunk, (long long)(1 << 28));
    chunk = std::min(chunk, 0x7fffffffll / per);          // shadow rays of a wavefront fit an int
    bool good = true;
    if (v->c_cap < chunk) {
        const long long c = std::max(chunk, v->c_cap * 3 / 2);
        for (int k = 0; k < 2 && good; ++k)
            good = realloc_exact(&v->c_rays[k], 2 * (size_t)c) && realloc_exact(&v->c_pixel[k], (size_t)c) &&
                   realloc_exact(&v->c_rng[k], (size_t)c) && realloc_exact(&v->c_thr[k], (size_t)c) &&
                   realloc_exact(&v->c_w[k], (size_t)c);
        good = good && realloc_exact(&v->c_hits, (size_t)c) && realloc_exact(&v->c_merge, (size_t)kMergeRec * c);
        v->c_cap = good ? c : 0;
    }
    good = good && ensure_shadow(v, chunk * per);
    if (!good) { cudaSetDevice(prev); return IMBART_ERR_OUT_OF_MEMORY; }
    const VcmParams p = make_params(v, sh, cam, st, image);
    long long n_closest = 0, n_shadow = 0, n_waves = 0;
    int rc = 0;
    for (long long first = 0; first < total && !rc; first += chunk) {
        int n = (int)std::min(chunk, total - first);
        int cur = 0;
        vcm_camera_kernel<<<(n + 127) / 128, 128, 0, s>>>(p, st->camera_seed, st->spp, first_sample + first, n,
                                                         v->c_rays[cur],
                                                         v->c_pixel[cur], v->c_rng[cur], v->c_thr[cur], v->c_w[cur]);
        note_launches(1);
        while (n > 0 && !rc) {
            rc = launch_trace_internal(scene, v->c_rays[cur], v->c_hits, nullptr, n, IMBART_TRACE_CLOSEST, s, nullptr);
            if (rc) break;
            n_closest += n;
            ++n_waves;
            if (!ok(cudaMemsetAsync(v->counts, 0, sizeof(int) * 4, s), "cudaMemsetAsync")) { rc = IMBART_ERR_CUDA; break; }
            const int nxt = 1 - cur;
            if (!group_paths(v, sh, n, s, [&](uint8_t* keys) {
                    pt::shade_key_kernel<<<(n + 255) / 256, 256, 0, s>>>(p.s, v->c_hits, n, nullptr, keys);
                })) {
                rc = IMBART_ERR_CUDA;
                break;
            }
            vcm_camera_shade_kernel<<<(n + 127) / 128, 128, 0, s>>>(
                p, n, v->c_rays[cur], v->c_hits, v->c_pixel[cur], v->c_rng[cur], v->c_thr[cur], v->c_w[cur],
                v->c_rays[nxt], v->c_pixel[nxt], v->c_rng[nxt], v->c_thr[nxt], v->c_w[nxt], v->s_rays, v->s_pixel,
                v->s_contrib, v->c_merge, v->use_perm ? v->perm : nullptr);
            note_launches(1);
            if (p.merging && (st->algorithm == IMBART_VCM || st->algorithm == IMBART_PPM)) {
                if (st->num_knn <= 32)   // one warp per queued vertex
                    vcm_merge_warp_kernel<<<(int)(((long long)n * 32 + 127) / 128), 128, 0, s>>>(p, v->counts + 3,
                                                                                               v->c_merge);
                else
                    vcm_merge_kernel<<<(n + 127) / 128, 128, 0, s>>>(p, v->counts + 3, v->c_merge);
                note_launches(1);
            }
            const int bound = n * per;
            rc = launch_trace_internal(scene, v->s_rays, v->s_hits, nullptr, bound, IMBART_TRACE_ANY, s, nullptr,
                                       nullptr, v->counts + 1);
            if (rc) break;
            vcm_shadow_kernel<<<(bound + 127) / 128, 128, 0, s>>>(v->counts + 1, v->s_hits, v->s_pixel, v->s_contrib,
                                                                   image);
            note_launches(1);
            if (!ok(cudaGetLastError(), "camera pass kernels") ||
                !ok(cudaMemcpyAsync(v->host_counts, v->counts, sizeof(int) * 2, cudaMemcpyDeviceToHost, s),
                    "cudaMemcpyAsync") ||
                !ok(cudaStreamSynchronize(s), "cudaStreamSynchronize")) {
                rc = IMBART_ERR_CUDA;
                break;
            }
            n_shadow += v->host_counts[1];
            n = v->host_counts[0];
            cur = nxt;
        }
    }
    if (stats) { stats[0] = n_closest; stats[1] = n_shadow; stats[2] = n_waves; }
    cudaSetDevice(prev);
    return rc;
}

int imbart_vcm_render(imbart_vcm* v, const imbart_scene* scene, const imbart_shading* sh, const imbart_camera* cam,
                      const imbart_vcm_settings* st, int iteration, float* image, long long max_paths_in_flight,
                      long long* stats, void* stream) {
    int rc = imbart_vcm_begin_iteration(v, st, iteration, nullptr);
    long long a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
    if (!rc) rc = imbart_vcm_light_pass(v, scene, sh, cam, st, image, a, stream);
    if (!rc) rc = imbart_vcm_camera_pass(v, scene, sh, cam, st, image, max_paths_in_flight, b, stream);
    if (stats)
        for (int k = 0; k < 3; ++k) stats[k] = a[k] + b[k];
    return rc;
}

int imbart_estimate_pixel_size(const imbart_scene* scene, const imbart_camera* cam, float* pixel_size, void* stream) {
    PixelProbe probe;
    const int rc = estimate_pixel_size(scene, cam, pixel_size, (cudaStream_t)stream, probe);
    probe.release();
    return rc;
}

}  // extern "C"
