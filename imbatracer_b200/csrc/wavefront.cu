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
// run with a tile at least as large as the image. By default the bounce loop of a sample
// range runs as a CUDA graph whose kernels read their queue sizes on the device (see
// build_range_graph); the host-driven loop remains for measurement and on request.
//
// This file is compiled with -fmad=false (see build.py): the shading arithmetic rounds like
// the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "imbart_internal.h"
#include "pt_kernels.cuh"

using imbart::Rng;
using namespace imbart::sh;
using namespace imbart::pt;

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
    uint8_t* keys = nullptr;                 // material grouping: key per path
    int* perm = nullptr;                     // shading order
    int* tile_counts = nullptr;              // grouping sort: 8 counts (then offsets) per tile
    // The bounce loop of one sample range as a CUDA graph, replayed once per range.
    int graphs = -1;                         // -1: IMBART_PT_GRAPH (default 2); 0 host loop, 1 graph, 2 forked graph
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> graph_key;    // the launch parameters the graph was built with
    int graph_kernels = 0;                   // kernel launches per replay
    int graph_bounces = 0;                   // range state sized for this many bounces
    long long* range_state = nullptr;        // next sample, per-slot totals, waves; then the range's counts
    int* graph_work = nullptr;               // (next, done) counters of the graph's traversal launches
    CameraParams* camera = nullptr;          // the frame's camera and seeding, copied in before the replays
    // Forked form: a second shadow queue, so that a bounce's shadow rays are traced beside the
    // next bounce's closest hits.
    float4* srays2 = nullptr;
    int4* shits2 = nullptr;
    int* spixel2 = nullptr;
    float4* scontrib2 = nullptr;
};

namespace imbart {
namespace {

bool ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? IMBART_ERR_OUT_OF_MEMORY : IMBART_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
    return false;
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
    cudaFree(c->keys); cudaFree(c->perm); cudaFree(c->tile_counts);
    c->keys = nullptr; c->perm = nullptr; c->tile_counts = nullptr;
    cudaFree(c->srays2); cudaFree(c->shits2); cudaFree(c->spixel2); cudaFree(c->scontrib2);
    c->srays2 = nullptr; c->shits2 = nullptr; c->spixel2 = nullptr; c->scontrib2 = nullptr;
    c->cap = 0;
}

// Grouping of each wavefront's paths by material before shading: IMBART_PT_SORT=0 turns it
// off (for comparison); on by default.
bool sort_by_material() {
    static const int v = [] {
        const char* e = std::getenv("IMBART_PT_SORT");
        return e && *e ? std::atoi(e) : 1;
    }();
    return v != 0;
}

bool ensure_capacity(imbart_pt_context* c, long long n) {
    if (c->cap >= n) return true;
    free_ctx_buffers(c);
    bool good = true;
    for (int k = 0; k < 2 && good; ++k)
        good = dev_alloc(&c->rays[k], 2 * n) && dev_alloc(&c->pixel[k], n) && dev_alloc(&c->rng[k], n) &&
               dev_alloc(&c->thr[k], n) && dev_alloc(&c->bounces[k], n);
    good = good && dev_alloc(&c->hits, n) && dev_alloc(&c->srays, 2 * n) && dev_alloc(&c->shits, n) &&
           dev_alloc(&c->spixel, n) && dev_alloc(&c->scontrib, n) && dev_alloc(&c->keys, n) &&
           dev_alloc(&c->perm, n) && dev_alloc(&c->tile_counts, (size_t)kShadeKeys * group_tiles(n));
    if (!good) { free_ctx_buffers(c); return false; }
    c->cap = n;
    c->graph_key.clear();   // the frame graph names the old buffers
    return true;
}

// How the bounce loop runs: 0 driven from the host, 1 as a CUDA graph (one chain of
// launches), 2 as a CUDA graph whose shadow-ray work (each bounce's any-hit launch and
// accumulation) runs on a branch beside the next bounce's closest-hit launch (measured best:
// the launches fill each other's tails). The caller's choice, else IMBART_PT_GRAPH, else 2.
int graph_mode(const imbart_pt_context* c) {
    if (c->graphs >= 0) return c->graphs;
    static const int v = [] {
        const char* e = std::getenv("IMBART_PT_GRAPH");
        const int x = e && *e ? std::atoi(e) : 2;
        return x < 0 || x > 2 ? 2 : x;
    }();
    return v;
}

// ---------------------------------------------------------------------------------------
// The bounce loop as a CUDA graph. The host loop reads each wavefront's queue sizes back
// before it launches the next wavefront (one synchronization per bounce). Captured, every
// kernel of a sample range reads its queue size on the device instead and walks its queue
// with a grid stride: camera samples, then per bounce b < max_path_len the closest-hit
// launch, the material grouping, the shading launch, the any-hit launch and the shadow
// accumulation, each sized for the largest queue; a bounce whose queue is empty costs a few
// microseconds of launches that exit at once. The range state (next sample index, the
// range's queue sizes, totals for the statistics) lives on the device, so the same graph is
// replayed once per range and the frame runs without host synchronization.
//
// Range state: [0] first sample of the next range, [1 + k] total of count slot k over the
// ranges, [1 + n_slots] wavefronts traced; then n_slots ints: slot 2b = paths entering
// bounce b, slot 2b + 3 = shadow rays of bounce b.
// ---------------------------------------------------------------------------------------
__global__ void range_begin_kernel(const long long* first, int* counts, int n_slots, long long total,
                                   long long chunk) {
    const long long left = total - *first;
    const int n = (int)(left < chunk ? left : chunk);
    for (int k = threadIdx.x; k < n_slots; k += blockDim.x) counts[k] = k == 0 ? n : 0;
}

__global__ void range_end_kernel(long long* state, const int* counts, int n_slots, int bounces, long long chunk) {
    for (int k = threadIdx.x; k < n_slots; k += blockDim.x) state[1 + k] += counts[k];
    if (threadIdx.x == 0) {
        int waves = 0;
        for (int b = 0; b < bounces; ++b) waves += counts[2 * b] > 0;
        state[1 + n_slots] += waves;
        state[0] += chunk;
    }
}

// Everything the graph's kernels take into their parameters: equal keys, same graph. The
// camera and the seed are read on the device, so a new view or seed replays the same graph.
struct FrameGraphKey {
    unsigned long long scene[12];
    ShadingScene s;
    float* image;
    long long total, chunk;
    int max_path_len, rr_start, group, fork, trace_cfg[10];
};

std::vector<unsigned char> frame_key(const imbart_scene* scene, const imbart_shading* sh, float* image, long long total,
                                     long long chunk, int max_path_len, int rr_start, bool group, bool fork) {
    FrameGraphKey k;
    std::memset(&k, 0, sizeof(k));
    scene_launch_key(scene, k.scene);
    std::memcpy(&k.s, &sh->s, sizeof(k.s));
    k.image = image;
    k.total = total;
    k.chunk = chunk;
    k.max_path_len = max_path_len;
    k.rr_start = rr_start;
    k.group = group ? 1 : 0;
    k.fork = fork ? 1 : 0;
    trace_config_snapshot(k.trace_cfg);
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&k);
    return std::vector<unsigned char>(b, b + sizeof(k));
}

bool ensure_range_state(imbart_pt_context* c, int bounces, cudaStream_t st) {
    if (!c->camera && !ok(cudaMalloc((void**)&c->camera, sizeof(CameraParams)), "cudaMalloc")) return false;
    if (c->graph_bounces >= bounces) return true;
    cudaFree(c->range_state);
    cudaFree(c->graph_work);
    c->range_state = nullptr;
    c->graph_work = nullptr;
    c->graph_bounces = 0;
    c->graph_key.clear();
    const int n_slots = 2 * bounces + 2;
    const size_t state_bytes = sizeof(long long) * (n_slots + 2) + sizeof(int) * n_slots;
    if (!ok(cudaMalloc((void**)&c->range_state, state_bytes), "cudaMalloc") ||
        !ok(cudaMalloc((void**)&c->graph_work, sizeof(int) * 4 * bounces), "cudaMalloc") ||
        !ok(cudaMemsetAsync(c->graph_work, 0, sizeof(int) * 4 * bounces, st), "cudaMemsetAsync"))
        return false;
    c->graph_bounces = bounces;
    return true;
}

int device_sms(int device) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return std::max(sms, 1);
}

// Explicit construction of a graph's kernel nodes. The graph is built with the graph API, not
// by stream capture: a capture in progress would make device-wide synchronization by any other
// thread of the process (cudaDeviceSynchronize, cudaFree) fail and invalidate the capture.
struct GraphBuilder {
    cudaGraph_t graph = nullptr;
    int kernels = 0;
    bool good = true;

    // Adds kernel `k` with the given arguments after `deps` (null nodes are skipped).
    template <typename... KArgs, typename... Args>
    cudaGraphNode_t kernel(std::initializer_list<cudaGraphNode_t> deps, void (*k)(KArgs...), dim3 grid, dim3 block,
                           Args&&... args) {
        if (!good) return nullptr;
        return add(deps, (const void*)k, grid, block, std::tuple<KArgs...>(std::forward<Args>(args)...),
                   std::index_sequence_for<KArgs...>{});
    }

    template <typename Tuple, size_t... I>
    cudaGraphNode_t add(std::initializer_list<cudaGraphNode_t> deps, const void* func, dim3 grid, dim3 block,
                        Tuple args, std::index_sequence<I...>) {
        void* ptrs[] = {(void*)&std::get<I>(args)..., nullptr};
        std::vector<cudaGraphNode_t> d;
        for (cudaGraphNode_t x : deps)
            if (x) d.push_back(x);
        cudaKernelNodeParams np{};
        np.func = const_cast<void*>(func);
        np.gridDim = grid;
        np.blockDim = block;
        np.kernelParams = ptrs;
        cudaGraphNode_t node = nullptr;
        good = ok(cudaGraphAddKernelNode(&node, graph, d.data(), d.size(), &np), "cudaGraphAddKernelNode");
        kernels += good ? 1 : 0;
        return good ? node : nullptr;
    }

    cudaGraphNode_t trace(std::initializer_list<cudaGraphNode_t> deps, const imbart_scene* scene, const void* rays,
                          void* hits, int bound, int flags, const int* count_ptr, int* work) {
        if (!good) return nullptr;
        std::vector<cudaGraphNode_t> d;
        for (cudaGraphNode_t x : deps)
            if (x) d.push_back(x);
        cudaGraphNode_t node = nullptr;
        good = add_trace_node(graph, d.data(), (int)d.size(), &node, scene, rays, hits, bound, flags, count_ptr,
                              work) == 0;
        kernels += good ? 1 : 0;
        return good ? node : nullptr;
    }
};

// Builds the bounce loop of one sample range (`chunk` samples at most) into ctx->exec.
int build_range_graph(imbart_pt_context* ctx, const imbart_scene* scene, const imbart_shading* sh, int max_path_len,
                  int rr_start, float* image, long long total, long long chunk, bool group, bool fork) {
    const int sms = device_sms(ctx->device);
    // Shading: one thread per entry of the queue's bound, blocks past the queue's size doing
    // nothing. (A block-stride loop over one wave measured no faster: the loop costs the
    // shading kernel registers, 86 instead of 71, or spills under a 7-block bound.)
    const int shade_grid = (int)((chunk + 127) / 128);
    const int small_grid = 16 * sms;
    const int n = (int)chunk;
    const int n_slots = 2 * max_path_len + 2;
    long long* state = ctx->range_state;
    int* counts = reinterpret_cast<int*>(state + n_slots + 2);
    if (fork && !ctx->srays2 &&
        !(dev_alloc(&ctx->srays2, 2 * chunk) && dev_alloc(&ctx->shits2, chunk) && dev_alloc(&ctx->spixel2, chunk) &&
          dev_alloc(&ctx->scontrib2, chunk)))
        return IMBART_ERR_OUT_OF_MEMORY;
    GraphBuilder gb;
    if (!ok(cudaGraphCreate(&gb.graph, 0), "cudaGraphCreate")) return IMBART_ERR_CUDA;
    cudaGraphNode_t main = gb.kernel({}, range_begin_kernel, dim3(1), dim3(64), state, counts, n_slots, total, chunk);
    main = gb.kernel({main}, camera_range_kernel, dim3(small_grid), dim3(128), ctx->camera, state, counts,
                     ctx->rays[0], ctx->pixel[0], ctx->rng[0], ctx->thr[0], ctx->bounces[0]);
    // Shadow-ray work: on the main chain, or (forked) on a branch of its own beside the next
    // bounce's closest hits; acc[b] = accumulation node of bounce b.
    std::vector<cudaGraphNode_t> acc(max_path_len, nullptr);
    cudaGraphNode_t side = nullptr;
    int cur = 0;
    for (int b = 0; b < max_path_len && gb.good; ++b) {
        const int* n_in = counts + 2 * b;
        int* out = counts + 2 * b + 2;   // [0] next paths, [1] shadow rays
        main = gb.trace({main}, scene, ctx->rays[cur], ctx->hits, n,
                        b == 0 ? (IMBART_TRACE_CLOSEST | IMBART_TRACE_COHERENT) : IMBART_TRACE_CLOSEST, n_in,
                        ctx->graph_work + 4 * b);
        ShadeParams p{};
        p.s = sh->s;
        p.n = n;
        p.n_ptr = n_in;
        p.max_path_len = max_path_len;
        p.rr_start = rr_start;
        p.rays = ctx->rays[cur]; p.hits = ctx->hits; p.pixel = ctx->pixel[cur]; p.rng = ctx->rng[cur];
        p.thr = ctx->thr[cur]; p.bounces = ctx->bounces[cur];
        const int nxt = 1 - cur;
        p.o_rays = ctx->rays[nxt]; p.o_pixel = ctx->pixel[nxt]; p.o_rng = ctx->rng[nxt];
        p.o_thr = ctx->thr[nxt]; p.o_bounces = ctx->bounces[nxt];
        // Shadow queue of this bounce (the forked form alternates two).
        const bool second = fork && (b & 1);
        float4* srays = second ? ctx->srays2 : ctx->srays;
        int4* shits = second ? ctx->shits2 : ctx->shits;
        int* spixel = second ? ctx->spixel2 : ctx->spixel;
        float4* scontrib = second ? ctx->scontrib2 : ctx->scontrib;
        p.s_rays = srays; p.s_pixel = spixel; p.s_contrib = scontrib;
        p.counts = out;
        p.image = image;
        if (group) {
            main = gb.kernel({main}, shade_key_kernel, dim3(small_grid), dim3(256), sh->s, ctx->hits, n, n_in,
                             ctx->keys);
            const int tiles = group_tiles(n);
            main = gb.kernel({main}, group_count_kernel, dim3(tiles), dim3(256), ctx->keys, n, n_in, ctx->tile_counts);
            main = gb.kernel({main}, group_scan_kernel, dim3(1), dim3(1024), ctx->tile_counts, n, n_in);
            main = gb.kernel({main}, group_scatter_kernel, dim3(tiles), dim3(256), ctx->keys, n, n_in,
                             ctx->tile_counts, ctx->perm);
            p.perm = ctx->perm;
        }
        // The shadow queue this bounce fills was last read by the shadow work of bounce b - 2
        // (forked), or of bounce b - 1 (on the main chain already).
        const cudaGraphNode_t reuse = fork && b >= 2 ? acc[b - 2] : nullptr;
        main = gb.kernel({main, reuse}, pt_shade_kernel<false>, dim3(shade_grid), dim3(128), p);
        const cudaGraphNode_t shaded = main;
        cudaGraphNode_t t = gb.trace({shaded, fork ? side : nullptr}, scene, srays, shits, n, IMBART_TRACE_ANY,
                                     out + 1, ctx->graph_work + 4 * b + 2);
        t = gb.kernel({t}, shadow_accumulate_kernel<false>, dim3(small_grid), dim3(128), (const int*)(out + 1),
                      (const int4*)shits, (const int*)spixel, (const float4*)scontrib, image, (const int*)nullptr,
                      (const ReqDev*)nullptr);
        acc[b] = t;
        if (fork) side = t;
        else main = t;
        cur = nxt;
    }
    gb.kernel({main, side}, range_end_kernel, dim3(1), dim3(64), state, (const int*)counts, n_slots, max_path_len,
              chunk);
    int rc = gb.good ? 0 : (imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA);
    if (!rc && ctx->exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ctx->exec, gb.graph, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(ctx->exec);
            ctx->exec = nullptr;
        }
    }
    if (!rc && !ctx->exec && !ok(cudaGraphInstantiate(&ctx->exec, gb.graph, 0), "cudaGraphInstantiate")) {
        ctx->exec = nullptr;
        rc = IMBART_ERR_CUDA;
    }
    cudaGraphDestroy(gb.graph);
    ctx->graph_kernels = gb.kernels;
    return rc;
}

// A frame through the bounce-loop graph: the graph is (re)built when a launch parameter
// changed, then replayed once per sample range.
int render_graph(imbart_pt_context* ctx, const imbart_scene* scene, const imbart_shading* sh, const CameraParams& c,
                 int max_path_len, int rr_start, float* image, long long first, long long total, long long chunk,
                 bool group, bool fork, long long* stats, cudaStream_t st) {
    if (!ensure_range_state(ctx, max_path_len, st)) return IMBART_ERR_OUT_OF_MEMORY;
    std::vector<unsigned char> key = frame_key(scene, sh, image, total, chunk, max_path_len, rr_start, group, fork);
    if (!ctx->exec || key != ctx->graph_key) {
        ctx->graph_key.clear();
        const int rc = build_range_graph(ctx, scene, sh, max_path_len, rr_start, image, total, chunk, group, fork);
        if (rc) return rc;
        ctx->graph_key = std::move(key);
    }
    const int n_slots = 2 * max_path_len + 2;
    // A copy from pageable memory is staged before the call returns: `c` may go out of scope.
    // The ranges cover samples [first, total): state[0] is the first sample of the next range.
    if (!ok(cudaMemcpyAsync(ctx->camera, &c, sizeof(CameraParams), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync") ||
        !ok(cudaMemsetAsync(ctx->range_state, 0, sizeof(long long) * (n_slots + 2), st), "cudaMemsetAsync") ||
        (first != 0 &&
         !ok(cudaMemcpyAsync(ctx->range_state, &first, sizeof(long long), cudaMemcpyHostToDevice, st),
             "cudaMemcpyAsync")))
        return IMBART_ERR_CUDA;
    const long long ranges = (total - first + chunk - 1) / chunk;
    for (long long r = 0; r < ranges; ++r)
        if (!ok(cudaGraphLaunch(ctx->exec, st), "cudaGraphLaunch")) return IMBART_ERR_CUDA;
    note_launches((int)(ctx->graph_kernels * ranges));
    if (stats) {
        std::vector<long long> tot(n_slots + 2);
        if (!ok(cudaMemcpyAsync(tot.data(), ctx->range_state, sizeof(long long) * tot.size(), cudaMemcpyDeviceToHost,
                                st), "cudaMemcpyAsync") ||
            !ok(cudaStreamSynchronize(st), "cudaStreamSynchronize"))
            return IMBART_ERR_CUDA;
        long long closest = 0, shadow = 0;
        for (int b = 0; b < max_path_len; ++b) { closest += tot[1 + 2 * b]; shadow += tot[1 + 2 * b + 3]; }
        stats[0] = closest; stats[1] = shadow; stats[2] = tot[1 + n_slots];
    }
    return 0;
}

}  // namespace
}  // namespace imbart

using namespace imbart;

extern "C" {

imbart_shading* imbart_shading_create_ex(int device, const float* vertices, int n_vertices, const float* normals,
                                         const float* texcoords, const int* tris, const float* geom_normals,
                                         int n_tris, const float* inst_inv, int n_inst, const int* mat_kind,
                                         const float* mat_params, int n_mats, const int* light_kinds,
                                         const float* lights_in, int n_lights, const float* env_color,
                                         const float* bsphere, const int* tex_dims, const float* tex_pixels,
                                         int n_textures) {
    if (!vertices || !normals || !texcoords || !tris || !geom_normals || !inst_inv || !mat_kind || !mat_params ||
        n_vertices <= 0 || n_tris <= 0 || n_inst <= 0 || n_mats <= 0 || n_lights < 0 ||
        (n_lights > 0 && !lights_in) || (n_lights == 0 && !env_color) || !valid_light_kinds(light_kinds, n_lights) ||
        n_textures < 0 || (n_textures > 0 && (!tex_dims || !tex_pixels))) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_shading_create: invalid argument");
        return nullptr;
    }
    std::vector<int4> tex_info(std::max(n_textures, 1), make_int4(0, 0, 0, 0));
    long long texels = 0;
    for (int t = 0; t < n_textures; ++t) {
        if (tex_dims[2 * t] <= 0 || tex_dims[2 * t + 1] <= 0 || texels + (long long)tex_dims[2 * t] * tex_dims[2 * t + 1] > INT_MAX) {
            set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_shading_create: invalid texture size");
            return nullptr;
        }
        tex_info[t] = make_int4((int)texels, tex_dims[2 * t], tex_dims[2 * t + 1], 0);
        texels += (long long)tex_dims[2 * t] * tex_dims[2 * t + 1];
    }
    const std::vector<Material> mats = decode_materials(mat_kind, mat_params, n_mats, n_textures > 0);
    for (const Material& m : mats)
        if (m.tex >= n_textures || m.bump >= n_textures) {
            set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_shading_create: texture index out of range");
            return nullptr;
        }
    const std::vector<LightSrc> lights = decode_lights(light_kinds, lights_in, n_lights);
    int prev = 0;
    cudaGetDevice(&prev);
    if (!ok(cudaSetDevice(device), "cudaSetDevice")) return nullptr;
    imbart_shading* h = new imbart_shading;
    h->device = device;
    h->kind_mask = material_kind_mask(mats);
    ShadingScene& s = h->s;
    auto upl = [&](const void* src, size_t bytes) -> void* {
        void* d = nullptr;
        if (!ok(cudaMalloc(&d, std::max<size_t>(bytes, 16)), "cudaMalloc")) return nullptr;
        h->allocations.push_back(d);
        if (bytes > 0 && !ok(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy")) return nullptr;
        return d;
    };
    s.vertices = (const float*)upl(vertices, sizeof(float) * 3 * (size_t)n_vertices);
    s.normals = (const float*)upl(normals, sizeof(float) * 3 * (size_t)n_vertices);
    s.texcoords = (const float*)upl(texcoords, sizeof(float) * 2 * (size_t)n_vertices);
    s.tris = (const int4*)upl(tris, sizeof(int4) * (size_t)n_tris);
    s.geom_normals = (const float*)upl(geom_normals, sizeof(float) * 3 * (size_t)n_tris);
    s.inst_inv = (const float*)upl(inst_inv, sizeof(float) * 12 * (size_t)n_inst);
    Material* dmats = (Material*)upl(mats.data(), sizeof(Material) * mats.size());
    LightSrc* dlights = (LightSrc*)upl(lights.data(), sizeof(LightSrc) * lights.size());
    s.tex_pixels = (const float4*)upl(tex_pixels, sizeof(float4) * (size_t)texels);
    s.tex_info = (const int4*)upl(tex_info.data(), sizeof(int4) * tex_info.size());
    s.n_textures = n_textures;
    s.materials = dmats;
    s.n_materials = n_mats;
    s.lights = dlights;
    s.n_lights = n_lights;
    s.has_env = env_color ? 1 : 0;
    s.light_count = n_lights + s.has_env;
    for (int k = 0; k < 3; ++k) s.env_color[k] = env_color ? env_color[k] : 0.0f;
    for (int k = 0; k < 5; ++k) s.bsphere[k] = bsphere ? bsphere[k] : 0.0f;
    const bool good = s.vertices && s.normals && s.texcoords && s.tris && s.geom_normals && s.inst_inv && dmats &&
                      dlights && s.tex_pixels && s.tex_info;
    if (good) {
        if (n_lights > 0) setup_lights_kernel<<<(n_lights + 127) / 128, 128>>>(dlights, n_lights);
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

imbart_shading* imbart_shading_create(int device, const float* vertices, int n_vertices, const float* normals,
                                      const float* texcoords, const int* tris, const float* geom_normals, int n_tris,
                                      const float* inst_inv, int n_inst, const int* mat_kind,
                                      const float* mat_params, int n_mats, const float* tri_lights,
                                      int n_tri_lights, const float* env_color, const float* bsphere) {
    return imbart_shading_create_ex(device, vertices, n_vertices, normals, texcoords, tris, geom_normals, n_tris,
                                    inst_inv, n_inst, mat_kind, mat_params, n_mats, nullptr, tri_lights, n_tri_lights,
                                    env_color, bsphere, nullptr, nullptr, 0);
}

int imbart_shading_set_env_map(imbart_shading* h, int texture, float intensity) {
    if (!h || texture < 0 || texture >= h->s.n_textures || !(intensity >= 0.0f)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_shading_set_env_map: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (!h->s.has_env) {
        h->s.has_env = 1;
        h->s.light_count += 1;
    }
    h->s.env_map = texture + 1;
    h->s.env_intensity = intensity;
    return 0;
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
    if (c->exec) cudaGraphExecDestroy(c->exec);
    cudaFree(c->range_state);
    cudaFree(c->graph_work);
    cudaFree(c->camera);
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

int imbart_pt_render_range(imbart_pt_context* ctx, const imbart_scene* scene, const imbart_shading* sh,
                           const float* raster_to_world, const float* cam_pos, int width, int height, int spp,
                           int max_path_len, int rr_start, unsigned long long seed_base, float* image,
                           long long max_paths_in_flight, long long first_sample, long long n_samples,
                           long long* stats, void* stream) {
    if (!ctx || !scene || !sh || !raster_to_world || !cam_pos || !image || width <= 0 || height <= 0 || spp <= 0 ||
        max_path_len < 1 || first_sample < 0 || n_samples <= 0 ||
        first_sample > (long long)width * height * spp - n_samples) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_pt_render: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // Samples [first_sample, total) of the frame's width * height * spp sample indices.
    const long long total = first_sample + n_samples;
    long long chunk = max_paths_in_flight > 0 ? max_paths_in_flight : (16ll << 20);
    chunk = std::min(chunk, n_samples);
    chunk = std::min(chunk, (long long)(1 << 30));
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(ctx->device);
    if (!ensure_capacity(ctx, chunk)) { cudaSetDevice(prev); return IMBART_ERR_OUT_OF_MEMORY; }
    CameraParams c;
    std::memset(&c, 0, sizeof(c));
    std::memcpy(c.r2w, raster_to_world, sizeof(c.r2w));
    std::memcpy(c.pos, cam_pos, sizeof(c.pos));
    c.width = width; c.height = height; c.spp = spp;
    c.tile_left = 0; c.tile_top = 0; c.tile_w = width; c.full_w = width;
    c.seed_base = seed_base;
    long long n_closest = 0, n_shadow = 0, n_waves = 0;
    int rc = 0;
    imbart_pt_profile* prof = ctx->profile;
    const bool group = sort_by_material() && __builtin_popcount(sh->kind_mask) > 1;
    const int mode = graph_mode(ctx);
    if (!prof && mode > 0) {
        // Measurement (per-launch events, host-side ray counts) keeps the host-driven loop.
        rc = render_graph(ctx, scene, sh, c, max_path_len, rr_start, image, first_sample, total, chunk, group, mode == 2,
                          stats, st);
        cudaSetDevice(prev);
        return rc;
    }
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
        const bool any = (flags & IMBART_TRACE_ANY) != 0;
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
    for (long long first = first_sample; first < total && !rc; first += chunk) {
        int n = (int)std::min(chunk, total - first);
        int cur = 0;
        camera_kernel<<<(n + 127) / 128, 128, 0, st>>>(c, first, n, ctx->rays[cur], ctx->pixel[cur], ctx->rng[cur],
                                                       ctx->thr[cur], ctx->bounces[cur], nullptr);
        note_launches(1);
        bool camera_rays = true;   // the first wavefront of a sample range: coherent camera rays
        while (n > 0) {
            rc = trace(ctx->rays[cur], ctx->hits, n,
                       camera_rays ? (IMBART_TRACE_CLOSEST | IMBART_TRACE_COHERENT) : IMBART_TRACE_CLOSEST);
            camera_rays = false;
            if (rc) break;
            n_closest += n;
            ++n_waves;
            if (!ok(cudaMemsetAsync(ctx->counts, 0, sizeof(int) * 2, st), "cudaMemsetAsync")) { rc = IMBART_ERR_CUDA; break; }
            ShadeParams p{};
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
            if (group) {
                // Group the wavefront's paths by material kind before shading.
                shade_key_kernel<<<(n + 255) / 256, 256, 0, st>>>(sh->s, ctx->hits, n, nullptr, ctx->keys);
                launch_grouping(ctx->keys, n, nullptr, ctx->tile_counts, ctx->perm, st);
                note_launches(1);
                p.perm = ctx->perm;
            }
            pt_shade_kernel<false><<<(n + 127) / 128, 128, 0, st>>>(p);
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
                shadow_accumulate_kernel<false><<<(n_sh + 127) / 128, 128, 0, st>>>(
                    ctx->counts + 1, ctx->shits, ctx->spixel, ctx->scontrib, image, nullptr, nullptr);
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

int imbart_pt_render(imbart_pt_context* ctx, const imbart_scene* scene, const imbart_shading* sh,
                     const float* raster_to_world, const float* cam_pos, int width, int height, int spp,
                     int max_path_len, int rr_start, unsigned long long seed_base, float* image,
                     long long max_paths_in_flight, long long* stats, void* stream) {
    if (width <= 0 || height <= 0 || spp <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_pt_render: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    return imbart_pt_render_range(ctx, scene, sh, raster_to_world, cam_pos, width, height, spp, max_path_len,
                                  rr_start, seed_base, image, max_paths_in_flight, 0,
                                  (long long)width * height * spp, stats, stream);
}

int imbart_group_by_key(const unsigned char* keys, int n, int* perm, void* stream) {
    if (n < 0 || (n > 0 && (!keys || !perm))) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_group_by_key: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    int* tiles = nullptr;
    if (!ok(cudaMallocAsync((void**)&tiles, sizeof(int) * kShadeKeys * group_tiles(n), st), "cudaMallocAsync"))
        return IMBART_ERR_OUT_OF_MEMORY;
    launch_grouping(keys, n, nullptr, tiles, perm, st);
    const bool good = ok(cudaGetLastError(), "grouping kernels");
    cudaFreeAsync(tiles, st);
    return good ? 0 : IMBART_ERR_CUDA;
}

int imbart_pt_set_graphs(imbart_pt_context* ctx, int enable) {
    if (!ctx || enable < -1 || enable > 2) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_pt_set_graphs: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    ctx->graphs = enable;
    return 0;
}

int imbart_pt_set_profile(imbart_pt_context* ctx, imbart_pt_profile* profile) {
    if (!ctx) { set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_pt_set_profile"); return IMBART_ERR_INVALID_ARGUMENT; }
    ctx->profile = profile;
    return 0;
}

}  // extern "C"
