// Request server: continuous batching of path-traced frames and ray batches on one GPU.
//
// The reference renders one frame per process (its TileScheduler / QueueScheduler loops,
// tile_scheduler.h:100-144, queue_scheduler.h:177-275, fill a queue, trace, shade, repeat);
// serving many requests is new here. The server keeps that loop but feeds it from many
// requests at once:
//
//  * Scene residency. Every resident scene occupies one block of a single device pool:
//    [8-wide nodes | triangles | instances | shading arrays]. Node, triangle and instance
//    indices are rebased on upload so that they index the pool itself in units of their own
//    record size; the traversal kernels then serve rays of any resident scene in one launch,
//    each ray starting at its scene's root. Blocks start at multiples of 3840 bytes (the
//    least common multiple of the 80, 48 and 64-byte record sizes and 256), so every array of
//    a block starts on a record boundary of the pool. When the pool is full the least
//    recently used scene without outstanding requests is evicted.
//  * Wavefronts. Between wavefronts the worker admits requests in arrival order (scene
//    resident, accumulation image allocated in the pool), tops the path queue up with new
//    camera samples shared max-min fairly among the admitted renders, and gathers ray-batch
//    rays. Each wavefront is then one closest-hit launch, one shading launch, one any-hit
//    launch and one accumulation launch over the paths of every request (plus one launch per
//    query type for the ray batches), followed by one host synchronization that reads the
//    next queue size and each request's count of finished paths. A render request is done
//    when all its samples were generated and as many paths finished.
//  * Completion. Finished images are copied to the caller's buffer by a completion thread on
//    its own stream, overlapping the next wavefronts.
//
//  * VCM-family frames (VCM, BPT, PPM, LT, VCM-PT) keep a light-vertex cache and a photon
//    grid per iteration, so they are not merged into the path-tracing wavefronts. Admitted
//    ones are advanced by a few VCM lanes (threads, each with its own stream and VCM
//    context): a lane takes the request at the head of the round robin, renders one iteration
//    (imbart_vcm_render on the pool's copy of its scene) and puts it back. Small frames are
//    latency-bound (one host synchronization per wavefront), so several lanes keep the GPU
//    busy where one request alone cannot.
//
// The plain mode runs the same requests one at a time through imbart_pt_render /
// imbart_trace / imbart_vcm_render, for comparison on the same GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "hashgrid_query.cuh"
#include "imbart_internal.h"
#include "pt_kernels.cuh"

using namespace imbart;
using namespace imbart::pt;
using namespace imbart::sh;

namespace imbart {
namespace {

constexpr size_t kBlockAlign = 3840;        // lcm(80, 48, 64, 256)
constexpr size_t kArrayAlign = 256;
constexpr int kMaxReqSlots = 4096;          // admitted requests at once
constexpr int kMaxSceneSlots = 1024;        // resident scenes at once
// Registered scenes. The record vector is reserved once, so the worker threads can read it
// while scenes are added (a push_back never reallocates).
constexpr size_t kMaxScenes = 1 << 16;
constexpr size_t kMaxPoolBytes = 160ull << 30;   // node indices of the pool stay below 2^31

bool cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? IMBART_ERR_OUT_OF_MEMORY : IMBART_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// First-fit allocator over the byte range [0, size) with coalescing of freed ranges.
class RangeAllocator {
public:
    void reset(size_t size) {
        free_.clear();
        if (size) free_[0] = size;
        size_ = size;
        used_ = 0;
    }
    // Returns the offset of `bytes` aligned to `align` and ending at or below `limit`, or
    // SIZE_MAX.
    size_t alloc(size_t bytes, size_t align, size_t limit = SIZE_MAX) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            const size_t start = align_up(it->first, align), end = it->first + it->second;
            if (start + bytes > limit) break;
            if (start + bytes > end) continue;
            const size_t off = it->first;
            free_.erase(it);
            if (start > off) free_[off] = start - off;
            if (start + bytes < end) free_[start + bytes] = end - (start + bytes);
            used_ += bytes;
            return start;
        }
        return SIZE_MAX;
    }
    void release(size_t off, size_t bytes) {
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t used() const { return used_; }
    size_t size() const { return size_; }

private:
    std::map<size_t, size_t> free_;
    size_t size_ = 0, used_ = 0;
};

// Adds the block's index offsets to a scene's node, triangle and instance references.
// Top-level nodes (the last `n_top` of the node array) reference instances, the others
// triangles.
__global__ void rebase_kernel(WideNode* nodes, int n_nodes, int n_top, uint32_t node_off, uint32_t tri_off,
                              uint32_t inst_off, WideInst* insts, int n_insts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_nodes) {
        nodes[i].child_base += node_off;
        nodes[i].prim_base += (i >= n_nodes - n_top) ? inst_off : tri_off;
    }
    if (i < n_insts) insts[i].root += (int32_t)node_off;
}

// Root node of each ray of a gathered ray batch: runs of equal roots.
struct RootRun {
    int begin;
    int root;
};

__global__ void fill_roots_kernel(const RootRun* runs, int n_runs, int n, int* roots) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int lo = 0, hi = n_runs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (runs[mid].begin <= j) lo = mid;
        else hi = mid - 1;
    }
    roots[j] = runs[lo].root;
}

enum class MemKind { Device, Pinned, Pageable };

MemKind mem_kind(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return MemKind::Pageable;
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return MemKind::Device;
    if (a.type == cudaMemoryTypeHost) return MemKind::Pinned;
    return MemKind::Pageable;
}

// VCM lanes of a batched server: IMBART_SERVE_VCM_LANES, default 4.
int env_lanes() {
    const char* e = std::getenv("IMBART_SERVE_VCM_LANES");
    return e && *e ? std::atoi(e) : 4;
}

// A share of the resident block slots from the environment: a finite number in (0, 1];
// anything else (unset, text, NaN, out of range) gives `dflt`.
float env_share(const char* name, float dflt) {
    const char* e = std::getenv(name);
    if (!e || !*e) return dflt;
    char* end = nullptr;
    const float v = std::strtof(e, &end);
    if (end == e || *end != '\0' || !std::isfinite(v) || !(v > 0.0f) || v > 1.0f) return dflt;
    return v;
}

double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

struct SceneRec {
    HostWideScene wide;
    std::vector<float> vertices, normals, texcoords, geom_normals, inst_inv, mat_params, tri_lights, tex_pixels;
    std::vector<int> mesh_tris, mat_kind, light_kinds, tex_dims;
    std::vector<Material> mats;
    std::vector<LightSrc> lights;
    std::vector<int4> tex_info;
    int n_tri_lights = 0;     // lights of every kind
    int n_textures = 0;
    bool has_env = false;
    float env[3] = {0, 0, 0};
    int env_map = 0;              // 1 + environment image texture, 0: constant
    unsigned kind_mask = 0;       // material kinds present (bit per kind)
    float env_intensity = 0.0f;
    float bsphere[5] = {0, 0, 0, 0, 0};
    // Block layout (byte offsets from the block start).
    size_t bytes = 0, o_nodes = 0, o_tris = 0, o_insts = 0, o_vert = 0, o_nrm = 0, o_tc = 0, o_mtris = 0,
           o_gn = 0, o_inv = 0, o_mats = 0, o_lights = 0, o_tex = 0, o_texinfo = 0;
    // Residency (batched mode).
    bool resident = false;
    size_t block = 0;
    int slot = -1;
    int root = 0;                 // top-level root in the pool
    int start_root = 0;           // per-ray root word: root, or the mesh root | kDirectRootBit
    int direct_root = -1;         // mesh root of a top level that is one identity instance of id 0
    long long last_used = 0;
    int refs = 0;
    // Plain mode.
    imbart_scene* plain_scene = nullptr;
    imbart_shading* plain_shading = nullptr;
};

struct Request {
    long long ticket = 0;
    int kind = 0;                  // 0 render, 1 ray batch, 2 VCM-family frame
    int scene = 0;
    // render
    imbart_render_request rr{};
    long long total = 0, generated = 0;
    // VCM-family frame
    imbart_vcm_request vq{};
    int iter_done = 0;             // iterations finished
    int iter_claimed = 0;          // iterations handed to lanes (several lanes may run one request)
    int iter_running = 0;          // iterations in progress
    int failed = 0;                // first error of an iteration (the last running lane completes it)
    cudaEvent_t ready = nullptr;   // recorded on the worker stream after the scene upload and image clear
    // ray batch
    const imbart_ray* rays = nullptr;
    imbart_hit* hits = nullptr;
    int count = 0, flags = 0, done_rays = 0;
    MemKind rays_kind = MemKind::Pageable, hits_kind = MemKind::Pageable;
    // bookkeeping
    int slot = -1;
    size_t img_off = SIZE_MAX, img_bytes = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int status = 0;
    bool complete = false;
};

// One ray-batch piece gathered into a wavefront.
struct BatchPiece {
    Request* r;
    int src_first;    // first ray of the request
    int dst;          // position in the gathered buffer
    int n;
};

}  // namespace
}  // namespace imbart

struct imbart_server {
    int device = 0;
    int mode = IMBART_SERVE_BATCHED;
    long long cap = 0;                    // paths per wavefront, rays per batch wavefront
    std::chrono::steady_clock::time_point t0;

    // Device pool and tables (batched mode).
    uint8_t* pool = nullptr;
    size_t pool_bytes = 0;
    RangeAllocator alloc;                 // guarded by mu
    imbart_scene* pool_scene = nullptr;   // traversal view of the pool
    ReqDev* d_reqs = nullptr;
    ReqDev* h_reqs = nullptr;             // pinned mirror
    ShadingScene* d_scenes = nullptr;
    ShadingScene* h_scenes = nullptr;     // pinned mirror
    int* d_terminated = nullptr;
    int* h_terminated = nullptr;          // pinned
    GenChunk* d_chunks = nullptr;
    GenChunk* h_chunks = nullptr;         // pinned
    RootRun* d_runs = nullptr;
    RootRun* h_runs = nullptr;            // pinned
    int* d_counts = nullptr;
    int* h_counts = nullptr;              // pinned
    uint8_t* keys = nullptr;              // material grouping of a wavefront
    int* perm = nullptr;
    int* tile_counts = nullptr;           // grouping sort: 8 counts (then offsets) per tile
    std::vector<int> free_req_slots, free_scene_slots;

    // Path queues (double-buffered), shadow queue, hits.
    float4* rays[2] = {nullptr, nullptr};
    int* pixel[2] = {nullptr, nullptr};
    unsigned long long* rng[2] = {nullptr, nullptr};
    float4* thr[2] = {nullptr, nullptr};
    int* bounces[2] = {nullptr, nullptr};
    int* req[2] = {nullptr, nullptr};
    int* root[2] = {nullptr, nullptr};
    int4* hits = nullptr;
    float4* srays = nullptr;
    int4* shits = nullptr;
    int* spixel = nullptr;
    float4* scontrib = nullptr;
    int* sreq = nullptr;
    int* sroot = nullptr;
    int cur = 0;
    long long n_cur = 0;

    // Ray-batch gather buffers.
    imbart_ray* b_rays = nullptr;
    imbart_hit* b_hits = nullptr;
    int* b_roots = nullptr;
    imbart_ray* stage_rays = nullptr;     // pinned
    imbart_hit* stage_hits = nullptr;     // pinned

    // VCM-family frames: plain mode runs them on the worker thread with lane 0; batched mode
    // runs them on `vcm_lanes` threads of their own, each with its own stream, VCM context and
    // traversal view of the pool.
    struct VcmLane {
        cudaStream_t stream = nullptr;
        imbart_vcm* vcm = nullptr;
        imbart_scene* view = nullptr;
    };
    std::vector<VcmLane> vcm_lanes;
    std::vector<std::thread> vcm_threads;
    std::condition_variable cv_vcm;
    int vcm_running = 0;                  // iterations in progress (their requests are off active_vcm)

    // Plain mode.
    imbart_pt_context* pt = nullptr;
    float* plain_image = nullptr;
    size_t plain_image_bytes = 0;
    imbart_ray* plain_rays = nullptr;
    imbart_hit* plain_hits = nullptr;
    long long plain_ray_cap = 0;

    cudaStream_t stream = nullptr;        // worker
    cudaStream_t copy_stream = nullptr;   // completion thread

    // Scenes and requests.
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::vector<std::unique_ptr<SceneRec>> scenes;
    std::map<long long, std::unique_ptr<Request>> requests;
    std::deque<Request*> incoming;
    long long next_ticket = 1;
    long long outstanding = 0;
    bool stop = false;
    int broken = 0;
    imbart_server_stats stats{};
    long long tick = 0;

    // Worker-only state.
    std::deque<Request*> pending;
    std::vector<Request*> active_renders;
    std::deque<Request*> active_rays;
    std::deque<Request*> active_vcm;

    // Completion thread.
    struct Job {
        Request* r;
        float* dst;
        const float* src;
        size_t bytes;
    };
    std::deque<Job> jobs;
    std::condition_variable cv_jobs;
    std::thread worker, completer;
};

namespace imbart {
namespace {

template <typename T>
bool dalloc(T** p, size_t n) {
    *p = nullptr;
    return cuda_check(cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(n, 1)), "cudaMalloc");
}

template <typename T>
bool halloc(T** p, size_t n) {
    *p = nullptr;
    return cuda_check(cudaMallocHost((void**)p, sizeof(T) * std::max<size_t>(n, 1)), "cudaMallocHost");
}

void layout_scene(SceneRec& s) {
    size_t o = 0;
    s.o_nodes = o; o = align_up(o + s.wide.nodes.size() * sizeof(WideNode), kBlockAlign);
    s.o_tris = o; o = align_up(o + s.wide.tris.size() * sizeof(WideTri), kBlockAlign);
    s.o_insts = o; o = align_up(o + s.wide.insts.size() * sizeof(WideInst), kArrayAlign);
    s.o_vert = o; o = align_up(o + s.vertices.size() * sizeof(float), kArrayAlign);
    s.o_nrm = o; o = align_up(o + s.normals.size() * sizeof(float), kArrayAlign);
    s.o_tc = o; o = align_up(o + s.texcoords.size() * sizeof(float), kArrayAlign);
    s.o_mtris = o; o = align_up(o + s.mesh_tris.size() * sizeof(int), kArrayAlign);
    s.o_gn = o; o = align_up(o + s.geom_normals.size() * sizeof(float), kArrayAlign);
    s.o_inv = o; o = align_up(o + s.inst_inv.size() * sizeof(float), kArrayAlign);
    s.o_mats = o; o = align_up(o + s.mats.size() * sizeof(Material), kArrayAlign);
    s.o_lights = o; o = align_up(o + s.lights.size() * sizeof(LightSrc), kArrayAlign);
    s.o_tex = o; o = align_up(o + s.tex_pixels.size() * sizeof(float), kArrayAlign);
    s.o_texinfo = o; o = align_up(o + s.tex_info.size() * sizeof(int4), kBlockAlign);
    s.bytes = o;
}

void complete_locked(imbart_server* S, Request* r, int status) {
    r->status = status;
    r->t_done = now_ms(S->t0);
    r->complete = true;
    S->outstanding -= 1;
    if (status == 0) S->stats.completed += 1;
    else S->stats.failed += 1;
    S->cv_done.notify_all();
}

// Evicts the least recently used resident scene that no admitted request uses.
bool evict_one_locked(imbart_server* S) {
    SceneRec* victim = nullptr;
    for (auto& sp : S->scenes) {
        SceneRec* s = sp.get();
        if (s->resident && s->refs == 0 && (!victim || s->last_used < victim->last_used)) victim = s;
    }
    if (!victim) return false;
    S->alloc.release(victim->block, victim->bytes);
    S->free_scene_slots.push_back(victim->slot);
    victim->resident = false;
    victim->slot = -1;
    S->stats.scene_evictions += 1;
    return true;
}

// Scene blocks must end below this pool offset: the traversal kernels keep node, triangle
// and instance indices in 30 bits (the stack's entry type takes the top two), and the
// 48-byte triangles reach 2^30 records first.
constexpr size_t kSceneIndexLimit = (size_t(1) << 30) * sizeof(WideTri);

// Allocates pool bytes below `limit`, evicting unused scenes as needed. SIZE_MAX when it
// cannot.
size_t pool_alloc_locked(imbart_server* S, size_t bytes, size_t align, size_t limit = SIZE_MAX) {
    for (;;) {
        const size_t off = S->alloc.alloc(bytes, align, limit);
        if (off != SIZE_MAX) return off;
        if (!evict_one_locked(S)) return SIZE_MAX;
    }
}

// Uploads a scene into a pool block (stream-ordered) and registers its shading table entry.
// Returns 0, 1 when the pool has no room now, or an error code.
int make_resident_locked(imbart_server* S, SceneRec& s) {
    if (s.resident) return 0;
    if (S->free_scene_slots.empty()) return evict_one_locked(S) ? make_resident_locked(S, s) : 1;
    const size_t block = pool_alloc_locked(S, s.bytes, kBlockAlign, kSceneIndexLimit);
    if (block == SIZE_MAX) return 1;
    uint8_t* b = S->pool + block;
    cudaStream_t st = S->stream;
    auto put = [&](size_t off, const void* src, size_t bytes) {
        return bytes == 0 || cuda_check(cudaMemcpyAsync(b + off, src, bytes, cudaMemcpyHostToDevice, st), "upload");
    };
    bool good = put(s.o_nodes, s.wide.nodes.data(), s.wide.nodes.size() * sizeof(WideNode)) &&
                put(s.o_tris, s.wide.tris.data(), s.wide.tris.size() * sizeof(WideTri)) &&
                put(s.o_insts, s.wide.insts.data(), s.wide.insts.size() * sizeof(WideInst)) &&
                put(s.o_vert, s.vertices.data(), s.vertices.size() * sizeof(float)) &&
                put(s.o_nrm, s.normals.data(), s.normals.size() * sizeof(float)) &&
                put(s.o_tc, s.texcoords.data(), s.texcoords.size() * sizeof(float)) &&
                put(s.o_mtris, s.mesh_tris.data(), s.mesh_tris.size() * sizeof(int)) &&
                put(s.o_gn, s.geom_normals.data(), s.geom_normals.size() * sizeof(float)) &&
                put(s.o_inv, s.inst_inv.data(), s.inst_inv.size() * sizeof(float)) &&
                put(s.o_mats, s.mats.data(), s.mats.size() * sizeof(Material)) &&
                put(s.o_lights, s.lights.data(), s.lights.size() * sizeof(LightSrc)) &&
                put(s.o_tex, s.tex_pixels.data(), s.tex_pixels.size() * sizeof(float)) &&
                put(s.o_texinfo, s.tex_info.data(), s.tex_info.size() * sizeof(int4));
    if (!good) {
        S->alloc.release(block, s.bytes);
        return IMBART_ERR_CUDA;
    }
    const uint32_t node_off = (uint32_t)((block + s.o_nodes) / sizeof(WideNode));
    const uint32_t tri_off = (uint32_t)((block + s.o_tris) / sizeof(WideTri));
    const uint32_t inst_off = (uint32_t)((block + s.o_insts) / sizeof(WideInst));
    const int n_nodes = (int)s.wide.nodes.size(), n_insts = (int)s.wide.insts.size();
    const int n = std::max(n_nodes, n_insts);
    WideNode* nodes = reinterpret_cast<WideNode*>(b + s.o_nodes);
    WideInst* insts = reinterpret_cast<WideInst*>(b + s.o_insts);
    rebase_kernel<<<(n + 255) / 256, 256, 0, st>>>(nodes, n_nodes, s.wide.top_nodes, node_off, tri_off, inst_off,
                                                  insts, n_insts);
    Material* mats = reinterpret_cast<Material*>(b + s.o_mats);
    LightSrc* lights = reinterpret_cast<LightSrc*>(b + s.o_lights);
    const int4* mtris = reinterpret_cast<const int4*>(b + s.o_mtris);
    const int n_mtris = (int)(s.mesh_tris.size() / 4);
    const float* verts = reinterpret_cast<const float*>(b + s.o_vert);
    int launches = 1;
    if (s.n_tri_lights > 0) {
        setup_lights_kernel<<<(s.n_tri_lights + 127) / 128, 128, 0, st>>>(lights, s.n_tri_lights);
        ++launches;
    }
    emitter_area_kernel<<<(n_mtris + 127) / 128, 128, 0, st>>>(verts, mtris, n_mtris, mats);
    note_launches(launches + 1);
    const int slot = S->free_scene_slots.back();
    S->free_scene_slots.pop_back();
    ShadingScene& ss = S->h_scenes[slot];
    ss.vertices = verts;
    ss.normals = reinterpret_cast<const float*>(b + s.o_nrm);
    ss.texcoords = reinterpret_cast<const float*>(b + s.o_tc);
    ss.tris = mtris;
    ss.geom_normals = reinterpret_cast<const float*>(b + s.o_gn);
    ss.inst_inv = reinterpret_cast<const float*>(b + s.o_inv);
    ss.materials = mats;
    ss.n_materials = (int)s.mats.size();
    ss.lights = lights;
    ss.n_lights = s.n_tri_lights;
    ss.tex_pixels = reinterpret_cast<const float4*>(b + s.o_tex);
    ss.tex_info = reinterpret_cast<const int4*>(b + s.o_texinfo);
    ss.n_textures = s.n_textures;
    ss.has_env = s.has_env ? 1 : 0;
    ss.light_count = s.n_tri_lights + ss.has_env;
    for (int k = 0; k < 3; ++k) ss.env_color[k] = s.env[k];
    ss.env_map = s.env_map;
    ss.env_intensity = s.env_intensity;
    for (int k = 0; k < 5; ++k) ss.bsphere[k] = s.bsphere[k];
    if (!cuda_check(cudaMemcpyAsync(S->d_scenes + slot, &ss, sizeof(ShadingScene), cudaMemcpyHostToDevice, st),
                    "upload") ||
        !cuda_check(cudaGetLastError(), "scene upload kernels")) {
        S->alloc.release(block, s.bytes);
        S->free_scene_slots.push_back(slot);
        return IMBART_ERR_CUDA;
    }
    s.resident = true;
    s.block = block;
    s.slot = slot;
    s.root = s.wide.root + (int)node_off;
    // A top level that is one identity instance of id 0: rays start in the mesh tree.
    const bool direct = s.wide.insts.size() == 1 && s.wide.insts[0].id == 0 && identity_instance(s.wide.insts[0]);
    s.direct_root = direct ? s.wide.insts[0].root + (int)node_off : -1;
    s.start_root = direct ? (s.direct_root | kDirectRootBit) : s.root;
    S->stats.scene_uploads += 1;
    return 0;
}

void release_request_locked(imbart_server* S, Request* r) {
    if (r->slot >= 0) {
        S->free_req_slots.push_back(r->slot);
        r->slot = -1;
    }
    SceneRec& s = *S->scenes[r->scene];
    s.refs -= 1;
}

// Admission in arrival order; stops at the first request that does not fit now.
void admit(imbart_server* S) {
    std::lock_guard<std::mutex> lk(S->mu);
    while (!S->pending.empty()) {
        Request* r = S->pending.front();
        SceneRec& s = *S->scenes[r->scene];
        if (r->kind == 0 && S->free_req_slots.empty()) break;
        s.refs += 1;           // pins the scene while memory for the image is found
        const int rc = make_resident_locked(S, s);
        if (rc > 1) { s.refs -= 1; S->broken = rc; return; }
        if (rc == 1) {
            s.refs -= 1;
            const bool idle = S->active_renders.empty() && S->active_rays.empty() && S->active_vcm.empty() &&
                              S->vcm_running == 0 && S->n_cur == 0 && S->jobs.empty();
            if (idle) {
                // Nothing left to finish or evict: the scene can never fit.
                S->pending.pop_front();
                set_error(IMBART_ERR_LIMIT, "imbart_server: scene larger than the pool");
                complete_locked(S, r, IMBART_ERR_LIMIT);
                continue;
            }
            break;
        }
        if (r->kind == 2) {
            const size_t bytes = (size_t)r->vq.camera.width * r->vq.camera.height * 3 * sizeof(float);
            const size_t off = pool_alloc_locked(S, bytes, kArrayAlign);
            if (off == SIZE_MAX) {
                s.refs -= 1;
                const bool idle = S->active_renders.empty() && S->active_rays.empty() && S->active_vcm.empty() &&
                                  S->vcm_running == 0 && S->n_cur == 0 && S->jobs.empty();
                if (idle) {
                    S->pending.pop_front();
                    complete_locked(S, r, IMBART_ERR_LIMIT);
                    continue;
                }
                break;
            }
            r->img_off = off;
            r->img_bytes = bytes;
            if (!cuda_check(cudaMemsetAsync(S->pool + off, 0, bytes, S->stream), "cudaMemsetAsync") ||
                !cuda_check(cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming), "cudaEventCreate") ||
                !cuda_check(cudaEventRecord(r->ready, S->stream), "cudaEventRecord")) {
                S->broken = IMBART_ERR_CUDA;
                return;
            }
            S->active_vcm.push_back(r);
            S->cv_vcm.notify_one();
        } else if (r->kind == 0) {
            const size_t bytes = (size_t)r->rr.width * r->rr.height * 3 * sizeof(float);
            const size_t off = pool_alloc_locked(S, bytes, kArrayAlign);
            if (off == SIZE_MAX) {
                s.refs -= 1;
                const bool idle = S->active_renders.empty() && S->active_rays.empty() && S->active_vcm.empty() &&
                                  S->vcm_running == 0 && S->n_cur == 0 && S->jobs.empty();
                if (idle) {
                    S->pending.pop_front();
                    complete_locked(S, r, IMBART_ERR_LIMIT);
                    continue;
                }
                break;
            }
            r->img_off = off;
            r->img_bytes = bytes;
            r->slot = S->free_req_slots.back();
            S->free_req_slots.pop_back();
            ReqDev& d = S->h_reqs[r->slot];
            std::memcpy(d.r2w, r->rr.raster_to_world, sizeof(d.r2w));
            std::memcpy(d.pos, r->rr.cam_pos, sizeof(d.pos));
            d.width = r->rr.width; d.height = r->rr.height; d.spp = r->rr.spp;
            d.max_path_len = r->rr.max_path_len; d.rr_start = r->rr.rr_start;
            d.scene_slot = s.slot; d.root = s.start_root;
            d.seed_base = r->rr.seed_base;
            d.image = reinterpret_cast<float*>(S->pool + off);
            if (!cuda_check(cudaMemsetAsync(d.image, 0, bytes, S->stream), "cudaMemsetAsync") ||
                !cuda_check(cudaMemsetAsync(S->d_terminated + r->slot, 0, sizeof(int), S->stream), "cudaMemsetAsync") ||
                !cuda_check(cudaMemcpyAsync(S->d_reqs + r->slot, &d, sizeof(ReqDev), cudaMemcpyHostToDevice, S->stream),
                            "cudaMemcpyAsync")) {
                S->broken = IMBART_ERR_CUDA;
                return;
            }
            S->active_renders.push_back(r);
        } else {
            S->active_rays.push_back(r);
        }
        s.last_used = ++S->tick;
        r->t_start = now_ms(S->t0);
        S->pending.pop_front();
    }
}

// Max-min fair split of `free_slots` new camera samples over the admitted renders.
int plan_generation(imbart_server* S, long long free_slots) {
    std::vector<Request*> want;
    for (Request* r : S->active_renders)
        if (r->generated < r->total) want.push_back(r);
    std::sort(want.begin(), want.end(), [](const Request* a, const Request* b) {
        return a->total - a->generated < b->total - b->generated;
    });
    int n_chunks = 0;
    long long out = 0;
    for (size_t k = 0; k < want.size() && free_slots > 0; ++k) {
        Request* r = want[k];
        const long long share = free_slots / (long long)(want.size() - k);
        const long long take = std::min(r->total - r->generated, std::max(share, 1ll));
        if (take <= 0) continue;
        GenChunk& c = S->h_chunks[n_chunks++];
        c.first_sample = r->generated;
        c.req = r->slot;
        c.count = (int)take;
        c.out_begin = (int)out;
        c.pad = 0;
        r->generated += take;
        out += take;
        free_slots -= take;
    }
    return n_chunks;
}

bool copy_rays_in(imbart_server* S, const BatchPiece& p) {
    const size_t bytes = (size_t)p.n * sizeof(imbart_ray);
    const imbart_ray* src = p.r->rays + p.src_first;
    if (p.r->rays_kind == MemKind::Pageable) {
        std::memcpy(S->stage_rays + p.dst, src, bytes);
        return cuda_check(cudaMemcpyAsync(S->b_rays + p.dst, S->stage_rays + p.dst, bytes, cudaMemcpyHostToDevice,
                                          S->stream), "cudaMemcpyAsync");
    }
    return cuda_check(cudaMemcpyAsync(S->b_rays + p.dst, src, bytes, cudaMemcpyDefault, S->stream), "cudaMemcpyAsync");
}

bool copy_hits_out(imbart_server* S, const BatchPiece& p) {
    const size_t bytes = (size_t)p.n * sizeof(imbart_hit);
    imbart_hit* dst = p.r->hits + p.src_first;
    if (p.r->hits_kind == MemKind::Pageable)
        return cuda_check(cudaMemcpyAsync(S->stage_hits + p.dst, S->b_hits + p.dst, bytes, cudaMemcpyDeviceToHost,
                                          S->stream), "cudaMemcpyAsync");
    return cuda_check(cudaMemcpyAsync(dst, S->b_hits + p.dst, bytes, cudaMemcpyDefault, S->stream), "cudaMemcpyAsync");
}

// Gathers ray-batch pieces (closest-hit first, then any-hit) up to the wavefront's ray limit.
void plan_batches(imbart_server* S, std::vector<BatchPiece>& pieces, int& n_closest, int& n_any) {
    pieces.clear();
    long long used = 0;
    n_closest = n_any = 0;
    for (int pass = 0; pass < 2; ++pass) {
        for (Request* r : S->active_rays) {
            const bool any = (r->flags & IMBART_TRACE_ANY) != 0;
            if (any != (pass == 1)) continue;
            // Pieces already planned for this request in this wavefront.
            int planned = 0;
            for (const BatchPiece& p : pieces) if (p.r == r) planned += p.n;
            const long long left = (long long)r->count - r->done_rays - planned;
            const long long take = std::min(left, S->cap - used);
            if (take <= 0) continue;
            pieces.push_back(BatchPiece{r, r->done_rays + planned, (int)used, (int)take});
            used += take;
            (pass == 0 ? n_closest : n_any) += (int)take;
        }
    }
}

void fail_all_active(imbart_server* S, int code) {
    std::lock_guard<std::mutex> lk(S->mu);
    for (Request* r : S->active_renders) {
        if (r->img_off != SIZE_MAX) S->alloc.release(r->img_off, r->img_bytes);
        release_request_locked(S, r);
        complete_locked(S, r, code);
    }
    S->active_renders.clear();
    for (Request* r : S->active_rays) {
        release_request_locked(S, r);
        complete_locked(S, r, code);
    }
    S->active_rays.clear();
    for (Request* r : S->active_vcm) {
        if (r->iter_running > 0) {   // a lane still renders into its image: that lane completes it
            if (!r->failed) r->failed = code;
            continue;
        }
        if (r->ready) { cudaEventDestroy(r->ready); r->ready = nullptr; }
        if (r->img_off != SIZE_MAX) S->alloc.release(r->img_off, r->img_bytes);
        release_request_locked(S, r);
        complete_locked(S, r, code);
    }
    S->active_vcm.clear();
    for (Request* r : S->pending) complete_locked(S, r, code);
    S->pending.clear();
    S->n_cur = 0;
}

float serve_grid_share() {
    static const float v = env_share("IMBART_SERVE_GRID_SHARE", 0.75f);
    return v;
}

// One merged wavefront. Returns false when there was nothing to do.
bool batched_wave(imbart_server* S) {
    cudaStream_t st = S->stream;
    admit(S);
    if (S->broken) { fail_all_active(S, S->broken); return true; }
    const int cur = S->cur, nxt = 1 - cur;
    // New camera samples behind the paths still in flight.
    const long long free_slots = S->cap - S->n_cur;
    const int n_chunks = free_slots > 0 ? plan_generation(S, free_slots) : 0;
    int n_gen = 0;
    if (n_chunks > 0) {
        const GenChunk& last = S->h_chunks[n_chunks - 1];
        n_gen = last.out_begin + last.count;
        if (!cuda_check(cudaMemcpyAsync(S->d_chunks, S->h_chunks, sizeof(GenChunk) * n_chunks, cudaMemcpyHostToDevice,
                                        st), "cudaMemcpyAsync")) { S->broken = IMBART_ERR_CUDA; return true; }
        camera_multi_kernel<<<(n_gen + 127) / 128, 128, 0, st>>>(
            S->d_reqs, S->d_chunks, n_chunks, n_gen, (int)S->n_cur, S->rays[cur], S->pixel[cur], S->rng[cur],
            S->thr[cur], S->bounces[cur], S->req[cur], S->root[cur]);
        note_launches(1);
    }
    const int n = (int)(S->n_cur + n_gen);
    // While VCM-family iterations run on the lanes, the merged wavefront's persistent
    // traversal launches leave a share of the SMs to the lanes' launches, which would
    // otherwise wait for whole persistent launches to drain (config-4 mix: 177 -> 188 req/s
    // at a share of 0.75; IMBART_SERVE_GRID_SHARE).
    {
        bool lanes_busy;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            lanes_busy = S->vcm_running > 0 || !S->active_vcm.empty();
        }
        scene_set_grid_share(S->pool_scene, lanes_busy ? serve_grid_share() : 1.0f);
    }
    std::vector<BatchPiece> pieces;
    int n_bc = 0, n_ba = 0;
    plan_batches(S, pieces, n_bc, n_ba);
    if (n == 0 && pieces.empty()) return false;
    bool good = true;
    if (n > 0) {
        good = launch_trace_internal(S->pool_scene, S->rays[cur], S->hits, nullptr, n, IMBART_TRACE_CLOSEST, st,
                                     nullptr, S->root[cur]) == 0 &&
               cuda_check(cudaMemsetAsync(S->d_counts, 0, sizeof(int) * 2, st), "cudaMemsetAsync");
        if (good) {
            ShadeParams p{};
            p.n = n;
            p.rays = S->rays[cur]; p.hits = S->hits; p.pixel = S->pixel[cur]; p.rng = S->rng[cur];
            p.thr = S->thr[cur]; p.bounces = S->bounces[cur];
            p.o_rays = S->rays[nxt]; p.o_pixel = S->pixel[nxt]; p.o_rng = S->rng[nxt];
            p.o_thr = S->thr[nxt]; p.o_bounces = S->bounces[nxt];
            p.s_rays = S->srays; p.s_pixel = S->spixel; p.s_contrib = S->scontrib;
            p.counts = S->d_counts;
            p.reqs = S->d_reqs; p.scenes = S->d_scenes;
            p.req = S->req[cur]; p.root = S->root[cur];
            p.o_req = S->req[nxt]; p.o_root = S->root[nxt]; p.s_req = S->sreq; p.s_root = S->sroot;
            p.terminated = S->d_terminated;
            // Group the paths by material kind (RayQueue::sort_by_material) before shading.
            // Only when the active renders' scenes hold more than one material kind.
            unsigned kinds = 0;
            for (Request* r : S->active_renders) kinds |= S->scenes[r->scene]->kind_mask;
            const bool group = __builtin_popcount(kinds) > 1;
            if (group) {
                shade_key_multi_kernel<<<(n + 255) / 256, 256, 0, st>>>(S->d_reqs, S->d_scenes, S->req[cur], S->hits,
                                                                         n, nullptr, S->keys);
                launch_grouping(S->keys, n, nullptr, S->tile_counts, S->perm, st);
                note_launches(1);
                p.perm = S->perm;
            }
            pt_shade_kernel<true><<<(n + 127) / 128, 128, 0, st>>>(p);
            note_launches(1);
            good = cuda_check(cudaGetLastError(), "shade kernel") &&
                   launch_trace_internal(S->pool_scene, S->srays, S->shits, nullptr, n, IMBART_TRACE_ANY, st, nullptr,
                                         S->sroot, S->d_counts + 1) == 0;
            if (good) {
                shadow_accumulate_kernel<true><<<(n + 127) / 128, 128, 0, st>>>(
                    S->d_counts + 1, S->shits, S->spixel, S->scontrib, nullptr, S->sreq, S->d_reqs);
                note_launches(1);
                good = cuda_check(cudaGetLastError(), "accumulate kernel");
            }
        }
    }
    if (good && !pieces.empty()) {
        // Gather rays and their roots, trace both query types, scatter hits.
        int n_runs = 0;
        for (const BatchPiece& p : pieces) {
            good = good && copy_rays_in(S, p);
            S->h_runs[n_runs++] = RootRun{p.dst, S->scenes[p.r->scene]->start_root};
        }
        const int nb = n_bc + n_ba;
        good = good &&
               cuda_check(cudaMemcpyAsync(S->d_runs, S->h_runs, sizeof(RootRun) * n_runs, cudaMemcpyHostToDevice, st),
                          "cudaMemcpyAsync");
        if (good) {
            fill_roots_kernel<<<(nb + 255) / 256, 256, 0, st>>>(S->d_runs, n_runs, nb, S->b_roots);
            note_launches(1);
        }
        if (good && n_bc > 0)
            good = launch_trace_internal(S->pool_scene, S->b_rays, S->b_hits, nullptr, n_bc, IMBART_TRACE_CLOSEST, st,
                                         nullptr, S->b_roots) == 0;
        if (good && n_ba > 0)
            good = launch_trace_internal(S->pool_scene, S->b_rays + n_bc, S->b_hits + n_bc, nullptr, n_ba,
                                         IMBART_TRACE_ANY, st, nullptr, S->b_roots + n_bc) == 0;
        for (const BatchPiece& p : pieces) good = good && copy_hits_out(S, p);
    }
    // One synchronization: next queue size, shadow count, finished paths per request.
    int max_slot = 0;
    for (Request* r : S->active_renders) max_slot = std::max(max_slot, r->slot + 1);
    good = good &&
           cuda_check(cudaMemcpyAsync(S->h_counts, S->d_counts, sizeof(int) * 2, cudaMemcpyDeviceToHost, st),
                      "cudaMemcpyAsync") &&
           (max_slot == 0 ||
            cuda_check(cudaMemcpyAsync(S->h_terminated, S->d_terminated, sizeof(int) * max_slot,
                                       cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync")) &&
           cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    if (!good) {
        S->broken = IMBART_ERR_CUDA;
        fail_all_active(S, IMBART_ERR_CUDA);
        return true;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->stats.waves += 1;
    if (n > 0) {
        S->stats.closest_rays += n;
        S->stats.shadow_rays += S->h_counts[1];
        S->n_cur = S->h_counts[0];
        S->cur = nxt;
    }
    S->stats.batch_rays += n_bc + n_ba;
    for (const BatchPiece& p : pieces) {
        if (p.r->hits_kind == MemKind::Pageable)
            std::memcpy(p.r->hits + p.src_first, S->stage_hits + p.dst, (size_t)p.n * sizeof(imbart_hit));
        p.r->done_rays += p.n;
    }
    for (auto it = S->active_rays.begin(); it != S->active_rays.end();) {
        Request* r = *it;
        if (r->done_rays >= r->count) {
            release_request_locked(S, r);
            complete_locked(S, r, 0);
            it = S->active_rays.erase(it);
        } else {
            ++it;
        }
    }
    // Finished renders go to the completion thread.
    for (auto it = S->active_renders.begin(); it != S->active_renders.end();) {
        Request* r = *it;
        if (r->generated == r->total && (long long)S->h_terminated[r->slot] == r->total) {
            const float* img = reinterpret_cast<const float*>(S->pool + r->img_off);
            release_request_locked(S, r);
            S->jobs.push_back(imbart_server::Job{r, r->rr.image_host, img, r->img_bytes});
            S->cv_jobs.notify_one();
            it = S->active_renders.erase(it);
        } else {
            ++it;
        }
    }
    return true;
}

// Iteration k + 1 (k = 0, 1, ...) of a VCM-family request: its settings (seeds advanced by
// k * seed_step; the photon radius from the estimated pixel size when the request gave none,
// estimated by the lane that runs iteration 1 before any other lane takes the request)
// rendered by imbart_vcm_render on `scene` / `sh` into `image`. Iterations depend on their
// index only, so several lanes may render iterations of one request at once.
int vcm_iteration(imbart_server* S, imbart_server::VcmLane& lane, Request* r, int k_iter, const imbart_scene* scene,
                  const imbart_shading* sh, float* image, long long* stats) {
    if (!lane.vcm) {
        lane.vcm = imbart_vcm_create(S->device);
        if (!lane.vcm) return imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA;
    }
    imbart_vcm_request& q = r->vq;
    if (!(q.settings.base_radius > 0.0f)) {
        float pixel = 0.0f;
        const int rc = vcm_estimate_pixel_size(lane.vcm, scene, &q.camera, &pixel, lane.stream);
        if (rc) return rc;
        q.settings.base_radius = pixel * q.radius_factor;
        if (!(q.settings.base_radius > 0.0f)) {
            set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server: VCM photon radius is not positive");
            return IMBART_ERR_INVALID_ARGUMENT;
        }
    }
    imbart_vcm_settings st = q.settings;
    const unsigned long long k = (unsigned long long)k_iter;
    st.light_seed = q.settings.light_seed + k * q.seed_step;
    st.camera_seed = q.settings.camera_seed + k * q.seed_step;
    // Camera paths in flight: the frame's samples of one iteration, at most the server's cap.
    const long long paths = std::min<long long>(S->cap, (long long)q.camera.width * q.camera.height * st.spp);
    return imbart_vcm_render(lane.vcm, scene, sh, &q.camera, &st, k_iter + 1, image, paths, stats, lane.stream);
}

// Batched mode: a VCM lane takes the admitted VCM-family request at the head of the round
// robin, claims its next iteration and puts it back at once (so that other lanes can run
// later iterations of it meanwhile: a long request near the end of a batch is spread over
// every lane), renders the iteration on the pool's copy of its scene, and the lane that ends
// the last running iteration hands the finished image to the completion thread. Iteration 1
// goes first alone when the photon radius still has to be estimated.
void vcm_lane_main(imbart_server* S, int index) {
    cudaSetDevice(S->device);
    imbart_server::VcmLane& lane = S->vcm_lanes[index];
    for (;;) {
        Request* r;
        int k = 0;
        bool estimate = false;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_vcm.wait(lk, [&] { return S->stop || !S->active_vcm.empty(); });
            if (S->active_vcm.empty()) return;
            r = S->active_vcm.front();
            S->active_vcm.pop_front();
            if (r->failed || r->iter_claimed >= r->vq.iterations) continue;   // the running lanes complete it
            k = r->iter_claimed++;
            estimate = !(r->vq.settings.base_radius > 0.0f);
            r->iter_running += 1;
            S->vcm_running += 1;
            if (!estimate && r->iter_claimed < r->vq.iterations) {
                S->active_vcm.push_back(r);
                S->cv_vcm.notify_one();
            }
        }
        SceneRec& s = *S->scenes[r->scene];
        // The lane's stream waits for the upload and the image clear on the worker stream.
        if (r->ready) cudaStreamWaitEvent(lane.stream, r->ready, 0);
        scene_pool_view_set_root(lane.view, s.root, s.direct_root, s.direct_root >= 0 ? 0 : -1);
        imbart_shading sh;
        sh.device = S->device;
        sh.s = S->h_scenes[s.slot];
        long long stats[3] = {0, 0, 0};
        int rc = vcm_iteration(S, lane, r, k, lane.view, &sh, reinterpret_cast<float*>(S->pool + r->img_off), stats);
        if (!rc && !cuda_check(cudaStreamSynchronize(lane.stream), "cudaStreamSynchronize")) rc = IMBART_ERR_CUDA;
        std::lock_guard<std::mutex> lk(S->mu);
        S->vcm_running -= 1;
        r->iter_running -= 1;
        S->stats.closest_rays += stats[0];
        S->stats.shadow_rays += stats[1];
        S->stats.waves += stats[2];
        if (rc && !r->failed) r->failed = rc;
        if (!rc) r->iter_done += 1;
        if (estimate && !r->failed && r->iter_claimed < r->vq.iterations) {
            S->active_vcm.push_back(r);   // the radius is known now: the other lanes may join
            S->cv_vcm.notify_all();
        }
        if (r->iter_running > 0 || (!r->failed && r->iter_done < r->vq.iterations)) continue;
        // The last running iteration of a finished or failed request (a failed one may still
        // sit in the round robin).
        S->active_vcm.erase(std::remove(S->active_vcm.begin(), S->active_vcm.end(), r), S->active_vcm.end());
        if (r->ready) { cudaEventDestroy(r->ready); r->ready = nullptr; }
        if (r->failed) {
            // A failed request gives its memory back; the others go on.
            S->alloc.release(r->img_off, r->img_bytes);
            r->img_off = SIZE_MAX;
            release_request_locked(S, r);
            complete_locked(S, r, r->failed);
            S->cv_work.notify_all();
        } else {
            release_request_locked(S, r);
            S->jobs.push_back(imbart_server::Job{r, r->vq.image_host,
                                                 reinterpret_cast<const float*>(S->pool + r->img_off), r->img_bytes});
            S->cv_jobs.notify_one();
        }
    }
}

// Plain mode: one request through the single-request entry points.
int plain_request(imbart_server* S, Request* r) {
    SceneRec& s = *S->scenes[r->scene];
    cudaStream_t st = S->stream;
    if (!s.plain_scene) {
        s.plain_scene = upload_wide_scene(s.wide, S->device);
        if (!s.plain_scene) return imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA;
        s.plain_shading = imbart_shading_create_ex(
            S->device, s.vertices.data(), (int)(s.vertices.size() / 3), s.normals.data(), s.texcoords.data(),
            s.mesh_tris.data(), s.geom_normals.data(), (int)(s.mesh_tris.size() / 4), s.inst_inv.data(),
            (int)(s.inst_inv.size() / 12), s.mat_kind.data(), s.mat_params.data(), (int)s.mat_kind.size(),
            s.light_kinds.empty() ? nullptr : s.light_kinds.data(), s.tri_lights.empty() ? nullptr : s.tri_lights.data(),
            s.n_tri_lights, s.has_env ? s.env : nullptr, s.bsphere, s.tex_dims.empty() ? nullptr : s.tex_dims.data(),
            s.tex_pixels.empty() ? nullptr : s.tex_pixels.data(), s.n_textures);
        if (!s.plain_shading) return imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA;
        if (s.env_map > 0) {
            const int rc = imbart_shading_set_env_map(s.plain_shading, s.env_map - 1, s.env_intensity);
            if (rc) return rc;
        }
        S->stats.scene_uploads += 1;
    }
    if (r->kind == 0 || r->kind == 2) {
        const size_t bytes = r->kind == 0 ? (size_t)r->rr.width * r->rr.height * 3 * sizeof(float)
                                          : (size_t)r->vq.camera.width * r->vq.camera.height * 3 * sizeof(float);
        if (bytes > S->plain_image_bytes) {
            cudaFree(S->plain_image);
            S->plain_image = nullptr;
            S->plain_image_bytes = 0;
            if (!dalloc((uint8_t**)&S->plain_image, bytes)) return IMBART_ERR_OUT_OF_MEMORY;
            S->plain_image_bytes = bytes;
        }
        if (!cuda_check(cudaMemsetAsync(S->plain_image, 0, bytes, st), "cudaMemsetAsync")) return IMBART_ERR_CUDA;
        long long stats[3] = {0, 0, 0};
        if (r->kind == 0) {
            const int rc = imbart_pt_render(S->pt, s.plain_scene, s.plain_shading, r->rr.raster_to_world,
                                            r->rr.cam_pos, r->rr.width, r->rr.height, r->rr.spp, r->rr.max_path_len,
                                            r->rr.rr_start, r->rr.seed_base, S->plain_image, S->cap, stats, st);
            if (rc) return rc;
        } else {
            while (r->iter_done < r->vq.iterations) {
                long long it[3] = {0, 0, 0};
                const int rc = vcm_iteration(S, S->vcm_lanes[0], r, r->iter_done, s.plain_scene, s.plain_shading,
                                             S->plain_image, it);
                if (rc) return rc;
                r->iter_done += 1;
                for (int k = 0; k < 3; ++k) stats[k] += it[k];
            }
        }
        float* dst = r->kind == 0 ? r->rr.image_host : r->vq.image_host;
        if (!cuda_check(cudaMemcpyAsync(dst, S->plain_image, bytes, cudaMemcpyDeviceToHost, st),
                        "cudaMemcpyAsync") ||
            !cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize"))
            return IMBART_ERR_CUDA;
        std::lock_guard<std::mutex> lk(S->mu);
        S->stats.closest_rays += stats[0];
        S->stats.shadow_rays += stats[1];
        S->stats.waves += stats[2];
        return 0;
    }
    if (r->count > S->plain_ray_cap) {
        cudaFree(S->plain_rays); cudaFree(S->plain_hits);
        S->plain_rays = nullptr; S->plain_hits = nullptr; S->plain_ray_cap = 0;
        if (!dalloc(&S->plain_rays, r->count) || !dalloc(&S->plain_hits, r->count)) return IMBART_ERR_OUT_OF_MEMORY;
        S->plain_ray_cap = r->count;
    }
    const size_t rb = (size_t)r->count * sizeof(imbart_ray), hb = (size_t)r->count * sizeof(imbart_hit);
    if (!cuda_check(cudaMemcpyAsync(S->plain_rays, r->rays, rb, cudaMemcpyDefault, st), "cudaMemcpyAsync"))
        return IMBART_ERR_CUDA;
    const int rc = launch_trace_internal(s.plain_scene, S->plain_rays, S->plain_hits, nullptr, r->count, r->flags, st,
                                         nullptr);
    if (rc) return rc;
    if (!cuda_check(cudaMemcpyAsync(r->hits, S->plain_hits, hb, cudaMemcpyDefault, st), "cudaMemcpyAsync") ||
        !cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize"))
        return IMBART_ERR_CUDA;
    std::lock_guard<std::mutex> lk(S->mu);
    S->stats.batch_rays += r->count;
    return 0;
}

void worker_main(imbart_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            for (;;) {
                while (!S->incoming.empty()) {
                    S->pending.push_back(S->incoming.front());
                    S->incoming.pop_front();
                }
                const bool busy = !S->pending.empty() || !S->active_renders.empty() || !S->active_rays.empty() ||
                                  S->n_cur > 0;
                if (busy) break;
                if (S->stop) return;
                S->cv_work.wait(lk);
            }
        }
        if (S->mode == IMBART_SERVE_PLAIN) {
            Request* r = S->pending.front();
            S->pending.pop_front();
            r->t_start = now_ms(S->t0);
            const int rc = plain_request(S, r);
            std::lock_guard<std::mutex> lk(S->mu);
            complete_locked(S, r, rc);
            continue;
        }
        if (!batched_wave(S)) {
            // Admission is blocked on memory held by images still being copied out.
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->broken) continue;
            S->cv_work.wait_for(lk, std::chrono::milliseconds(1));
        }
    }
}

void completer_main(imbart_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        imbart_server::Job job;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_jobs.wait(lk, [&] { return S->stop || !S->jobs.empty(); });
            if (S->jobs.empty()) return;
            job = S->jobs.front();
        }
        const bool good =
            cuda_check(cudaMemcpyAsync(job.dst, job.src, job.bytes, cudaMemcpyDeviceToHost,
                                       S->copy_stream), "cudaMemcpyAsync") &&
            cuda_check(cudaStreamSynchronize(S->copy_stream), "cudaStreamSynchronize");
        std::lock_guard<std::mutex> lk(S->mu);
        S->jobs.pop_front();
        S->alloc.release(job.r->img_off, job.r->img_bytes);
        job.r->img_off = SIZE_MAX;
        complete_locked(S, job.r, good ? 0 : IMBART_ERR_CUDA);
        S->cv_work.notify_all();
    }
}

void free_server(imbart_server* S) {
    cudaSetDevice(S->device);
    for (auto& sp : S->scenes) {
        if (sp->plain_scene) imbart_scene_destroy(sp->plain_scene);
        if (sp->plain_shading) imbart_shading_destroy(sp->plain_shading);
    }
    if (S->pool_scene) scene_pool_view_destroy(S->pool_scene);
    if (S->pt) imbart_pt_destroy(S->pt);
    for (auto& lane : S->vcm_lanes) {
        if (lane.vcm) imbart_vcm_destroy(lane.vcm);
        if (lane.view) scene_pool_view_destroy(lane.view);
        if (lane.stream && lane.stream != S->stream) cudaStreamDestroy(lane.stream);
    }
    void* dev[] = {S->pool, S->d_reqs, S->d_scenes, S->d_terminated, S->d_chunks, S->d_runs, S->d_counts,
                   S->keys, S->perm, S->tile_counts,
                   S->hits, S->srays, S->shits, S->spixel, S->scontrib, S->sreq, S->sroot, S->b_rays, S->b_hits,
                   S->b_roots, S->plain_image, S->plain_rays, S->plain_hits};
    for (void* p : dev) cudaFree(p);
    for (int k = 0; k < 2; ++k) {
        void* q[] = {S->rays[k], S->pixel[k], S->rng[k], S->thr[k], S->bounces[k], S->req[k], S->root[k]};
        for (void* p : q) cudaFree(p);
    }
    void* host[] = {S->h_reqs, S->h_scenes, S->h_terminated, S->h_chunks, S->h_runs, S->h_counts, S->stage_rays,
                    S->stage_hits};
    for (void* p : host) cudaFreeHost(p);
    if (S->stream) cudaStreamDestroy(S->stream);
    if (S->copy_stream) cudaStreamDestroy(S->copy_stream);
    delete S;
}

}  // namespace
}  // namespace imbart

extern "C" {

imbart_server* imbart_server_create(int device, int mode, long long hbm_budget_bytes, long long max_paths_in_flight) {
    if (mode != IMBART_SERVE_BATCHED && mode != IMBART_SERVE_PLAIN) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_create: unknown mode");
        return nullptr;
    }
    int prev = 0;
    cudaGetDevice(&prev);
    if (!cuda_check(cudaSetDevice(device), "cudaSetDevice")) return nullptr;
    imbart_server* S = new imbart_server;
    S->device = device;
    S->mode = mode;
    S->t0 = std::chrono::steady_clock::now();
    S->scenes.reserve(kMaxScenes);
    S->cap = max_paths_in_flight > 0 ? std::min(max_paths_in_flight, (long long)(1 << 30)) : (4ll << 20);
    bool good = cuda_check(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking), "cudaStreamCreate") &&
                cuda_check(cudaStreamCreateWithFlags(&S->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (good && mode == IMBART_SERVE_PLAIN) {
        S->pt = imbart_pt_create(device);
        good = S->pt != nullptr;
        S->vcm_lanes.resize(1);
        S->vcm_lanes[0].stream = S->stream;
    } else if (good) {
        const long long budget = hbm_budget_bytes > 0 ? hbm_budget_bytes : (4ll << 30);
        S->pool_bytes = std::min<size_t>(align_up((size_t)budget, kBlockAlign), kMaxPoolBytes);
        const size_t cap = (size_t)S->cap;
        good = dalloc(&S->pool, S->pool_bytes) && dalloc(&S->d_reqs, kMaxReqSlots) && halloc(&S->h_reqs, kMaxReqSlots) &&
               dalloc(&S->d_scenes, kMaxSceneSlots) && halloc(&S->h_scenes, kMaxSceneSlots) &&
               dalloc(&S->d_terminated, kMaxReqSlots) && halloc(&S->h_terminated, kMaxReqSlots) &&
               dalloc(&S->d_chunks, kMaxReqSlots) && halloc(&S->h_chunks, kMaxReqSlots) &&
               dalloc(&S->d_runs, kMaxReqSlots) && halloc(&S->h_runs, kMaxReqSlots) &&
               dalloc(&S->d_counts, 4) && halloc(&S->h_counts, 4) &&
               dalloc(&S->hits, cap) && dalloc(&S->srays, 2 * cap) && dalloc(&S->shits, cap) &&
               dalloc(&S->keys, cap) && dalloc(&S->perm, cap) && dalloc(&S->tile_counts, (size_t)kShadeKeys * group_tiles(cap)) &&
               dalloc(&S->spixel, cap) && dalloc(&S->scontrib, cap) && dalloc(&S->sreq, cap) &&
               dalloc(&S->sroot, cap) && dalloc(&S->b_rays, cap) && dalloc(&S->b_hits, cap) &&
               dalloc(&S->b_roots, cap) && halloc(&S->stage_rays, cap) && halloc(&S->stage_hits, cap);
        for (int k = 0; k < 2 && good; ++k)
            good = dalloc(&S->rays[k], 2 * cap) && dalloc(&S->pixel[k], cap) && dalloc(&S->rng[k], cap) &&
                   dalloc(&S->thr[k], cap) && dalloc(&S->bounces[k], cap) && dalloc(&S->req[k], cap) &&
                   dalloc(&S->root[k], cap);
        if (good) {
            S->pool_scene = scene_pool_view(device, S->pool, S->pool_bytes);
            good = S->pool_scene != nullptr;
        }
        S->vcm_lanes.resize(std::max(1, std::min(env_lanes(), 16)));
        for (auto& lane : S->vcm_lanes) {
            if (!good) break;
            good = cuda_check(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking), "cudaStreamCreate") &&
                   (lane.view = scene_pool_view(device, S->pool, S->pool_bytes)) != nullptr;
            // Share of the resident block slots a lane's persistent traversal launches take
            // (IMBART_SERVE_LANE_GRID_SHARE, default all).
            if (good) scene_set_grid_share(lane.view, env_share("IMBART_SERVE_LANE_GRID_SHARE", 1.0f));
        }
        S->alloc.reset(S->pool_bytes);
        for (int i = kMaxReqSlots - 1; i >= 0; --i) S->free_req_slots.push_back(i);
        for (int i = kMaxSceneSlots - 1; i >= 0; --i) S->free_scene_slots.push_back(i);
    }
    if (!good) {
        free_server(S);
        cudaSetDevice(prev);
        return nullptr;
    }
    S->stats.pool_bytes = (long long)S->pool_bytes;
    S->worker = std::thread(worker_main, S);
    S->completer = std::thread(completer_main, S);
    if (mode == IMBART_SERVE_BATCHED)
        for (int k = 0; k < (int)S->vcm_lanes.size(); ++k) S->vcm_threads.emplace_back(vcm_lane_main, S, k);
    cudaSetDevice(prev);
    return S;
}

void imbart_server_destroy(imbart_server* S) {
    if (!S) return;
    imbart_server_drain(S);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    S->cv_jobs.notify_all();
    S->cv_vcm.notify_all();
    S->worker.join();
    S->completer.join();
    for (auto& t : S->vcm_threads) t.join();
    int prev = 0;
    cudaGetDevice(&prev);
    free_server(S);
    cudaSetDevice(prev);
}

}  // extern "C"

namespace imbart {
namespace {
bool valid_shading_source(const imbart_scene_source* src) {
    return src && src->vertices && src->n_vertices > 0 && src->normals && src->texcoords && src->mesh_tris &&
           src->geom_normals && src->n_mesh_tris > 0 && src->inst_inv && src->n_inst_inv > 0 && src->mat_kind &&
           src->mat_params && src->n_mats > 0 && src->n_tri_lights >= 0 &&
           !(src->n_tri_lights > 0 && !src->tri_lights) &&
           !(src->n_tri_lights == 0 && !src->env_color && src->env_map <= 0) &&
           valid_light_kinds(src->light_kinds, src->n_tri_lights) && src->n_textures >= 0 &&
           !(src->n_textures > 0 && (!src->tex_dims || !src->tex_pixels));
}

int register_scene(imbart_server* S, const imbart_scene_source* src, std::unique_ptr<SceneRec> s);
}  // namespace
}  // namespace imbart

extern "C" {

int imbart_server_add_scene(imbart_server* S, const imbart_scene_source* src) {
    if (!S || !valid_shading_source(src) || !src->nodes || src->n_nodes <= 0 || !src->instances ||
        src->n_instances <= 0 || !src->tris || src->n_tri_vec4 <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_add_scene: invalid argument");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    auto s = std::make_unique<SceneRec>();
    // The pool's scenes share one traversal view, so they are all 8-wide.
    const std::string err = convert_node2(src->root, src->nodes, src->n_nodes, src->instances, src->n_instances,
                                          src->tris, src->n_tri_vec4, s->wide, 8);
    if (!err.empty()) {
        set_error(IMBART_ERR_BAD_SCENE, "imbart_server_add_scene: " + err);
        return -IMBART_ERR_BAD_SCENE;
    }
    return register_scene(S, src, std::move(s));
}

int imbart_server_add_scene_gpu_build(imbart_server* S, const imbart_scene_source* src, const imbart_mesh_desc* meshes,
                                      int n_meshes, const imbart_instance_desc* instances, int n_instances,
                                      float* build_ms) {
    if (!S || !valid_shading_source(src) || !meshes || n_meshes <= 0 || !instances || n_instances <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_add_scene_gpu_build: invalid argument");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    const auto t0 = std::chrono::steady_clock::now();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(S->device);
    cudaStream_t st = nullptr;
    auto s = std::make_unique<SceneRec>();
    imbart_scene* g = nullptr;
    bool good = cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate") &&
                (g = imbart_scene_build_gpu(meshes, n_meshes, instances, n_instances, S->device, st, nullptr)) != nullptr;
    if (good) {
        // The built arrays come to the host like a converted scene's: the pool uploads and
        // evicts scenes from their host copies.
        imbart_scene_info info;
        const void *vn = nullptr, *vt = nullptr, *vi = nullptr;
        good = imbart_scene_get_info(g, &info) == 0 && imbart_scene_get_device_arrays(g, &vn, &vt, &vi) == 0;
        if (good) {
            s->wide.nodes.resize((size_t)info.wide_nodes);
            s->wide.tris.resize((size_t)info.triangles);
            s->wide.insts.resize((size_t)info.instances);
            s->wide.root = info.root;
            s->wide.top_nodes = (int)info.top_nodes;
            good = cuda_check(cudaMemcpyAsync(s->wide.nodes.data(), vn, sizeof(WideNode) * s->wide.nodes.size(),
                                              cudaMemcpyDeviceToHost, st), "D2H") &&
                   cuda_check(cudaMemcpyAsync(s->wide.tris.data(), vt, sizeof(WideTri) * s->wide.tris.size(),
                                              cudaMemcpyDeviceToHost, st), "D2H") &&
                   cuda_check(cudaMemcpyAsync(s->wide.insts.data(), vi, sizeof(WideInst) * s->wide.insts.size(),
                                              cudaMemcpyDeviceToHost, st), "D2H") &&
                   cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        }
    }
    if (g) imbart_scene_destroy(g);
    if (st) cudaStreamDestroy(st);
    cudaSetDevice(prev);
    if (!good) return -(imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA);
    if (build_ms) *build_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return register_scene(S, src, std::move(s));
}

}  // extern "C"

namespace imbart {
namespace {
int register_scene(imbart_server* S, const imbart_scene_source* src, std::unique_ptr<SceneRec> s) {
    auto vec = [](const auto* p, size_t n) { return std::vector<std::remove_const_t<std::remove_pointer_t<decltype(p)>>>(p, p + n); };
    s->vertices = vec(src->vertices, 3 * (size_t)src->n_vertices);
    s->normals = vec(src->normals, 3 * (size_t)src->n_vertices);
    s->texcoords = vec(src->texcoords, 2 * (size_t)src->n_vertices);
    s->mesh_tris = vec(src->mesh_tris, 4 * (size_t)src->n_mesh_tris);
    s->geom_normals = vec(src->geom_normals, 3 * (size_t)src->n_mesh_tris);
    s->inst_inv = vec(src->inst_inv, 12 * (size_t)src->n_inst_inv);
    s->mat_kind = vec(src->mat_kind, (size_t)src->n_mats);
    s->mat_params = vec(src->mat_params, 16 * (size_t)src->n_mats);
    if (src->n_tri_lights > 0) s->tri_lights = vec(src->tri_lights, 12 * (size_t)src->n_tri_lights);
    if (src->light_kinds && src->n_tri_lights > 0) s->light_kinds = vec(src->light_kinds, (size_t)src->n_tri_lights);
    s->n_textures = src->n_textures;
    long long texels = 0;
    s->tex_info.assign(std::max(src->n_textures, 1), make_int4(0, 0, 0, 0));
    for (int t = 0; t < src->n_textures; ++t) {
        const int w = src->tex_dims[2 * t], h = src->tex_dims[2 * t + 1];
        if (w <= 0 || h <= 0 || texels + (long long)w * h > INT_MAX) {
            set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_add_scene: invalid texture size");
            return -IMBART_ERR_INVALID_ARGUMENT;
        }
        s->tex_info[t] = make_int4((int)texels, w, h, 0);
        texels += (long long)w * h;
    }
    if (src->n_textures > 0) {
        s->tex_dims = vec(src->tex_dims, 2 * (size_t)src->n_textures);
        s->tex_pixels = vec(src->tex_pixels, 4 * (size_t)texels);
    }
    s->mats = decode_materials(src->mat_kind, src->mat_params, src->n_mats, src->n_textures > 0);
    s->kind_mask = material_kind_mask(s->mats);
    for (const Material& m : s->mats)
        if (m.tex >= src->n_textures || m.bump >= src->n_textures) {
            set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_add_scene: texture index out of range");
            return -IMBART_ERR_INVALID_ARGUMENT;
        }
    s->lights = decode_lights(src->light_kinds, src->tri_lights, src->n_tri_lights);
    s->n_tri_lights = src->n_tri_lights;
    s->has_env = src->env_color != nullptr || src->env_map > 0;
    for (int k = 0; k < 3; ++k) s->env[k] = src->env_color ? src->env_color[k] : 0.0f;
    if (src->env_map < 0 || src->env_map > src->n_textures || !(src->env_intensity >= 0.0f)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_add_scene: invalid environment image");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    s->env_map = src->env_map;
    s->env_intensity = src->env_intensity;
    for (int k = 0; k < 5; ++k) s->bsphere[k] = src->bsphere ? src->bsphere[k] : 0.0f;
    for (int i = 0; i < src->n_mesh_tris; ++i) {
        const int* t = src->mesh_tris + 4 * i;
        if (t[0] < 0 || t[1] < 0 || t[2] < 0 || t[0] >= src->n_vertices || t[1] >= src->n_vertices ||
            t[2] >= src->n_vertices || t[3] < 0 || t[3] >= src->n_mats) {
            set_error(IMBART_ERR_BAD_SCENE, "imbart_server_add_scene: triangle index out of range");
            return -IMBART_ERR_BAD_SCENE;
        }
    }
    layout_scene(*s);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->mode == IMBART_SERVE_BATCHED && s->bytes > std::min(S->pool_bytes, kSceneIndexLimit)) {
        set_error(IMBART_ERR_LIMIT, "imbart_server_add_scene: scene larger than the pool (or its scene region)");
        return -IMBART_ERR_LIMIT;
    }
    if (S->scenes.size() >= kMaxScenes) {
        set_error(IMBART_ERR_LIMIT, "imbart_server_add_scene: too many scenes");
        return -IMBART_ERR_LIMIT;
    }
    S->scenes.push_back(std::move(s));
    return (int)S->scenes.size() - 1;
}
}  // namespace
}  // namespace imbart

extern "C" {

static long long submit(imbart_server* S, std::unique_ptr<Request> r) {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->broken) {
        set_error(S->broken, "imbart_server: the server failed earlier");
        return -S->broken;
    }
    if (r->scene < 0 || r->scene >= (int)S->scenes.size()) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server: unknown scene");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    r->ticket = S->next_ticket++;
    r->t_submit = now_ms(S->t0);
    Request* raw = r.get();
    S->requests[r->ticket] = std::move(r);
    S->incoming.push_back(raw);
    S->outstanding += 1;
    S->stats.submitted += 1;
    S->cv_work.notify_all();
    return raw->ticket;
}

long long imbart_server_submit_render(imbart_server* S, const imbart_render_request* q) {
    if (!S || !q || !q->image_host || q->width <= 0 || q->height <= 0 || q->spp <= 0 || q->max_path_len < 1 ||
        (long long)q->width * q->height * q->spp > 2147483647ll) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_submit_render: invalid argument");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    auto r = std::make_unique<Request>();
    r->kind = 0;
    r->scene = q->scene;
    r->rr = *q;
    r->total = (long long)q->width * q->height * q->spp;
    return submit(S, std::move(r));
}

long long imbart_server_submit_rays(imbart_server* S, int scene, const imbart_ray* rays, imbart_hit* hits, int count,
                                    int flags) {
    if (!S || count <= 0 || !rays || !hits || (flags != IMBART_TRACE_CLOSEST && flags != IMBART_TRACE_ANY)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_submit_rays: invalid argument");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    auto r = std::make_unique<Request>();
    r->kind = 1;
    r->scene = scene;
    r->rays = rays;
    r->hits = hits;
    r->count = count;
    r->flags = flags;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(S->device);
    r->rays_kind = mem_kind(rays);
    r->hits_kind = mem_kind(hits);
    cudaSetDevice(prev);
    return submit(S, std::move(r));
}

long long imbart_server_submit_vcm(imbart_server* S, const imbart_vcm_request* q) {
    if (!S || !q || !q->image_host || q->camera.width <= 0 || q->camera.height <= 0 || q->iterations <= 0 ||
        (long long)q->camera.width * q->camera.height > 2147483647ll / 3) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_submit_vcm: invalid argument");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    // The settings are checked as imbart_vcm_begin_iteration checks them, with a positive
    // radius (given, or radius_factor > 0 for the estimate).
    imbart_vcm_settings st = q->settings;
    if (!(st.base_radius > 0.0f)) st.base_radius = q->radius_factor > 0.0f ? 1.0f : 0.0f;
    if (st.algorithm < IMBART_VCM || st.algorithm > IMBART_VCM_PT || st.spp <= 0 || st.max_path_len < 1 ||
        st.light_path_count <= 0 || st.num_connections < 0 || st.num_knn < 1 || st.num_knn > kGridMaxK ||
        st.light_tile_size < 0 || !(st.base_radius > 0.0f)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_submit_vcm: invalid settings");
        return -IMBART_ERR_INVALID_ARGUMENT;
    }
    auto r = std::make_unique<Request>();
    r->kind = 2;
    r->scene = q->scene;
    r->vq = *q;
    return submit(S, std::move(r));
}

int imbart_server_wait(imbart_server* S, long long ticket, imbart_request_result* out) {
    if (!S) return IMBART_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->requests.find(ticket);
    if (it == S->requests.end()) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_server_wait: unknown ticket");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    Request* r = it->second.get();
    S->cv_done.wait(lk, [&] { return r->complete; });
    if (out) {
        out->status = r->status;
        out->kind = r->kind;
        out->submit_ms = r->t_submit;
        out->start_ms = r->t_start;
        out->done_ms = r->t_done;
    }
    const int status = r->status;
    S->requests.erase(it);
    return status;
}

int imbart_server_drain(imbart_server* S) {
    if (!S) return IMBART_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->outstanding == 0; });
    return S->broken;
}

int imbart_server_get_stats(imbart_server* S, imbart_server_stats* out) {
    if (!S || !out) return IMBART_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->pool_used_bytes = (long long)S->alloc.used();
    out->kernel_launches = launches_total();
    return 0;
}

}  // extern "C"
