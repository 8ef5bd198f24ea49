// Host side of the traversal: scene preparation and upload, the stream-ordered trace entry
// points and the four drop-in symbols of the reference boundary (ray_queue.h:247-343).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "imbart_internal.h"
#include "trace_kernel.cuh"
#include "trace_launch.cuh"

struct imbart_scene {
    int device = 0;
    imbart::WideNode* nodes = nullptr;
    imbart::WideTri* tris = nullptr;
    imbart::WideInst* insts = nullptr;
    int* indices = nullptr;
    float2* texcoords = nullptr;
    int* masks = nullptr;
    uint8_t* mask_buffer = nullptr;
    int n_masks = 0;
    int* error_flags = nullptr;
    imbart_scene_info info{};
    bool owns_arrays = true;   // false for views into a node pool shared by several scenes
    float grid_share = 1.0f;   // persistent launches use this share of the resident block slots
    // Top level = one identity instance: its wide root and id (TraceParams::direct_root).
    int direct_root = -1, direct_inst = -1;
    imbart_scene() { info.node_width = 8; }   // converted scenes overwrite it
};

namespace imbart {
namespace {


bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? IMBART_ERR_OUT_OF_MEMORY : IMBART_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

template <typename T>
bool upload(T** dst, const T* src, size_t n, int64_t* bytes) {
    *dst = nullptr;
    if (n == 0) return true;
    if (!cuda_ok(cudaMalloc((void**)dst, n * sizeof(T)), "cudaMalloc")) return false;
    *bytes += (int64_t)(n * sizeof(T));
    return cuda_ok(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
}

void free_scene(imbart_scene* s) {
    if (!s) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    if (s->owns_arrays) {
        cudaFree(s->nodes); cudaFree(s->tris); cudaFree(s->insts);
        cudaFree(s->indices); cudaFree(s->texcoords); cudaFree(s->masks); cudaFree(s->mask_buffer);
    }
    cudaFree(s->error_flags);
    cudaSetDevice(prev);
    delete s;
}

imbart_scene* upload_scene(const HostWideScene& h, int device) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return nullptr;
    std::unique_ptr<imbart_scene, void (*)(imbart_scene*)> s(new imbart_scene, free_scene);
    s->device = device;
    int64_t bytes = 0;
    bool ok = upload(&s->nodes, h.nodes.data(), h.nodes.size(), &bytes) &&
              upload(&s->tris, h.tris.data(), h.tris.size(), &bytes) &&
              upload(&s->insts, h.insts.data(), h.insts.size(), &bytes);
    if (ok && h.masked) {
        std::vector<int> m(3 * h.masks.size());
        for (size_t i = 0; i < h.masks.size(); ++i) {
            m[3 * i] = h.masks[i].width; m[3 * i + 1] = h.masks[i].height; m[3 * i + 2] = h.masks[i].offset;
        }
        ok = upload(&s->indices, h.indices.data(), h.indices.size(), &bytes) &&
             upload(&s->texcoords, reinterpret_cast<const float2*>(h.texcoords.data()), h.texcoords.size(), &bytes) &&
             upload(&s->masks, m.data(), m.size(), &bytes) &&
             upload(&s->mask_buffer, h.mask_buffer.data(), h.mask_buffer.size(), &bytes);
        s->n_masks = (int)h.masks.size();
    }
    if (ok) ok = cuda_ok(cudaMalloc((void**)&s->error_flags, 4 * sizeof(int)), "cudaMalloc") &&
                 cuda_ok(cudaMemset(s->error_flags, 0, 4 * sizeof(int)), "cudaMemset");
    cudaSetDevice(prev);
    if (!ok) return nullptr;
    s->info.wide_nodes = (int64_t)h.nodes.size();
    s->info.top_nodes = h.top_nodes;
    s->info.triangles = (int64_t)h.tris.size();
    s->info.instances = (int64_t)h.insts.size();
    s->info.device_bytes = bytes;
    s->info.root = h.root;
    s->info.masked = h.masked ? 1 : 0;
    s->info.node_width = h.node_width;
    if (h.insts.size() == 1 && identity_instance(h.insts[0])) {
        s->direct_root = h.insts[0].root;
        s->direct_inst = h.insts[0].id;
    }
    return s.release();
}

template <typename Node, typename Convert>
imbart_scene* prepare(Convert convert, int root, const Node* nodes, int n_nodes,
                      const imbart_instance_node* insts, int n_insts, const imbart_vec4* tris, int n_tri_vec4,
                      const int* indices, int n_indices, const imbart_vec2* texcoords, int n_texcoords,
                      const imbart_mask_desc* masks, int n_masks, const char* mask_buffer, int mask_buffer_size,
                      int device) {
    if (!nodes || !insts || !tris || n_nodes <= 0 || n_insts <= 0 || n_tri_vec4 <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "scene preparation: missing arrays");
        return nullptr;
    }
    HostWideScene h;
    const std::string err = convert(root, nodes, n_nodes, insts, n_insts, tris, n_tri_vec4, h, -1);
    if (!err.empty()) {
        set_error(IMBART_ERR_BAD_SCENE, "scene preparation: " + err);
        return nullptr;
    }
    attach_masks(h, indices, n_indices, texcoords, n_texcoords, masks, n_masks, mask_buffer, mask_buffer_size);
    return upload_scene(h, device);
}

// ---------------------------------------------------------------------------------------
// Kernel variants. Variant 0 is the one-ray-per-thread kernel; variants 1..10 are the
// persistent-warp kernel at different block sizes / register budgets / shared stack depths.
// Closest-hit and any-hit queries pick their variants separately (measured on the B200:
// persistent warps win on incoherent closest-hit rays, the one-ray-per-thread kernel on
// short any-hit traversals). The configuration is process-wide (imbart_set_trace_config /
// imbart_set_trace_variant_any, or IMBART_TRACE_VARIANT, IMBART_TRACE_VARIANT_ANY,
// IMBART_TRACE_REFILL and IMBART_TRACE_POSTPONE in the environment).
// ---------------------------------------------------------------------------------------
// Three query classes keep their own variant and refill threshold: incoherent closest hit,
// any hit, and closest hit over coherent rays (camera rays, flag IMBART_TRACE_COHERENT),
// which traverse best in static batches (refill only when the whole warp is idle).
constexpr int kTraceVariants = 17;   // persistent-kernel shapes 1..17 (0: one ray per thread)
constexpr int kFirstCoopVariant = 11; // 11..17: the shapes with the cooperative triangle phase

// Each class also keeps its triangle batch: in the per-lane shapes, the triangles a lane
// tests per loop trip before the lanes with node work take their next node step (0: the
// whole group at once; two measured best there: secondary rays +13 %, camera rays +7 % over
// 0); the cooperative shapes ignore it. Defaults: the cooperative 256 x 3 shape for every
// class (on the frame's ray sets of the instanced scene: camera / secondary / shadow rays
// +2 / +9 / +10 % over the best per-lane shapes).
struct TraceConfig {
    int variant, refill, postpone, variant_any;
    int refill_any, variant_coh, refill_coh;
    int tri_batch = 0, tri_batch_any = 0, tri_batch_coh = 0;
};

std::mutex g_cfg_mutex;
bool g_cfg_init = false;
TraceConfig g_cfg{11, 24, 0, 11, 8, 11, 32};

int env_int(const char* name, int dflt) {
    const char* v = getenv(name);
    return v && *v ? atoi(v) : dflt;
}

TraceConfig current_config() {
    std::lock_guard<std::mutex> lk(g_cfg_mutex);
    if (!g_cfg_init) {
        g_cfg.variant = env_int("IMBART_TRACE_VARIANT", g_cfg.variant);
        g_cfg.variant_any = env_int("IMBART_TRACE_VARIANT_ANY", g_cfg.variant_any);
        g_cfg.refill = env_int("IMBART_TRACE_REFILL", g_cfg.refill);
        g_cfg.refill_any = env_int("IMBART_TRACE_REFILL_ANY", g_cfg.refill_any);
        g_cfg.variant_coh = env_int("IMBART_TRACE_VARIANT_COHERENT", g_cfg.variant_coh);
        g_cfg.refill_coh = env_int("IMBART_TRACE_REFILL_COHERENT", g_cfg.refill_coh);
        g_cfg.postpone = env_int("IMBART_TRACE_POSTPONE", g_cfg.postpone);
        g_cfg.tri_batch = env_int("IMBART_TRACE_TRI_BATCH", g_cfg.tri_batch);
        g_cfg.tri_batch_any = g_cfg.tri_batch_coh = g_cfg.tri_batch;
        g_cfg_init = true;
    }
    return g_cfg;
}

// Work counters of the persistent kernel: a ring of self-resetting (next, done) pairs per
// device. A launch takes the next slot; the kernel's last warp zeroes it on exit, so slots
// are reusable in stream order and concurrent launches on different streams use different
// slots (a collision would need 4096 launches in flight).
constexpr int kWorkSlots = 4096;
std::mutex g_work_mutex;
std::map<int, int*> g_work_pool;
std::atomic<uint32_t> g_work_next{0};

int* work_slot(int device) {
    int* pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_work_mutex);
        auto it = g_work_pool.find(device);
        if (it == g_work_pool.end()) {
            int prev = 0;
            cudaGetDevice(&prev);
            cudaSetDevice(device);
            const bool ok = cuda_ok(cudaMalloc((void**)&pool, sizeof(int) * 2 * kWorkSlots), "cudaMalloc") &&
                            cuda_ok(cudaMemset(pool, 0, sizeof(int) * 2 * kWorkSlots), "cudaMemset");
            cudaSetDevice(prev);
            if (!ok) return nullptr;
            g_work_pool[device] = pool;
        } else {
            pool = it->second;
        }
    }
    const uint32_t slot = g_work_next.fetch_add(1, std::memory_order_relaxed) % kWorkSlots;
    return pool + 2 * slot;
}

template <bool kStats>
const void* simple_kernel(bool any, bool masked) {
    if (any && masked) return (const void*)trace_kernel<true, true, kStats>;
    if (any) return (const void*)trace_kernel<true, false, kStats>;
    if (masked) return (const void*)trace_kernel<false, true, kStats>;
    return (const void*)trace_kernel<false, false, kStats>;
}

// The launch of one traversal query (kernel, grid, block and parameters) under the current
// configuration; false with the error set on invalid arguments. `count` = 0: nothing to launch.
bool trace_spec(const imbart_scene* s, const imbart_ray* rays, imbart_hit* hits, float* v_out, int count, int flags,
                unsigned long long* stats, const int* roots, const int* count_ptr, int* work_override, TraceParams& p,
                LaunchSpec& spec) {
    if (!s || (!rays && count > 0) || (!hits && count > 0) || count < 0 || (roots && s->info.masked)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_trace: invalid argument");
        return false;
    }
    spec = LaunchSpec{};
    if (count == 0) return true;
    p.nodes = s->nodes; p.tris = s->tris; p.insts = s->insts; p.root = s->info.root;
    p.indices = s->indices; p.texcoords = s->texcoords; p.masks = s->masks; p.mask_buffer = s->mask_buffer;
    p.n_masks = s->n_masks;
    p.rays = reinterpret_cast<const float4*>(rays);
    p.hits = reinterpret_cast<int4*>(hits);
    p.v_out = v_out;
    p.count = count;
    p.roots = roots;
    p.count_ptr = count_ptr;
    p.direct_root = roots ? -1 : s->direct_root;
    p.direct_inst = s->direct_inst;
    p.error_flags = s->error_flags;
    p.stats = stats;
    const bool any = (flags & IMBART_TRACE_ANY) != 0;
    const bool coherent = !any && (flags & IMBART_TRACE_COHERENT) != 0;
    const bool masked = s->info.masked != 0;
    const TraceConfig cfg = current_config();
    const int variant = any ? cfg.variant_any : coherent ? cfg.variant_coh : cfg.variant;
    const int refill = any ? cfg.refill_any : coherent ? cfg.refill_coh : cfg.refill;
    if (variant == 0) {
        const int block = 128;
        spec.func = stats ? simple_kernel<true>(any, masked) : simple_kernel<false>(any, masked);
        spec.grid = dim3((count + block - 1) / block);
        spec.block = dim3(block);
    } else {
        int* work = work_override ? work_override : work_slot(s->device);
        if (!work) return false;
        p.work = work;
        p.refill_lanes = std::min(std::max(refill, 1), 32);
        p.postpone_lanes = std::min(std::max(cfg.postpone, 0), 32);
        p.tri_batch = std::max(any ? cfg.tri_batch_any : coherent ? cfg.tri_batch_coh : cfg.tri_batch, 0);
        // 4-wide scenes take the 4-slot kernels (trace_w4.cu); the 8-slot kernels also trace
        // them correctly (empty slots never hit), only with twice the box tests. Single
        // identity-instance scenes take the flat kernels (trace_flat.cu).
        if (s->info.node_width == 4)
            spec = persistent_kernel_spec_w4(stats != nullptr, variant, any, masked, count, s->device,
                                             s->grid_share, p);
        else if (p.direct_root >= 0)
            spec = persistent_kernel_spec_flat(stats != nullptr, variant, any, masked, count, s->device,
                                               s->grid_share, p);
        else
            spec = stats ? persistent_kernel_spec<true, 8>(variant, any, masked, count, s->device, s->grid_share, p)
                         : persistent_kernel_spec<false, 8>(variant, any, masked, count, s->device, s->grid_share, p);
    }
    if (!spec.func) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_trace: unknown kernel variant");
        return false;
    }
    return true;
}

int launch_trace(const imbart_scene* s, const imbart_ray* rays, imbart_hit* hits, float* v_out,
                 int count, int flags, cudaStream_t stream, unsigned long long* stats = nullptr,
                 const int* roots = nullptr, const int* count_ptr = nullptr, int* work_override = nullptr) {
    TraceParams p;
    LaunchSpec spec;
    if (!trace_spec(s, rays, hits, v_out, count, flags, stats, roots, count_ptr, work_override, p, spec))
        return imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA;
    if (!spec.func) return 0;
    void* args[] = {&p};
    if (!cuda_ok(cudaLaunchKernel(spec.func, spec.grid, spec.block, args, 0, stream), "trace kernel launch"))
        return IMBART_ERR_CUDA;
    note_launches(1);
    return 0;
}

// Per-thread stream for the synchronous drop-in entry points: the reference calls them
// concurrently from its tile-scheduler threads (tile_scheduler.h:120-130).
cudaStream_t thread_stream() {
    thread_local cudaStream_t st = nullptr;
    if (!st) cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    return st;
}

// ---------------------------------------------------------------------------------------
// Drop-in scene cache. The reference passes raw pointers without sizes; device arrays are
// sized through their allocation range, host arrays are walked from the root.
// ---------------------------------------------------------------------------------------
using CacheKey = std::tuple<const void*, int, const void*, const void*, const void*, const void*, int>;
std::mutex g_cache_mutex;
std::map<CacheKey, imbart_scene*> g_cache;

void clear_cache() {
    std::lock_guard<std::mutex> lk(g_cache_mutex);
    for (auto& kv : g_cache) free_scene(kv.second);
    g_cache.clear();
}

// cuMemGetAddressRange through the runtime's driver entry-point table, so that the library
// loads on machines without a driver (the CPU-only build and test host).
using MemGetAddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
MemGetAddressRangeFn mem_get_address_range() {
    static MemGetAddressRangeFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<MemGetAddressRangeFn>(f);
    }();
    return fn;
}

// Copies the tail of the device allocation that starts at or before `ptr` to the host.
template <typename T>
bool fetch_device_array(const T* ptr, std::vector<T>& out) {
    out.clear();
    if (!ptr) return true;
    cudaFree(0);  // make the primary context current for the driver call
    MemGetAddressRangeFn range = mem_get_address_range();
    if (!range) {
        set_error(IMBART_ERR_CUDA, "drop-in traversal: cuMemGetAddressRange unavailable");
        return false;
    }
    CUdeviceptr base = 0;
    size_t size = 0;
    if (range(&base, &size, (CUdeviceptr)ptr) != CUDA_SUCCESS) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "drop-in traversal: pointer is not a device allocation");
        return false;
    }
    const size_t off = (size_t)((CUdeviceptr)ptr - base);
    const size_t n = (size - off) / sizeof(T);
    out.resize(n);
    return n == 0 || cuda_ok(cudaMemcpy(out.data(), ptr, n * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
}

imbart_scene* cached_device_scene(int root, const imbart_node2* nodes, const imbart_instance_node* insts,
                                  const imbart_vec4* tris, const int* indices, const imbart_vec2* texcoords,
                                  const imbart_mask_desc* masks, const char* mask_buffer) {
    int device = 0;
    cudaGetDevice(&device);
    const CacheKey key{nodes, root, insts, tris, masks, mask_buffer, device};
    std::lock_guard<std::mutex> lk(g_cache_mutex);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;
    std::vector<imbart_node2> hn;
    std::vector<imbart_instance_node> hi;
    std::vector<imbart_vec4> ht;
    std::vector<int> hidx;
    std::vector<imbart_vec2> htc;
    std::vector<imbart_mask_desc> hm;
    std::vector<char> hmb;
    if (!fetch_device_array(nodes, hn) || !fetch_device_array(insts, hi) || !fetch_device_array(tris, ht) ||
        !fetch_device_array(indices, hidx) || !fetch_device_array(texcoords, htc) ||
        !fetch_device_array(masks, hm) || !fetch_device_array(mask_buffer, hmb))
        return nullptr;
    imbart_scene* s = prepare<imbart_node2>(convert_node2, root, hn.data(), (int)hn.size(), hi.data(), (int)hi.size(),
                                            ht.data(), (int)ht.size(), hidx.data(), (int)hidx.size(),
                                            htc.data(), (int)htc.size(), hm.data(), (int)hm.size(),
                                            hmb.data(), (int)hmb.size(), device);
    if (s) g_cache[key] = s;
    return s;
}

imbart_scene* cached_host_scene(int root, const imbart_node4* nodes, const imbart_instance_node* insts,
                                const imbart_vec4* tris, const int* indices, const imbart_vec2* texcoords,
                                const imbart_mask_desc* masks, const char* mask_buffer) {
    int device = 0;
    cudaGetDevice(&device);
    const CacheKey key{nodes, root, insts, tris, masks, mask_buffer, device};
    std::lock_guard<std::mutex> lk(g_cache_mutex);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;
    // Host arrays carry no size: the converter only touches what is reachable from the root.
    // Index and texcoord arrays are only needed when masks are active; their extent is the
    // largest index reachable through the triangles (computed by the converter's caller).
    HostWideScene h;
    const std::string err = convert_node4(root, nodes, INT_MAX, insts, INT_MAX, tris, INT_MAX, h);
    if (!err.empty()) {
        set_error(IMBART_ERR_BAD_SCENE, "scene preparation: " + err);
        return nullptr;
    }
    if (masks && mask_buffer && indices) {
        int max_tri = 0;
        for (const WideTri& t : h.tris) max_tri = std::max(max_tri, t.id);
        int n_idx = 4 * (max_tri + 1), max_mat = 0, max_tc = 0;
        for (int i = 0; i < n_idx; ++i) {
            if (i % 4 == 3) max_mat = std::max(max_mat, indices[i]);
            else max_tc = std::max(max_tc, indices[i]);
        }
        int buf = 0;
        for (int m = 0; m <= max_mat; ++m) buf = std::max(buf, masks[m].offset + masks[m].width * masks[m].height);
        attach_masks(h, indices, n_idx, texcoords, texcoords ? max_tc + 1 : 0, masks, max_mat + 1, mask_buffer, buf);
    }
    imbart_scene* s = upload_scene(h, device);
    if (s) g_cache[key] = s;
    return s;
}

void dropin_device(bool any, int root, imbart_node2* nodes, imbart_instance_node* insts, imbart_vec4* tris,
                   imbart_ray* rays, imbart_hit* hits, int* indices, imbart_vec2* texcoords,
                   imbart_mask_desc* masks, char* mask_buffer, int count) {
    imbart_scene* s = cached_device_scene(root, nodes, insts, tris, indices, texcoords, masks, mask_buffer);
    if (!s) return;
    cudaStream_t st = thread_stream();
    if (launch_trace(s, rays, hits, nullptr, count, any ? IMBART_TRACE_ANY : IMBART_TRACE_CLOSEST, st) == 0)
        cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

void dropin_host(bool any, int root, imbart_node4* nodes, imbart_instance_node* insts, imbart_vec4* tris,
                 imbart_ray* rays, imbart_hit* hits, int* indices, imbart_vec2* texcoords,
                 imbart_mask_desc* masks, char* mask_buffer, int count) {
    imbart_scene* s = cached_host_scene(root, nodes, insts, tris, indices, texcoords, masks, mask_buffer);
    if (!s) return;
    imbart_trace_host(s, rays, hits, count, any ? IMBART_TRACE_ANY : IMBART_TRACE_CLOSEST, thread_stream());
}

}  // namespace

int launch_trace_internal(const imbart_scene* scene, const void* rays, void* hits, float* v_out, int count,
                          int flags, void* stream, unsigned long long* stats, const int* roots,
                          const int* count_ptr, int* work) {
    return launch_trace(scene, reinterpret_cast<const imbart_ray*>(rays), reinterpret_cast<imbart_hit*>(hits), v_out,
                        count, flags, (cudaStream_t)stream, stats, roots, count_ptr, work);
}

int add_trace_node(cudaGraph_t graph, const cudaGraphNode_t* deps, int n_deps, cudaGraphNode_t* node,
                   const imbart_scene* scene, const void* rays, void* hits, int count, int flags,
                   const int* count_ptr, int* work) {
    TraceParams p;
    LaunchSpec spec;
    if (!trace_spec(scene, reinterpret_cast<const imbart_ray*>(rays), reinterpret_cast<imbart_hit*>(hits), nullptr,
                    count, flags, nullptr, nullptr, count_ptr, work, p, spec))
        return imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA;
    if (!spec.func) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "add_trace_node: empty launch");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    void* args[] = {&p};
    cudaKernelNodeParams np{};
    np.func = const_cast<void*>(spec.func);
    np.gridDim = spec.grid;
    np.blockDim = spec.block;
    np.sharedMemBytes = 0;
    np.kernelParams = args;
    np.extra = nullptr;
    return cuda_ok(cudaGraphAddKernelNode(node, graph, deps, (size_t)n_deps, &np), "cudaGraphAddKernelNode")
               ? 0
               : IMBART_ERR_CUDA;
}

void scene_set_grid_share(imbart_scene* s, float share) {
    // Written so that NaN takes the lower bound too.
    s->grid_share = !(share > 0.05f) ? 0.05f : (share < 1.0f ? share : 1.0f);
}

void scene_launch_key(const imbart_scene* s, unsigned long long out[12]) {
    out[0] = (unsigned long long)(uintptr_t)s->nodes; out[1] = (unsigned long long)(uintptr_t)s->tris;
    out[2] = (unsigned long long)(uintptr_t)s->insts; out[3] = (unsigned long long)(uintptr_t)s->indices;
    out[4] = (unsigned long long)(uintptr_t)s->texcoords; out[5] = (unsigned long long)(uintptr_t)s->masks;
    out[6] = (unsigned long long)(uintptr_t)s->mask_buffer; out[7] = (unsigned long long)(uintptr_t)s->error_flags;
    out[8] = (unsigned long long)s->n_masks; out[9] = (unsigned long long)(unsigned)s->info.root;
    uint32_t share_bits;
    std::memcpy(&share_bits, &s->grid_share, sizeof(share_bits));
    out[10] = (unsigned long long)s->info.masked | ((unsigned long long)share_bits << 32);
    out[11] = (unsigned long long)s->device;
}

void trace_config_snapshot(int out[10]) {
    const TraceConfig c = current_config();
    out[0] = c.variant; out[1] = c.refill; out[2] = c.postpone; out[3] = c.variant_any;
    out[4] = c.refill_any; out[5] = c.variant_coh; out[6] = c.refill_coh;
    out[7] = c.tri_batch; out[8] = c.tri_batch_any; out[9] = c.tri_batch_coh;
}

imbart_scene* upload_wide_scene(const HostWideScene& h, int device) { return upload_scene(h, device); }

imbart_scene* scene_pool_view(int device, const void* pool, size_t pool_bytes) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return nullptr;
    imbart_scene* s = new imbart_scene;
    s->device = device;
    s->owns_arrays = false;
    s->nodes = (WideNode*)pool;
    s->tris = (WideTri*)pool;
    s->insts = (WideInst*)pool;
    s->info.device_bytes = (int64_t)pool_bytes;
    const bool ok = cuda_ok(cudaMalloc((void**)&s->error_flags, 4 * sizeof(int)), "cudaMalloc") &&
                    cuda_ok(cudaMemset(s->error_flags, 0, 4 * sizeof(int)), "cudaMemset");
    cudaSetDevice(prev);
    if (!ok) { free_scene(s); return nullptr; }
    return s;
}

void scene_pool_view_destroy(imbart_scene* s) { free_scene(s); }

void scene_pool_view_set_root(imbart_scene* s, int root, int direct_root, int direct_inst) {
    s->info.root = root;
    s->direct_root = direct_root;
    s->direct_inst = direct_inst;
}

imbart_scene* scene_adopt_device_arrays(int device, WideNode* nodes, int64_t n_nodes, int64_t top_nodes,
                                        WideTri* tris, int64_t n_tris, WideInst* insts, int64_t n_insts, int root) {
    imbart_scene* s = new imbart_scene;
    s->device = device;
    s->nodes = nodes;
    s->tris = tris;
    s->insts = insts;
    s->owns_arrays = false;
    if (!cuda_ok(cudaMalloc((void**)&s->error_flags, 4 * sizeof(int)), "cudaMalloc") ||
        !cuda_ok(cudaMemset(s->error_flags, 0, 4 * sizeof(int)), "cudaMemset")) {
        free_scene(s);
        return nullptr;
    }
    s->owns_arrays = true;
    s->info.wide_nodes = n_nodes;
    s->info.top_nodes = top_nodes;
    s->info.triangles = n_tris;
    s->info.instances = n_insts;
    s->info.device_bytes = n_nodes * (int64_t)sizeof(WideNode) + n_tris * (int64_t)sizeof(WideTri) +
                           n_insts * (int64_t)sizeof(WideInst);
    s->info.root = root;
    s->info.masked = 0;
    return s;
}

}  // namespace imbart

using namespace imbart;

extern "C" {

imbart_scene* imbart_scene_from_node2(int root, const imbart_node2* nodes, int n_nodes,
                                      const imbart_instance_node* instances, int n_instances,
                                      const imbart_vec4* tris, int n_tri_vec4,
                                      const int* indices, int n_indices,
                                      const imbart_vec2* texcoords, int n_texcoords,
                                      const imbart_mask_desc* masks, int n_masks,
                                      const char* mask_buffer, int mask_buffer_size, int device) {
    return prepare<imbart_node2>(convert_node2, root, nodes, n_nodes, instances, n_instances, tris, n_tri_vec4,
                                 indices, n_indices, texcoords, n_texcoords, masks, n_masks, mask_buffer,
                                 mask_buffer_size, device);
}

imbart_scene* imbart_scene_from_node4(int root, const imbart_node4* nodes, int n_nodes,
                                      const imbart_instance_node* instances, int n_instances,
                                      const imbart_vec4* tris, int n_tri_vec4,
                                      const int* indices, int n_indices,
                                      const imbart_vec2* texcoords, int n_texcoords,
                                      const imbart_mask_desc* masks, int n_masks,
                                      const char* mask_buffer, int mask_buffer_size, int device) {
    return prepare<imbart_node4>(convert_node4, root, nodes, n_nodes, instances, n_instances, tris, n_tri_vec4,
                                 indices, n_indices, texcoords, n_texcoords, masks, n_masks, mask_buffer,
                                 mask_buffer_size, device);
}

void imbart_scene_destroy(imbart_scene* scene) { free_scene(scene); }

int imbart_scene_get_info(const imbart_scene* scene, imbart_scene_info* out) {
    if (!scene || !out) { set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_scene_get_info"); return IMBART_ERR_INVALID_ARGUMENT; }
    *out = scene->info;
    return 0;
}

int imbart_scene_get_device_arrays(const imbart_scene* scene, const void** nodes, const void** tris,
                                   const void** instances) {
    if (!scene) { set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_scene_get_device_arrays"); return IMBART_ERR_INVALID_ARGUMENT; }
    if (nodes) *nodes = scene->nodes;
    if (tris) *tris = scene->tris;
    if (instances) *instances = scene->insts;
    return 0;
}

int imbart_trace(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits, int count, int flags,
                 void* stream) {
    return launch_trace(scene, rays, hits, nullptr, count, flags, (cudaStream_t)stream);
}

int imbart_trace_uv(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits, float* v_out, int count,
                    int flags, void* stream) {
    return launch_trace(scene, rays, hits, v_out, count, flags, (cudaStream_t)stream);
}

int imbart_trace_host(const imbart_scene* scene, const imbart_ray* rays_host, imbart_hit* hits_host, int count,
                      int flags, void* stream) {
    if (!scene || count < 0 || (count > 0 && (!rays_host || !hits_host))) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_trace_host: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (count == 0) return 0;
    // Per-thread device staging buffers, grown on demand.
    thread_local imbart_ray* d_rays = nullptr;
    thread_local imbart_hit* d_hits = nullptr;
    thread_local int cap = 0;
    thread_local int cap_device = -1;
    if (cap < count || cap_device != scene->device) {
        cudaFree(d_rays); cudaFree(d_hits);
        d_rays = nullptr; d_hits = nullptr; cap = 0;
        if (!cuda_ok(cudaMalloc((void**)&d_rays, sizeof(imbart_ray) * (size_t)count), "cudaMalloc") ||
            !cuda_ok(cudaMalloc((void**)&d_hits, sizeof(imbart_hit) * (size_t)count), "cudaMalloc"))
            return IMBART_ERR_OUT_OF_MEMORY;
        cap = count;
        cap_device = scene->device;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (!cuda_ok(cudaMemcpyAsync(d_rays, rays_host, sizeof(imbart_ray) * (size_t)count, cudaMemcpyHostToDevice, st),
                 "cudaMemcpyAsync H2D"))
        return IMBART_ERR_CUDA;
    const int rc = launch_trace(scene, d_rays, d_hits, nullptr, count, flags, st);
    if (rc) return rc;
    if (!cuda_ok(cudaMemcpyAsync(hits_host, d_hits, sizeof(imbart_hit) * (size_t)count, cudaMemcpyDeviceToHost, st),
                 "cudaMemcpyAsync D2H"))
        return IMBART_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize")) return IMBART_ERR_CUDA;
    return 0;
}

int imbart_trace_stats(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits, int count, int flags,
                       unsigned long long* stats, void* stream) {
    if (!stats) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_trace_stats: stats is NULL");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    return launch_trace(scene, rays, hits, nullptr, count, flags, (cudaStream_t)stream, stats);
}

int imbart_scene_error_count(const imbart_scene* scene) {
    if (!scene) return -1;
    int v = 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    const bool ok = cuda_ok(cudaMemcpy(&v, scene->error_flags, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
    cudaSetDevice(prev);
    return ok ? v : -1;
}

int64_t imbart_kernel_launch_count(void) { return launches_total(); }

int imbart_set_trace_config(int variant, int refill_lanes, int postpone_lanes) {
    if (variant < 0 || variant > kTraceVariants || refill_lanes < 1 || refill_lanes > 32 || postpone_lanes < 0 ||
        postpone_lanes > 32) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_set_trace_config: out of range");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    current_config();
    std::lock_guard<std::mutex> lk(g_cfg_mutex);
    g_cfg.variant = variant;
    g_cfg.refill = refill_lanes;
    g_cfg.postpone = postpone_lanes;
    g_cfg.variant_any = variant;
    g_cfg.variant_coh = variant;
    return 0;
}

int imbart_set_trace_class(int flags, int variant, int refill_lanes) {
    if (variant < 0 || variant > kTraceVariants || refill_lanes < 1 || refill_lanes > 32 || flags < 0 || flags > 3) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_set_trace_class: out of range");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    current_config();
    std::lock_guard<std::mutex> lk(g_cfg_mutex);
    if (flags & IMBART_TRACE_ANY) { g_cfg.variant_any = variant; g_cfg.refill_any = refill_lanes; }
    else if (flags & IMBART_TRACE_COHERENT) { g_cfg.variant_coh = variant; g_cfg.refill_coh = refill_lanes; }
    else { g_cfg.variant = variant; g_cfg.refill = refill_lanes; }
    return 0;
}

int imbart_set_trace_tri_batch(int flags, int tri_batch) {
    if (tri_batch < 0 || tri_batch > 24 || flags < 0 || flags > 3) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_set_trace_tri_batch: out of range");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    current_config();
    std::lock_guard<std::mutex> lk(g_cfg_mutex);
    if (flags & IMBART_TRACE_ANY) g_cfg.tri_batch_any = tri_batch;
    else if (flags & IMBART_TRACE_COHERENT) g_cfg.tri_batch_coh = tri_batch;
    else g_cfg.tri_batch = tri_batch;
    return 0;
}

int imbart_get_trace_tri_batch(int flags) {
    const TraceConfig c = current_config();
    const bool any = (flags & IMBART_TRACE_ANY) != 0, coh = !any && (flags & IMBART_TRACE_COHERENT) != 0;
    return any ? c.tri_batch_any : coh ? c.tri_batch_coh : c.tri_batch;
}

int imbart_get_trace_class(int flags, int* variant, int* refill_lanes) {
    const TraceConfig c = current_config();
    const bool any = (flags & IMBART_TRACE_ANY) != 0, coh = !any && (flags & IMBART_TRACE_COHERENT) != 0;
    if (variant) *variant = any ? c.variant_any : coh ? c.variant_coh : c.variant;
    if (refill_lanes) *refill_lanes = any ? c.refill_any : coh ? c.refill_coh : c.refill;
    return 0;
}

int imbart_trace_autotune(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits, int count, int flags,
                          void* stream, imbart_trace_tuning* out) {
    if (!scene || !rays || !hits || count <= 0 || flags < 0 || flags > 3) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_trace_autotune: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int v0 = 0, r0 = 0;
    imbart_get_trace_class(flags, &v0, &r0);
    const int b0 = imbart_get_trace_tri_batch(flags);
    // Time one configuration: a warm-up launch, then the mean of three.
    auto time_config = [&](int variant, int refill, float* ms) -> int {
        int rc = imbart_set_trace_class(flags, variant, refill);
        for (int k = 0; k < 4 && !rc; ++k) {
            if (k == 1) cudaEventRecord(e0, st);
            rc = launch_trace(scene, rays, hits, nullptr, count, flags, st);
        }
        if (rc) return rc;
        cudaEventRecord(e1, st);
        if (!cuda_ok(cudaEventSynchronize(e1), "cudaEventSynchronize")) return IMBART_ERR_CUDA;
        cudaEventElapsedTime(ms, e0, e1);
        *ms /= 3.0f;
        return 0;
    };
    static const int kRefills[] = {4, 8, 16, 24, 32};
    float default_ms = 0.0f, best_ms = FLT_MAX;
    int best_v = v0, best_r = r0;
    int rc = time_config(v0, r0, &default_ms);
    if (!rc) { best_ms = default_ms; }
    for (int v = 1; v <= kTraceVariants && !rc; ++v)
        for (int r : kRefills) {
            float ms = 0.0f;
            rc = time_config(v, r, &ms);
            if (rc) break;
            if (ms < best_ms) { best_ms = ms; best_v = v; best_r = r; }
        }
    imbart_set_trace_class(flags, rc ? v0 : best_v, rc ? r0 : best_r);
    // Then the triangle batch of the chosen shape.
    int best_b = b0;
    static const int kTriBatches[] = {0, 1, 2, 3, 4};
    for (int b : kTriBatches) {
        if (rc || b == b0) continue;
        if (best_v >= kFirstCoopVariant && b > 0) continue;   // the cooperative shapes ignore it
        imbart_set_trace_tri_batch(flags, b);
        float ms = 0.0f;
        rc = time_config(best_v, best_r, &ms);
        if (!rc && ms < best_ms) { best_ms = ms; best_b = b; }
    }
    if (rc) imbart_set_trace_class(flags, v0, r0);
    imbart_set_trace_tri_batch(flags, rc ? b0 : best_b);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaSetDevice(prev);
    if (!rc && out) {
        out->variant = best_v;
        out->refill = best_r;
        out->ms = best_ms;
        out->default_ms = default_ms;
        out->tri_batch = best_b;
    }
    return rc;
}

int imbart_set_trace_variant_any(int variant) {
    if (variant < 0 || variant > kTraceVariants) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_set_trace_variant_any: out of range");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    current_config();
    std::lock_guard<std::mutex> lk(g_cfg_mutex);
    g_cfg.variant_any = variant;
    return 0;
}

int imbart_get_trace_config(int* variant, int* refill_lanes, int* postpone_lanes) {
    const TraceConfig c = current_config();
    if (variant) *variant = c.variant;
    if (refill_lanes) *refill_lanes = c.refill;
    if (postpone_lanes) *postpone_lanes = c.postpone;
    return 0;
}

int imbart_get_trace_variant_any(void) { return current_config().variant_any; }

void imbart_invalidate_scenes(void) { clear_cache(); }

void intersect_gpu_masked_instanced(int root, imbart_node2* nodes, imbart_instance_node* instances, imbart_vec4* tris,
                                    imbart_ray* rays, imbart_hit* hits, int* indices, imbart_vec2* texcoords,
                                    imbart_mask_desc* masks, char* mask_buffer, int count) {
    dropin_device(false, root, nodes, instances, tris, rays, hits, indices, texcoords, masks, mask_buffer, count);
}

void occluded_gpu_masked_instanced(int root, imbart_node2* nodes, imbart_instance_node* instances, imbart_vec4* tris,
                                   imbart_ray* rays, imbart_hit* hits, int* indices, imbart_vec2* texcoords,
                                   imbart_mask_desc* masks, char* mask_buffer, int count) {
    dropin_device(true, root, nodes, instances, tris, rays, hits, indices, texcoords, masks, mask_buffer, count);
}

void intersect_cpu_masked_instanced(int root, imbart_node4* nodes, imbart_instance_node* instances, imbart_vec4* tris,
                                    imbart_ray* rays, imbart_hit* hits, int* indices, imbart_vec2* texcoords,
                                    imbart_mask_desc* masks, char* mask_buffer, int count) {
    dropin_host(false, root, nodes, instances, tris, rays, hits, indices, texcoords, masks, mask_buffer, count);
}

void occluded_cpu_masked_instanced(int root, imbart_node4* nodes, imbart_instance_node* instances, imbart_vec4* tris,
                                   imbart_ray* rays, imbart_hit* hits, int* indices, imbart_vec2* texcoords,
                                   imbart_mask_desc* masks, char* mask_buffer, int count) {
    dropin_host(true, root, nodes, instances, tris, rays, hits, indices, texcoords, masks, mask_buffer, count);
}

}  // extern "C"
