// Photon hash grid on the GPU: build (bounding box, hashed counting sort) and batched
// k-capped radius queries, with the semantics of the reference's HashGrid
// (src/imbatracer/rangesearch/rangesearch.h):
//   build  :25-75   r^2, cell size (2r in the reference, a parameter here), bbox of the
//                   photon positions inflated by 0.1 % of its extent per side, counting sort
//                   into `table_size` buckets (2 * photon count in the reference)
//   hash   :137-148 ((x*73856093) ^ (y*19349663) ^ (z*83492791)) mod table_size on unsigned
//                   coordinates, coordinates = floor((p - bbox.min) / cell size)
//   query  :77-129  outside the bbox -> nothing; home cell plus the nearer neighbour per
//                   axis (8 buckets in the reference's order, a bucket hit twice is scanned
//                   twice), squared distance <= r^2, k nearest kept by insertion sort
// Every float operation is explicitly rounded (no contraction) so that cell indices and
// distances equal the reference's bit for bit. Within a bucket photons are placed by an
// atomic cursor, as in the reference's parallel scatter (rangesearch.h:68-74); the query
// returns its k photons ordered by (distance, photon index).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cfloat>
#include <mutex>
#include <string>

#include "hashgrid_query.cuh"
#include "imbart_internal.h"

struct imbart_hashgrid {
    int device = 0;
    int n = 0;              // photons in the current build
    int table = 0;          // buckets in the current build
    int sorted_cap = 0, cell_of_cap = 0, ends_cap = 0, cursor_cap = 0;
    float4* sorted = nullptr;   // position xyz + original index (int bits) in bucket order
    int* cell_ends = nullptr;   // inclusive end of each bucket
    int* cell_of = nullptr;     // bucket of each photon (scratch)
    int* cursor = nullptr;      // scatter cursor per bucket (scratch)
    int* block_sums = nullptr;  // scan scratch
    int block_sums_cap = 0;
    float* params = nullptr;    // device: lo[3], hi[3], radius, r^2, cell, inv_cell
    float host_params[10] = {};
    float cell_factor = 2.0f;   // cell size / radius of the current build
};

namespace imbart {
namespace {

constexpr int kBlock = 256;
constexpr int kScanItems = 8;                 // items per thread in the scan kernels
constexpr int kScanTile = kBlock * kScanItems;
constexpr int kMaxK = kGridMaxK;

bool ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? IMBART_ERR_OUT_OF_MEMORY : IMBART_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// Order-preserving float <-> int mapping for atomicMin/atomicMax on floats.
__device__ __forceinline__ int float_to_ordered(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ordered_to_float(int i) {
    return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

__global__ void bbox_init_kernel(int* box) {
    if (threadIdx.x < 3) box[threadIdx.x] = float_to_ordered(FLT_MAX);
    else if (threadIdx.x < 6) box[threadIdx.x] = float_to_ordered(-FLT_MAX);
}

// Exact min/max of the positions (order-independent, so bit-identical to a serial pass).
__global__ void bbox_kernel(const float* __restrict__ pos, int stride, int n, int* __restrict__ box) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* p = pos + (size_t)i * stride;
        for (int a = 0; a < 3; ++a) {
            const float v = p[a];
            lo[a] = lo[a] < v ? lo[a] : v;
            hi[a] = hi[a] > v ? hi[a] : v;
        }
    }
    for (int a = 0; a < 3; ++a) {
        for (int off = 16; off > 0; off >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(box + a, float_to_ordered(lo[a]));
            atomicMax(box + 3 + a, float_to_ordered(hi[a]));
        }
    }
}

// Inflates the box (rangesearch.h:44-46) and derives the cell parameters (:27-30).
__global__ void params_kernel(const int* __restrict__ box, float radius, float cell_factor, float* __restrict__ prm) {
    if (threadIdx.x != 0) return;
    float lo[3], hi[3], ext[3];
    for (int a = 0; a < 3; ++a) { lo[a] = ordered_to_float(box[a]); hi[a] = ordered_to_float(box[3 + a]); }
    for (int a = 0; a < 3; ++a) ext[a] = __fsub_rn(hi[a], lo[a]);
    for (int a = 0; a < 3; ++a) hi[a] = __fadd_rn(hi[a], __fmul_rn(ext[a], 0.001f));
    for (int a = 0; a < 3; ++a) lo[a] = __fsub_rn(lo[a], __fmul_rn(ext[a], 0.001f));
    const float cell = __fmul_rn(radius, cell_factor);
    for (int a = 0; a < 3; ++a) { prm[a] = lo[a]; prm[3 + a] = hi[a]; }
    prm[6] = radius;
    prm[7] = __fmul_rn(radius, radius);
    prm[8] = cell;
    prm[9] = __fdiv_rn(1.0f, cell);
}


__device__ __forceinline__ int cell_of_point(const float* prm, float px, float py, float pz, uint32_t table) {
    const float inv = prm[9];
    const int cx = (int)floorf(__fmul_rn(inv, __fsub_rn(px, prm[0])));
    const int cy = (int)floorf(__fmul_rn(inv, __fsub_rn(py, prm[1])));
    const int cz = (int)floorf(__fmul_rn(inv, __fsub_rn(pz, prm[2])));
    return hash_cell((uint32_t)cx, (uint32_t)cy, (uint32_t)cz, table);
}

__global__ void count_kernel(const float* __restrict__ pos, int stride, int n, const float* __restrict__ prm,
                             uint32_t table, int* __restrict__ counts, int* __restrict__ cell_of) {
    __shared__ float sp[10];
    if (threadIdx.x < 10) sp[threadIdx.x] = prm[threadIdx.x];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* p = pos + (size_t)i * stride;
        const int c = cell_of_point(sp, p[0], p[1], p[2], table);
        cell_of[i] = c;
        atomicAdd(counts + c, 1);
    }
}

// Three-phase exclusive scan: per-tile sums, scan of the tile sums, tile-local scan + offset.
__global__ void scan_tiles_kernel(const int* __restrict__ in, int n, int* __restrict__ tile_sums) {
    __shared__ int warp_sums[kBlock / 32];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int s = 0;
    for (int k = 0; k < kScanItems; ++k) s += (base + k < n) ? in[base + k] : 0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kBlock / 32; ++w) t += warp_sums[w];
        tile_sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the tile sums by one block (tiles <= kBlock * kScanItems * ... looped).
__global__ void scan_sums_kernel(int* __restrict__ sums, int n_tiles) {
    __shared__ int buf[kBlock];
    int carry = 0;
    for (int base = 0; base < n_tiles; base += kBlock) {
        const int i = base + threadIdx.x;
        const int v = i < n_tiles ? sums[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < kBlock; off <<= 1) {
            const int t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < n_tiles) sums[i] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        carry += buf[kBlock - 1];
        __syncthreads();
    }
}

// Writes inclusive ends (cell_ends) and exclusive starts (cursor) of every bucket. `starts`
// may alias `counts_in`: every thread reads its items before writing them.
__global__ void scan_apply_kernel(const int* counts_in, int n, const int* __restrict__ tile_off,
                                  int* __restrict__ ends, int* starts) {
    __shared__ int warp_sums[kBlock / 32];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
    for (int k = 0; k < kScanItems; ++k) { v[k] = (base + k < n) ? counts_in[base + k] : 0; s += v[k]; }
    // exclusive scan of per-thread sums within the block
    int incl = s;
    for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, off);
        if ((int)(threadIdx.x & 31) >= off) incl += t;
    }
    if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = incl;
    __syncthreads();
    int warp_off = 0;
    for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) warp_off += warp_sums[w];
    int run = tile_off[blockIdx.x] + warp_off + incl - s;
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) {
            starts[base + k] = run;
            run += v[k];
            ends[base + k] = run;
        }
    }
}

__global__ void scatter_kernel(const float* __restrict__ pos, int stride, int n, const int* __restrict__ cell_of,
                               int* __restrict__ cursor, float4* __restrict__ sorted) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* p = pos + (size_t)i * stride;
        const int slot = atomicAdd(cursor + cell_of[i], 1);
        sorted[slot] = make_float4(p[0], p[1], p[2], __int_as_float(i));
    }
}

// One query per thread (the search itself is grid_query_knn, hashgrid_query.cuh).
__global__ void query_kernel(const float4* __restrict__ sorted, const int* __restrict__ ends,
                             const float* __restrict__ prm, uint32_t table, const float* __restrict__ queries,
                             int nq, int k, int* __restrict__ out_ids, int* __restrict__ out_count,
                             float* __restrict__ out_d2) {
    __shared__ float sp[10];
    if (threadIdx.x < 10) sp[threadIdx.x] = prm[threadIdx.x];
    __syncthreads();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const float qx = queries[3 * (size_t)q + 0], qy = queries[3 * (size_t)q + 1], qz = queries[3 * (size_t)q + 2];
    float dist[kMaxK];
    int ids[kMaxK];
    const int count = grid_query_knn(sorted, ends, sp, table, qx, qy, qz, k, dist, ids);
    out_count[q] = count;
    int* o = out_ids + (size_t)q * k;
    for (int i = 0; i < k; ++i) o[i] = i < count ? ids[i] : -1;
    if (out_d2) {
        float* od = out_d2 + (size_t)q * k;
        for (int i = 0; i < k; ++i) od[i] = i < count ? dist[i] : 0.0f;
    }
}

// One warp per query (k <= 32; the search is grid_query_knn_warp): lane i writes entry i.
__global__ void __launch_bounds__(128) query_warp_kernel(const float4* __restrict__ sorted,
                                                         const int* __restrict__ ends, const float* __restrict__ prm,
                                                         uint32_t table, const float* __restrict__ queries, int nq,
                                                         int k, int* __restrict__ out_ids, int* __restrict__ out_count,
                                                         float* __restrict__ out_d2) {
    __shared__ float sp[10];
    if (threadIdx.x < 10) sp[threadIdx.x] = prm[threadIdx.x];
    __syncthreads();
    const long long q = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (q >= nq) return;   // uniform across the warp
    const int lane = threadIdx.x & 31;
    const float qx = queries[3 * q + 0], qy = queries[3 * q + 1], qz = queries[3 * q + 2];
    float my_d;
    int my_id;
    const int count = grid_query_knn_warp(sorted, ends, sp, table, qx, qy, qz, k, my_d, my_id);
    if (lane == 0) out_count[q] = count;
    if (lane < k) {
        out_ids[q * k + lane] = lane < count ? my_id : -1;
        if (out_d2) out_d2[q * k + lane] = lane < count ? my_d : 0.0f;
    }
}

// Grid-stride launches over n items: at most 8 blocks per SM of the current device (SM
// counts cached per device index).
int grid_for(int n) {
    static std::mutex mu;
    static int sms_of[64] = {};
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64) {
        std::lock_guard<std::mutex> lk(mu);
        if (!sms_of[dev]) cudaDeviceGetAttribute(&sms_of[dev], cudaDevAttrMultiProcessorCount, dev);
        sms = sms_of[dev];
    } else {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return std::max(1, std::min((n + kBlock - 1) / kBlock, std::max(sms, 1) * 8));
}

// Grows geometrically: reallocation synchronizes the device, and a grid rebuilt every
// iteration over a slowly growing photon count would otherwise reallocate every time.
template <typename T>
bool grow(T** p, int* cap, int need) {
    if (*cap >= need) return true;
    const int n = (int)std::min<long long>(std::max<long long>(need, (long long)*cap * 3 / 2), INT_MAX);
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (!ok(cudaMalloc((void**)p, sizeof(T) * (size_t)std::max(n, 1)), "cudaMalloc")) return false;
    *cap = n;
    return true;
}

}  // namespace

bool hashgrid_device_view(const imbart_hashgrid* g, const void** sorted, const int** cell_ends, const float** params,
                          int* table, int* n) {
    if (!g || g->table == 0) return false;
    *sorted = g->sorted;
    *cell_ends = g->cell_ends;
    *params = g->params;
    *table = g->table;
    *n = g->n;
    return true;
}

}  // namespace imbart

using namespace imbart;

extern "C" {

imbart_hashgrid* imbart_hashgrid_create(int device) {
    imbart_hashgrid* g = new imbart_hashgrid;
    g->device = device;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    const bool good = ok(cudaMalloc((void**)&g->params, sizeof(float) * 16), "cudaMalloc");
    cudaSetDevice(prev);
    if (!good) { delete g; return nullptr; }
    return g;
}

void imbart_hashgrid_destroy(imbart_hashgrid* g) {
    if (!g) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    cudaFree(g->sorted); cudaFree(g->cell_ends); cudaFree(g->cell_of); cudaFree(g->cursor);
    cudaFree(g->block_sums); cudaFree(g->params);
    cudaSetDevice(prev);
    delete g;
}

int imbart_hashgrid_build(imbart_hashgrid* g, const float* positions, int stride, int n, float radius,
                          float cell_factor, int table_size, void* stream) {
    if (!g || n < 0 || (n > 0 && !positions) || stride < 3 || !(radius > 0.0f) || !(cell_factor > 0.0f)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_build: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (table_size <= 0) table_size = std::max(2 * n, 1);   // reference: 2 * photons (rangesearch.h:26)
    cudaStream_t st = (cudaStream_t)stream;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    int rc = 0;
    const int n_tiles = (table_size + kScanTile - 1) / kScanTile;
    int* box = nullptr;
    if (!grow(&g->sorted, &g->sorted_cap, n) || !grow(&g->cell_of, &g->cell_of_cap, n) ||
        !grow(&g->cell_ends, &g->ends_cap, table_size) || !grow(&g->cursor, &g->cursor_cap, table_size) ||
        !grow(&g->block_sums, &g->block_sums_cap, n_tiles + 8))
        rc = IMBART_ERR_OUT_OF_MEMORY;
    if (!rc) {
        box = g->block_sums + n_tiles;   // 6 ints after the tile sums
        const int grid = grid_for(std::max(n, 1));
        bbox_init_kernel<<<1, 32, 0, st>>>(box);
        if (n > 0) bbox_kernel<<<grid, kBlock, 0, st>>>(positions, stride, n, box);
        params_kernel<<<1, 32, 0, st>>>(box, radius, cell_factor, g->params);
        ok(cudaMemsetAsync(g->cursor, 0, sizeof(int) * (size_t)table_size, st), "cudaMemsetAsync");
        if (n > 0) count_kernel<<<grid, kBlock, 0, st>>>(positions, stride, n, g->params, (uint32_t)table_size,
                                                         g->cursor, g->cell_of);
        scan_tiles_kernel<<<n_tiles, kBlock, 0, st>>>(g->cursor, table_size, g->block_sums);
        scan_sums_kernel<<<1, kBlock, 0, st>>>(g->block_sums, n_tiles);
        scan_apply_kernel<<<n_tiles, kBlock, 0, st>>>(g->cursor, table_size, g->block_sums, g->cell_ends, g->cursor);
        if (n > 0) scatter_kernel<<<grid, kBlock, 0, st>>>(positions, stride, n, g->cell_of, g->cursor, g->sorted);
        note_launches(n > 0 ? 8 : 5);
        if (!ok(cudaGetLastError(), "hash grid build")) rc = IMBART_ERR_CUDA;
        g->n = n;
        g->table = table_size;
        g->cell_factor = cell_factor;
    }
    cudaSetDevice(prev);
    return rc;
}

int imbart_hashgrid_query(const imbart_hashgrid* g, const float* queries, int nq, int k, int* out_ids,
                          int* out_counts, float* out_d2, void* stream) {
    if (!g || nq < 0 || k < 1 || k > kMaxK || (nq > 0 && (!queries || !out_ids || !out_counts)) || g->table == 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_query: invalid argument (k must be 1..64, grid built)");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (!(g->cell_factor >= 1.0f)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_query: the grid's cells are smaller than the radius "
                                               "(build with cell_factor >= 1)");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (nq == 0) return 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    if (k <= 32) {
        // One warp per query: coalesced photon loads and the list in registers.
        const long long grid = ((long long)nq * 32 + 127) / 128;
        query_warp_kernel<<<(unsigned)grid, 128, 0, (cudaStream_t)stream>>>(
            g->sorted, g->cell_ends, g->params, (uint32_t)g->table, queries, nq, k, out_ids, out_counts, out_d2);
    } else {
        const int grid = (nq + 127) / 128;
        query_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(g->sorted, g->cell_ends, g->params, (uint32_t)g->table,
                                                             queries, nq, k, out_ids, out_counts, out_d2);
    }
    note_launches(1);
    const bool good = ok(cudaGetLastError(), "hash grid query");
    cudaSetDevice(prev);
    return good ? 0 : IMBART_ERR_CUDA;
}

}  // extern "C"

namespace imbart {
namespace {
// Staging buffers and a stream of one host thread for the host-array entry points (on one
// device at a time; they move to another device when the grid does).
struct HostStaging {
    int device = -1;
    cudaStream_t stream = nullptr;
    float* in = nullptr;
    size_t in_cap = 0;
    int* ids = nullptr;
    size_t out_cap = 0;
    float* d2 = nullptr;
    size_t d2_cap = 0;
    int* counts = nullptr;
    size_t count_cap = 0;

    void release() {
        cudaFree(in); cudaFree(ids); cudaFree(d2); cudaFree(counts);
        if (stream) cudaStreamDestroy(stream);
        in = nullptr; ids = nullptr; d2 = nullptr; counts = nullptr; stream = nullptr;
        in_cap = out_cap = d2_cap = count_cap = 0;
    }
    ~HostStaging() { if (device >= 0) release(); }

    bool on(int dev) {
        if (device == dev) return true;
        if (device >= 0) {
            int prev = 0;
            cudaGetDevice(&prev);
            cudaSetDevice(device);
            release();
            cudaSetDevice(prev);
        }
        device = dev;
        return ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    }
};

template <typename T>
bool stage(T** p, size_t* cap, size_t need) {
    if (*cap >= need) return true;
    const size_t n = std::max(need, *cap * 3 / 2);
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (!ok(cudaMalloc((void**)p, sizeof(T) * n), "cudaMalloc")) return false;
    *cap = n;
    return true;
}

thread_local HostStaging t_staging;
}  // namespace
}  // namespace imbart

extern "C" {

int imbart_hashgrid_build_host(imbart_hashgrid* g, const float* positions, int stride, int n, float radius,
                               float cell_factor, int table_size) {
    if (!g || n < 0 || (n > 0 && !positions) || stride < 3) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_build_host: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    HostStaging& h = t_staging;
    const size_t floats = (size_t)std::max(n, 1) * (size_t)stride;
    int rc = 0;
    if (!h.on(g->device) || !stage(&h.in, &h.in_cap, floats)) rc = IMBART_ERR_CUDA;
    if (!rc && n > 0 &&
        !ok(cudaMemcpyAsync(h.in, positions, sizeof(float) * (size_t)n * stride, cudaMemcpyHostToDevice, h.stream),
            "cudaMemcpyAsync"))
        rc = IMBART_ERR_CUDA;
    if (!rc) rc = imbart_hashgrid_build(g, h.in, stride, n, radius, cell_factor, table_size, h.stream);
    if (!rc && !ok(cudaStreamSynchronize(h.stream), "imbart_hashgrid_build_host")) rc = IMBART_ERR_CUDA;
    cudaSetDevice(prev);
    return rc;
}

int imbart_hashgrid_query_host(const imbart_hashgrid* g, const float* queries, int nq, int k, int* out_ids,
                               int* out_counts, float* out_d2) {
    if (!g || nq < 0 || k < 1 || k > kMaxK || (nq > 0 && (!queries || !out_ids || !out_counts))) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_query_host: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (nq == 0) return 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    HostStaging& h = t_staging;
    const size_t nk = (size_t)nq * (size_t)k;
    int rc = 0;
    if (!h.on(g->device) || !stage(&h.in, &h.in_cap, (size_t)nq * 3) || !stage(&h.ids, &h.out_cap, nk) ||
        !stage(&h.counts, &h.count_cap, (size_t)nq))
        rc = IMBART_ERR_CUDA;
    if (!rc && out_d2 && !stage(&h.d2, &h.d2_cap, nk)) rc = IMBART_ERR_CUDA;
    if (!rc && !ok(cudaMemcpyAsync(h.in, queries, sizeof(float) * 3 * (size_t)nq, cudaMemcpyHostToDevice, h.stream),
                   "cudaMemcpyAsync"))
        rc = IMBART_ERR_CUDA;
    if (!rc) rc = imbart_hashgrid_query(g, h.in, nq, k, h.ids, h.counts, out_d2 ? h.d2 : nullptr, h.stream);
    if (!rc && !(ok(cudaMemcpyAsync(out_ids, h.ids, sizeof(int) * nk, cudaMemcpyDeviceToHost, h.stream), "D2H") &&
                 ok(cudaMemcpyAsync(out_counts, h.counts, sizeof(int) * (size_t)nq, cudaMemcpyDeviceToHost, h.stream),
                    "D2H") &&
                 (!out_d2 || ok(cudaMemcpyAsync(out_d2, h.d2, sizeof(float) * nk, cudaMemcpyDeviceToHost, h.stream),
                                "D2H")) &&
                 ok(cudaStreamSynchronize(h.stream), "imbart_hashgrid_query_host")))
        rc = IMBART_ERR_CUDA;
    cudaSetDevice(prev);
    return rc;
}

int imbart_hashgrid_get_params(const imbart_hashgrid* g, float* params10, int* n, int* table_size) {
    if (!g) { set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_get_params"); return IMBART_ERR_INVALID_ARGUMENT; }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    bool good = true;
    if (params10) good = ok(cudaMemcpy(params10, g->params, sizeof(float) * 10, cudaMemcpyDeviceToHost), "cudaMemcpy");
    cudaSetDevice(prev);
    if (n) *n = g->n;
    if (table_size) *table_size = g->table;
    return good ? 0 : IMBART_ERR_CUDA;
}

int imbart_hashgrid_get_arrays(const imbart_hashgrid* g, const void** sorted, const int** cell_ends) {
    if (!g) { set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_get_arrays"); return IMBART_ERR_INVALID_ARGUMENT; }
    if (sorted) *sorted = g->sorted;
    if (cell_ends) *cell_ends = g->cell_ends;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Hash-grid build that allocates nothing.
//
// Some callers must not allocate device memory at all: a server that admits work against a
// fixed HBM budget accounts for every byte up front, and cudaMalloc / cudaFree synchronize
// the device, stalling the other requests' streams; hosts that own all device memory
// through their own arena hand out only buffers they sized themselves. For them the build's
// scratch (bucket id per photon, bucket cursors, scan tile sums, bounding box) lives in one
// statically sized device array below, held by every GPU that loads the library until the
// process exits: 4 * (2^20 + 2^21 + 1024 + 8) bytes, about 12 MiB. The caller passes the
// inputs and the outputs it allocated itself.
// ---------------------------------------------------------------------------------------
namespace imbart {
namespace {
constexpr int kNoAllocMaxPhotons = 1 << 20;
constexpr int kNoAllocMaxTable = 1 << 21;
constexpr int kNoAllocTiles = (kNoAllocMaxTable + kScanTile - 1) / kScanTile;
constexpr size_t kNoAllocInts = (size_t)kNoAllocMaxPhotons + kNoAllocMaxTable + kNoAllocTiles + 8;

static __device__ __align__(256) int g_noalloc_scratch[kNoAllocInts];

// Device address of the scratch array, looked up once per device with that device current.
std::mutex g_noalloc_mutex;
int* g_noalloc_addr[64] = {};
}  // namespace
}  // namespace imbart

extern "C" int imbart_hashgrid_build_noalloc(const float* positions, int stride, int n, float radius,
                                             float cell_factor, int table_size, void* sorted_out,
                                             int* cell_ends_out, float* params_out, void* stream) {
    if (n < 0 || (n > 0 && (!positions || !sorted_out)) || stride < 3 || !(radius > 0.0f) || !(cell_factor > 0.0f) ||
        !cell_ends_out || !params_out) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_hashgrid_build_noalloc: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    if (table_size <= 0) table_size = std::max(2 * n, 1);
    if (n > kNoAllocMaxPhotons || table_size > kNoAllocMaxTable) {
        set_error(IMBART_ERR_LIMIT, "imbart_hashgrid_build_noalloc: at most 1048576 photons and 2097152 buckets "
                                    "(the size of its static scratch); use imbart_hashgrid_build for more");
        return IMBART_ERR_LIMIT;
    }
    // A launch error left pending by earlier work on this thread is cleared here, so that
    // the status returned below describes this call's own launches.
    (void)cudaGetLastError();
    int device = 0;
    if (!ok(cudaGetDevice(&device), "cudaGetDevice")) return IMBART_ERR_CUDA;
    if (device < 0 || device >= 64) {
        set_error(IMBART_ERR_LIMIT, "imbart_hashgrid_build_noalloc: device index above 63");
        return IMBART_ERR_LIMIT;
    }
    int* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mutex);
        if (!g_noalloc_addr[device]) {
            void* addr = nullptr;
            if (!ok(cudaGetSymbolAddress(&addr, g_noalloc_scratch), "cudaGetSymbolAddress")) return IMBART_ERR_CUDA;
            g_noalloc_addr[device] = static_cast<int*>(addr);
        }
        scratch = g_noalloc_addr[device];
    }
    int* cell_of = scratch;
    int* cursor = cell_of + kNoAllocMaxPhotons;
    int* tile_sums = cursor + kNoAllocMaxTable;
    const int n_tiles = (table_size + kScanTile - 1) / kScanTile;
    int* box = tile_sums + kNoAllocTiles;
    float4* sorted = static_cast<float4*>(sorted_out);
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = grid_for(std::max(n, 1));
    // The scratch keeps the previous call's contents: the box and the bucket counts are
    // reset here; bucket ids, tile sums and cursors are fully rewritten before they are read.
    bbox_init_kernel<<<1, 32, 0, st>>>(box);
    if (n > 0) bbox_kernel<<<grid, kBlock, 0, st>>>(positions, stride, n, box);
    params_kernel<<<1, 32, 0, st>>>(box, radius, cell_factor, params_out);
    if (!ok(cudaMemsetAsync(cursor, 0, sizeof(int) * (size_t)table_size, st), "cudaMemsetAsync")) return IMBART_ERR_CUDA;
    if (n > 0) count_kernel<<<grid, kBlock, 0, st>>>(positions, stride, n, params_out, (uint32_t)table_size, cursor,
                                                     cell_of);
    scan_tiles_kernel<<<n_tiles, kBlock, 0, st>>>(cursor, table_size, tile_sums);
    scan_sums_kernel<<<1, kBlock, 0, st>>>(tile_sums, n_tiles);
    scan_apply_kernel<<<n_tiles, kBlock, 0, st>>>(cursor, table_size, tile_sums, cell_ends_out, cursor);
    if (n > 0) scatter_kernel<<<grid, kBlock, 0, st>>>(positions, stride, n, cell_of, cursor, sorted);
    note_launches(n > 0 ? 8 : 5);
    return ok(cudaGetLastError(), "imbart_hashgrid_build_noalloc") ? 0 : IMBART_ERR_CUDA;
}
