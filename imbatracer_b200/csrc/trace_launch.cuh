// Launch shapes of the persistent traversal kernel, shared by the translation units of the
// 8-slot kernels (trace.cu), the 4-slot kernels for 4-wide scenes (trace_w4.cu) and the flat
// kernels for single identity-instance scenes (trace_flat.cu).
// Variants 1..10 are per-lane shapes, 11..17 the shapes with the cooperative triangle phase.
#pragma once

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "trace_kernel.cuh"

namespace imbart {

// A traversal launch: kernel, grid, block (the parameters are the TraceParams beside it).
struct LaunchSpec {
    const void* func = nullptr;
    dim3 grid, block;
};

template <typename Kernel>
int max_grid(Kernel k, int block, int device) {
    static std::mutex m;
    static std::map<std::pair<const void*, int>, int> cache;
    std::lock_guard<std::mutex> lk(m);
    const auto key = std::make_pair((const void*)k, device);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int g = std::max(1, per_sm) * std::max(1, sms);
    cache[key] = g;
    return g;
}

// One persistent block per resident slot (fewer for short queues).
template <int kSlots, bool kFlat, bool kAny, bool kMasked, bool kStats, int kBlock, int kMinBlocks, int kSh,
          bool kCoop = false>
LaunchSpec persistent_spec(int count, int device, float share, TraceParams& p) {
    auto k = trace_persistent<kAny, kMasked, kStats, kBlock, kMinBlocks, kSh, kCoop, kSlots, kFlat>;
    const int slots = std::max(1, (int)(max_grid(k, kBlock, device) * share));
    const int grid = std::min(slots, (count + kBlock - 1) / kBlock);
    p.total_warps = grid * (kBlock / 32);
    return {(const void*)k, dim3(grid), dim3(kBlock)};
}

template <int kSlots, bool kFlat, bool kAny, bool kMasked, bool kStats>
LaunchSpec variant_spec(int variant, int count, int device, float share, TraceParams& p) {
    switch (variant) {
        case 1: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 4, 16>(count, device, share, p);
        case 2: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 6, 12>(count, device, share, p);
        case 3: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 2, 16>(count, device, share, p);
        case 4: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 3, 12>(count, device, share, p);
        case 5: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 64, 8, 16>(count, device, share, p);
        case 6: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 4, 8>(count, device, share, p);
        case 7: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 7, 10>(count, device, share, p);
        case 8: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 4, 12>(count, device, share, p);
        case 9: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 4, 16>(count, device, share, p);
        case 10: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 8, 12>(count, device, share, p);
        // Cooperative triangle phase (all lanes test the warp's pending ray/triangle pairs).
        case 11: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 3, 12, true>(count, device, share, p);
        case 12: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 4, 8, true>(count, device, share, p);
        case 13: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 6, 12, true>(count, device, share, p);
        case 14: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 4, 16, true>(count, device, share, p);
        case 15: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 8, 12, true>(count, device, share, p);
        case 16: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 256, 4, 12, true>(count, device, share, p);
        case 17: return persistent_spec<kSlots, kFlat, kAny, kMasked, kStats, 128, 7, 10, true>(count, device, share, p);
        default: return {};
    }
}

template <bool kStats, int kSlots, bool kFlat = false>
LaunchSpec persistent_kernel_spec(int variant, bool any, bool masked, int count, int device, float share,
                                  TraceParams& p) {
    if (any && masked) return variant_spec<kSlots, kFlat, true, true, kStats>(variant, count, device, share, p);
    if (any) return variant_spec<kSlots, kFlat, true, false, kStats>(variant, count, device, share, p);
    if (masked) return variant_spec<kSlots, kFlat, false, true, kStats>(variant, count, device, share, p);
    return variant_spec<kSlots, kFlat, false, false, kStats>(variant, count, device, share, p);
}

// The 4-slot kernels (trace_w4.cu): the same shapes, for scenes converted 4-wide.
LaunchSpec persistent_kernel_spec_w4(bool stats, int variant, bool any, bool masked, int count, int device,
                                     float share, TraceParams& p);
// The flat kernels (trace_flat.cu): the same shapes for 8-wide scenes whose top level is one
// identity instance (TraceParams::direct_root >= 0, no per-ray roots).
LaunchSpec persistent_kernel_spec_flat(bool stats, int variant, bool any, bool masked, int count, int device,
                                       float share, TraceParams& p);

}  // namespace imbart
