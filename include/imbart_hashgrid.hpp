/* C++ adapter with the interface of the reference's photon hash grid, HashGrid<Iter, Photon>
 * (src/imbatracer/rangesearch/rangesearch.h:21-129), over libimbart's GPU grid
 * (imbart_hashgrid_build_host / imbart_hashgrid_query_host in imbart.h).
 *
 *   build(begin, end, radius)  rangesearch.h:24-75   photons converted with Photon(*it) and
 *                                                     kept on the host in build order; their
 *                                                     positions (it->position()) go to the
 *                                                     GPU grid: cell size 2r, 2n buckets
 *   query(pos, out, k)         rangesearch.h:77-129  at most the k nearest photons within the
 *                                                     radius into out[0..count) as pointers
 *                                                     into the photon array; returns count
 *
 * The neighbour sets are the reference's bit for bit (same box, cells, hash and k-nearest
 * rule); within equal distances the order is by build index. query() is one device round
 * trip per call and may be called from several threads at once (the reference calls it from
 * its shading threads, vcm.cpp:571-576); query_batch() serves many positions per round trip.
 * The reference's HashGrid reports no errors; the adapter keeps that interface, so a failed
 * build leaves an empty grid (queries find nothing) and imbart_last_error() says why.
 *
 * Only <vector> and imbart.h are needed: no CUDA headers. Link with libimbart.
 */
#pragma once

#include <cstddef>
#include <vector>

#include "imbart.h"

namespace imbart {

template <typename Iter, typename Photon>
class GpuHashGrid {
public:
    explicit GpuHashGrid(int device = 0) : device_(device) {}
    ~GpuHashGrid() {
        if (grid_) imbart_hashgrid_destroy(grid_);
    }
    GpuHashGrid(const GpuHashGrid&) = delete;
    GpuHashGrid& operator=(const GpuHashGrid&) = delete;

    void build(const Iter& photons_begin, const Iter& photons_end, float radius) {
        photons_.clear();
        positions_.clear();
        built_ = false;
        radius_ = radius;
        if (!grid_) grid_ = imbart_hashgrid_create(device_);
        if (!grid_) return;
        const std::ptrdiff_t n = photons_end - photons_begin;
        photons_.reserve((size_t)n);
        positions_.reserve(3 * (size_t)n);
        for (Iter it = photons_begin; it != photons_end; ++it) {
            photons_.emplace_back(*it);
            const auto& p = it->position();
            positions_.push_back(p.x);
            positions_.push_back(p.y);
            positions_.push_back(p.z);
        }
        built_ = imbart_hashgrid_build_host(grid_, positions_.data(), 3, (int)n, radius, 2.0f, 0) == 0;
    }

    template <typename Vec3, typename Container>
    int query(const Vec3& query_pos, Container& out, int k) const {
        if (!built_ || k < 1 || k > 64) return 0;
        const float q[3] = {query_pos.x, query_pos.y, query_pos.z};
        int ids[64];
        int count = 0;
        if (imbart_hashgrid_query_host(grid_, q, 1, k, ids, &count, nullptr) != 0) return 0;
        for (int i = 0; i < count; ++i) out[i] = &photons_[(size_t)ids[i]];
        return count;
    }

    /* nq queries (xyz packed) in one round trip: ids (nq*k, build indices, -1 padded) and
     * counts (nq). Returns 0 or an imbart error code. */
    int query_batch(const float* positions, int nq, int k, int* ids, int* counts) const {
        if (!built_) return IMBART_ERR_INVALID_ARGUMENT;
        return imbart_hashgrid_query_host(grid_, positions, nq, k, ids, counts, nullptr);
    }

    const Photon* photons() const { return photons_.data(); }
    size_t size() const { return photons_.size(); }
    float radius() const { return radius_; }

private:
    int device_;
    imbart_hashgrid* grid_ = nullptr;
    bool built_ = false;
    float radius_ = 0.0f;
    std::vector<Photon> photons_;
    std::vector<float> positions_;
};

}  // namespace imbart
