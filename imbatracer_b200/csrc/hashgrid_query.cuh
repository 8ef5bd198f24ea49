// The photon hash grid's k-capped radius query for one point, shared by the batched query
// kernel (hashgrid.cu) and the vertex-merging step of the VCM camera pass (vcm.cu).
// HashGrid::query (src/imbatracer/rangesearch/rangesearch.h:77-129): outside the grid's box
// nothing is found; otherwise the home cell and, per axis, the neighbour on the side of the
// nearer face are scanned (8 buckets in the reference's order; a bucket reached twice is
// scanned twice), photons with squared distance <= r^2 are kept, at most k of them by the
// reference's insertion rule (a tie with the current k-th replaces it once the list is full).
// The list is then ordered by (distance, photon index). Every float operation is explicitly
// rounded, so cells and distances equal the reference's bit for bit.
//
// Those eight cells hold every photon within r only while the cell size is at least 2r (the
// reference's grid: cell = 2r). Grids with smaller cells (r <= cell < 2r, e.g. cell = r) are
// queried over every cell the box [q - r, q + r] touches instead — up to 4 per axis, bounds
// rounded outward and mapped to cells with the build's own rounding, so no photon within r
// is missed — in x-major order, each bucket once.
#pragma once

#include <stdint.h>

namespace imbart {

constexpr int kGridMaxK = 64;

__device__ __forceinline__ int hash_cell(uint32_t x, uint32_t y, uint32_t z, uint32_t table) {
    return (int)(((x * 73856093u) ^ (y * 19349663u) ^ (z * 83492791u)) % table);
}

// The cells a query scans. Reference mode (cell >= 2r): cell j of 8 is (j&4 ? xo : x0,
// j&2 ? yo : y0, j&1 ? zo : z0) with (x0, y0, z0) the home cell and (xo, yo, zo) the nearer
// neighbours. Range mode: cell j is (x0 + j / (ny nz), y0 + (j / nz) % ny, z0 + j % nz).
struct GridCells {
    bool ref_mode;
    int n;                       // cells to visit
    int x0, y0, z0;              // home cell / range start
    int xo, yo, zo;              // reference mode: neighbours
    int ny, nz;                  // range mode: extent in y and z
};

// Cell coordinate of a coordinate value, rounded as the build rounds it.
__device__ __forceinline__ int grid_coord(float v, float lo, float inv) {
    return (int)floorf(__fmul_rn(inv, __fsub_rn(v, lo)));
}

// prm: lo xyz, hi xyz, radius, r^2, cell size, 1 / cell size. False outside the grid's box.
__device__ __forceinline__ bool grid_cells(const float* prm, float qx, float qy, float qz, GridCells& g) {
    const bool inside = qx >= prm[0] && qy >= prm[1] && qz >= prm[2] && qx <= prm[3] && qy <= prm[4] && qz <= prm[5];
    if (!inside) return false;
    const float inv = prm[9], r = prm[6];
    g.ref_mode = prm[8] >= __fmul_rn(2.0f, r);
    if (g.ref_mode) {
        const float cx = __fmul_rn(inv, __fsub_rn(qx, prm[0]));
        const float cy = __fmul_rn(inv, __fsub_rn(qy, prm[1]));
        const float cz = __fmul_rn(inv, __fsub_rn(qz, prm[2]));
        const float fx = floorf(cx), fy = floorf(cy), fz = floorf(cz);
        g.x0 = (int)fx; g.y0 = (int)fy; g.z0 = (int)fz;
        g.xo = g.x0 + (__fsub_rn(cx, fx) < 0.5f ? -1 : 1);
        g.yo = g.y0 + (__fsub_rn(cy, fy) < 0.5f ? -1 : 1);
        g.zo = g.z0 + (__fsub_rn(cz, fz) < 0.5f ? -1 : 1);
        g.n = 8;
    } else {
        // A photon within r has each coordinate in [q - r, q + r]; the bounds are rounded
        // outward and mapped like photon coordinates (a monotone map), so its cell is inside.
        g.x0 = grid_coord(__fsub_rd(qx, r), prm[0], inv);
        g.y0 = grid_coord(__fsub_rd(qy, r), prm[1], inv);
        g.z0 = grid_coord(__fsub_rd(qz, r), prm[2], inv);
        const int nx = min(grid_coord(__fadd_ru(qx, r), prm[0], inv) - g.x0 + 1, 4);
        g.ny = min(grid_coord(__fadd_ru(qy, r), prm[1], inv) - g.y0 + 1, 4);
        g.nz = min(grid_coord(__fadd_ru(qz, r), prm[2], inv) - g.z0 + 1, 4);
        g.n = nx * g.ny * g.nz;
    }
    return true;
}

__device__ __forceinline__ int grid_cell_bucket(const GridCells& g, int j, uint32_t table) {
    int x, y, z;
    if (g.ref_mode) {
        x = (j & 4) ? g.xo : g.x0;
        y = (j & 2) ? g.yo : g.y0;
        z = (j & 1) ? g.zo : g.z0;
    } else {
        x = g.x0 + j / (g.ny * g.nz);
        y = g.y0 + (j / g.nz) % g.ny;
        z = g.z0 + j % g.nz;
    }
    return hash_cell((uint32_t)x, (uint32_t)y, (uint32_t)z, table);
}

// Range mode visits each bucket once: a cell whose bucket an earlier cell already had is skipped.
__device__ __forceinline__ bool grid_bucket_seen(const GridCells& g, int j, int c, uint32_t table) {
    if (g.ref_mode) return false;
    for (int i = 0; i < j; ++i)
        if (grid_cell_bucket(g, i, table) == c) return true;
    return false;
}

// sorted: photons in bucket order (xyz + original index bits), ends: inclusive bucket ends.
// Returns the count; dist / ids (capacity k <= kGridMaxK) hold the result.
__device__ __forceinline__ int grid_query_knn(const float4* __restrict__ sorted, const int* __restrict__ ends,
                                              const float* prm, uint32_t table, float qx, float qy, float qz, int k,
                                              float* dist, int* ids) {
    int count = 0;
    GridCells g;
    if (!grid_cells(prm, qx, qy, qz, g)) return 0;
    const float r2 = prm[7];
    for (int j = 0; j < g.n; ++j) {
        const int c = grid_cell_bucket(g, j, table);
        if (grid_bucket_seen(g, j, c, table)) continue;
        const int b = c == 0 ? 0 : __ldg(ends + c - 1);
        const int e = __ldg(ends + c);
        for (int s = b; s < e; ++s) {
            const float4 ph = __ldg(sorted + s);
            const float dx = __fsub_rn(qx, ph.x), dy = __fsub_rn(qy, ph.y), dz = __fsub_rn(qz, ph.z);
            const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            if (!(d2 <= r2)) continue;
            if (count == k) {
                if (dist[count - 1] < d2) continue;
            } else {
                count++;
            }
            dist[count - 1] = d2;
            ids[count - 1] = __float_as_int(ph.w);
            for (int l = count - 2; l >= 0; --l) {
                if (dist[l] > d2) {
                    const float td = dist[l]; dist[l] = dist[l + 1]; dist[l + 1] = td;
                    const int ti = ids[l]; ids[l] = ids[l + 1]; ids[l + 1] = ti;
                } else {
                    break;
                }
            }
        }
    }
    // Deterministic order among equal distances: by photon index.
    for (int i = 1; i < count; ++i) {
        const float d = dist[i];
        const int id = ids[i];
        int l = i - 1;
        while (l >= 0 && dist[l] == d && ids[l] > id) { dist[l + 1] = dist[l]; ids[l + 1] = ids[l]; --l; }
        dist[l + 1] = d;
        ids[l + 1] = id;
    }
    return count;
}

// The same query with one warp per point (k <= 32; every lane of the warp calls it with the
// same point). The 32 lanes scan each bucket together, in the reference's order; photons
// inside the radius are inserted in scan order into a k-nearest list held one entry per lane
// (lane i: entry i), with the reference's insertion rule (after every kept photon at distance
// <= d2; when the list is full the last entry leaves first). Equal distances are then ordered
// by photon index, so the list equals grid_query_knn's. Returns the count (warp-uniform).
__device__ __forceinline__ int grid_query_knn_warp(const float4* __restrict__ sorted, const int* __restrict__ ends,
                                                   const float* prm, uint32_t table, float qx, float qy, float qz,
                                                   int k, float& my_d, int& my_id) {
    const int lane = threadIdx.x & 31;
    my_d = 0.0f;
    my_id = -1;
    int count = 0;
    GridCells gc;
    if (!grid_cells(prm, qx, qy, qz, gc)) return 0;
    const float r2 = prm[7];
    // Lane j of a chunk computes cell (chunk + j)'s bucket; in range mode buckets met before
    // (lower lane or the previous chunk) are dropped, so each is scanned once.
    int prev_bucket = -1;
    for (int c0 = 0; c0 < gc.n; c0 += 32) {
        const int jj = c0 + lane;
        const int my_bucket = jj < gc.n ? grid_cell_bucket(gc, jj, table) : -2 - lane;
        bool seen = false;
        if (!gc.ref_mode) {
            const unsigned same = __match_any_sync(0xffffffffu, my_bucket);
            seen = (same & ((1u << lane) - 1u)) != 0u;
            if (c0 > 0)
                for (int l = 0; l < 32; ++l) seen |= __shfl_sync(0xffffffffu, prev_bucket, l) == my_bucket;
        }
        unsigned todo = __ballot_sync(0xffffffffu, jj < gc.n && !seen);
        prev_bucket = my_bucket;
        while (todo) {
            const int cl = __ffs(todo) - 1;
            todo &= todo - 1;
            const int c = __shfl_sync(0xffffffffu, my_bucket, cl);
            const int b = c == 0 ? 0 : __ldg(ends + c - 1);
            const int e = __ldg(ends + c);
            for (int base = b; base < e; base += 32) {
                const int s = base + lane;
                float d2 = 0.0f;
                int id = -1;
                bool within = false;
                if (s < e) {
                    const float4 ph = __ldg(sorted + s);
                    const float dx = __fsub_rn(qx, ph.x), dy = __fsub_rn(qy, ph.y), dz = __fsub_rn(qz, ph.z);
                    d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                    id = __float_as_int(ph.w);
                    within = d2 <= r2;
                }
                unsigned cand = __ballot_sync(0xffffffffu, within);
                while (cand) {
                    const int src = __ffs(cand) - 1;
                    cand &= cand - 1;
                    const float cd = __shfl_sync(0xffffffffu, d2, src);
                    const int cid = __shfl_sync(0xffffffffu, id, src);
                    int kept;
                    if (count == k) {
                        const float last = __shfl_sync(0xffffffffu, my_d, k - 1);
                        if (last < cd) continue;
                        kept = k - 1;
                    } else {
                        kept = count;
                        count++;
                    }
                    const int pos = __popc(__ballot_sync(0xffffffffu, lane < kept && my_d <= cd));
                    const float up_d = __shfl_up_sync(0xffffffffu, my_d, 1);
                    const int up_id = __shfl_up_sync(0xffffffffu, my_id, 1);
                    if (lane > pos && lane <= kept) { my_d = up_d; my_id = up_id; }
                    if (lane == pos) { my_d = cd; my_id = cid; }
                }
            }
        }
    }
    // Equal distances by photon index (odd-even transposition over adjacent equal pairs).
    const float next_d = __shfl_down_sync(0xffffffffu, my_d, 1);
    const unsigned ties = __ballot_sync(0xffffffffu, lane + 1 < count && my_d == next_d);
    if (ties) {
        for (int pass = 0; pass < count; ++pass) {
            const float nd = __shfl_down_sync(0xffffffffu, my_d, 1);
            const int nid = __shfl_down_sync(0xffffffffu, my_id, 1);
            const float pd = __shfl_up_sync(0xffffffffu, my_d, 1);
            const int pid = __shfl_up_sync(0xffffffffu, my_id, 1);
            const bool left = ((lane & 1) == (pass & 1));   // this lane is the left of its pair
            if (left) {
                if (lane + 1 < count && my_d == nd && my_id > nid) my_id = nid;
            } else if (lane >= 1 && lane < count) {
                if (pd == my_d && pid > my_id) my_id = pid;
            }
        }
    }
    return count;
}

}  // namespace imbart
