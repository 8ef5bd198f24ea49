// The photon hash grid's k-capped radius query for one point, shared by the batched query
// kernel (hashgrid.cu) and the vertex-merging step of the VCM camera pass (vcm.cu).
// HashGrid::query (src/imbatracer/rangesearch/rangesearch.h:77-129): outside the grid's box
// nothing is found; otherwise the home cell and, per axis, the neighbour on the side of the
// nearer face are scanned (8 buckets in the reference's order; a bucket reached twice is
// scanned twice), photons with squared distance <= r^2 are kept, at most k of them by the
// reference's insertion rule (a tie with the current k-th replaces it once the list is full).
// The list is then ordered by (distance, photon index). Every float operation is explicitly
// rounded, so cells and distances equal the reference's bit for bit.
#pragma once

#include <stdint.h>

namespace imbart {

constexpr int kGridMaxK = 64;

__device__ __forceinline__ int hash_cell(uint32_t x, uint32_t y, uint32_t z, uint32_t table) {
    return (int)(((x * 73856093u) ^ (y * 19349663u) ^ (z * 83492791u)) % table);
}

// prm: lo xyz, hi xyz, radius, r^2, cell size, 1 / cell size. sorted: photons in bucket order
// (xyz + original index bits), ends: inclusive bucket ends. Returns the count; dist / ids
// (capacity k <= kGridMaxK) hold the result.
__device__ __forceinline__ int grid_query_knn(const float4* __restrict__ sorted, const int* __restrict__ ends,
                                              const float* prm, uint32_t table, float qx, float qy, float qz, int k,
                                              float* dist, int* ids) {
    int count = 0;
    const bool inside = qx >= prm[0] && qy >= prm[1] && qz >= prm[2] && qx <= prm[3] && qy <= prm[4] && qz <= prm[5];
    if (!inside) return 0;
    const float inv = prm[9], r2 = prm[7];
    const float cx = __fmul_rn(inv, __fsub_rn(qx, prm[0]));
    const float cy = __fmul_rn(inv, __fsub_rn(qy, prm[1]));
    const float cz = __fmul_rn(inv, __fsub_rn(qz, prm[2]));
    const float fx = floorf(cx), fy = floorf(cy), fz = floorf(cz);
    const int px = (int)fx, py = (int)fy, pz = (int)fz;
    const int pxo = px + (__fsub_rn(cx, fx) < 0.5f ? -1 : 1);
    const int pyo = py + (__fsub_rn(cy, fy) < 0.5f ? -1 : 1);
    const int pzo = pz + (__fsub_rn(cz, fz) < 0.5f ? -1 : 1);
    for (int j = 0; j < 8; ++j) {
        const int x = (j & 4) ? pxo : px;
        const int y = (j & 2) ? pyo : py;
        const int z = (j & 1) ? pzo : pz;
        const int c = hash_cell((uint32_t)x, (uint32_t)y, (uint32_t)z, table);
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

}  // namespace imbart
