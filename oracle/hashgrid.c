/*
 * Oracle: CPU restatement of the reference's photon hash grid (HashGrid in
 * src/imbatracer/rangesearch/rangesearch.h). TEST INFRASTRUCTURE ONLY.
 *
 *   build  rangesearch.h:25-75   radius, r^2, cell size (2r in the reference), inverse cell
 *                                 size; bbox of the photon positions inflated by 0.1 % of its
 *                                 extent per side; counting sort of photons into
 *                                 `table_size` hashed cells (2 * photon count in the reference)
 *   hash   rangesearch.h:137-148 ((x*73856093) ^ (y*19349663) ^ (z*83492791)) mod size on
 *                                 unsigned cell coordinates, coords = floor((p - min) / cell)
 *   query  rangesearch.h:77-129  home cell plus the nearer neighbour per axis (8 cells, in
 *                                 the reference's order), squared distance <= r^2, at most k
 *                                 nearest kept by insertion sort (ties keep the earlier photon,
 *                                 an equal distance replaces the last one when full)
 * Within a cell photons are ordered by ascending original index (the reference's order there
 * depends on its parallel scatter, rangesearch.h:68-74); query results are compared as sets.
 * Compiled with -ffp-contract=off so every float operation rounds as in the reference.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    float lo[3], hi[3];
    float radius, radius_sqr, cell_size, inv_cell_size;
    uint32_t table_size;
    int32_t n;
} o_grid;

static int cell_index_u(const o_grid* g, uint32_t x, uint32_t y, uint32_t z) {
    return (int)(((x * 73856093u) ^ (y * 19349663u) ^ (z * 83492791u)) % g->table_size);
}

static int cell_index_p(const o_grid* g, const float* p) {
    const float dx = g->inv_cell_size * (p[0] - g->lo[0]);
    const float dy = g->inv_cell_size * (p[1] - g->lo[1]);
    const float dz = g->inv_cell_size * (p[2] - g->lo[2]);
    const int cx = (int)floorf(dx), cy = (int)floorf(dy), cz = (int)floorf(dz);
    return cell_index_u(g, (uint32_t)cx, (uint32_t)cy, (uint32_t)cz);
}

/* Builds the grid over n positions (xyz at pos + i * stride floats). cell_ends receives
 * table_size inclusive ends, sorted_ids the original photon index of each sorted slot. */
void oracle_hashgrid_build(const float* pos, int stride, int n, float radius, float cell_factor,
                           int table_size, o_grid* g, int* cell_ends, int* sorted_ids) {
    g->radius = radius;
    g->radius_sqr = radius * radius;
    g->cell_size = radius * cell_factor;
    g->inv_cell_size = 1.0f / g->cell_size;
    g->table_size = (uint32_t)table_size;
    g->n = n;
    for (int a = 0; a < 3; ++a) { g->lo[a] = FLT_MAX; g->hi[a] = -FLT_MAX; }
    for (int i = 0; i < n; ++i) {
        const float* p = pos + (size_t)i * stride;
        for (int a = 0; a < 3; ++a) {
            g->lo[a] = g->lo[a] < p[a] ? g->lo[a] : p[a];
            g->hi[a] = g->hi[a] > p[a] ? g->hi[a] : p[a];
        }
    }
    float ext[3];
    for (int a = 0; a < 3; ++a) ext[a] = g->hi[a] - g->lo[a];
    for (int a = 0; a < 3; ++a) g->hi[a] = g->hi[a] + ext[a] * 0.001f;
    for (int a = 0; a < 3; ++a) g->lo[a] = g->lo[a] - ext[a] * 0.001f;

    int* cell = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    memset(cell_ends, 0, sizeof(int) * (size_t)table_size);
    for (int i = 0; i < n; ++i) {
        cell[i] = cell_index_p(g, pos + (size_t)i * stride);
        cell_ends[cell[i]]++;
    }
    int sum = 0;
    for (int c = 0; c < table_size; ++c) { const int t = cell_ends[c]; cell_ends[c] = sum; sum += t; }
    for (int i = 0; i < n; ++i) sorted_ids[cell_ends[cell[i]]++] = i;
    free(cell);
}

/* Cell coordinate of a coordinate value with the build's rounding. */
static int grid_coord(const o_grid* g, float v, int axis) {
    return (int)floorf(g->inv_cell_size * (v - g->lo[axis]));
}

/* q - r rounded down and q + r rounded up (the box a photon within r lies in). */
static float sub_down(float q, float r) {
    float a = q - r;
    if ((double)a > (double)q - (double)r) a = nextafterf(a, -INFINITY);
    return a;
}
static float add_up(float q, float r) {
    float b = q + r;
    if ((double)b < (double)q + (double)r) b = nextafterf(b, INFINITY);
    return b;
}

/* Queries nq positions; out_ids gets up to k original photon indices per query (ordered by
 * distance as the reference's insertion sort leaves them), out_count the count and
 * out_d2 (optional) the squared distances. Grids whose cell is at least 2r (the reference's)
 * scan the reference's eight cells; grids with r <= cell < 2r scan every cell the box
 * [q - r, q + r] touches (bounds rounded outward, at most 4 per axis), x-major, each bucket
 * once — the same cells and order as the GPU query. */
void oracle_hashgrid_query(const o_grid* g, const int* cell_ends, const int* sorted_ids,
                           const float* pos, int stride, const float* queries, int nq, int k,
                           int* out_ids, int* out_count, float* out_d2, int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(threads)
    for (int q = 0; q < nq; ++q) {
        const float* qp = queries + 3 * (size_t)q;
        int* ids = out_ids + (size_t)q * k;
        float dist[256];
        int count = 0;
        const int inside = qp[0] >= g->lo[0] && qp[1] >= g->lo[1] && qp[2] >= g->lo[2] &&
                           qp[0] <= g->hi[0] && qp[1] <= g->hi[1] && qp[2] <= g->hi[2];
        if (inside && k > 0 && k <= 256) {
            const int ref_mode = g->cell_size >= 2.0f * g->radius;
            int cells[64];
            int n = 0;
            if (ref_mode) {
                const float cx = g->inv_cell_size * (qp[0] - g->lo[0]);
                const float cy = g->inv_cell_size * (qp[1] - g->lo[1]);
                const float cz = g->inv_cell_size * (qp[2] - g->lo[2]);
                const float fx = floorf(cx), fy = floorf(cy), fz = floorf(cz);
                const int px = (int)fx, py = (int)fy, pz = (int)fz;
                const int pxo = px + ((cx - fx) < 0.5f ? -1 : 1);
                const int pyo = py + ((cy - fy) < 0.5f ? -1 : 1);
                const int pzo = pz + ((cz - fz) < 0.5f ? -1 : 1);
                for (int j = 0; j < 8; ++j)
                    cells[n++] = cell_index_u(g, (uint32_t)((j & 4) ? pxo : px), (uint32_t)((j & 2) ? pyo : py),
                                              (uint32_t)((j & 1) ? pzo : pz));
            } else {
                int lo_c[3], cnt[3];
                for (int a = 0; a < 3; ++a) {
                    lo_c[a] = grid_coord(g, sub_down(qp[a], g->radius), a);
                    cnt[a] = grid_coord(g, add_up(qp[a], g->radius), a) - lo_c[a] + 1;
                    if (cnt[a] > 4) cnt[a] = 4;
                }
                for (int x = 0; x < cnt[0]; ++x)
                    for (int y = 0; y < cnt[1]; ++y)
                        for (int z = 0; z < cnt[2]; ++z) {
                            const int c = cell_index_u(g, (uint32_t)(lo_c[0] + x), (uint32_t)(lo_c[1] + y),
                                                       (uint32_t)(lo_c[2] + z));
                            int seen = 0;
                            for (int i = 0; i < n; ++i) seen |= cells[i] == c;
                            if (!seen) cells[n++] = c;
                        }
            }
            for (int j = 0; j < n; ++j) {
                const int c = cells[j];
                const int b = c == 0 ? 0 : cell_ends[c - 1];
                const int e = cell_ends[c];
                for (int s = b; s < e; ++s) {
                    const int id = sorted_ids[s];
                    const float* pp = pos + (size_t)id * stride;
                    const float dx = qp[0] - pp[0], dy = qp[1] - pp[1], dz = qp[2] - pp[2];
                    const float d2 = (dx * dx + dy * dy) + dz * dz;
                    if (!(d2 <= g->radius_sqr)) continue;
                    if (count == k) {
                        if (dist[count - 1] < d2) continue;
                    } else {
                        count++;
                    }
                    dist[count - 1] = d2;
                    ids[count - 1] = id;
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
        }
        out_count[q] = count;
        for (int i = count; i < k; ++i) ids[i] = -1;
        if (out_d2)
            for (int i = 0; i < k; ++i) out_d2[(size_t)q * k + i] = i < count ? dist[i] : 0.0f;
    }
}
