// GPU BVH builder: builds a whole scene (one BVH per mesh, a top-level BVH over the
// instances) on the device, directly in the compressed 8-wide layout the traversal kernels
// read, so that admitting a scene does not wait for a CPU build and a host-side conversion.
//
// The reference builds its mesh BVHs on the CPU, serially, with SBVH (sbvh_builder.h:29-165)
// and its top level with binned SAH (fast_bvh_builder.h); here every step runs in parallel
// kernels:
//   1. primitive boxes and the box of their centroids;
//   2. 63-bit Morton codes of the centroids, radix-sorted (CUB);
//   3. PLOC clustering (Meister and Bittner, "Parallel Locally-Ordered Clustering for
//      Bounding Volume Hierarchy Construction", TVCG 2018): every cluster finds its nearest
//      neighbour (smallest union surface area) among the 16 clusters on either side in Morton
//      order, mutual nearest neighbours merge, the cluster array is compacted; repeated until
//      one cluster is left. Merged nodes are numbered by prefix sums, so the tree does not
//      depend on thread timing;
//   4. a bottom-up pass computing surface-area costs (traversal cost 1, one unit per
//      primitive) that turns subtrees of at most three triangles into leaves where that is
//      cheaper (one instance per leaf at the top level);
//   5. a top-down collapse into 8-wide nodes, one level per launch: a wide node takes its
//      binary node's children and opens the largest-area internal child until it has 8,
//      assigns slots by direction octant, quantizes the child boxes conservatively (the same
//      arithmetic as the host converter, convert.cpp) and writes the leaves' triangle or
//      instance records.
// Hits do not depend on the tree: traversal over this layout finds the same closest hit
// as over any other BVH of the same triangles.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "imbart_internal.h"

namespace imbart {
namespace {

constexpr int kRadius = 16;          // PLOC search radius
constexpr int kBlock = 256;
constexpr int kMaxLeafTris = 3;

struct Box6 {
    float lo[3], hi[3];
};

__device__ __forceinline__ float half_area(const Box6& b) {
    const float dx = fmaxf(b.hi[0] - b.lo[0], 0.0f), dy = fmaxf(b.hi[1] - b.lo[1], 0.0f),
                dz = fmaxf(b.hi[2] - b.lo[2], 0.0f);
    return dx * (dy + dz) + dy * dz;
}

__device__ __forceinline__ Box6 merge(const Box6& a, const Box6& b) {
    Box6 r;
    for (int k = 0; k < 3; ++k) { r.lo[k] = fminf(a.lo[k], b.lo[k]); r.hi[k] = fmaxf(a.hi[k], b.hi[k]); }
    return r;
}

// Order-preserving int encoding of floats for atomicMin / atomicMax.
__device__ __forceinline__ int f2ord(float f) { const int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7fffffff; }
__device__ __forceinline__ float ord2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// ---------------------------------------------------------------------------------------
// 1-2. Boxes, centroid bounds, Morton codes
// ---------------------------------------------------------------------------------------
__global__ void tri_boxes_kernel(const float* __restrict__ v, const int4* __restrict__ idx, int n, Box6* boxes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 t = idx[i];
    Box6 b;
    for (int k = 0; k < 3; ++k) {
        const float a = v[3 * t.x + k], c = v[3 * t.y + k], d = v[3 * t.z + k];
        b.lo[k] = fminf(a, fminf(c, d));
        b.hi[k] = fmaxf(a, fmaxf(c, d));
    }
    boxes[i] = b;
}

// World boxes of instances, one block per instance: the bound of the instanced mesh's
// vertices through the 3x4 object-to-world matrix in double precision, rounded outward and
// widened by 2^-20 of its magnitude (tighter than transforming the mesh box for rotated
// instances).
__global__ void __launch_bounds__(kBlock) inst_boxes_kernel(const float* __restrict__ o2w, const int* __restrict__ mesh,
                                                            const float* __restrict__ verts,
                                                            const long long* __restrict__ vert_first,
                                                            const int* __restrict__ vert_count, Box6* boxes) {
    __shared__ double red[6][kBlock / 32];
    const int i = blockIdx.x;
    const float* m = o2w + 12 * i;
    const float* v = verts + 3 * vert_first[mesh[i]];
    const int nv = vert_count[mesh[i]];
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int k = threadIdx.x; k < nv; k += kBlock) {
        const double p[3] = {v[3 * k], v[3 * k + 1], v[3 * k + 2]};
        for (int r = 0; r < 3; ++r) {
            const double w = (double)m[4 * r] * p[0] + (double)m[4 * r + 1] * p[1] + (double)m[4 * r + 2] * p[2] +
                             (double)m[4 * r + 3];
            lo[r] = fmin(lo[r], w);
            hi[r] = fmax(hi[r], w);
        }
    }
    for (int r = 0; r < 3; ++r)
        for (int o = 16; o > 0; o >>= 1) {
            lo[r] = fmin(lo[r], __shfl_xor_sync(0xffffffffu, lo[r], o));
            hi[r] = fmax(hi[r], __shfl_xor_sync(0xffffffffu, hi[r], o));
        }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int r = 0; r < 3; ++r) { red[r][warp] = lo[r]; red[3 + r][warp] = hi[r]; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < kBlock / 32; ++w)
        for (int r = 0; r < 3; ++r) { lo[r] = fmin(lo[r], red[r][w]); hi[r] = fmax(hi[r], red[3 + r][w]); }
    double mag = 0.0;
    for (int r = 0; r < 3; ++r) mag = fmax(mag, fmax(fabs(lo[r]), fabs(hi[r])));
    const double pad = mag * 9.5367431640625e-07 + 1e-30;
    Box6 b;
    for (int r = 0; r < 3; ++r) { b.lo[r] = __double2float_rd(lo[r] - pad); b.hi[r] = __double2float_ru(hi[r] + pad); }
    boxes[i] = b;
}

__global__ void centroid_bounds_kernel(const Box6* __restrict__ boxes, int n, int* cb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    if (i < n) {
        const Box6 b = boxes[i];
        for (int k = 0; k < 3; ++k) { lo[k] = hi[k] = 0.5f * (b.lo[k] + b.hi[k]); }
    }
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) { atomicMin(cb + k, f2ord(lo[k])); atomicMax(cb + 3 + k, f2ord(hi[k])); }
    }
}

__device__ __forceinline__ uint64_t spread21(uint32_t x) {
    uint64_t v = x & 0x1fffffu;
    v = (v | (v << 32)) & 0x001f00000000ffffull;
    v = (v | (v << 16)) & 0x001f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void morton_kernel(const Box6* __restrict__ boxes, int n, const int* __restrict__ cb, uint64_t* keys,
                              int* vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Box6 b = boxes[i];
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
        const float lo = ord2f(cb[k]), hi = ord2f(cb[3 + k]);
        const float ext = hi - lo;
        const float c = 0.5f * (b.lo[k] + b.hi[k]);
        const float t = ext > 0.0f ? (c - lo) / ext : 0.0f;
        q[k] = (uint32_t)fminf(fmaxf(t * 2097152.0f, 0.0f), 2097151.0f);
    }
    keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    vals[i] = i;
}

// ---------------------------------------------------------------------------------------
// 3. PLOC
// ---------------------------------------------------------------------------------------
__global__ void ploc_init_kernel(const int* __restrict__ sorted, int n, const Box6* __restrict__ boxes, int* cl,
                                 Box6* clbox, Box6* nbox, int* parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = sorted[i];
    cl[i] = p;
    clbox[i] = boxes[p];
    nbox[i] = boxes[i];
    parent[i] = -1;
}

// Nearest neighbour of every cluster within kRadius positions (boxes staged in shared
// memory); ties go to the smaller position.
__global__ void __launch_bounds__(kBlock) ploc_nn_kernel(const Box6* __restrict__ clbox, int m, int* nn) {
    __shared__ Box6 sb[kBlock + 2 * kRadius];
    const int first = blockIdx.x * kBlock - kRadius;
    for (int t = threadIdx.x; t < kBlock + 2 * kRadius; t += kBlock) {
        const int j = first + t;
        if (j >= 0 && j < m) sb[t] = clbox[j];
    }
    __syncthreads();
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= m) return;
    const Box6 bi = sb[threadIdx.x + kRadius];
    float best = FLT_MAX;
    int bj = -1;
    const int lo = max(0, i - kRadius), hi = min(m - 1, i + kRadius);
    for (int j = lo; j <= hi; ++j) {
        if (j == i) continue;
        const float d = half_area(merge(bi, sb[j - first]));
        if (d < best) { best = d; bj = j; }
    }
    nn[i] = bj;
}

__global__ void ploc_flags_kernel(const int* __restrict__ nn, int m, int* mflag, int* kflag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    mflag[i] = (mutual && i < j) ? 1 : 0;
    kflag[i] = (mutual && i > j) ? 0 : 1;
}

__global__ void totals_kernel(const int* a, const int* as, const int* b, const int* bs, int m, int* out) {
    out[0] = as[m - 1] + a[m - 1];
    out[1] = b ? bs[m - 1] + b[m - 1] : 0;
}

__global__ void ploc_compact_kernel(const int* __restrict__ cl, const Box6* __restrict__ clbox, const int* __restrict__ nn,
                                    int m, const int* __restrict__ mflag, const int* __restrict__ mrank,
                                    const int* __restrict__ kflag, const int* __restrict__ kpos, int node_base,
                                    int* cl2, Box6* clbox2, Box6* nbox, int* left, int* right, int* parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !kflag[i]) return;
    const int o = kpos[i];
    if (mflag[i]) {
        const int j = nn[i];
        const int node = node_base + mrank[i];
        const int l = cl[i], r = cl[j];
        const Box6 b = merge(clbox[i], clbox[j]);
        nbox[node] = b;
        left[node] = l;
        right[node] = r;
        parent[l] = node;
        parent[r] = node;
        parent[node] = -1;
        cl2[o] = node;
        clbox2[o] = b;
    } else {
        cl2[o] = cl[i];
        clbox2[o] = clbox[i];
    }
}

// ---------------------------------------------------------------------------------------
// 4. Leaves by surface-area cost (bottom-up; the second child to finish continues)
// ---------------------------------------------------------------------------------------
__global__ void leaf_cost_kernel(int n, const Box6* __restrict__ nbox, const int* __restrict__ left,
                                 const int* __restrict__ right, const int* __restrict__ parent, int max_leaf,
                                 float* cost, int* cnt, uint8_t* leafy, int* visit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cnt[i] = 1;
    cost[i] = half_area(nbox[i]);
    leafy[i] = 1;
    int node = i;
    for (int guard = 0; guard < n; ++guard) {
        const int p = parent[node];
        if (p < 0) return;
        __threadfence();
        if (atomicAdd(visit + p, 1) == 0) return;
        __threadfence();
        const int l = left[p], r = right[p];
        const int c = __ldcg(cnt + l) + __ldcg(cnt + r);
        const float a = half_area(nbox[p]);
        const float inner = a + __ldcg(cost + l) + __ldcg(cost + r);
        const float leaf = a * (float)c;
        const bool lf = c <= max_leaf && leaf <= inner;
        cnt[p] = c;
        cost[p] = lf ? leaf : inner;
        leafy[p] = lf ? 1 : 0;
        node = p;
    }
}

// ---------------------------------------------------------------------------------------
// 5. Collapse into 8-wide nodes
// ---------------------------------------------------------------------------------------
__global__ void wide_gather_kernel(const int* __restrict__ qb, int q, const Box6* __restrict__ nbox,
                                   const int* __restrict__ left, const int* __restrict__ right,
                                   const uint8_t* __restrict__ leafy, const int* __restrict__ cnt, int* kids,
                                   int* nkids, int* n_int, int* n_prims) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= q) return;
    const int b = qb[e];
    int k[8];
    int nk;
    if (leafy[b]) {
        k[0] = b;
        nk = 1;
    } else {
        k[0] = left[b];
        k[1] = right[b];
        nk = 2;
        while (nk < 8) {
            int best = -1;
            float best_area = -1.0f;
            for (int i = 0; i < nk; ++i) {
                if (leafy[k[i]]) continue;
                const float a = half_area(nbox[k[i]]);
                if (a > best_area) { best_area = a; best = i; }
            }
            if (best < 0) break;
            const int c = k[best];
            for (int t = best; t < nk - 1; ++t) k[t] = k[t + 1];
            k[nk - 1] = left[c];
            k[nk] = right[c];
            ++nk;
        }
    }
    int ni = 0, np = 0;
    for (int i = 0; i < nk; ++i) {
        kids[8 * e + i] = k[i];
        if (leafy[k[i]]) np += cnt[k[i]];
        else ++ni;
    }
    nkids[e] = nk;
    n_int[e] = ni;
    n_prims[e] = np;
}

// Conservative 8-bit quantization of one axis (convert.cpp quantize_axis, same arithmetic).
__device__ void quantize_axis_dev(const float* lo, const float* hi, const bool* valid, float pad, float* p_out,
                                  uint8_t* bexp_out, uint8_t* qlo, uint8_t* qhi) {
    double nlo = DBL_MAX, nhi = -DBL_MAX;
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        nlo = fmin(nlo, (double)lo[i] - pad);
        nhi = fmax(nhi, (double)hi[i] + pad);
    }
    if (nlo > nhi) { nlo = 0.0; nhi = 0.0; }
    const double ext = nhi - nlo;
    int e = -126;
    if (ext > 0.0) {
        int ex;
        frexp(ext / 252.0, &ex);
        e = max(ex - 1, -126);
        while (e < 127 && ldexp(252.0, e) < ext) ++e;
    }
    float P = 0.0f;
    for (;;) {
        const double s = ldexp(1.0, e);
        const double margin = s / 128.0;
        const double origin = nlo - margin - 32768.0 * s;
        P = (float)origin;
        if ((double)P > origin) P = nextafterf(P, -FLT_MAX);
        bool ok = true;
        for (int i = 0; i < 8; ++i) {
            if (!valid[i]) { qlo[i] = 1; qhi[i] = 0; continue; }
            const double L = (double)lo[i] - pad - margin, H = (double)hi[i] + pad + margin;
            double ql = floor((L - (double)P) / s) - 32768.0;
            double qh = ceil((H - (double)P) / s) - 32768.0;
            for (int g = 0; g < 64 && (double)P + (32768.0 + ql) * s > L; ++g) ql -= 1;
            for (int g = 0; g < 64 && (double)P + (32768.0 + qh) * s < H; ++g) qh += 1;
            if (!(ql >= 0 && qh <= 255)) { ok = false; break; }
            qlo[i] = (uint8_t)ql;
            qhi[i] = (uint8_t)qh;
        }
        if (ok || e >= 127) break;
        ++e;
    }
    *p_out = P;
    *bexp_out = (uint8_t)(e + 127);
}

struct LeafOut {
    // Triangles (mode 0) or instances (mode 1).
    int mode;
    const float* verts;
    const int4* idx;
    int tri_offset;
    WideTri* tris;
    const float* w2o;       // 12 floats per instance
    const int* inst_id;
    const int* inst_mesh;
    const int* mesh_root;   // wide root per mesh
    WideInst* insts;
};

__device__ void emit_prim(const LeafOut& o, int prim, int at) {
    if (o.mode == 0) {
        const int4 t = o.idx[prim];
        WideTri r;
        for (int k = 0; k < 3; ++k) {
            r.v0[k] = o.verts[3 * t.x + k];
            r.v1[k] = o.verts[3 * t.y + k];
            r.v2[k] = o.verts[3 * t.z + k];
        }
        r.id = o.tri_offset + prim;
        r.pad0 = 0;
        r.pad1 = 0;
        o.tris[at] = r;
    } else {
        WideInst r;
        for (int k = 0; k < 12; ++k) r.m[k] = o.w2o[12 * prim + k];
        r.id = o.inst_id[prim];
        r.root = o.mesh_root[o.inst_mesh[prim]];
        r.pad[0] = 0;
        r.pad[1] = 0;
        o.insts[at] = r;
    }
}

__global__ void wide_write_kernel(const int* __restrict__ qb, int q, const int* __restrict__ kids,
                                  const int* __restrict__ nkids, const int* __restrict__ int_off,
                                  const int* __restrict__ prim_off, int wide_first, int child_first, int prim_first,
                                  const Box6* __restrict__ nbox, const int* __restrict__ left,
                                  const int* __restrict__ right, const uint8_t* __restrict__ leafy,
                                  const int* __restrict__ cnt, int n_leaves, WideNode* out, int* next_qb, LeafOut lo) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= q) return;
    const int nk = nkids[e];
    int k[8];
    for (int i = 0; i < nk; ++i) k[i] = kids[8 * e + i];

    // Slot assignment: slot s prefers children towards (s&1 ? +x : -x, s&2 ? +y : -y,
    // s&4 ? +z : -z); greedy over (score, kid, slot) in decreasing score, ties in kid/slot order.
    Box6 all = nbox[k[0]];
    for (int i = 1; i < nk; ++i) all = merge(all, nbox[k[i]]);
    float pc[3];
    for (int a = 0; a < 3; ++a) pc[a] = 0.5f * (all.lo[a] + all.hi[a]);
    float d[8][3];
    for (int i = 0; i < nk; ++i) {
        const Box6 b = nbox[k[i]];
        for (int a = 0; a < 3; ++a) d[i][a] = 0.5f * (b.lo[a] + b.hi[a]) - pc[a];
    }
    int slot_of[8];
    unsigned kid_done = 0, slot_used = 0;
    for (int round = 0; round < nk; ++round) {
        float best = -FLT_MAX;
        int bi = -1, bs = -1;
        for (int i = 0; i < nk; ++i) {
            if (kid_done & (1u << i)) continue;
            for (int s = 0; s < 8; ++s) {
                if (slot_used & (1u << s)) continue;
                const float score = (s & 1 ? d[i][0] : -d[i][0]) + (s & 2 ? d[i][1] : -d[i][1]) +
                                    (s & 4 ? d[i][2] : -d[i][2]);
                if (score > best || bi < 0) { best = score; bi = i; bs = s; }
            }
        }
        kid_done |= 1u << bi;
        slot_used |= 1u << bs;
        slot_of[bi] = bs;
    }
    int in_slot[8];
    for (int s = 0; s < 8; ++s) in_slot[s] = -1;
    for (int i = 0; i < nk; ++i) in_slot[slot_of[i]] = k[i];

    WideNode nd;
    memset(&nd, 0, sizeof(nd));
    const int child_base = child_first + int_off[e];
    const int prim_base = prim_first + prim_off[e];
    nd.child_base = (uint32_t)child_base;
    nd.prim_base = (uint32_t)prim_base;
    int rank = 0, poff = 0;
    for (int s = 0; s < 8; ++s) {
        const int c = in_slot[s];
        if (c < 0) continue;
        if (!leafy[c]) {
            nd.imask |= (uint8_t)(1u << s);
            next_qb[int_off[e] + rank] = c;
            ++rank;
            continue;
        }
        // The leaf's primitives, left to right (at most kMaxLeafTris).
        int stack[8], sp = 0, count = 0;
        stack[sp++] = c;
        while (sp > 0) {
            const int x = stack[--sp];
            if (x < n_leaves) {
                emit_prim(lo, x, prim_base + poff + count);
                ++count;
            } else {
                stack[sp++] = right[x];
                stack[sp++] = left[x];
            }
        }
        nd.meta[s] = (uint8_t)((count << 5) | poff);
        poff += count;
    }
    float blo[3][8], bhi[3][8];
    bool valid[8];
    float mag = 0.0f;
    for (int s = 0; s < 8; ++s) {
        valid[s] = in_slot[s] >= 0;
        for (int a = 0; a < 3; ++a) { blo[a][s] = 0.0f; bhi[a][s] = 0.0f; }
        if (!valid[s]) continue;
        const Box6 b = nbox[in_slot[s]];
        for (int a = 0; a < 3; ++a) {
            blo[a][s] = b.lo[a];
            bhi[a][s] = b.hi[a];
            mag = fmaxf(mag, fmaxf(fabsf(b.lo[a]), fabsf(b.hi[a])));
            mag = fmaxf(mag, b.hi[a] - b.lo[a]);
        }
    }
    const float pad = mag * 9.5367431640625e-07f + 1e-30f;
    float p[3];
    uint8_t bexp[3];
    quantize_axis_dev(blo[0], bhi[0], valid, pad, &p[0], &bexp[0], nd.qlo_x, nd.qhi_x);
    quantize_axis_dev(blo[1], bhi[1], valid, pad, &p[1], &bexp[1], nd.qlo_y, nd.qhi_y);
    quantize_axis_dev(blo[2], bhi[2], valid, pad, &p[2], &bexp[2], nd.qlo_z, nd.qhi_z);
    nd.px = p[0]; nd.py = p[1]; nd.pz = p[2];
    nd.ex = bexp[0]; nd.ey = bexp[1]; nd.ez = bexp[2];
    out[wide_first + e] = nd;
}

// ---------------------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------------------
bool ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? IMBART_ERR_OUT_OF_MEMORY : IMBART_ERR_CUDA,
              std::string("imbart_scene_build_gpu: ") + what + ": " + cudaGetErrorString(e));
    return false;
}

template <typename T>
bool dmalloc(T** p, size_t n) { *p = nullptr; return ck(cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(n, 1)), "cudaMalloc"); }

int grid(long long n) { return (int)std::max<long long>(1, (n + kBlock - 1) / kBlock); }

struct Scratch {
    long long cap = 0;
    Box6 *boxes = nullptr, *clbox = nullptr, *clbox2 = nullptr, *nbox = nullptr;
    uint64_t *keys = nullptr, *keys2 = nullptr;
    int *vals = nullptr, *vals2 = nullptr, *cl = nullptr, *cl2 = nullptr, *nn = nullptr;
    int *mflag = nullptr, *mrank = nullptr, *kflag = nullptr, *kpos = nullptr;
    int *left = nullptr, *right = nullptr, *parent = nullptr, *cnt = nullptr, *visit = nullptr;
    float* cost = nullptr;
    uint8_t* leafy = nullptr;
    int *qb = nullptr, *qb2 = nullptr, *kids = nullptr, *nkids = nullptr, *n_int = nullptr, *n_prims = nullptr,
        *int_off = nullptr, *prim_off = nullptr;
    int* cb = nullptr;
    int* totals = nullptr;
    int* h_totals = nullptr;   // pinned
    void* temp = nullptr;
    size_t temp_bytes = 0;

    bool alloc(long long n) {
        cap = n;
        const size_t m = (size_t)n, nodes = 2 * (size_t)n;
        bool ok = dmalloc(&boxes, m) && dmalloc(&clbox, m) && dmalloc(&clbox2, m) && dmalloc(&nbox, nodes) &&
                  dmalloc(&keys, m) && dmalloc(&keys2, m) && dmalloc(&vals, m) && dmalloc(&vals2, m) &&
                  dmalloc(&cl, m) && dmalloc(&cl2, m) && dmalloc(&nn, m) && dmalloc(&mflag, m) && dmalloc(&mrank, m) &&
                  dmalloc(&kflag, m) && dmalloc(&kpos, m) && dmalloc(&left, nodes) && dmalloc(&right, nodes) &&
                  dmalloc(&parent, nodes) && dmalloc(&cnt, nodes) && dmalloc(&visit, nodes) && dmalloc(&cost, nodes) &&
                  dmalloc(&leafy, nodes) && dmalloc(&qb, m) && dmalloc(&qb2, m) && dmalloc(&kids, 8 * m) &&
                  dmalloc(&nkids, m) && dmalloc(&n_int, m) && dmalloc(&n_prims, m) && dmalloc(&int_off, m) &&
                  dmalloc(&prim_off, m) && dmalloc(&cb, 8) && dmalloc(&totals, 4) &&
                  ck(cudaMallocHost((void**)&h_totals, 4 * sizeof(int)), "cudaMallocHost");
        if (!ok) return false;
        size_t a = 0, b = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, a, keys, keys2, vals, vals2, (int)n, 0, 63);
        cub::DeviceScan::ExclusiveSum(nullptr, b, mflag, mrank, (int)n);
        temp_bytes = std::max(a, b);
        return ck(cudaMalloc(&temp, temp_bytes), "cudaMalloc");
    }
    void release() {
        void* ps[] = {boxes, clbox, clbox2, nbox, keys, keys2, vals, vals2, cl, cl2, nn, mflag, mrank, kflag, kpos,
                      left, right, parent, cnt, visit, cost, leafy, qb, qb2, kids, nkids, n_int, n_prims, int_off,
                      prim_off, cb, totals, temp};
        for (void* p : ps) cudaFree(p);
        cudaFreeHost(h_totals);
    }
};

bool read_totals(Scratch& S, cudaStream_t st) {
    return ck(cudaMemcpyAsync(S.h_totals, S.totals, 2 * sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync") &&
           ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

bool scan(Scratch& S, const int* in, int* out, int n, cudaStream_t st) {
    size_t bytes = S.temp_bytes;
    return ck(cub::DeviceScan::ExclusiveSum(S.temp, bytes, in, out, n, st), "DeviceScan");
}

// Builds the binary tree over S.boxes[0, n) (steps 1-4); returns the root node or -1.
int build_binary(Scratch& S, int n, int max_leaf, cudaStream_t st) {
    // The atomics start at the extreme encodings (f2ord is monotonic over the ints).
    static const int init[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, (int)0x80000000, (int)0x80000000, (int)0x80000000};
    if (!ck(cudaMemcpyAsync(S.cb, init, sizeof(init), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync")) return -1;
    centroid_bounds_kernel<<<grid(n), kBlock, 0, st>>>(S.boxes, n, S.cb);
    morton_kernel<<<grid(n), kBlock, 0, st>>>(S.boxes, n, S.cb, S.keys, S.vals);
    size_t bytes = S.temp_bytes;
    if (!ck(cub::DeviceRadixSort::SortPairs(S.temp, bytes, S.keys, S.keys2, S.vals, S.vals2, n, 0, 63, st), "SortPairs"))
        return -1;
    ploc_init_kernel<<<grid(n), kBlock, 0, st>>>(S.vals2, n, S.boxes, S.cl, S.clbox, S.nbox, S.parent);
    note_launches(4);
    int m = n, node_base = n;
    int* cl = S.cl;
    int* cl2 = S.cl2;
    Box6* cb1 = S.clbox;
    Box6* cb2 = S.clbox2;
    for (int iter = 0; m > 1; ++iter) {
        if (iter > n) { set_error(IMBART_ERR_CUDA, "imbart_scene_build_gpu: clustering made no progress"); return -1; }
        ploc_nn_kernel<<<grid(m), kBlock, 0, st>>>(cb1, m, S.nn);
        ploc_flags_kernel<<<grid(m), kBlock, 0, st>>>(S.nn, m, S.mflag, S.kflag);
        if (!scan(S, S.mflag, S.mrank, m, st) || !scan(S, S.kflag, S.kpos, m, st)) return -1;
        ploc_compact_kernel<<<grid(m), kBlock, 0, st>>>(cl, cb1, S.nn, m, S.mflag, S.mrank, S.kflag, S.kpos, node_base,
                                                        cl2, cb2, S.nbox, S.left, S.right, S.parent);
        totals_kernel<<<1, 1, 0, st>>>(S.mflag, S.mrank, S.kflag, S.kpos, m, S.totals);
        note_launches(6);
        if (!ck(cudaGetLastError(), "clustering kernels") || !read_totals(S, st)) return -1;
        const int merges = S.h_totals[0], kept = S.h_totals[1];
        if (merges <= 0 || kept != m - merges) {
            set_error(IMBART_ERR_CUDA, "imbart_scene_build_gpu: clustering made no progress");
            return -1;
        }
        node_base += merges;
        m = kept;
        std::swap(cl, cl2);
        std::swap(cb1, cb2);
    }
    int root = 0;
    if (!ck(cudaMemcpyAsync(&root, cl, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync") ||
        !ck(cudaMemsetAsync(S.visit, 0, sizeof(int) * (size_t)node_base, st), "cudaMemsetAsync"))
        return -1;
    leaf_cost_kernel<<<grid(n), kBlock, 0, st>>>(n, S.nbox, S.left, S.right, S.parent, max_leaf, S.cost, S.cnt,
                                                 S.leafy, S.visit);
    note_launches(1);
    if (!ck(cudaGetLastError(), "leaf kernel") || !ck(cudaStreamSynchronize(st), "cudaStreamSynchronize")) return -1;
    return root;
}

// Collapses the binary tree rooted at `root` into wide nodes from *wide_count on (the
// root first) and leaf records from *prim_count on. Returns the wide root or -1.
int collapse(Scratch& S, int root, int n_leaves, WideNode* out, int* wide_count, int* prim_count, const LeafOut& lo,
             cudaStream_t st) {
    const int wroot = *wide_count;
    if (!ck(cudaMemcpyAsync(S.qb, &root, sizeof(int), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync")) return -1;
    int q = 1;
    int level_first = wroot;     // wide index of the level's first node
    int next_free = wroot + 1;   // first wide index after the nodes allocated so far
    int* qb = S.qb;
    int* qb2 = S.qb2;
    for (int level = 0; q > 0; ++level) {
        if (level > 4 * n_leaves + 8) { set_error(IMBART_ERR_CUDA, "imbart_scene_build_gpu: collapse did not end"); return -1; }
        wide_gather_kernel<<<grid(q), kBlock, 0, st>>>(qb, q, S.nbox, S.left, S.right, S.leafy, S.cnt, S.kids,
                                                       S.nkids, S.n_int, S.n_prims);
        if (!scan(S, S.n_int, S.int_off, q, st) || !scan(S, S.n_prims, S.prim_off, q, st)) return -1;
        totals_kernel<<<1, 1, 0, st>>>(S.n_int, S.int_off, S.n_prims, S.prim_off, q, S.totals);
        wide_write_kernel<<<grid(q), kBlock, 0, st>>>(qb, q, S.kids, S.nkids, S.int_off, S.prim_off, level_first,
                                                      next_free, *prim_count, S.nbox, S.left, S.right, S.leafy, S.cnt,
                                                      n_leaves, out, qb2, lo);
        note_launches(5);
        if (!ck(cudaGetLastError(), "collapse kernels") || !read_totals(S, st)) return -1;
        const int n_int = S.h_totals[0], n_prims = S.h_totals[1];
        *prim_count += n_prims;
        level_first = next_free;
        next_free += n_int;
        q = n_int;
        std::swap(qb, qb2);
    }
    *wide_count = next_free;
    return wroot;
}

int build_scene_gpu(const imbart_mesh_desc* meshes, int n_meshes, const imbart_instance_desc* insts, int n_insts,
                    int device, void* stream, imbart_scene** out, float* build_ms) {
    *out = nullptr;
    if (!meshes || n_meshes <= 0 || !insts || n_insts <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_scene_build_gpu: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    long long total_tris = 0, max_n = n_insts;
    for (int k = 0; k < n_meshes; ++k) {
        const imbart_mesh_desc& m = meshes[k];
        if (!m.vertices || !m.indices || m.n_vertices <= 0 || m.n_tris <= 0) {
            set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_scene_build_gpu: empty mesh");
            return IMBART_ERR_INVALID_ARGUMENT;
        }
        for (long long t = 0; t < 4ll * m.n_tris; ++t) {
            if ((t & 3) == 3) continue;
            if (m.indices[t] < 0 || m.indices[t] >= m.n_vertices) {
                set_error(IMBART_ERR_BAD_SCENE, "imbart_scene_build_gpu: vertex index out of range");
                return IMBART_ERR_BAD_SCENE;
            }
        }
        total_tris += m.n_tris;
        max_n = std::max<long long>(max_n, m.n_tris);
    }
    for (int i = 0; i < n_insts; ++i)
        if (insts[i].mesh < 0 || insts[i].mesh >= n_meshes) {
            set_error(IMBART_ERR_BAD_SCENE, "imbart_scene_build_gpu: instance of an unknown mesh");
            return IMBART_ERR_BAD_SCENE;
        }
    if (total_tris >= (1ll << 30) || max_n >= (1ll << 29)) {
        set_error(IMBART_ERR_LIMIT, "imbart_scene_build_gpu: scene too large");
        return IMBART_ERR_LIMIT;
    }
    int prev = 0;
    cudaGetDevice(&prev);
    if (!ck(cudaSetDevice(device), "cudaSetDevice")) return IMBART_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const auto t0 = std::chrono::steady_clock::now();
    Scratch S;
    WideNode* nodes = nullptr;
    WideTri* tris = nullptr;
    WideInst* winsts = nullptr;
    float* d_verts = nullptr;
    int4* d_idx = nullptr;
    float *d_o2w = nullptr, *d_w2o = nullptr;
    int *d_mesh = nullptr, *d_id = nullptr, *d_roots = nullptr;
    // Wide nodes: at most one per binary internal node, plus one per mesh (and the top).
    const long long node_cap = total_tris + n_insts + n_meshes + 2;
    long long total_verts = 0;
    std::vector<long long> vert_first(n_meshes);
    std::vector<int> vert_count(n_meshes);
    for (int k = 0; k < n_meshes; ++k) {
        vert_first[k] = total_verts;
        vert_count[k] = meshes[k].n_vertices;
        total_verts += meshes[k].n_vertices;
    }
    long long* d_vfirst = nullptr;
    int* d_vcount = nullptr;
    bool good = S.alloc(max_n) && dmalloc(&nodes, node_cap) && dmalloc(&tris, total_tris) && dmalloc(&winsts, n_insts) &&
                dmalloc(&d_verts, 3 * total_verts) && dmalloc(&d_idx, max_n) &&
                dmalloc(&d_vfirst, n_meshes) && dmalloc(&d_vcount, n_meshes) &&
                dmalloc(&d_o2w, 12 * (size_t)n_insts) && dmalloc(&d_w2o, 12 * (size_t)n_insts) &&
                dmalloc(&d_mesh, n_insts) && dmalloc(&d_id, n_insts) && dmalloc(&d_roots, n_meshes);
    int wide_count = 0, prim_count = 0, root = -1;
    std::vector<int> mesh_root(n_meshes, 0);
    for (int k = 0; k < n_meshes && good; ++k) {
        const imbart_mesh_desc& m = meshes[k];
        float* mv = d_verts + 3 * vert_first[k];
        good = ck(cudaMemcpyAsync(mv, m.vertices, sizeof(float) * 3 * (size_t)m.n_vertices, cudaMemcpyDefault, st),
                  "cudaMemcpyAsync") &&
               ck(cudaMemcpyAsync(d_idx, m.indices, sizeof(int4) * (size_t)m.n_tris, cudaMemcpyDefault, st),
                  "cudaMemcpyAsync");
        if (!good) break;
        tri_boxes_kernel<<<grid(m.n_tris), kBlock, 0, st>>>(mv, d_idx, m.n_tris, S.boxes);
        note_launches(1);
        const int broot = build_binary(S, m.n_tris, kMaxLeafTris, st);
        if (broot < 0) { good = false; break; }
        LeafOut lo{};
        lo.mode = 0;
        lo.verts = mv;
        lo.idx = d_idx;
        lo.tri_offset = m.tri_offset;
        lo.tris = tris;
        mesh_root[k] = collapse(S, broot, m.n_tris, nodes, &wide_count, &prim_count, lo, st);
        if (mesh_root[k] < 0) good = false;
    }
    const int bottom_nodes = wide_count;
    if (good) {
        std::vector<float> o2w(12 * (size_t)n_insts), w2o(12 * (size_t)n_insts);
        std::vector<int> mesh(n_insts), id(n_insts);
        for (int i = 0; i < n_insts; ++i) {
            std::memcpy(&o2w[12 * i], insts[i].obj_to_world, 12 * sizeof(float));
            std::memcpy(&w2o[12 * i], insts[i].world_to_obj, 12 * sizeof(float));
            mesh[i] = insts[i].mesh;
            id[i] = insts[i].id;
        }
        good = ck(cudaMemcpyAsync(d_o2w, o2w.data(), o2w.size() * sizeof(float), cudaMemcpyHostToDevice, st), "copy") &&
               ck(cudaMemcpyAsync(d_w2o, w2o.data(), w2o.size() * sizeof(float), cudaMemcpyHostToDevice, st), "copy") &&
               ck(cudaMemcpyAsync(d_mesh, mesh.data(), mesh.size() * sizeof(int), cudaMemcpyHostToDevice, st), "copy") &&
               ck(cudaMemcpyAsync(d_id, id.data(), id.size() * sizeof(int), cudaMemcpyHostToDevice, st), "copy") &&
               ck(cudaMemcpyAsync(d_roots, mesh_root.data(), mesh_root.size() * sizeof(int), cudaMemcpyHostToDevice, st),
                  "copy") &&
               ck(cudaMemcpyAsync(d_vfirst, vert_first.data(), vert_first.size() * sizeof(long long),
                                  cudaMemcpyHostToDevice, st), "copy") &&
               ck(cudaMemcpyAsync(d_vcount, vert_count.data(), vert_count.size() * sizeof(int), cudaMemcpyHostToDevice,
                                  st), "copy");
        if (good) {
            inst_boxes_kernel<<<n_insts, kBlock, 0, st>>>(d_o2w, d_mesh, d_verts, d_vfirst, d_vcount, S.boxes);
            note_launches(1);
            const int broot = build_binary(S, n_insts, 1, st);
            if (broot < 0) good = false;
            if (good) {
                LeafOut lo{};
                lo.mode = 1;
                lo.w2o = d_w2o;
                lo.inst_id = d_id;
                lo.inst_mesh = d_mesh;
                lo.mesh_root = d_roots;
                lo.insts = winsts;
                int inst_count = 0;
                root = collapse(S, broot, n_insts, nodes, &wide_count, &inst_count, lo, st);
                good = root >= 0 && ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
            }
        }
    }
    S.release();
    cudaFree(d_verts); cudaFree(d_idx); cudaFree(d_o2w); cudaFree(d_w2o);
    cudaFree(d_vfirst); cudaFree(d_vcount);
    cudaFree(d_mesh); cudaFree(d_id); cudaFree(d_roots);
    int rc = 0;
    if (good) {
        imbart_scene* s = scene_adopt_device_arrays(device, nodes, wide_count, wide_count - bottom_nodes, tris,
                                                    prim_count, winsts, n_insts, root);
        if (s) {
            *out = s;
            if (build_ms)
                *build_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        } else {
            good = false;
        }
    }
    if (!good) {
        cudaFree(nodes); cudaFree(tris); cudaFree(winsts);
        rc = imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA;
    }
    cudaSetDevice(prev);
    return rc;
}

// ---------------------------------------------------------------------------------------
// Refit: the vertices moved, the topology did not. Triangle records take their triangle's
// new vertices; node boxes are recomputed bottom-up (bottom levels, then the instances'
// world boxes, then the top level) and requantized with the build's conservative
// arithmetic. Each leaf-only node starts a thread that refits it and climbs: the last child
// of a parent to finish refits the parent (a counter per node).
// ---------------------------------------------------------------------------------------
__global__ void refit_tris_kernel(WideTri* tris, long long n, const float* __restrict__ verts,
                                  const int4* __restrict__ tri_verts, int n_tri_ids, long long n_verts, int* error) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    WideTri t = tris[i];
    if (t.id < 0 || t.id >= n_tri_ids) { atomicExch(error, 1); return; }
    const int4 v = tri_verts[t.id];
    if (v.x < 0 || v.y < 0 || v.z < 0 || v.x >= n_verts || v.y >= n_verts || v.z >= n_verts) {
        atomicExch(error, 2);
        return;
    }
    for (int k = 0; k < 3; ++k) {
        t.v0[k] = verts[3 * (long long)v.x + k];
        t.v1[k] = verts[3 * (long long)v.y + k];
        t.v2[k] = verts[3 * (long long)v.z + k];
    }
    tris[i] = t;
}

// Parent of every internal child and the count of internal children of nodes [first, last).
__global__ void refit_links_kernel(const WideNode* __restrict__ nodes, int first, int last, int* parent, int* pending) {
    const int n = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= last) return;
    const WideNode nd = nodes[n];
    pending[n] = __popc(nd.imask);
    int rank = 0;
    for (int s = 0; s < 8; ++s)
        if (nd.imask & (1u << s)) parent[nd.child_base + rank++] = n;
}

__device__ __forceinline__ Box6 empty_box() {
    Box6 b;
    for (int a = 0; a < 3; ++a) { b.lo[a] = FLT_MAX; b.hi[a] = -FLT_MAX; }
    return b;
}

// Another thread's finished box, read past the L1 cache.
__device__ __forceinline__ Box6 load_box_cg(const Box6* p) {
    const float* f = reinterpret_cast<const float*>(p);
    Box6 b;
    for (int a = 0; a < 3; ++a) { b.lo[a] = __ldcg(f + a); b.hi[a] = __ldcg(f + 3 + a); }
    return b;
}

// Requantizes node n from its children (leaf slots: their triangles or instances; internal
// slots: the boxes their refits stored) and stores its own box.
__device__ void refit_node(WideNode* nodes, int n, const WideTri* __restrict__ tris, const Box6* inst_boxes, bool top,
                           Box6* exact) {
    WideNode nd = nodes[n];
    float blo[3][8], bhi[3][8];
    bool valid[8];
    float mag = 0.0f;
    Box6 all = empty_box();
    int rank = 0;
    for (int s = 0; s < 8; ++s) {
        Box6 b = empty_box();
        if (nd.imask & (1u << s)) {
            b = load_box_cg(exact + nd.child_base + rank++);
            valid[s] = true;
        } else {
            const int count = nd.meta[s] >> 5, off = nd.meta[s] & 31;
            valid[s] = count > 0;
            for (int k = 0; k < count; ++k) {
                const long long r = (long long)nd.prim_base + off + k;
                if (top) {
                    b = merge(b, inst_boxes[r]);
                } else {
                    const WideTri t = tris[r];
                    for (int a = 0; a < 3; ++a) {
                        b.lo[a] = fminf(b.lo[a], fminf(t.v0[a], fminf(t.v1[a], t.v2[a])));
                        b.hi[a] = fmaxf(b.hi[a], fmaxf(t.v0[a], fmaxf(t.v1[a], t.v2[a])));
                    }
                }
            }
        }
        for (int a = 0; a < 3; ++a) { blo[a][s] = valid[s] ? b.lo[a] : 0.0f; bhi[a][s] = valid[s] ? b.hi[a] : 0.0f; }
        if (!valid[s]) continue;
        all = merge(all, b);
        for (int a = 0; a < 3; ++a) {
            mag = fmaxf(mag, fmaxf(fabsf(b.lo[a]), fabsf(b.hi[a])));
            mag = fmaxf(mag, b.hi[a] - b.lo[a]);
        }
    }
    const float pad = mag * 9.5367431640625e-07f + 1e-30f;
    float p[3];
    uint8_t bexp[3];
    quantize_axis_dev(blo[0], bhi[0], valid, pad, &p[0], &bexp[0], nd.qlo_x, nd.qhi_x);
    quantize_axis_dev(blo[1], bhi[1], valid, pad, &p[1], &bexp[1], nd.qlo_y, nd.qhi_y);
    quantize_axis_dev(blo[2], bhi[2], valid, pad, &p[2], &bexp[2], nd.qlo_z, nd.qhi_z);
    nd.px = p[0]; nd.py = p[1]; nd.pz = p[2];
    nd.ex = bexp[0]; nd.ey = bexp[1]; nd.ez = bexp[2];
    nodes[n] = nd;
    exact[n] = all;
}

__global__ void refit_up_kernel(WideNode* nodes, int first, int last, const int* __restrict__ parent, int* pending,
                                const WideTri* __restrict__ tris, const Box6* inst_boxes, bool top, Box6* exact) {
    int n = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= last || nodes[n].imask != 0) return;
    for (;;) {
        refit_node(nodes, n, tris, inst_boxes, top, exact);
        __threadfence();
        const int p = parent[n];
        if (p < 0) return;
        if (atomicSub(pending + p, 1) != 1) return;   // the parent's last child to finish goes on
        __threadfence();
        n = p;
    }
}

// World box of each instance record: its mesh root's box through the object-to-world
// transform (the inverse of the stored world-to-object rows, in double precision), corners
// rounded outward and widened by 2^-20 of their magnitude.
__global__ void refit_inst_boxes_kernel(const WideInst* __restrict__ insts, int n, const Box6* exact, Box6* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const WideInst w = insts[i];
    const Box6 b = load_box_cg(exact + w.root);
    double a[3][3], t[3];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) a[r][c] = w.m[4 * r + c];
        t[r] = w.m[4 * r + 3];
    }
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                       a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                       a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int c = 0; c < 8; ++c) {
        const double x = (c & 1) ? b.hi[0] : b.lo[0], y = (c & 2) ? b.hi[1] : b.lo[1], z = (c & 4) ? b.hi[2] : b.lo[2];
        const double px = x - t[0], py = y - t[1], pz = z - t[2];   // object = A world + t  =>  world = A^-1 (object - t)
        for (int r = 0; r < 3; ++r) {
            const double v = inv[r][0] * px + inv[r][1] * py + inv[r][2] * pz;
            lo[r] = fmin(lo[r], v);
            hi[r] = fmax(hi[r], v);
        }
    }
    Box6 o;
    double m = 0.0;
    for (int r = 0; r < 3; ++r) m = fmax(m, fmax(fabs(lo[r]), fabs(hi[r])));
    const double pad = m * 9.5367431640625e-07 + 1e-30;
    for (int r = 0; r < 3; ++r) {
        o.lo[r] = __double2float_rd(lo[r] - pad);
        o.hi[r] = __double2float_ru(hi[r] + pad);
    }
    out[i] = o;
}

int refit_scene(imbart_scene* scene, const float* verts, long long n_verts, const int* tri_verts, int n_tri_ids,
                cudaStream_t st) {
    imbart_scene_info info;
    const void *vn = nullptr, *vt = nullptr, *vi = nullptr;
    if (imbart_scene_get_info(scene, &info) != 0 || imbart_scene_get_device_arrays(scene, &vn, &vt, &vi) != 0)
        return imbart_last_error() ? imbart_last_error() : IMBART_ERR_INVALID_ARGUMENT;
    if (!vn || info.wide_nodes <= 0 || info.wide_nodes > INT_MAX || info.top_nodes <= 0 ||
        info.top_nodes > info.wide_nodes) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_scene_refit: scene without its own node array");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    WideNode* nodes = static_cast<WideNode*>(const_cast<void*>(vn));
    WideTri* tris = static_cast<WideTri*>(const_cast<void*>(vt));
    const WideInst* insts = static_cast<const WideInst*>(vi);
    const int n_nodes = (int)info.wide_nodes, first_top = (int)(info.wide_nodes - info.top_nodes);
    Box6 *exact = nullptr, *inst_boxes = nullptr;
    int *parent = nullptr, *pending = nullptr, *error = nullptr;
    bool good = dmalloc(&exact, n_nodes) && dmalloc(&inst_boxes, info.instances) && dmalloc(&parent, n_nodes) &&
                dmalloc(&pending, n_nodes) && dmalloc(&error, 1) &&
                ck(cudaMemsetAsync(parent, 0xff, sizeof(int) * (size_t)n_nodes, st), "cudaMemsetAsync") &&
                ck(cudaMemsetAsync(error, 0, sizeof(int), st), "cudaMemsetAsync");
    if (good) {
        refit_tris_kernel<<<grid(info.triangles), kBlock, 0, st>>>(tris, info.triangles, verts,
                                                                    reinterpret_cast<const int4*>(tri_verts), n_tri_ids,
                                                                    n_verts, error);
        refit_links_kernel<<<grid(n_nodes), kBlock, 0, st>>>(nodes, 0, n_nodes, parent, pending);
        if (first_top > 0)
            refit_up_kernel<<<grid(first_top), kBlock, 0, st>>>(nodes, 0, first_top, parent, pending, tris, nullptr,
                                                               false, exact);
        refit_inst_boxes_kernel<<<grid(info.instances), kBlock, 0, st>>>(insts, (int)info.instances, exact,
                                                                        inst_boxes);
        refit_up_kernel<<<grid(info.top_nodes), kBlock, 0, st>>>(nodes, first_top, n_nodes, parent, pending, tris,
                                                                inst_boxes, true, exact);
        note_launches(first_top > 0 ? 5 : 4);
        int h_error = 0;
        good = ck(cudaGetLastError(), "refit launch") &&
               ck(cudaMemcpyAsync(&h_error, error, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync") &&
               ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        if (good && h_error) {
            set_error(IMBART_ERR_INVALID_ARGUMENT, h_error == 1 ? "imbart_scene_refit: a triangle id beyond n_tri_ids"
                                                                : "imbart_scene_refit: a vertex index out of range");
            good = false;
        }
    }
    cudaFree(exact); cudaFree(inst_boxes); cudaFree(parent); cudaFree(pending); cudaFree(error);
    return good ? 0 : (imbart_last_error() ? imbart_last_error() : IMBART_ERR_CUDA);
}

}  // namespace
}  // namespace imbart

extern "C" int imbart_scene_refit(imbart_scene* scene, const float* vertices, long long n_vertices,
                                  const int* tri_vertices, int n_tri_ids, void* stream) {
    if (!scene || !vertices || !tri_vertices || n_vertices <= 0 || n_tri_ids <= 0) {
        imbart::set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_scene_refit: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    imbart_scene_info info;
    if (imbart_scene_get_info(scene, &info) != 0) return imbart_last_error();
    int prev = 0;
    cudaGetDevice(&prev);
    int dev = prev;
    // The scene's device: the one its arrays live on (pointer attributes).
    const void* vn = nullptr;
    const void* vt = nullptr;
    const void* vi = nullptr;
    imbart_scene_get_device_arrays(scene, &vn, &vt, &vi);
    cudaPointerAttributes attr;
    if (vn && cudaPointerGetAttributes(&attr, vn) == cudaSuccess && attr.type == cudaMemoryTypeDevice) dev = attr.device;
    cudaSetDevice(dev);
    const int rc = imbart::refit_scene(scene, vertices, n_vertices, tri_vertices, n_tri_ids, (cudaStream_t)stream);
    cudaSetDevice(prev);
    return rc;
}

extern "C" imbart_scene* imbart_scene_build_gpu(const imbart_mesh_desc* meshes, int n_meshes,
                                                const imbart_instance_desc* instances, int n_instances, int device,
                                                void* stream, float* build_ms) {
    imbart_scene* s = nullptr;
    imbart::build_scene_gpu(meshes, n_meshes, instances, n_instances, device, stream, &s, build_ms);
    return s;
}
